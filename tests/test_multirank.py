"""World-size-2 gloo test of the particle-sharded statistics merge (CPU only).

Each rank accumulates its shard of a mu cache (with the oracle, standing in
for the per-GPU kernel) and the ranks merge with
shard.reduce_dmumu_accumulators; the merged result must equal a single pass
over all particles: counts exactly, sums and Welford moments to 1e-12."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import random_mu_cache, zero_dmumu
from particle_transport_b200 import shard
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


KEYMAP = {"counts": "dmumu_counts", "sum_d": "dmumu_sum_delta", "sum_d2": "dmumu_sum_delta2",
          "w_count": "particle_counts", "w_mean": "particle_means", "w_m2": "particle_m2s",
          "pair_ss": "pair_sum_squares", "pair_n": "pair_counts"}


def _worker(rank, world, port, out_q):
    import torch.distributed as dist

    from oracle import oracle as o
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mu = random_mu_cache(301, 90, seed=7, nan_frac=0.02)
    lags = log_spaced_lag_steps(89, 9)
    edges, _ = build_mu_edges_full(0.0, 1.0, 12)
    a, b = shard.shard_range(mu.shape[0], rank, world)
    acc = zero_dmumu(len(lags), 12)
    o.dmumu_accumulate(np.ascontiguousarray(mu[a:b]), lags, edges, acc, nthreads=1)
    merged = shard.reduce_dmumu_accumulators({KEYMAP[k]: v for k, v in acc.items()})
    dist.barrier()
    dist.destroy_process_group()
    out_q.put((rank, merged))


def test_sharded_merge_matches_single_pass(oracle):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mu = random_mu_cache(301, 90, seed=7, nan_frac=0.02)
    lags = log_spaced_lag_steps(89, 9)
    edges, _ = build_mu_edges_full(0.0, 1.0, 12)
    ref = zero_dmumu(len(lags), 12)
    oracle.dmumu_accumulate(mu, lags, edges, ref, nthreads=1)
    for r in range(world):
        m = res[r]
        assert np.array_equal(m["dmumu_counts"], ref["counts"])
        assert np.array_equal(m["pair_counts"], ref["pair_n"])
        assert np.array_equal(m["particle_counts"], ref["w_count"])
        assert np.allclose(m["dmumu_sum_delta2"], ref["sum_d2"], rtol=1e-12, atol=0)
        assert np.allclose(m["particle_means"], ref["w_mean"], rtol=1e-12, atol=0)
        assert np.allclose(m["particle_m2s"], ref["w_m2"], rtol=1e-10, atol=0)
    # both ranks hold the identical merged result
    for k in res[0]:
        assert np.array_equal(res[0][k], res[1][k])


@pytest.mark.parametrize("n,world", [(10, 3), (16_777_216, 8), (1, 2), (0, 4)])
def test_shard_ranges_cover(n, world):
    rs = [shard.shard_range(n, r, world) for r in range(world)]
    assert rs[0][0] == 0 and rs[-1][1] == n
    assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
    sizes = [b - a for a, b in rs]
    assert max(sizes) - min(sizes) <= 1
