"""World-size-2 gloo test of the particle-sharded statistics merge (CPU only).

Each rank accumulates its shard of a mu cache and of a momentum cache (with
the oracle, standing in for the per-GPU kernels), takes the D_pp
normalisation p0 from rank 0 (shard.broadcast_p0) and the ranks merge with
shard.reduce_dmumu_accumulators / shard.reduce_dpp_accumulators, the calls
bench.py makes under torchrun; the merged result must equal a single pass
over all particles: counts exactly, sums and Welford moments to 1e-12."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import random_mu_cache, zero_dmumu, zero_dpp
from particle_transport_b200 import shard
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


DPP_KEYMAP = {"counts": "counts", "sum_dp": "sum_delta_p", "sum_dp2": "sum_delta_p2", "sum_dpn": "sum_delta_p_norm",
              "sum_dpn2": "sum_delta_p_norm2"}


def random_momenta(n, nsave, seed=11):
    """float32 momenta shaped (nsave, 3, n) with a slow random walk of |p|."""
    rng = np.random.default_rng(seed)
    p = np.abs(1.0 + 0.01 * np.cumsum(rng.normal(size=(nsave, n)), axis=0))
    d = rng.normal(size=(nsave, 3, n))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    mom = (d * p[:, None, :] * 5.3e-18).astype(np.float32)
    mom[rng.random(mom.shape) < 0.01] = np.nan
    mom[0, :, 0] = np.abs(mom[0, :, 0])  # particle 0 is finite at the first save (it defines p0)
    return mom


def p0_of(mom):
    m = mom[0, :, 0].astype(np.float64)
    return float(np.sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]))


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
    mom = random_momenta(301, 90)
    p0 = shard.broadcast_p0(p0_of(np.ascontiguousarray(mom[:, :, a:b])) if a < b else float("nan"))
    dacc = zero_dpp(len(lags))
    o.dpp_accumulate(np.ascontiguousarray(mom[:, :, a:b]), lags, p0, dacc, nthreads=1)
    dmerged = shard.reduce_dpp_accumulators({DPP_KEYMAP[k]: v for k, v in dacc.items()})
    dist.barrier()
    dist.destroy_process_group()
    out_q.put((rank, (merged, dmerged, p0)))


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
    mom = random_momenta(301, 90)
    dref = zero_dpp(len(lags))
    oracle.dpp_accumulate(mom, lags, p0_of(mom), dref, nthreads=1)
    for r in range(world):
        m, d, p0 = res[r]
        assert p0 == p0_of(mom)  # rank 1 took rank 0's p0
        assert np.array_equal(d["counts"], dref["counts"]) and d["counts"].sum() > 0
        for k in ("sum_dp", "sum_dp2", "sum_dpn", "sum_dpn2"):
            assert np.allclose(d[DPP_KEYMAP[k]], dref[k], rtol=1e-12, atol=0), k
        assert np.array_equal(m["dmumu_counts"], ref["counts"])
        assert np.array_equal(m["pair_counts"], ref["pair_n"])
        assert np.array_equal(m["particle_counts"], ref["w_count"])
        assert np.allclose(m["dmumu_sum_delta2"], ref["sum_d2"], rtol=1e-12, atol=0)
        assert np.allclose(m["particle_means"], ref["w_mean"], rtol=1e-12, atol=0)
        assert np.allclose(m["particle_m2s"], ref["w_m2"], rtol=1e-10, atol=0)
    # both ranks hold the identical merged result
    for part in (0, 1):
        for k in res[0][part]:
            assert np.array_equal(res[0][part][k], res[1][part][k])


@pytest.mark.parametrize("n,world", [(10, 3), (16_777_216, 8), (1, 2), (0, 4)])
def test_shard_ranges_cover(n, world):
    rs = [shard.shard_range(n, r, world) for r in range(world)]
    assert rs[0][0] == 0 and rs[-1][1] == n
    assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
    sizes = [b - a for a, b in rs]
    assert max(sizes) - min(sizes) <= 1
