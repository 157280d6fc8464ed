"""Batched campaigns (pt_batch_*) on a B200.

Every campaign's mu cache and final state must be bit-identical to the
same campaign run alone through pt_push_advance_fast: the batch changes only
which slot and which CTA a particle lands on, never its arithmetic.  That
holds with the per-campaign brick sort, with CUDA-graph epochs, and when
campaigns join and leave between epochs (continuous batching)."""
import math

import numpy as np
import pytest

from helpers import small_problem
from particle_transport_b200 import runner as R
from particle_transport_b200.batch import Batch, autotune, tune_batch
from particle_transport_b200.fields import FieldLibrary
from particle_transport_b200.particles import energy_to_gamma, init_particles
from particle_transport_b200.time_units import reference_Omega0
from particle_transport_b200 import fields as F

pytestmark = pytest.mark.gpu


def campaigns(torch, storage="brick_bf16"):
    pa = small_problem(n=16, n_particles=1000, u_over_c=1e-4, seed=3)
    pb = small_problem(n=16, n_particles=10, u_over_c=2e-4, seed=8)
    fa = FieldLibrary(pa.fields, pa.grid, storage)
    fb = FieldLibrary(pb.fields, pb.grid, storage)
    out = []
    for i, (fl, pbm, E, n, nsteps, stride) in enumerate([(fa, pa, 1.0, 1000, 301, 4), (fb, pb, 10.0, 700, 129, 8),
                                                          (fa, pa, 3.0, 257, 200, 5), (fb, pb, 1.0, 3, 77, 1)]):
        g0 = energy_to_gamma(E)
        Om = reference_Omega0(pa.B0, g0, F.Q_E, F.M_P)
        dt = (2 * math.pi / 64) / Om
        st = init_particles(n, pbm.grid, E, seed=100 + i)
        out.append(dict(field=fl, state=st, dt=dt, nsteps=nsteps, stride=stride))
    return out


def run_alone(torch, c):
    ens = R.FastEnsemble(c["field"], c["state"], np.ones(len(c["state"]["x1"]), np.uint8))
    nsave = R.n_saves(c["nsteps"], c["stride"])
    cache = torch.full((nsave, ens.n), float("nan"), dtype=torch.float32, device="cuda")
    ens.advance(R.push_params(c["dt"], c["nsteps"], c["stride"], cache="mu", precision="f32"), 0, c["nsteps"],
                cache, 0, nsave)
    st, al = ens.export()
    torch.cuda.synchronize()
    return cache.cpu().numpy(), {k: v.cpu().numpy() for k, v in st.items()}


def new_cache(torch, c):
    return torch.full((R.n_saves(c["nsteps"], c["stride"]), len(c["state"]["x1"])), float("nan"),
                      dtype=torch.float32, device="cuda")


@pytest.mark.parametrize("sort,graph,K,every", [(True, True, 64, (1, 1, 1, 1)), (True, False, 32, (1, 1, 1, 1)),
                                               (False, True, 50, (1, 1, 1, 1)), (True, True, 16, (1, 3, 2, 5)),
                                               (True, False, 16, (4, 1, 0, 2))])
def test_batch_bit_identical_to_single_runs(cuda, sort, graph, K, every):
    """Every campaign ends with the cache and state of its run alone, with a
    sort before every epoch, on per-campaign cadences (each campaign then
    holds its slots in its own buffer of the pair), or without sorting."""
    torch = cuda
    cs = campaigns(torch)
    ref = [run_alone(torch, c) for c in cs]
    b = Batch(5000, max_campaigns=8, steps_per_epoch=K, sort=sort)
    caches = [new_cache(torch, c) for c in cs]
    ids = [b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ch, sort_every=e)
           for c, ch, e in zip(cs, caches, every)]
    epochs = max(math.ceil(c["nsteps"] / K) for c in cs)
    b.run(epochs, use_graph=graph)
    for c, cid, ch, (mu_ref, st_ref) in zip(cs, ids, caches, ref):
        assert b.step(cid) == c["nsteps"]
        assert np.array_equal(ch.cpu().numpy(), mu_ref, equal_nan=True)
        st, _ = b.export(cid)
        for k in st:
            assert np.array_equal(st[k].cpu().numpy(), st_ref[k]), k
    b.close()


def test_batch_join_and_leave(cuda):
    torch = cuda
    cs = campaigns(torch)
    ref = [run_alone(torch, c) for c in cs]
    b = Batch(1300, max_campaigns=3, steps_per_epoch=64)
    caches = [new_cache(torch, c) for c in cs]
    live = {}
    live[0] = b.add(cs[0]["field"], cs[0]["state"], cs[0]["dt"], cs[0]["nsteps"], cs[0]["stride"], cache=caches[0])
    b.run(2)
    live[2] = b.add(cs[2]["field"], cs[2]["state"], cs[2]["dt"], cs[2]["nsteps"], cs[2]["stride"], cache=caches[2])
    b.run(1)
    live[3] = b.add(cs[3]["field"], cs[3]["state"], cs[3]["dt"], cs[3]["nsteps"], cs[3]["stride"], cache=caches[3])
    finished = {}
    pending = [1]
    for _ in range(40):
        b.run(1)
        for j, cid in list(live.items()):
            if b.done(cid):
                st, _ = b.export(cid)
                finished[j] = {k: v.cpu().numpy() for k, v in st.items()}
                b.remove(cid)
                del live[j]
        # campaign 1 joins when slots free up (capacity 1300 < sum of all)
        if pending:
            try:
                j = pending[0]
                live[j] = b.add(cs[j]["field"], cs[j]["state"], cs[j]["dt"], cs[j]["nsteps"], cs[j]["stride"],
                                cache=caches[j])
                pending.pop()
            except Exception:
                pass
        if not live and not pending:
            break
    assert sorted(finished) == [0, 1, 2, 3]
    for j, (mu_ref, st_ref) in enumerate(ref):
        assert np.array_equal(caches[j].cpu().numpy(), mu_ref, equal_nan=True), j
        for k in st_ref:
            assert np.array_equal(finished[j][k], st_ref[k]), (j, k)
    b.close()


@pytest.mark.parametrize("sort", [True, False])
def test_batch_pause_and_resume(cuda, sort):
    """Campaigns paused for some epochs (pt_batch_set_running) and resumed --
    after an odd number of epochs, so that the sort buffers changed parity
    while they waited -- end with the caches and states of their runs alone."""
    torch = cuda
    cs = campaigns(torch)
    ref = [run_alone(torch, c) for c in cs]
    K = 32
    b = Batch(5000, max_campaigns=8, steps_per_epoch=K, sort=sort)
    caches = [new_cache(torch, c) for c in cs]
    ids = [b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ch) for c, ch in zip(cs, caches)]
    b.run(1)
    b.set_running([ids[1], ids[3]])
    st0 = {k: v.cpu().numpy() for k, v in b.export(ids[0])[0].items()}
    b.run(3)
    assert b.step(ids[0]) == K and b.step(ids[2]) == K
    assert b.step(ids[1]) == min(4 * K, cs[1]["nsteps"])
    # a paused campaign exports the state it stopped with
    st0b = {k: v.cpu().numpy() for k, v in b.export(ids[0])[0].items()}
    for k in st0:
        assert np.array_equal(st0[k], st0b[k]), k
    b.set_running([ids[0]])
    b.run(2)
    b.set_running([ids[2], ids[0]])
    b.run(1)
    b.set_running(None)
    b.run(max(math.ceil(c["nsteps"] / K) for c in cs))
    for c, cid, ch, (mu_ref, st_ref) in zip(cs, ids, caches, ref):
        assert b.step(cid) == c["nsteps"]
        assert np.array_equal(ch.cpu().numpy(), mu_ref, equal_nan=True)
        st, _ = b.export(cid)
        for k in st:
            assert np.array_equal(st[k].cpu().numpy(), st_ref[k]), k
    from particle_transport_b200._lib import PtError
    b.remove(ids[3])
    with pytest.raises(PtError, match="no such campaign"):
        b.set_running([ids[3]])
    b.close()


def test_batch_ring_cache(cuda):
    torch = cuda
    c = campaigns(torch)[1]
    mu_ref, _ = run_alone(torch, c)
    b = Batch(1000, max_campaigns=2, steps_per_epoch=64)
    ring = torch.full((5, len(c["state"]["x1"])), float("nan"), dtype=torch.float32, device="cuda")
    cid = b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ring, ring=True)
    b.run(math.ceil(c["nsteps"] / 64))
    nsave = mu_ref.shape[0]
    got = ring.cpu().numpy()
    for r in range(nsave - 5, nsave):
        assert np.array_equal(got[r % 5], mu_ref[r], equal_nan=True)
    b.close()


def test_batch_rejects_bad_input(cuda):
    torch = cuda
    from particle_transport_b200._lib import PtError
    c = campaigns(torch)[0]
    b = Batch(100, max_campaigns=1)
    with pytest.raises(PtError, match="no free slot"):
        b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"])
    fr = FieldLibrary(*[small_problem(n=8, n_particles=2).__dict__[k] for k in ("fields", "grid")], "ref_f64")
    st = {k: v[:10] for k, v in c["state"].items()}
    with pytest.raises(PtError, match="storage"):
        b.add(fr, st, c["dt"], c["nsteps"], c["stride"])
    b.close()


def test_autotune_picks_a_candidate(cuda, tmp_path, monkeypatch):
    torch = cuda
    monkeypatch.setenv("PTB200_TUNE_CACHE", str(tmp_path))
    cs = campaigns(torch)
    best, timings = autotune(cs, "brick_bf16", 5000, epochs=1, candidates=((64, 2), (32, 1)))
    assert best in ((64, 2), (32, 1)) and len(timings) == 2
    best2, _ = autotune(cs, "brick_bf16", 5000, epochs=1, candidates=((64, 2), (32, 1)))
    assert best2 == best  # served from the cache file


def test_tune_batch_picks_cadences(cuda, tmp_path, monkeypatch):
    torch = cuda
    monkeypatch.setenv("PTB200_TUNE_CACHE", str(tmp_path))
    cs = campaigns(torch)
    shapes = ((256, 1), (128, 2), (64, 4))
    t = tune_batch(cs, "brick_bf16", 5000, cadences=(16, 32), shapes=shapes, steps=64)
    assert t["K"] in (16, 32) and (t["threads_per_block"], t["blocks_per_sm"]) in shapes and not t["cached"]
    assert len(t["sort_every"]) == len(cs) and all(v >= 1 for v in t["sort_every"])
    assert all(v in (16, 32) for v in t["cadence_steps"].values())
    t2 = tune_batch(cs, "brick_bf16", 5000, cadences=(16, 32), shapes=shapes, steps=64)
    assert t2["cached"] and t2["K"] == t["K"] and t2["sort_every"] == t["sort_every"]
    # the tuned batch gives every campaign the result of its run alone
    ref = [run_alone(torch, c) for c in cs]
    b = Batch(5000, max_campaigns=8, steps_per_epoch=t["K"], blocks_per_sm=t["blocks_per_sm"],
              threads_per_block=t["threads_per_block"])
    caches = [new_cache(torch, c) for c in cs]
    for c, ch, e in zip(cs, caches, t["sort_every"]):
        b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ch, sort_every=e)
    b.run(max(math.ceil(c["nsteps"] / t["K"]) for c in cs))
    for ch, (mu_ref, _) in zip(caches, ref):
        assert np.array_equal(ch.cpu().numpy(), mu_ref, equal_nan=True)
    b.close()


@pytest.mark.parametrize("K,every", [(64, (1, 1, 1, 1)), (16, (1, 3, 2, 5))])
def test_batch_time_fastest_caches_bit_identical(cuda, K, every):
    """Campaigns with time-fastest mu caches ([n][pitch]: each particle's
    saves contiguous) hold the values of the row caches of their runs alone."""
    torch = cuda
    cs = campaigns(torch)
    ref = [run_alone(torch, c) for c in cs]
    b = Batch(5000, max_campaigns=8, steps_per_epoch=K, sort=True)
    caches = [torch.full((len(c["state"]["x1"]), R.n_saves(c["nsteps"], c["stride"]) + 3), float("inf"),
                         dtype=torch.float32, device="cuda") for c in cs]
    ids = [b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ch, sort_every=e, time_fastest=True)
           for c, ch, e in zip(cs, caches, every)]
    b.run(max(math.ceil(c["nsteps"] / K) for c in cs))
    for c, cid, ch, (mu_ref, _) in zip(cs, ids, caches, ref):
        assert b.step(cid) == c["nsteps"]
        got = ch.cpu().numpy()
        nsave = mu_ref.shape[0]
        assert np.array_equal(got[:, :nsave].T, mu_ref, equal_nan=True)
        assert np.all(np.isinf(got[:, nsave:]))  # the pad past the last save is left alone
    b.close()


def test_batch_time_fastest_ring(cuda):
    torch = cuda
    c = campaigns(torch)[1]
    mu_ref, _ = run_alone(torch, c)
    b = Batch(1000, max_campaigns=2, steps_per_epoch=64)
    ring = torch.full((len(c["state"]["x1"]), 8), float("nan"), dtype=torch.float32, device="cuda")
    cid = b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ring, ring=True, time_fastest=True)
    b.run(math.ceil(c["nsteps"] / 64))
    nsave = mu_ref.shape[0]
    got = ring.cpu().numpy()
    for r in range(nsave - 8, nsave):
        assert np.array_equal(got[:, r % 8], mu_ref[r], equal_nan=True)
    b.close()


@pytest.mark.parametrize("threads,bps", [(128, 4), (64, 8), (256, 3)])
def test_batch_launch_shapes_bit_identical(cuda, threads, bps):
    """Threads per block (particles per thread = 256 / threads) and blocks per
    SM change only which thread advances a particle: caches and states are
    those of the runs alone."""
    torch = cuda
    cs = campaigns(torch)
    ref = [run_alone(torch, c) for c in cs]
    b = Batch(5000, max_campaigns=8, steps_per_epoch=32, sort=True, blocks_per_sm=bps, threads_per_block=threads)
    caches = [new_cache(torch, c) for c in cs]
    ids = [b.add(c["field"], c["state"], c["dt"], c["nsteps"], c["stride"], cache=ch, sort_every=2)
           for c, ch in zip(cs, caches)]
    b.run(3)
    b.set_launch(256, 2)  # a new shape between epochs: the graph is captured again
    b.run(max(math.ceil(c["nsteps"] / 32) for c in cs))
    for c, cid, ch, (mu_ref, st_ref) in zip(cs, ids, caches, ref):
        assert np.array_equal(ch.cpu().numpy(), mu_ref, equal_nan=True)
        st, _ = b.export(cid)
        for k in st:
            assert np.array_equal(st[k].cpu().numpy(), st_ref[k]), k
    from particle_transport_b200._lib import PtError
    with pytest.raises(PtError, match="threads_per_block"):
        b.set_launch(96, 2)
    b.close()
