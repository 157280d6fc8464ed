"""Campaign server (continuous batching) on a B200.

A job's result must not depend on what else runs beside it: its mu cache
is bit-identical alone and in the mix, and its D_mumu products agree to the
statistics tolerance (counts exact, FP64 sums to 1e-12 -- they differ only
by summation order).  The HBM budget must hold jobs back until memory
frees up, and every job must still finish."""
import numpy as np
import pytest

from helpers import small_problem
from particle_transport_b200.fields import FieldLibrary, reference_B0_T
from particle_transport_b200.server import CampaignServer, JobSpec

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def library(cuda):
    pa = small_problem(n=16, n_particles=4, u_over_c=1e-4, seed=3)
    pb = small_problem(n=16, n_particles=4, u_over_c=2e-4, seed=9)
    libs = {"16": {"total": FieldLibrary(pa.fields, pa.grid, "brick_bf16"),
                   "alfven": FieldLibrary(pb.fields, pb.grid, "brick_bf16")}}
    B0 = {"16": reference_B0_T(*pa.fields[:3])}
    return libs, B0


@pytest.fixture(scope="module")
def library64b(cuda):
    pa = small_problem(n=16, n_particles=4, u_over_c=1e-4, seed=3)
    pb = small_problem(n=16, n_particles=4, u_over_c=2e-4, seed=9)
    libs = {"16": {"total": FieldLibrary(pa.fields, pa.grid, "brick_f64"),
                   "alfven": FieldLibrary(pb.fields, pb.grid, "brick_f64")}}
    return libs, {"16": reference_B0_T(*pa.fields[:3])}


@pytest.fixture(scope="module")
def library64(cuda):
    pa = small_problem(n=16, n_particles=4, u_over_c=1e-4, seed=3)
    pb = small_problem(n=16, n_particles=4, u_over_c=2e-4, seed=9)
    libs = {"16": {"total": FieldLibrary(pa.fields, pa.grid, "ref_f64"),
                   "alfven": FieldLibrary(pb.fields, pb.grid, "ref_f64")}}
    return libs, {"16": reference_B0_T(*pa.fields[:3])}


JOBS = [JobSpec("16", "total", 1.0, 3000, 6.0, seed=1),
        JobSpec("16", "alfven", 20.0, 777, 3.5, injection="fixed_mu", mu0=0.3, seed=2),
        JobSpec("16", "total", 5.0, 1500, 9.0, seed=3, n_lags=12, n_bins=10, dpp_particles=500),
        JobSpec("16", "alfven", 2.0, 64, 2.0, seed=4)]


def run_jobs(library, jobs, budget=150e9, stagger_ticks=0, push="f32", schedule="srpt", fill=1 << 22):
    libs, B0 = library
    srv = CampaignServer(libs, B0, hbm_budget_bytes=budget, capacity=20000, max_jobs=8, keep_cache=True, push=push,
                         schedule=schedule, fill_particles=fill)
    pending = list(jobs)
    ids = []
    while pending or not srv.idle():
        if pending:
            ids.append(srv.submit(pending.pop(0)))
            for _ in range(stagger_ticks):
                srv.tick()
        else:
            srv.tick()
    res = {r.job_id: r for r in srv.results}
    srv.close()
    return [res[i] for i in ids]


def same(a, b):
    assert np.array_equal(a.mu, b.mu, equal_nan=True)
    for k in ("dmumu_counts", "pair_counts", "particle_counts"):
        assert np.array_equal(a.acc[k], b.acc[k]), k
    for k in ("dmumu_sum_delta2", "pair_sum_squares", "particle_means"):
        assert np.allclose(a.acc[k], b.acc[k], rtol=1e-12, atol=0), k
    sc = 1e-12 * (np.sqrt(np.maximum(b.acc["dmumu_counts"], 1) * b.acc["dmumu_sum_delta2"]) + 1e-30)
    assert np.all(np.abs(a.acc["dmumu_sum_delta"] - b.acc["dmumu_sum_delta"]) <= sc)
    same_dpp(a.dpp, b.dpp)


def same_dpp(a, b):
    assert (a is None) == (b is None)
    if b is None:
        return
    assert a["p0"] == b["p0"]
    assert np.array_equal(a["counts"], b["counts"]) and a["counts"].sum() > 0
    for k in ("sum_delta_p2", "sum_delta_p_norm2"):
        assert np.allclose(a[k], b[k], rtol=1e-12, atol=0), k
    for k, k2 in (("sum_delta_p", "sum_delta_p2"), ("sum_delta_p_norm", "sum_delta_p_norm2")):
        sc = 1e-12 * (np.sqrt(np.maximum(b["counts"], 1) * b[k2]) + 1e-300)
        assert np.all(np.abs(a[k] - b[k]) <= sc), k


def test_job_results_same_alone_and_in_the_mix(library):
    alone = [run_jobs(library, [j])[0] for j in JOBS]
    mixed = run_jobs(library, JOBS, stagger_ticks=1)
    for a, m in zip(alone, mixed):
        same(m, a)
        assert m.particle_steps > 0 and m.latency > 0
    # the products are populated: pair counts equal sum over lags of valid starts
    assert all(r.acc["pair_counts"].sum() > 0 for r in mixed)


@pytest.mark.parametrize("schedule,fill", [("srpt", 1000), ("srpt", 1), ("all", 0)])
def test_schedules_give_the_same_results(library, schedule, fill):
    """Least-work-first epochs that hold back all but a few jobs (fill of
    1000 or 1 particles: the waiting jobs are paused in the batch) and the
    every-job schedule give every job the results of its run alone."""
    alone = [run_jobs(library, [j])[0] for j in JOBS]
    mixed = run_jobs(library, JOBS, stagger_ticks=1, schedule=schedule, fill=fill)
    for a, m in zip(alone, mixed):
        same(m, a)


def test_srpt_finishes_small_jobs_first(library):
    """With one job running at a time, jobs submitted together finish in the
    order of their work (particles x steps)."""
    res = run_jobs(library, JOBS, schedule="srpt", fill=1)
    by_finish = [r.job_id for r in sorted(res, key=lambda r: r.finished)]
    by_work = [r.job_id for r in sorted(res, key=lambda r: r.particle_steps)]
    assert by_finish == by_work


def test_budget_holds_jobs_back(library):
    sizes = [CampaignServer.job_bytes(j) for j in JOBS]
    budget = max(sizes) * 1.05  # the largest job must run without company
    res = run_jobs(library, JOBS, budget=budget)
    assert len(res) == len(JOBS)
    # at every admission the jobs in flight fit the budget
    for r in res:
        t = r.admitted
        in_flight = sum(CampaignServer.job_bytes(q.spec) for q in res if q.admitted <= t < q.finished)
        assert in_flight <= budget
    big = max(res, key=lambda r: CampaignServer.job_bytes(r.spec))
    assert all(not (q.admitted <= big.admitted < q.finished) for q in res if q is not big)
    alone = run_jobs(library, [JOBS[2]])[0]
    same([r for r in res if r.spec is JOBS[2]][0], alone)


def test_fp64_server_alone_mixed_and_direct(library64):
    """The plain FP64 push served: each job's result is the same alone and in
    the mix, and its mu cache is the one a direct FP64 run of the same initial
    state writes (bit for bit)."""
    import math

    import torch

    from particle_transport_b200 import runner as R
    from particle_transport_b200.fields import M_P, Q_E
    from particle_transport_b200.particles import energy_to_gamma, init_particles_device
    from particle_transport_b200.time_units import reference_Omega0

    alone = [run_jobs(library64, [j], push="f64")[0] for j in JOBS]
    mixed = run_jobs(library64, JOBS, stagger_ticks=1, push="f64")
    for a, m in zip(alone, mixed):
        same(m, a)
    libs, B0 = library64
    j = JOBS[1]
    fl = libs[j.library][j.mode]
    st = init_particles_device(fl, j.n_particles, j.energy_GeV, seed=j.seed, injection_mode=j.injection, mu0=j.mu0)
    dt = (2 * math.pi / j.steps_per_gyroperiod) / reference_Omega0(B0[j.library], energy_to_gamma(j.energy_GeV), Q_E,
                                                                   M_P)
    nsteps = int(round(j.duration_gyroperiods * j.steps_per_gyroperiod)) + 1
    stride = j.steps_per_gyroperiod // j.saves_per_gyroperiod
    nsave = R.n_saves(nsteps, stride)
    ens = R.DeviceEnsemble(fl, st, np.ones(j.n_particles, np.uint8))
    cache = torch.empty((nsave, j.n_particles), dtype=torch.float32, device="cuda")
    ens.advance(R.push_params(dt, nsteps, stride, cache="mu", precision="f64"), 0, nsteps, cache, 0, nsave)
    torch.cuda.synchronize()
    assert np.array_equal(mixed[1].mu, cache.cpu().numpy(), equal_nan=True)


def test_dpp_of_served_job_equals_direct_phase_space_run(library):
    """A served job's D_pp subset: the same momenta as a direct phase-space
    run of the same initial state, so the same D_pp sums."""
    import math

    import torch

    from particle_transport_b200 import runner as R
    from particle_transport_b200 import stats as S
    from particle_transport_b200.fields import M_P, Q_E
    from particle_transport_b200.particles import energy_to_gamma, init_particles_device
    from particle_transport_b200.time_units import reference_Omega0

    j = JOBS[2]
    res = run_jobs(library, [j])[0]
    libs, B0 = library
    fl = libs[j.library][j.mode]
    st = init_particles_device(fl, j.n_particles, j.energy_GeV, seed=j.seed, injection_mode=j.injection, mu0=j.mu0)
    dt = (2 * math.pi / j.steps_per_gyroperiod) / reference_Omega0(B0[j.library], energy_to_gamma(j.energy_GeV), Q_E,
                                                                   M_P)
    nsteps = int(round(j.duration_gyroperiods * j.steps_per_gyroperiod)) + 1
    stride = j.steps_per_gyroperiod // j.saves_per_gyroperiod
    nsave = R.n_saves(nsteps, stride)
    ens = R.FastEnsemble(fl, st, np.ones(j.n_particles, np.uint8))
    ps = torch.empty((nsave, 6, j.n_particles), dtype=torch.float32, device="cuda")
    ens.advance(R.push_params(dt, nsteps, stride, cache="phase_space", precision="f32", sort_every=64), 0, nsteps,
                ps, 0, nsave)
    mom = ps[:, 3:6, :j.dpp_particles].contiguous()
    m0 = mom[0, :, 0].double().cpu().numpy()
    p0 = math.sqrt(float(m0[0]) * float(m0[0]) + float(m0[1]) * float(m0[1]) + float(m0[2]) * float(m0[2]))
    acc = S.new_dpp_accumulators(len(res.lags), device="cuda")
    S.process_momenta_chunk_dpp(mom, res.lags, p0, acc["counts"], acc["sum_delta_p"], acc["sum_delta_p2"],
                                acc["sum_delta_p_norm"], acc["sum_delta_p_norm2"])
    direct = {k: v.cpu().numpy() for k, v in acc.items()}
    direct["p0"] = p0
    same_dpp(res.dpp, direct)


def test_fp64_server_over_bricks_same_as_reference_layout(library64, library64b):
    """The FP64 server over FP64 bricks (brick-sorted slots) returns what it
    returns over the reference layout: mu caches bit for bit, the same
    products."""
    ref = run_jobs(library64, JOBS, stagger_ticks=1, push="f64")
    brk = run_jobs(library64b, JOBS, stagger_ticks=1, push="f64")
    for a, b in zip(ref, brk):
        same(b, a)


def test_run_until_idle_returns_every_job(library):
    libs, B0 = library
    srv = CampaignServer(libs, B0, capacity=20000, max_jobs=8, keep_cache=True, fill_particles=1000)
    for j in JOBS:
        srv.submit(j)
    res = srv.run_until_idle(timeout_s=120)
    srv.close()
    assert sorted(r.job_id for r in res) == list(range(len(JOBS)))
    alone = run_jobs(library, [JOBS[1]])[0]
    same([r for r in res if r.job_id == 1][0], alone)
