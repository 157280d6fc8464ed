"""Parity of the CUDA push with the CPU oracle (needs a B200).

FP64 form: bit-identical to the oracle (and so to a Float64 run of the
reference) -- trajectories, mu cache, phase-space cache and alive counts.
FP32 form over Morton bricks: bounded deviation over the first gyroperiod,
exact |p| conservation with E = 0, results independent of the brick sort."""

import numpy as np
import pytest

from helpers import copy_state, fortran_fields, small_problem
from particle_transport_b200 import runner as R
from particle_transport_b200.fields import FieldLibrary

pytestmark = pytest.mark.gpu


# the FP64 push over the reference layout, over FP64 bricks with the slots in
# particle order, and over FP64 bricks re-sorted by brick every 16 steps:
# every one must be bit-identical to the oracle
F64_FORMS = [("ref_f64", 0), ("brick_f64", 0), ("brick_f64", 16)]


def run_both(pb, nsteps, stride, cache, periodic=True, f64_out=False, alive=None, storage="ref_f64", sort_every=0):
    from oracle import oracle as o
    n = len(pb.state["x1"])
    alive0 = np.ones(n, np.uint8) if alive is None else alive.copy()
    st_o = copy_state(pb.state)
    al_o = alive0.copy()
    out_o, ac_o = o.push_run(fortran_fields(pb.fields), pb.grid, st_o, al_o, pb.dt, nsteps, stride, periodic=periodic,
                             cache_mode={"mu": 1, "phase_space": 2}[cache], out_f64=f64_out)
    fl = FieldLibrary(pb.fields, pb.grid, storage)
    st_g = copy_state(pb.state)
    al_g = alive0.copy()
    col = R.CacheCollector(n, R.n_saves(nsteps, stride), cache, f64_out)
    params = R.push_params(pb.dt, nsteps, stride, periodic=periodic, cache=cache, cache_f64=f64_out,
                           sort_every=sort_every)
    ac_g = R.run_push_host(fl, st_g, al_g, params, col)
    return (out_o, ac_o, st_o, al_o), (col, ac_g, st_g, al_g)


@pytest.mark.parametrize("storage,sort_every", F64_FORMS)
def test_fp64_mu_cache_bit_exact(cuda, storage, sort_every):
    pb = small_problem(n=16, n_particles=700, u_over_c=1e-4)
    (mu_o, ac_o, st_o, al_o), (col, ac_g, st_g, al_g) = run_both(pb, 641, 4, "mu", storage=storage,
                                                                 sort_every=sort_every)
    assert np.array_equal(col.mu, mu_o, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(st_g[k], st_o[k]), k
    assert np.array_equal(ac_g, ac_o)
    assert np.array_equal(al_g, al_o)


@pytest.mark.parametrize("storage,sort_every", F64_FORMS)
@pytest.mark.parametrize("f64_out", [False, True])
def test_fp64_phase_space_bit_exact(cuda, f64_out, storage, sort_every):
    pb = small_problem(n=12, n_particles=300, energy_GeV=10.0, u_over_c=1e-4)
    ((pos_o, mom_o), ac_o, st_o, _), (col, ac_g, st_g, _) = run_both(pb, 257, 8, "phase_space", f64_out=f64_out,
                                                                     storage=storage, sort_every=sort_every)
    assert np.array_equal(col.positions, pos_o, equal_nan=True)
    assert np.array_equal(col.momenta, mom_o, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(st_g[k], st_o[k]), k


@pytest.mark.parametrize("storage,sort_every", F64_FORMS)
def test_fp64_open_boundary_bit_exact(cuda, storage, sort_every):
    pb = small_problem(n=10, n_particles=400, energy_GeV=30.0, u_over_c=1e-4)
    alive = np.ones(400, np.uint8)
    alive[::17] = 0  # some particles dead on entry
    (mu_o, ac_o, st_o, al_o), (col, ac_g, st_g, al_g) = run_both(pb, 400, 3, "mu", periodic=False, alive=alive,
                                                                 storage=storage, sort_every=sort_every)
    assert ac_o[-1] < ac_o[0]  # particles left the box
    assert np.array_equal(ac_g, ac_o)
    assert np.array_equal(al_g, al_o)
    assert np.array_equal(col.mu, mu_o, equal_nan=True)


@pytest.mark.parametrize("storage,sort_every", F64_FORMS)
def test_fp64_device_api_matches_host(cuda, storage, sort_every):
    torch = cuda
    pb = small_problem(n=16, n_particles=512)
    nsteps, stride = 333, 4
    (mu_o, _, st_o, _), _ = run_both(pb, nsteps, stride, "mu")
    fl = FieldLibrary(pb.fields, pb.grid, storage)
    ens = R.DeviceEnsemble(fl, pb.state, np.ones(512, np.uint8))
    nsave = R.n_saves(nsteps, stride)
    cache = torch.full((nsave, 512), float("nan"), dtype=torch.float32, device="cuda")
    params = R.push_params(pb.dt, nsteps, stride, cache="mu", steps_per_launch=16, sort_every=sort_every)
    s = 0
    for chunk in (5, 100, 1, 227):  # uneven chunks, each a separate call
        ens.advance(params, s, chunk, cache, 0, nsave)
        s += chunk
    assert s == nsteps
    torch.cuda.synchronize()
    assert np.array_equal(cache.cpu().numpy(), mu_o, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(ens.state[k].cpu().numpy(), st_o[k]), k


def _fast_mu(pb, storage, nsteps, stride, sort_every=0, u=True, variant=0):
    torch = __import__("torch")
    fl = FieldLibrary(pb.fields, pb.grid, storage)
    ens = R.FastEnsemble(fl, pb.state, np.ones(len(pb.state["x1"]), np.uint8))
    nsave = R.n_saves(nsteps, stride)
    cache = torch.full((nsave, ens.n), float("nan"), dtype=torch.float32, device="cuda")
    params = R.push_params(pb.dt, nsteps, stride, cache="mu", precision="f32", sort_every=sort_every,
                           kernel_variant=variant)
    ens.advance(params, 0, nsteps, cache, 0, nsave)
    st, al = ens.export()
    torch.cuda.synchronize()
    return cache.cpu().numpy(), {k: v.cpu().numpy() for k, v in st.items()}, fl


@pytest.mark.parametrize("storage,tol_particle,share,tol_med", [("brick_f32", 2e-3, 1.0, 1e-4),
                                                                ("brick_bf16", 0.05, 0.99, 0.02)])
def test_fast_push_close_over_one_gyroperiod(cuda, storage, tol_particle, share, tol_med):
    """mu of the FP32 push against the FP64 push over one gyroperiod: every
    particle within tol_particle over FP32 bricks.  Over BF16 bricks (B
    stored less its mean, 8 significant bits) a particle that passes a
    weak-field node sees a field error of ~2^-9 of the mean field there and
    can leave on another non-adiabatic branch, so the bound holds for 99 %
    of the particles, and the median sample error stays small."""
    pb = small_problem(n=16, n_particles=1000, u_over_c=1e-4)
    (mu_o, _, _, _), _ = run_both(pb, 65, 4, "mu")
    mu_f, _, _ = _fast_mu(pb, storage, 65, 4)
    d = np.abs(mu_f - mu_o)
    assert np.all(np.isfinite(mu_f))
    per_particle = d.max(axis=0)
    assert np.mean(per_particle < tol_particle) >= share, np.sort(per_particle)[-12:]
    assert np.median(d) < tol_med, np.median(d)


def test_bf16_mean_field_offset_off_axis(cuda):
    """BF16 bricks store B less its per-component mean and add the mean back
    after the interpolation.  With a uniform B0 added to Bx the mean field
    points between x and z, so all three offsets are in play; the BF16 push
    stays as close to the FP64 push over one gyroperiod as in the test above,
    and the FP32-brick push (no offset) stays within its own bound."""
    pb = small_problem(n=16, n_particles=1000, u_over_c=1e-4)
    pb.fields = [pb.fields[0] + pb.B0, *pb.fields[1:]]
    (mu_o, _, _, _), _ = run_both(pb, 65, 4, "mu")
    for storage, tol_particle, share in (("brick_f32", 2e-3, 0.99), ("brick_bf16", 0.05, 0.99)):
        mu_f, _, _ = _fast_mu(pb, storage, 65, 4)
        d = np.abs(mu_f - mu_o)
        assert np.all(np.isfinite(mu_f)), storage
        per_particle = d.max(axis=0)
        assert np.mean(per_particle < tol_particle) >= share, (storage, np.sort(per_particle)[-12:])
        assert np.median(d) < 0.02, (storage, np.median(d))


def test_xpair_layout_bit_identical_to_bf16(cuda):
    """The x-pair records hold the same BF16 values and the gather adds the
    corners in the same order: identical trajectories."""
    pb = small_problem(n=16, n_particles=1500, u_over_c=1e-4, energy_GeV=10.0)
    mu_a, st_a, _ = _fast_mu(pb, "brick_bf16", 300, 4, sort_every=32)
    mu_b, st_b, _ = _fast_mu(pb, "brick_bf16x", 300, 4, sort_every=32)
    assert np.array_equal(mu_a, mu_b, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(st_a[k], st_b[k]), k


@pytest.mark.parametrize("variant", [2, 3, 6, 9, 10, 11])
def test_launch_shapes_and_texture_fetches_bit_identical(cuda, variant):
    """Every launch shape, and corner fetches through the texture path
    (variants 9-11), give the same trajectories as the default shape."""
    pb = small_problem(n=16, n_particles=1200, u_over_c=1e-4, energy_GeV=10.0)
    mu_a, st_a, _ = _fast_mu(pb, "brick_bf16", 200, 4, sort_every=32, variant=1)
    mu_b, st_b, _ = _fast_mu(pb, "brick_bf16", 200, 4, sort_every=32, variant=variant)
    assert np.array_equal(mu_a, mu_b, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(st_a[k], st_b[k]), k


@pytest.mark.parametrize("storage", ["brick_f32", "brick_bf16", "brick_bf16x"])
def test_fast_push_non_pow2_brick_grid(cuda, storage):
    """20^3 nodes -> 3^3 bricks in x-fastest order (not a power-of-two cube)."""
    pb = small_problem(n=20, n_particles=800, u_over_c=1e-4)
    (mu_o, _, _, _), _ = run_both(pb, 65, 4, "mu")
    mu_f, _, _ = _fast_mu(pb, storage, 65, 4, sort_every=16)
    d = np.abs(mu_f - mu_o)
    tol = 2e-3 if storage == "brick_f32" else 0.2
    assert np.all(np.isfinite(mu_f)) and d.max() < tol, d.max()


def test_fast_push_energy_exact_with_E_zero(cuda):
    pb = small_problem(n=16, n_particles=800, u_over_c=0.0, energy_GeV=10.0)
    _, st, _ = _fast_mu(pb, "brick_bf16", 3000, 50)
    p_in = np.sqrt(pb.state["p1"] ** 2 + pb.state["p2"] ** 2 + pb.state["p3"] ** 2)
    p_out = np.sqrt(st["p1"] ** 2 + st["p2"] ** 2 + st["p3"] ** 2)
    assert np.max(np.abs(p_out / p_in - 1)) < 1e-13


def test_fast_push_sort_does_not_change_results(cuda):
    pb = small_problem(n=16, n_particles=2000, u_over_c=1e-4, energy_GeV=10.0)
    mu_a, st_a, _ = _fast_mu(pb, "brick_bf16", 300, 5, sort_every=0)
    mu_b, st_b, _ = _fast_mu(pb, "brick_bf16", 300, 5, sort_every=7)
    assert np.array_equal(mu_a, mu_b, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(st_a[k], st_b[k]), k


def test_fast_state_roundtrip(cuda):
    pb = small_problem(n=12, n_particles=333)
    _, st, _ = _fast_mu(pb, "brick_f32", 1, 1)  # one sample, no push
    for k in ("x1", "x2", "x3"):
        assert np.allclose(st[k], pb.state[k], rtol=1e-14, atol=1e-14 * pb.grid.xmax)
    for k in ("p1", "p2", "p3"):
        pm = np.sqrt(pb.state["p1"] ** 2 + pb.state["p2"] ** 2 + pb.state["p3"] ** 2)
        assert np.max(np.abs(st[k] - pb.state[k]) / pm) < 2e-7


def test_host_run_fast_matches_device(cuda):
    """pt_push_run (host buffers, pipelined egress) with the FP32 push gives
    the same mu cache as the device entry point."""
    pb = small_problem(n=16, n_particles=600, u_over_c=1e-4)
    mu_dev, _, fl = _fast_mu(pb, "brick_bf16", 500, 4)
    st = copy_state(pb.state)
    col = R.CacheCollector(600, R.n_saves(500, 4), "mu")
    R.run_push_host(fl, st, np.ones(600, np.uint8), R.push_params(pb.dt, 500, 4, cache="mu", precision="f32"), col)
    assert np.array_equal(col.mu, mu_dev, equal_nan=True)


def test_host_run_fast_matches_device_many_particles(cuda):
    """pt_push_run with more particles than 8 rows of the 512 MB egress slot
    hold (17M: 7 rows, i.e. 28-step chunks that do not line up with the
    64-step sort cadence) gives the same mu cache as the device entry point:
    the time-fastest chunks and their transpose to rows lose nothing."""
    n, nsteps, stride = 17_000_000, 100, 4
    pb = small_problem(n=16, n_particles=n, u_over_c=1e-4)
    mu_dev, _, fl = _fast_mu(pb, "brick_bf16", nsteps, stride, sort_every=64)
    col = R.CacheCollector(n, R.n_saves(nsteps, stride), "mu")
    R.run_push_host(fl, copy_state(pb.state), np.ones(n, np.uint8),
                    R.push_params(pb.dt, nsteps, stride, cache="mu", precision="f32", sort_every=64), col)
    assert np.array_equal(col.mu, mu_dev, equal_nan=True)


def test_errors_raise(cuda):
    from particle_transport_b200._lib import PtError
    pb = small_problem(n=8, n_particles=4)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    with pytest.raises(PtError, match="brick field"):
        R.run_push_host(fl, copy_state(pb.state), np.ones(4, np.uint8), R.push_params(pb.dt, 10, 1, precision="f32"))
    with pytest.raises(PtError, match="stride"):
        R.run_push_host(fl, copy_state(pb.state), np.ones(4, np.uint8), R.push_params(pb.dt, 10, 0))
    with pytest.raises(ValueError):
        R.run_push_host(fl, copy_state(pb.state), np.ones(3, np.uint8), R.push_params(pb.dt, 10, 1))
    # FP64 bricks are for the FP64 push only
    f64b = FieldLibrary(pb.fields, pb.grid, "brick_f64")
    with pytest.raises(PtError, match="brick field"):
        R.run_push_host(f64b, copy_state(pb.state), np.ones(4, np.uint8), R.push_params(pb.dt, 10, 1, precision="f32"))
    with pytest.raises(ValueError, match="FP32-push brick field"):
        R.FastEnsemble(f64b, pb.state, np.ones(4, np.uint8))


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_push_run_context_buffers_reused(cuda, precision):
    """pt_push_run keeps its device state, pinned staging and FP32 state in the
    context: calls of other sizes in between, and a call after pt_ctx_trim,
    give the same result as the first call."""
    pb = small_problem(n=16, n_particles=3000, u_over_c=1e-4)
    fl = FieldLibrary(pb.fields, pb.grid, "brick_bf16" if precision == "f32" else "ref_f64")
    params = R.push_params(pb.dt, 200, 4, cache="mu", precision=precision, sort_every=16 if precision == "f32" else 0)

    def run(n):
        st = {k: v[:n].copy() for k, v in pb.state.items()}
        col = R.CacheCollector(n, R.n_saves(200, 4), "mu")
        ac = R.run_push_host(fl, st, np.ones(n, np.uint8), params, col)
        return col.mu, st, ac

    first = run(3000)
    small = run(1000)
    again = run(3000)
    fl.ctx.trim()
    after_trim = run(3000)
    for res in (again, after_trim):
        assert np.array_equal(res[0], first[0], equal_nan=True)
        for k in R.KEYS:
            assert np.array_equal(res[1][k], first[1][k]), k
        assert np.array_equal(res[2], first[2])
    # the smaller run is the prefix of the larger one (particles are independent)
    assert np.array_equal(small[0], first[0][:, :1000], equal_nan=True)


@pytest.mark.parametrize("pitch_pad, steps_per_launch, row_base, f64", [
    (0, 0, 0, False),      # pitch = nsave: one call, aligned runs of 8 saves
    (5, 0, 0, False),      # pitch not a multiple of 8: runs aligned per element, not per particle
    (3, 24, 0, False),     # launches of 24 steps = 6 saves: runs split across launches
    (0, 64, 3, False),     # rows from a misaligned row_base
    (0, 40, 0, True),      # Float64 cache
])
def test_time_fastest_mu_cache_bit_identical_to_rows(cuda, pitch_pad, steps_per_launch, row_base, f64):
    """cache_pitch > 0: save row r of particle p at p * pitch + (r - row_base).
    The mu values are those of the row layout, bit for bit, under brick
    sorts, launch splits and any pitch."""
    torch = cuda
    pb = small_problem(n=16, n_particles=1700, u_over_c=1e-4, energy_GeV=10.0)
    fl = FieldLibrary(pb.fields, pb.grid, "brick_bf16")
    nsteps, stride = 401, 4
    nsave = R.n_saves(nsteps, stride)
    rows = nsave - row_base
    dt_ = torch.float64 if f64 else torch.float32
    out = {}
    for pitch in (0, rows + pitch_pad):
        ens = R.FastEnsemble(fl, pb.state, np.ones(1700, np.uint8))
        shape = (1700, pitch) if pitch else (rows, 1700)
        cache = torch.full(shape, float("inf"), dtype=dt_, device="cuda")
        params = R.push_params(pb.dt, nsteps, stride, cache="mu", cache_f64=f64, precision="f32", sort_every=32,
                               steps_per_launch=steps_per_launch, cache_pitch=pitch)
        ens.advance(params, 0, nsteps, cache, row_base, rows)
        torch.cuda.synchronize()
        c = cache.cpu().numpy()
        if pitch:
            assert np.all(np.isinf(c[:, rows:]))  # the pad past the last row is left alone
            c = c[:, :rows].T
        out[pitch] = c
        ens.close()
    a, b = out[0], out[rows + pitch_pad]
    assert np.isfinite(a).all()
    assert np.array_equal(a, b), np.argwhere(a != b)[:5]


def test_time_fastest_rejected_where_it_does_not_apply(cuda):
    from particle_transport_b200._lib import PtError
    pb = small_problem(n=8, n_particles=64)
    fb = FieldLibrary(pb.fields, pb.grid, "brick_bf16")
    ens = R.FastEnsemble(fb, pb.state, np.ones(64, np.uint8))
    torch = cuda
    cache = torch.empty((64, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(PtError, match="at least cache_rows"):
        ens.advance(R.push_params(pb.dt, 21, 4, cache="mu", precision="f32", cache_pitch=4), 0, 21, cache, 0, 6)
    with pytest.raises(PtError, match="FP32 push only"):
        ens.advance(R.push_params(pb.dt, 21, 4, cache="phase_space", precision="f32", cache_pitch=8), 0, 21, cache,
                    0, 6)
    with pytest.raises(PtError, match="cache_pitch must be 0"):
        R.run_push_host(fb, copy_state(pb.state), np.ones(64, np.uint8),
                        R.push_params(pb.dt, 21, 4, cache="mu", precision="f32", cache_pitch=8), lambda i, r: None)
