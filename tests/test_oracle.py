"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no fixtures for the push or the statistics, so the
oracle is pinned by analytic cases: the exact Boris rotation angle in a
uniform field, |p| conservation with E = 0, the E x B drift, hand-built
mu caches with closed-form bin counts and pair counts
(estimate_pair_visits, src/compute_delta_mu2_dmumu_full.jl:331-338), NaN
skipping and the kinetic-energy formula."""
import math

import numpy as np
import pytest

from helpers import copy_state, fortran_fields, random_mu_cache, small_problem, zero_dmumu, zero_dpp
from particle_transport_b200 import fields as F
from particle_transport_b200.particles import energy_to_gamma, energy_to_speed
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps

Q, M, C = F.Q_E, F.M_P, F.C_LIGHT


def uniform_problem(n=8, B_T=1e-10, u=(0.0, 0.0, 0.0), L=1e12):
    grid = F.build_uniform_grid(L, n, n, n)
    shp = (n, n, n)
    fields = [np.zeros(shp), np.zeros(shp), np.full(shp, B_T)] + [np.full(shp, float(v)) for v in u]
    return grid, fields


def one_particle(grid, p, x=None):
    x = x or (0.5 * grid.xmax, 0.5 * grid.ymax, 0.5 * grid.zmax)
    return {"x1": np.array([x[0]]), "x2": np.array([x[1]]), "x3": np.array([x[2]]),
            "p1": np.array([p[0]]), "p2": np.array([p[1]]), "p3": np.array([p[2]])}


def test_uniform_field_rotation_angle(oracle):
    grid, fields = uniform_problem()
    E = 1.0
    g0, v0 = energy_to_gamma(E), energy_to_speed(E)
    p0 = g0 * M * v0
    Om = Q * 1e-10 / (g0 * M)
    dt = 0.05 / Om
    st = one_particle(grid, (p0, 0.0, 0.0))
    alive = np.ones(1, np.uint8)
    nsteps = 40
    (pos, mom), _ = oracle.push_run(fortran_fields(fields), grid, st, alive, dt, nsteps, 1, cache_mode=2,
                                    out_f64=True)
    px, py = mom[:, 0, 0], mom[:, 1, 0]
    ang = np.unwrap(np.arctan2(py, px))
    t = Q * 1e-10 * dt / (2 * M * g0)
    expected = 2 * math.atan(t)
    # q > 0 in B along +z rotates p clockwise: angle decreases by 2 atan(t) per step
    assert np.allclose(np.diff(ang), -expected, rtol=0, atol=1e-13)
    pm = np.sqrt(px * px + py * py + mom[:, 2, 0] ** 2)
    assert np.max(np.abs(pm / p0 - 1)) < 1e-14


def test_energy_conserved_to_rounding_with_E_zero(oracle):
    pb = small_problem(n=12, n_particles=64, u_over_c=0.0)
    st = copy_state(pb.state)
    p_in = np.sqrt(st["p1"] ** 2 + st["p2"] ** 2 + st["p3"] ** 2)
    alive = np.ones(64, np.uint8)
    oracle.push_run(fortran_fields(pb.fields), pb.grid, st, alive, pb.dt, 2000, 50, cache_mode=0)
    p_out = np.sqrt(st["p1"] ** 2 + st["p2"] ** 2 + st["p3"] ** 2)
    assert np.max(np.abs(p_out / p_in - 1)) < 2000 * 4e-16


def test_exb_drift(oracle):
    u0 = 3.0e6  # m/s along x; E = -(u x B) = u0 B0 y;  E x B / B^2 = u0 x
    grid, fields = uniform_problem(B_T=1e-10, u=(u0, 0, 0), L=1e15)
    E = 1e-3  # 1 MeV: v ~ 1.4e7 m/s, non-relativistic
    g0, v0 = energy_to_gamma(E), energy_to_speed(E)
    Om = Q * 1e-10 / (g0 * M)
    dt = (2 * math.pi / 256) / Om
    st = one_particle(grid, (0.0, g0 * M * v0, 0.0))
    alive = np.ones(1, np.uint8)
    nper = 50
    x_start = st["x1"][0]
    oracle.push_run(fortran_fields(fields), grid, st, alive, dt, 256 * nper + 1, 256, periodic=False, cache_mode=0)
    drift = (st["x1"][0] - x_start) / (256 * nper * dt)
    assert abs(drift / u0 - 1) < 0.02


def test_open_boundary_kills_and_counts(oracle):
    grid, fields = uniform_problem(L=1e9)
    E = 1.0
    g0, v0 = energy_to_gamma(E), energy_to_speed(E)
    st = one_particle(grid, (0.0, 0.0, g0 * M * v0))  # along B: straight line out of the box
    alive = np.ones(1, np.uint8)
    dt = 0.3 * grid.dz / v0
    mu, alive_count = oracle.push_run(fortran_fields(fields), grid, st, alive, dt, 60, 1, periodic=False,
                                      cache_mode=1)
    assert alive[0] == 0
    die = int(np.argmax(alive_count == 0))
    assert alive_count[die - 1] == 1 and np.all(alive_count[die:] == 0)
    # mu = +1 (p along B) while alive, NaN after death (pre-push state of a dead particle)
    assert np.all(mu[: die + 1, 0] == 1.0)
    assert np.all(np.isnan(mu[die + 1:, 0]))


def test_push_threads_bit_identical(oracle):
    pb = small_problem(n=10, n_particles=97)
    outs = []
    for nt in (1, 3):
        st = copy_state(pb.state)
        mu, _ = oracle.push_run(fortran_fields(pb.fields), pb.grid, st, np.ones(97, np.uint8), pb.dt, 300, 7,
                                cache_mode=1, nthreads=nt)
        outs.append((mu, st))
    assert np.array_equal(outs[0][0], outs[1][0], equal_nan=True)
    for k in outs[0][1]:
        assert np.array_equal(outs[0][1][k], outs[1][1][k])


@pytest.mark.parametrize("v,expect", [
    (0.0, 1), (0.05, 2), (0.0499999, 1), (0.05000001, 2), (1.0, 20), (0.999, 20), (1.0000001, 0), (-0.1, 0),
    (float("nan"), 0), (float("inf"), 0)])
def test_mu_bin_index(oracle, v, expect):
    edges, _ = build_mu_edges_full(0.0, 1.0, 20)
    assert oracle.mu_bin_index(v, edges) == expect


def test_dmumu_closed_form_counts(oracle):
    n, nsave = 7, 50
    mu = np.full((n, nsave), 0.33, np.float32)  # constant: every pair in the same bin with dmu = 0
    lags = np.array([1, 2, 5, 49, 50, 60])
    edges, _ = build_mu_edges_full(0.0, 1.0, 10)
    for inj in (False, True):
        acc = zero_dmumu(len(lags), 10)
        oracle.dmumu_accumulate(mu, lags, edges, acc, injection=inj)
        b = 3  # 0.33 in [0.3, 0.4)
        for i, L in enumerate(lags):
            exp = 0 if L >= nsave else (n if inj else n * (nsave - L))
            assert acc["counts"][i, b] == exp
            assert acc["counts"][i].sum() == exp
            assert acc["pair_n"][i] == exp
            assert acc["w_count"][i] == (n if L < nsave else 0)
        assert np.all(acc["sum_d"] == 0) and np.all(acc["sum_d2"] == 0)


def test_dmumu_nan_skipping(oracle):
    n, nsave = 5, 30
    mu = random_mu_cache(n, nsave, seed=2, nan_frac=0.2)
    lags = np.array([1, 3, 7])
    edges, _ = build_mu_edges_full(0.0, 1.0, 8)
    acc = zero_dmumu(3, 8)
    oracle.dmumu_accumulate(mu, lags, edges, acc)
    fin = np.isfinite(mu)
    for i, L in enumerate(lags):
        valid = (fin[:, :-L] & fin[:, L:]).sum()
        assert acc["pair_n"][i] == valid
        assert acc["counts"][i].sum() == valid  # |mu| <= 1: every valid start is binned


def test_dmumu_signed_bins_exclude_out_of_range(oracle):
    n, nsave = 4, 40
    mu = random_mu_cache(n, nsave, seed=5)
    lags = np.array([1, 4])
    edges, _ = build_mu_edges_full(0.0, 1.0, 5, bin_abs=False)  # negative mu falls outside [0, 1]
    acc = zero_dmumu(2, 5)
    oracle.dmumu_accumulate(mu, lags, edges, acc, bin_abs=False)
    for i, L in enumerate(lags):
        starts = mu[:, : nsave - L]
        assert acc["counts"][i].sum() == (starts >= 0).sum()
        assert acc["pair_n"][i] == starts.size


def test_dmumu_welford_matches_numpy(oracle):
    n, nsave = 40, 60
    mu = random_mu_cache(n, nsave, seed=9)
    lags = log_spaced_lag_steps(nsave - 1, 6)
    edges, _ = build_mu_edges_full(0.0, 1.0, 10)
    acc = zero_dmumu(len(lags), 10)
    oracle.dmumu_accumulate(mu, lags, edges, acc, nthreads=3)
    m64 = mu.astype(np.float64)
    for i, L in enumerate(lags):
        d = m64[:, L:] - m64[:, :-L]
        per = (d * d).mean(axis=1)
        assert acc["w_count"][i] == n
        assert math.isclose(acc["w_mean"][i], per.mean(), rel_tol=1e-12)
        assert math.isclose(acc["w_m2"][i], ((per - per.mean()) ** 2).sum(), rel_tol=1e-10)
        assert math.isclose(acc["pair_ss"][i], (d * d).sum(), rel_tol=1e-12)
        assert math.isclose(acc["sum_d"][i].sum(), d.sum(), rel_tol=1e-9, abs_tol=1e-12)


def test_dpp_closed_form(oracle):
    n, nsave = 6, 20
    rng = np.random.default_rng(1)
    u = rng.normal(size=(3, n))
    u /= np.linalg.norm(u, axis=0)
    p = 5.4e-19
    mom = np.broadcast_to((p * u)[None], (nsave, 3, n)).astype(np.float32).copy()
    lags = np.array([1, 4, 19, 20])
    acc = zero_dpp(4)
    oracle.dpp_accumulate(mom, lags, p0=p, acc=acc)
    for i, L in enumerate(lags):
        assert acc["counts"][i] == (n * (nsave - L) if L < nsave else 0)
    assert np.all(acc["sum_dp"] == 0) and np.all(acc["sum_dpn2"] == 0)


def test_kinetic_energy(oracle):
    lib = oracle.lib()
    for E in (1.0, 10.0, 100.0):
        g, v = energy_to_gamma(E), energy_to_speed(E)
        assert math.isclose(lib.or_kinetic_energy_gev(g * M * v), E, rel_tol=1e-12)
    assert math.isnan(lib.or_kinetic_energy_gev(float("nan")))


def test_reconstruct_matches_cache(oracle):
    """mu reconstructed from a Float64 phase-space cache equals the mu cache."""
    pb = small_problem(n=10, n_particles=33)
    ff = fortran_fields(pb.fields)
    st1, st2 = copy_state(pb.state), copy_state(pb.state)
    mu, _ = oracle.push_run(ff, pb.grid, st1, np.ones(33, np.uint8), pb.dt, 200, 5, cache_mode=1, out_f64=True)
    (pos, mom), _ = oracle.push_run(ff, pb.grid, st2, np.ones(33, np.uint8), pb.dt, 200, 5, cache_mode=2,
                                    out_f64=True)
    rec = oracle.reconstruct_mu_f64(pos, mom, ff[:3], pb.grid)
    assert np.array_equal(rec.T, mu, equal_nan=True)
