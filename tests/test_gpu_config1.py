"""The reference's CPU-runnable configuration, end to end on the device.

64³ periodic box, B = B0 z + isotropic dB (|k| = 2..32, dB/B0 = 0.5), no
velocity field (E = 0), one cell = the 1 GeV gyroradius in B0 = 1 uG;
4096 protons at 1 GeV, uniform positions, isotropic momenta; 64 steps per
T_g0 for 50 T_g0 (3201 samples, 3200 pushes); mu cache every 4 steps (801
saves); D_mumu on 20 log-spaced lags x 20 |mu| bins.

FP64 push and binning on the device against the oracle on the same seeded
inputs: mu cache and final state bit-identical, bin and pair counts exact,
FP64 sums within 1e-12 (summation order).  The mixed-precision push over
FP32 / BF16 bricks conserves |p| exactly (E = 0) and reproduces <dmu^2>(tau)
to the sampling noise of 4096 particles."""
import math

import numpy as np
import pytest

from helpers import copy_state, fortran_fields, zero_dmumu
from particle_transport_b200 import fields as F
from particle_transport_b200 import runner as R
from particle_transport_b200 import stats as S
from particle_transport_b200.fields import FieldLibrary
from particle_transport_b200.particles import energy_to_gamma, init_particles
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps, reference_Omega0

pytestmark = pytest.mark.gpu

N, NP, SPG, DUR, STRIDE = 64, 4096, 64, 50, 4


@pytest.fixture(scope="module")
def config1():
    fields = [np.ascontiguousarray(f.numpy()) for f in F.to_si(F.synthetic_mhd_fields(N, 2, 32, 0.5, 1.0, 0.0, seed=1))]
    rg = F.gyroradius_m(1.0, 1e-10)
    grid = F.build_uniform_grid((N - 1) * rg, N, N, N)
    B0 = F.reference_B0_T(*fields[:3])
    dt = (2 * math.pi / SPG) / reference_Omega0(B0, energy_to_gamma(1.0), F.Q_E, F.M_P)
    state = init_particles(NP, grid, 1.0, seed=1)
    nsteps = SPG * DUR + 1
    lags = log_spaced_lag_steps((nsteps - 1) // STRIDE, 20)
    edges, _ = build_mu_edges_full(0.0, 1.0, 20)
    return dict(fields=fields, grid=grid, B0=B0, dt=dt, state=state, nsteps=nsteps, lags=lags, edges=edges)


def _gpu_dmumu(mu_rows, lags, edges):
    acc = S.new_dmumu_accumulators(len(lags), len(edges) - 1)
    S.process_mu_chunk_dmumu(np.ascontiguousarray(mu_rows, dtype=np.float32), lags, edges, acc["particle_counts"],
                             acc["particle_means"], acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                             acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"],
                             layout="particle_fastest")
    return acc


def test_config1_fp64_bit_exact_and_dmumu(cuda, oracle, config1):
    c = config1
    st_o = copy_state(c["state"])
    al_o = np.ones(NP, np.uint8)
    mu_o, ac_o = oracle.push_run(fortran_fields(c["fields"]), c["grid"], st_o, al_o, c["dt"], c["nsteps"], STRIDE,
                                 cache_mode=1)
    fl = FieldLibrary(c["fields"], c["grid"], "ref_f64")
    st_g = copy_state(c["state"])
    col = R.CacheCollector(NP, R.n_saves(c["nsteps"], STRIDE), "mu")
    ac_g = R.run_push_host(fl, st_g, np.ones(NP, np.uint8), R.push_params(c["dt"], c["nsteps"], STRIDE, cache="mu"),
                           col)
    assert col.mu.shape == (801, NP)
    assert np.array_equal(col.mu, mu_o, equal_nan=True)
    for k in R.KEYS:
        assert np.array_equal(st_g[k], st_o[k]), k
    assert np.array_equal(ac_g, ac_o) and ac_g[-1] == NP

    o = zero_dmumu(len(c["lags"]), 20)
    oracle.dmumu_accumulate(mu_o, c["lags"], c["edges"], o, time_fastest=False)
    g = _gpu_dmumu(col.mu, c["lags"], c["edges"])
    assert np.array_equal(g["dmumu_counts"], o["counts"])
    assert np.array_equal(g["pair_counts"], o["pair_n"])
    assert np.array_equal(g["particle_counts"], o["w_count"])
    assert np.allclose(g["dmumu_sum_delta2"], o["sum_d2"], rtol=1e-12, atol=0)
    assert np.allclose(g["pair_sum_squares"], o["pair_ss"], rtol=1e-12, atol=0)
    assert np.allclose(g["particle_means"], o["w_mean"], rtol=1e-11, atol=0)
    scale = 1e-12 * np.sqrt(np.maximum(o["counts"], 1) * o["sum_d2"]) + 1e-300
    assert np.all(np.abs(g["dmumu_sum_delta"] - o["sum_d"]) <= scale)
    # every save of every particle is finite with a periodic box
    assert g["pair_counts"].sum() == sum(NP * (801 - int(L)) for L in c["lags"])

    # derived products of the device accumulators against the oracle's derived arrays of its own accumulators:
    # the same cells survive the count cut, and the values agree to the summation-order differences of the sums
    t_s = c["dt"] * STRIDE * np.arange(801, dtype=np.float64)
    t_norm = (2 * math.pi / SPG) * STRIDE * np.arange(801, dtype=np.float64)
    tau_s = np.array([t_s[L] - t_s[0] for L in c["lags"]])
    tau_norm = np.array([t_norm[L] - t_norm[0] for L in c["lags"]])
    for min_count in (1, 5000):
        dg = S.compute_dmumu_arrays_full(g["dmumu_counts"], g["dmumu_sum_delta"], g["dmumu_sum_delta2"], tau_s,
                                         tau_norm, min_count)
        do = oracle.dmumu_arrays_full(o["counts"], o["sum_d"], o["sum_d2"], tau_s, tau_norm, min_count)
        for k in oracle.DMUMU_ARRAY_KEYS:
            assert np.array_equal(np.isnan(dg[k]), np.isnan(do[k])), k
        ok = ~np.isnan(do["mean_delta2"])
        assert ok.any() and (min_count == 1 or (~ok).any())
        for k in ("mean_delta2", "dmumu_raw_norm", "dmumu_raw_per_s"):
            assert np.allclose(dg[k][ok], do[k][ok], rtol=1e-12, atol=0), k
        raw = do["dmumu_raw_norm"][ok]
        assert np.all(np.abs(dg["dmumu_centered_norm"][ok] - do["dmumu_centered_norm"][ok]) <= 1e-11 * raw)
        mscale = scale[ok] / o["counts"][ok]
        assert np.all(np.abs(dg["mean_delta"][ok] - do["mean_delta"][ok]) <= mscale)
        for k in ("dmumu_raw_norm", "dmumu_centered_norm"):
            ug, wg = S.average_over_tau_full(dg[k], g["dmumu_counts"], min_count)
            uo, wo = oracle.average_over_tau_full(do[k], o["counts"], min_count)
            assert np.array_equal(np.isnan(ug), np.isnan(uo)) and np.array_equal(np.isnan(wg), np.isnan(wo))
            assert np.allclose(ug, uo, rtol=1e-11, equal_nan=True) and np.allclose(wg, wo, rtol=1e-11, equal_nan=True)
    tg = S.build_output_table(c["lags"], t_s, t_norm, g["particle_counts"], g["particle_means"], g["particle_m2s"],
                              g["pair_sum_squares"], g["pair_counts"])
    to = oracle.output_table(c["lags"], t_s, t_norm, o["w_count"], o["w_m2"], o["pair_ss"], o["pair_n"])
    for k in ("tau_s", "tau_norm", "tau_gyroperiods"):
        assert np.array_equal(tg[k], to[k]), k
    for k in ("delta_mu2_particle_std", "delta_mu2_particle_sem", "delta_mu2_pair_mean"):
        assert np.allclose(tg[k], to[k], rtol=1e-10, atol=0), k


@pytest.mark.parametrize("storage", ["brick_f32", "brick_bf16"])
def test_config1_mixed_precision(cuda, config1, storage):
    torch = cuda
    c = config1
    nsave = R.n_saves(c["nsteps"], STRIDE)
    fl64 = FieldLibrary(c["fields"], c["grid"], "ref_f64")
    col = R.CacheCollector(NP, nsave, "mu")
    R.run_push_host(fl64, copy_state(c["state"]), np.ones(NP, np.uint8),
                    R.push_params(c["dt"], c["nsteps"], STRIDE, cache="mu"), col)
    fl = FieldLibrary(c["fields"], c["grid"], storage)
    ens = R.FastEnsemble(fl, c["state"], np.ones(NP, np.uint8))
    cache = torch.empty((nsave, NP), dtype=torch.float32, device="cuda")
    ens.advance(R.push_params(c["dt"], c["nsteps"], STRIDE, cache="mu", precision="f32", sort_every=64), 0,
                c["nsteps"], cache, 0, nsave)
    st, _ = ens.export()
    torch.cuda.synchronize()
    p_in = np.sqrt(sum(c["state"][k] ** 2 for k in ("p1", "p2", "p3")))
    p_out = np.sqrt(sum(st[k].cpu().numpy() ** 2 for k in ("p1", "p2", "p3")))
    assert np.max(np.abs(p_out / p_in - 1)) < 1e-13  # E = 0: |p| conserved
    a = _gpu_dmumu(col.mu, c["lags"], c["edges"])
    b = _gpu_dmumu(cache.cpu().numpy(), c["lags"], c["edges"])
    # <dmu^2>(tau): mean over particles, within the sampling noise of 4096 particles
    rel = np.abs(b["particle_means"] / a["particle_means"] - 1)
    assert np.median(rel) < 0.02 and rel.max() < 0.08, rel
    assert np.array_equal(a["pair_counts"], b["pair_counts"])
