"""Derived product arrays against the oracle's restatement.

The accumulators of the lag statistics become the numbers the reference
writes into its products through compute_dmumu_arrays_full and
average_over_tau_full (src/compute_delta_mu2_dmumu_full.jl:706-776), the
computed columns of build_output_dataframe with sem_from_stats
(src/compute_delta_mu2_curve.jl:387-429) and compute_dpp_arrays
(src/compute_dpp_full.jl:301-330).  The host functions of
``particle_transport_b200.stats`` must give the same arrays bit for bit as
the C restatement, on accumulators from the oracle's own binning of seeded
caches (NaN samples, cells below the count cut, empty cells) and on
hand-built accumulators that exercise the max(0, .) centring and NaN
propagation."""
import math

import numpy as np
import pytest

from helpers import random_mu_cache, zero_dmumu, zero_dpp
from particle_transport_b200 import stats as S
from particle_transport_b200.time_units import build_mu_edges_full, log_spaced_lag_steps


def _same(a, b):
    return np.array_equal(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64), equal_nan=True)


def _time_axes(nsave, dt=0.37, omega0=2.9):
    t_s = dt * np.arange(nsave, dtype=np.float64)
    return t_s, t_s * omega0


@pytest.mark.parametrize("injection", [False, True])
@pytest.mark.parametrize("cut", ["none", "median", "all"])
def test_dmumu_derived_arrays_bit_identical(oracle, injection, cut):
    n, nsave = 300, 257
    mu = random_mu_cache(n, nsave, seed=7, nan_frac=0.05)
    lags = log_spaced_lag_steps(nsave - 1, 12)
    edges, _ = build_mu_edges_full(0.0, 1.0, 16)
    acc = zero_dmumu(len(lags), 16)
    oracle.dmumu_accumulate(mu, lags, edges, acc, injection=injection)
    t_s, t_norm = _time_axes(nsave)
    tau_s = np.array([t_s[l] - t_s[0] for l in lags])
    tau_norm = np.array([t_norm[l] - t_norm[0] for l in lags])
    nonzero = acc["counts"][acc["counts"] > 0]
    min_count = {"none": 1, "median": int(np.median(nonzero)), "all": int(acc["counts"].max()) + 1}[cut]

    got = S.compute_dmumu_arrays_full(acc["counts"], acc["sum_d"], acc["sum_d2"], tau_s, tau_norm, min_count)
    want = oracle.dmumu_arrays_full(acc["counts"], acc["sum_d"], acc["sum_d2"], tau_s, tau_norm, min_count)
    for k in oracle.DMUMU_ARRAY_KEYS:
        assert _same(got[k], want[k]), k
    below = acc["counts"] < min_count
    assert np.all(np.isnan(want["mean_delta2"][below])) and np.all(np.isfinite(want["mean_delta2"][~below]))
    if cut == "median":
        assert below.any() and (~below).any()  # the cut is exercised both ways
    assert np.all(want["dmumu_centered_norm"][~below] >= 0)

    for k in ("dmumu_raw_norm", "dmumu_centered_norm", "dmumu_raw_per_s", "mean_delta"):
        u, w = S.average_over_tau_full(got[k], acc["counts"], min_count)
        uo, wo = oracle.average_over_tau_full(want[k], acc["counts"], min_count)
        assert _same(u, uo) and _same(w, wo), k

    tab = S.build_output_table(lags, t_s, t_norm, acc["w_count"], acc["w_mean"], acc["w_m2"], acc["pair_ss"],
                               acc["pair_n"])
    tab_o = oracle.output_table(lags, t_s, t_norm, acc["w_count"], acc["w_m2"], acc["pair_ss"], acc["pair_n"])
    for k in oracle.TABLE_KEYS:
        assert _same(tab[k], tab_o[k]), k
    assert _same(tab["delta_mu2_particle_mean"], acc["w_mean"])
    assert np.array_equal(tab["n_pairs_used"], acc["pair_n"])


def test_dmumu_derived_edge_cells(oracle):
    """Hand-built accumulators: a cell whose centred second moment rounds
    below zero (clamped to 0), a NaN sum (propagates, as Julia's max does), an
    empty cell and an infinite value skipped by the tau average."""
    counts = np.array([[3, 0, 5, 2], [7, 1, 4, 9]], dtype=np.int64)
    sum_d = np.array([[0.3, 0.0, np.nan, 0.2], [0.7, 0.1, 1.0, -0.9]])
    # cell (0, 0): <d>^2 = 0.01 and <d^2> a hair below it -> centred value < 0 before the clamp
    sum_d2 = np.array([[3 * np.nextafter(0.01, 0.0), 0.0, 0.5, 0.1], [0.2, 0.3, 0.4, 0.5]])
    tau_s, tau_norm = np.array([2.0, 4.0]), np.array([0.5, 1.0])
    got = S.compute_dmumu_arrays_full(counts, sum_d, sum_d2, tau_s, tau_norm, 1)
    want = oracle.dmumu_arrays_full(counts, sum_d, sum_d2, tau_s, tau_norm, 1)
    for k in oracle.DMUMU_ARRAY_KEYS:
        assert _same(got[k], want[k]), k
    assert want["dmumu_centered_norm"][0, 0] == 0.0
    assert math.isnan(want["dmumu_centered_norm"][0, 2])  # NaN sum propagates through max(0, .)
    assert math.isnan(want["mean_delta"][0, 1])  # empty cell

    values = np.array([[1.0, np.inf, 2.0, np.nan], [3.0, 5.0, 4.0, 6.0]])
    for mc in (1, 2, 6):
        u, w = S.average_over_tau_full(values, counts, mc)
        uo, wo = oracle.average_over_tau_full(values, counts, mc)
        assert _same(u, uo) and _same(w, wo), mc
    u, w = oracle.average_over_tau_full(values, counts, 1)
    assert u[0] == 2.0 and w[0] == (1.0 * 3 + 3.0 * 7) / 10
    assert u[1] == 5.0  # the infinite value at lag 0 is skipped
    assert math.isnan(oracle.average_over_tau_full(values, counts, 10)[0][0])

    for c, m2 in ((0, 1.0), (1, 1.0), (2, 0.5), (1000, 3.25)):
        assert _same(S.sem_from_stats(c, m2), oracle.sem_from_stats(c, m2))


def test_dpp_derived_arrays_bit_identical(oracle):
    rng = np.random.default_rng(5)
    n, nsave = 200, 129
    p = np.abs(1.0 + 0.01 * np.cumsum(rng.normal(size=(nsave, n)), axis=0))
    dirs = rng.normal(size=(nsave, 3, n))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    mom = (dirs * p[:, None, :] * 5.3e-18).astype(np.float32)
    mom[rng.random(mom.shape) < 0.01] = np.nan
    lags = np.array([1, 2, 5, 17, 64, 128, 200], dtype=np.int64)  # the last lag has no pairs
    acc = zero_dpp(len(lags))
    p0 = float(np.linalg.norm(mom[0, :, 0].astype(np.float64)))
    oracle.dpp_accumulate(mom, lags, p0, acc)
    assert acc["counts"][-1] == 0
    tau_s = 0.25 * lags.astype(np.float64)
    tau_norm = 1.7 * lags.astype(np.float64)
    got = S.compute_dpp_arrays(acc["counts"], acc["sum_dp"], acc["sum_dp2"], acc["sum_dpn"], acc["sum_dpn2"], tau_s,
                               tau_norm)
    want = oracle.dpp_arrays(acc["counts"], acc["sum_dp"], acc["sum_dp2"], acc["sum_dpn"], acc["sum_dpn2"], tau_s,
                             tau_norm)
    for k in oracle.DPP_ARRAY_KEYS:
        assert _same(got[k], want[k]), k
    assert math.isnan(want["dpp_raw_per_s"][-1]) and np.all(np.isfinite(want["dpp_raw_per_s"][:-1]))
    # centring clamps a second moment that rounds below the squared mean
    c = np.array([3], np.int64)
    s1, s2 = np.array([0.3]), np.array([3 * np.nextafter(0.01, 0.0)])
    a = S.compute_dpp_arrays(c, s1, s2, s1, s2, np.ones(1), np.ones(1))
    b = oracle.dpp_arrays(c, s1, s2, s1, s2, np.ones(1), np.ones(1))
    for k in oracle.DPP_ARRAY_KEYS:
        assert _same(a[k], b[k]), k
    assert b["dpp_centered_norm"][0] == 0.0
