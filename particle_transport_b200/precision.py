"""The precision forms against the plain FP64 push.

The FP32 push over FP32 or BF16 bricks and the FP64 push run from the same
initial state on the same field; the transport products of each form are
compared cell by cell with those of the FP64 push:

- D_mumu(mu, tau): dmumu_raw_norm of compute_dmumu_arrays_full
  (src/compute_delta_mu2_dmumu_full.jl:706-744) over the cells holding at
  least ``min_count`` pairs;
- <dmu^2>(tau): the per-lag particle mean of the Welford triple
  (src/compute_delta_mu2_curve.jl:409-429);
- D_pp(tau): dpp_raw_norm of compute_dpp_arrays (src/compute_dpp_full.jl:301-330)
  over the first ``n_dpp`` particles, each form with its own p0, from a
  Float64 phase-space cache: the Float32 cache of the reference rounds |p|
  to ~6e-8 per sample, which at 1 GeV in a weakly scattering field is the
  size of the momentum changes themselves, so that rounding -- the same
  for either push -- would decide D_pp instead of the push;
- |dgamma|/gamma at the end against the FP64 push, and |gamma_end/gamma_0 - 1|
  of every form on the field with u = 0 (E = 0), where energy is conserved to
  rounding.

Each FP64 statistic carries a sampling error: once trajectories decorrelate
(chaos, or a field stored at lower precision) a form is a new draw of the
same statistic, not a rounding of the FP64 value.  The error is measured
per cell by batch means over independent batches of particles; a cell
passes when the form is within the tolerance (1 %), or -- where the
statistic is not resolved to 1 % by the particle count -- within K_SIGMA
standard errors of the difference of two runs.  Three more FP64 pushes are
held to the same test, which checks the test itself:
- f64_1ulp: x1 moved by one FP64 ulp (chaotic divergence alone);
- f64_f32ulp: x1 moved by one FP32 ulp of the box length, a perturbation of
  the size the FP32 push makes every step;
- f64_resample: an independent sample of initial states (another seed, the
  same distribution): the sampling noise itself.

The FP64 push runs over FP64 bricks with a brick sort every 64 steps; its
results are bit-identical to the reference-layout FP64 push (the parity
tests show this against the oracle).
"""
from __future__ import annotations

import math

import numpy as np

from . import fields as F
from . import runner as R
from . import stats as S
from .fields import FieldLibrary
from .particles import energy_to_gamma, init_particles_device
from .time_units import build_mu_edges_full, log_spaced_lag_steps, reference_Omega0

FORMS = {"f32": "brick_f32", "bf16": "brick_bf16"}
KEYS = R.KEYS


def build_libraries(fields_si, grid, forms=("f32", "bf16"), with_e0=True):
    """FP64-brick library plus one brick library per form, and (with_e0) the
    same libraries of the field with u = 0.  fields_si: six CUDA float64
    tensors (Bx, By, Bz, ux, uy, uz) in SI units."""
    import torch

    B0 = F.reference_B0_T(*fields_si[:3])
    libs = {"f64": FieldLibrary(fields_si, grid, "brick_f64")}
    for f in forms:
        libs[f] = FieldLibrary(fields_si, grid, FORMS[f], B_ref_T=B0)
    if with_e0:
        zero = [torch.zeros_like(fields_si[0])] * 3
        e0 = list(fields_si[:3]) + zero
        libs["f64_e0"] = FieldLibrary(e0, grid, "brick_f64")
        for f in forms:
            libs[f + "_e0"] = FieldLibrary(e0, grid, FORMS[f], B_ref_T=B0)
    return libs, B0


def dpp_sums_f64(pm, lags, p0):
    """The D_pp sums of process_momenta_chunk_dpp_cpu! (src/compute_dpp_full.jl:247-288)
    over |p| of every (save, particle) in FP64 (a CUDA tensor [nsave][n]):
    for each lag, pairs of finite ends, dp = |p|(s + L) - |p|(s)."""
    import torch

    out = {k: np.zeros(len(lags)) for k in ("sum_delta_p", "sum_delta_p2", "sum_delta_p_norm", "sum_delta_p_norm2")}
    out["counts"] = np.zeros(len(lags), np.int64)
    for i, L in enumerate(int(l) for l in lags):
        if L >= pm.shape[0]:
            continue
        d = pm[L:] - pm[:-L]
        d = d[torch.isfinite(d)]
        dn = d / p0
        out["counts"][i] = int(d.numel())
        out["sum_delta_p"][i] = float(d.sum().item())
        out["sum_delta_p2"][i] = float((d * d).sum().item())
        out["sum_delta_p_norm"][i] = float(dn.sum().item())
        out["sum_delta_p_norm2"][i] = float((dn * dn).sum().item())
    return out


def _push(lib, state, dt, nsteps, stride, cache_mode, n, cache_f64=False):
    """Push the first n particles of `state` (dict of CUDA float64 tensors);
    returns (cache, final state dict of CUDA tensors)."""
    import torch

    nsave = R.n_saves(nsteps, stride) if cache_mode != "none" else 0
    sub = {k: state[k][:n].clone() for k in KEYS}
    alive = torch.ones(n, dtype=torch.uint8, device="cuda")
    cache = None
    if cache_mode != "none":
        shape = (nsave, n) if cache_mode == "mu" else (nsave, 6, n)
        cache = torch.empty(shape, dtype=torch.float64 if cache_f64 else torch.float32, device="cuda")
    if lib.storage == "brick_f64":
        ens = R.DeviceEnsemble(lib, sub, alive)
        ens.advance(R.push_params(dt, nsteps, stride, cache=cache_mode, cache_f64=cache_f64, precision="f64",
                                  sort_every=64), 0, nsteps, cache, 0, nsave)
        return cache, ens.state
    ens = R.FastEnsemble(lib, sub, alive)
    ens.advance(R.push_params(dt, nsteps, stride, cache=cache_mode, cache_f64=cache_f64, precision="f32",
                              sort_every=64), 0, nsteps, cache, 0, nsave)
    final, _ = ens.export()
    ens.close()
    return cache, final


def _gamma(st):
    import torch

    p = torch.sqrt(st["p1"] * st["p1"] + st["p2"] * st["p2"] + st["p3"] * st["p3"])
    return torch.sqrt(1.0 + (p / (F.M_P * F.C_LIGHT)) ** 2)


K_SIGMA = 5.0  # sampling band: k standard errors of the difference of two runs
SE_CAP = 0.05  # cells whose FP64 standard error exceeds this are not measured by the sample


def rel(a, b):
    """|a - b| / |b| per cell (NaN where either is not finite or b is 0)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[~(np.isfinite(a) & np.isfinite(b) & (np.abs(b) > 0))] = np.nan
    return r


def ratio_se(S, C):
    """Relative standard error of sum(S) / sum(C) from per-batch sums S and
    counts C ([G, ...]; independent batches of particles): the linearised
    ratio-estimator variance G/(G-1) * sum_g (S_g - R C_g)^2 / (sum C)^2,
    which holds for batches of unequal counts and for the correlated pairs
    within one particle's series."""
    S, C = np.asarray(S, np.float64), np.asarray(C, np.float64)
    G = S.shape[0]
    with np.errstate(divide="ignore", invalid="ignore"):
        St, Ct = S.sum(0), C.sum(0)
        R = St / Ct
        se = np.sqrt(G / (G - 1.0) * ((S - R * C) ** 2).sum(0)) / Ct
        out = se / np.abs(R)
    out[~np.isfinite(out)] = np.nan
    return out


def rel_err(a, b, se, mask=None, tol=0.01, k=K_SIGMA, se_cap=SE_CAP):
    """Relative errors |a - b| / |b| over the cells finite in both (and in
    mask), judged against the reference's own relative standard error `se`
    per cell: a cell passes when its error is within tol, or within
    k * sqrt(2) * se where the statistic is not resolved to tol (two runs
    each carry the sampling error).  Cells whose standard error exceeds
    se_cap are held by a handful of particles (a few mirror crossings carry
    the sum); their spread is not Gaussian and they are counted, not judged.
    Returns the max and median error, the max over the resolved cells
    (k sqrt(2) se <= tol), the largest z = error / (sqrt(2) se), and the
    failing cells."""
    r = rel(a, b)
    m = np.isfinite(r) & np.isfinite(se)
    if mask is not None:
        m &= mask
    unmeasured = int((m & (se > se_cap)).sum())
    m &= se <= se_cap
    if not m.any():
        return {"max": math.nan, "median": math.nan, "cells": 0, "failing": []}
    band = k * math.sqrt(2.0) * se
    resolved = m & (band <= tol)
    z = np.where(m, r / (math.sqrt(2.0) * np.maximum(se, 1e-300)), 0.0)
    fail = m & (r > np.maximum(tol, band))
    out = {"max": float(r[m].max()), "median": float(np.median(r[m])), "cells": int(m.sum()),
           "unmeasured_cells": unmeasured, "resolved_cells": int(resolved.sum()),
           "max_resolved": float(r[resolved].max()) if resolved.any() else 0.0,
           "max_z": float(z.max()), "median_se": float(np.median(se[m])),
           "failing": [[int(v) for v in np.atleast_1d(i)] for i in zip(*np.nonzero(fail))][:8]}
    if fail.any():
        i = np.unravel_index(int(np.argmax(np.where(fail, r, -1.0))), r.shape)
        out.update(worst_cell=[int(v) for v in i], worst_ref=float(np.asarray(b)[i]),
                   worst_value=float(np.asarray(a)[i]), worst_se=float(se[i]))
    return out


PRODUCTS = ("D_mumu", "delta_mu2", "D_pp")
FLOORS = ("f64_1ulp", "f64_f32ulp", "f64_resample")


def check_forms(r, forms=("f32", "bf16")):
    """The tolerance test on one compare_forms result: every cell of every
    product of each form (and of each FP64 floor run, which checks the
    test itself) within the tolerance, or within the sampling band where
    the FP64 statistic is not resolved to the tolerance.  Returns the list
    of failures (empty when the result passes)."""
    bad = []
    for prod in PRODUCTS:
        for form in tuple(forms) + FLOORS:
            e = r[form][prod]
            if not e["cells"]:
                bad.append((form, prod, "no cells"))
            elif e["failing"]:
                bad.append((form, prod, e["worst_cell"], e["worst_value"], e["worst_ref"], e["worst_se"]))
    return bad


def compare_forms(libs, B0, grid, energy_GeV, n_particles, steps_per_gyroperiod=128, gyroperiods=50, stride=8,
                  n_lags=32, n_bins=20, n_dpp=131072, min_count=100, forms=("f32", "bf16"), seed=7, mu0=0.525,
                  tol=0.01, batches=16, arrays=None):
    """Errors of each form (and of the FP64 floor runs) against the FP64
    push for one energy; fixed-mu injection (mu0, random gyrophase) at
    random positions.  mu0 sits inside a |mu| bin (the default 0.525 is the
    centre of [0.5, 0.55) with 20 bins): injected exactly on an edge, the
    rounding of the initial field would move about half of the particles
    into the bin below, and the first saves of the two runs would fill
    different cells.

    The FP64 statistics carry a sampling error of their own; it is measured
    by batch means over `batches` independent batches of particles
    (ratio_se for D_mumu cells and D_pp lags, the Welford variance of the
    per-particle values for <dmu^2>).  Returns a dict keyed by form with
    rel_err of D_mumu, <dmu^2> and D_pp, |dgamma|/gamma at the end, and the
    E = 0 energy drift (when the libraries hold the u = 0 field).  A dict
    passed as `arrays` receives each run's product arrays ("f64" the
    reference) and the reference's relative standard errors ("se")."""
    import torch

    g0 = energy_to_gamma(energy_GeV)
    dt = (2 * math.pi / steps_per_gyroperiod) / reference_Omega0(B0, g0, F.Q_E, F.M_P)
    nsteps = steps_per_gyroperiod * gyroperiods + 1
    nsave = R.n_saves(nsteps, stride)
    lags = log_spaced_lag_steps(nsave - 1, n_lags)
    edges, _ = build_mu_edges_full(0.0, 1.0, n_bins)
    tau = np.array([l * stride * 2 * math.pi / steps_per_gyroperiod for l in lags])  # t Omega0
    n_dpp = min(n_dpp, n_particles)
    st = init_particles_device(libs["f64"], n_particles, energy_GeV, seed=seed, injection_mode="fixed_mu", mu0=mu0)
    st = {k: st[k].contiguous() for k in KEYS}
    st_ulp = dict(st, x1=torch.nextafter(st["x1"], torch.full_like(st["x1"], math.inf)))
    st_f32ulp = dict(st, x1=st["x1"] + (grid.xmax - grid.xmin) * 2.0 ** -24)
    st_resample = init_particles_device(libs["f64"], n_particles, energy_GeV, seed=seed + 7919,
                                        injection_mode="fixed_mu", mu0=mu0)
    st_resample = {k: st_resample[k].contiguous() for k in KEYS}

    def dmumu_acc(mu):
        acc = S.new_dmumu_accumulators(len(lags), n_bins, device="cuda")
        S.process_mu_chunk_dmumu(mu, lags, edges, acc["particle_counts"], acc["particle_means"],
                                 acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                                 acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"],
                                 layout="particle_fastest")
        return {k: v.cpu().numpy() for k, v in acc.items()}

    def products(lib, state, with_se=False):
        mu, final = _push(lib, state, dt, nsteps, stride, "mu", n_particles)
        a = dmumu_acc(mu)
        out = {}
        if with_se:
            cuts = np.linspace(0, n_particles, batches + 1).astype(int)
            parts = [dmumu_acc(mu[:, cuts[g]:cuts[g + 1]].contiguous()) for g in range(batches)]
            se_d = ratio_se([q["dmumu_sum_delta2"] for q in parts], [q["dmumu_counts"] for q in parts])
            with np.errstate(divide="ignore", invalid="ignore"):
                n_p = a["particle_counts"].astype(np.float64)
                se_pm = np.sqrt(a["particle_m2s"] / (n_p - 1.0) / n_p) / np.abs(a["particle_means"])
            out["se"] = {"D": se_d, "pm": se_pm}
        del mu
        d = S.compute_dmumu_arrays_full(a["dmumu_counts"], a["dmumu_sum_delta"], a["dmumu_sum_delta2"], tau, tau,
                                        min_count)
        ps, _ = _push(lib, state, dt, nsteps, stride, "phase_space", n_dpp, cache_f64=True)
        pm = torch.sqrt(ps[:, 3] * ps[:, 3] + ps[:, 4] * ps[:, 4] + ps[:, 5] * ps[:, 5])  # |p| per (save, particle)
        del ps
        p0 = float(pm[0, 0].item())
        b = dpp_sums_f64(pm, lags, p0)
        if with_se:
            cuts = np.linspace(0, n_dpp, batches + 1).astype(int)
            parts = [dpp_sums_f64(pm[:, cuts[g]:cuts[g + 1]], lags, p0) for g in range(batches)]
            out["se"]["Dpp"] = ratio_se([q["sum_delta_p_norm2"] for q in parts], [q["counts"] for q in parts])
        del pm
        dpp = S.compute_dpp_arrays(b["counts"], b["sum_delta_p"], b["sum_delta_p2"], b["sum_delta_p_norm"],
                                   b["sum_delta_p_norm2"], tau, tau)
        out.update(D=d["dmumu_raw_norm"], counts=a["dmumu_counts"], pm=a["particle_means"],
                   Dpp=dpp["dpp_raw_norm"], gamma=_gamma(final).cpu().numpy())
        return out

    ref = products(libs["f64"], st, with_se=True)
    se = ref["se"]
    out = {"energy_GeV": energy_GeV, "particles": n_particles, "dpp_particles": n_dpp, "saves": nsave,
           "lags": int(len(lags)), "mu_bins": n_bins, "min_count_per_cell": min_count, "mu0": mu0,
           "steps": nsteps - 1, "cells_counted": int((ref["counts"] >= min_count).sum()), "tolerance": tol,
           "k_sigma": K_SIGMA, "batches": batches}
    cells = ref["counts"] >= min_count
    results = {}
    for form, start in (("f64_1ulp", st_ulp), ("f64_f32ulp", st_f32ulp), ("f64_resample", st_resample)):
        results[form] = products(libs["f64"], start)
        torch.cuda.empty_cache()
    for form in forms:
        results[form] = products(libs[form], st)
        torch.cuda.empty_cache()
    if arrays is not None:
        arrays.update(results, f64=ref, se=se)
    for form, r in results.items():
        out[form] = {"D_mumu": rel_err(r["D"], ref["D"], se["D"], cells, tol),
                     "delta_mu2": rel_err(r["pm"], ref["pm"], se["pm"], None, tol),
                     "D_pp": rel_err(r["Dpp"], ref["Dpp"], se["Dpp"], None, tol),
                     "gamma_vs_f64_end": float(np.max(np.abs(r["gamma"] / ref["gamma"] - 1)))}
    # E = 0: every form conserves energy to rounding
    if "f64_e0" in libs:
        n_e0 = min(n_particles, 65536)
        for form in ("f64",) + tuple(forms):
            _, final = _push(libs[form + "_e0"], st, dt, nsteps, stride, "none", n_e0)
            g_start = _gamma({k: st[k][:n_e0] for k in KEYS})
            drift = float(torch.max(torch.abs(_gamma(final) / g_start - 1.0)).item())
            out.setdefault(form, {})["gamma_drift_E0"] = drift
    return out
