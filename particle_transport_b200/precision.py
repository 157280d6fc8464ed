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

Three more FP64 pushes give the floors a push is judged against:
- f64_1ulp: x1 moved by one FP64 ulp (chaotic divergence alone);
- f64_f32ulp: x1 moved by one FP32 ulp of the box length, a perturbation of
  the size the FP32 push makes every step;
- f64_resample: an independent sample of initial states (another seed, the
  same distribution), i.e. the sampling noise of each cell.  A product that
  differs between two samples by more than the tolerance is not resolved to
  that tolerance by the particle count, whatever the push: once trajectories
  decorrelate (chaos, or a field stored at lower precision) a form can only
  be held to that floor.

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


def rel(a, b):
    """|a - b| / |b| per cell (NaN where either is not finite or b is 0)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[~(np.isfinite(a) & np.isfinite(b) & (np.abs(b) > 0))] = np.nan
    return r


def rel_err(a, b, mask=None, resolved=None):
    """Relative errors |a - b| / |b| over the cells finite in both (and in
    mask): the max and median, and the max over the `resolved` cells with
    the worst resolved cell's index and values."""
    r = rel(a, b)
    m = np.isfinite(r)
    if mask is not None:
        m &= mask
    if not m.any():
        return {"max": math.nan, "median": math.nan, "cells": 0}
    out = {"max": float(r[m].max()), "median": float(np.median(r[m])), "cells": int(m.sum())}
    if resolved is not None:
        mr = m & resolved
        out["resolved_cells"] = int(mr.sum())
        if mr.any():
            w = np.where(mr, r, -1.0)
            i = np.unravel_index(int(np.argmax(w)), w.shape)
            out.update(max_resolved=float(r[i]), worst_cell=[int(v) for v in i],
                       worst_ref=float(np.asarray(b)[i]), worst_value=float(np.asarray(a)[i]))
        else:
            out["max_resolved"] = 0.0
    return out


PRODUCTS = ("D_mumu", "delta_mu2", "D_pp")
FLOORS = ("f64_f32ulp", "f64_resample")


def check_forms(r, forms=("f32", "bf16"), tol=0.01):
    """The tolerance test on one compare_forms result: for every product and
    form, (1) the cells FP64 resolves (both floors within resolve_tol) are
    within tol of the FP64 push, and (2) every cell is within tol, or within
    twice the larger FP64 floor where the statistic itself moves by more.
    Returns the list of failures (empty when the result passes)."""
    bad = []
    for prod in PRODUCTS:
        floor = max(r[f][prod]["max"] for f in FLOORS)
        for form in forms:
            e = r[form][prod]
            if not e["cells"]:
                bad.append((form, prod, "no cells"))
                continue
            if e.get("max_resolved", 0.0) > tol:
                bad.append((form, prod, "resolved", e["max_resolved"], e.get("worst_cell")))
            if e["max"] > max(tol, 2.0 * floor):
                bad.append((form, prod, "all cells", e["max"], floor))
    return bad


def compare_forms(libs, B0, grid, energy_GeV, n_particles, steps_per_gyroperiod=128, gyroperiods=50, stride=8,
                  n_lags=32, n_bins=20, n_dpp=131072, min_count=100, forms=("f32", "bf16"), seed=7, mu0=0.5,
                  resolve_tol=0.005, arrays=None):
    """Errors of each form (and of the FP64 floor runs) against the FP64
    push for one energy; fixed-mu injection (mu0, random gyrophase) at
    random positions.  Returns a dict keyed by form with the relative errors
    of D_mumu, <dmu^2> and D_pp -- over every cell, and over the resolved
    cells (those both FP64 floors f64_f32ulp and f64_resample reproduce
    within resolve_tol) with the worst one's index and values --,
    |dgamma|/gamma at the end, and the E = 0 energy drift (when the
    libraries hold the u = 0 field).  A dict passed as `arrays` receives
    each run's product arrays ("f64" the reference) and the resolved masks."""
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

    def products(lib, state):
        mu, final = _push(lib, state, dt, nsteps, stride, "mu", n_particles)
        acc = S.new_dmumu_accumulators(len(lags), n_bins, device="cuda")
        S.process_mu_chunk_dmumu(mu, lags, edges, acc["particle_counts"], acc["particle_means"],
                                 acc["particle_m2s"], acc["pair_sum_squares"], acc["pair_counts"],
                                 acc["dmumu_counts"], acc["dmumu_sum_delta"], acc["dmumu_sum_delta2"],
                                 layout="particle_fastest")
        del mu
        a = {k: v.cpu().numpy() for k, v in acc.items()}
        d = S.compute_dmumu_arrays_full(a["dmumu_counts"], a["dmumu_sum_delta"], a["dmumu_sum_delta2"], tau, tau,
                                        min_count)
        ps, _ = _push(lib, state, dt, nsteps, stride, "phase_space", n_dpp, cache_f64=True)
        pm = torch.sqrt(ps[:, 3] * ps[:, 3] + ps[:, 4] * ps[:, 4] + ps[:, 5] * ps[:, 5])  # |p| per (save, particle)
        del ps
        b = dpp_sums_f64(pm, lags, float(pm[0, 0].item()))
        del pm
        dpp = S.compute_dpp_arrays(b["counts"], b["sum_delta_p"], b["sum_delta_p2"], b["sum_delta_p_norm"],
                                   b["sum_delta_p_norm2"], tau, tau)
        return dict(D=d["dmumu_raw_norm"], counts=a["dmumu_counts"], pm=a["particle_means"],
                    Dpp=dpp["dpp_raw_norm"], gamma=_gamma(final).cpu().numpy())

    ref = products(libs["f64"], st)
    out = {"energy_GeV": energy_GeV, "particles": n_particles, "dpp_particles": n_dpp, "saves": nsave,
           "lags": int(len(lags)), "mu_bins": n_bins, "min_count_per_cell": min_count,
           "steps": nsteps - 1, "cells_counted": int((ref["counts"] >= min_count).sum()),
           "resolve_tolerance": resolve_tol}
    cells = ref["counts"] >= min_count
    floors = {}
    for form in ("f64_1ulp", "f64_f32ulp", "f64_resample"):
        start = {"f64_1ulp": st_ulp, "f64_f32ulp": st_f32ulp, "f64_resample": st_resample}[form]
        floors[form] = products(libs["f64"], start)
        torch.cuda.empty_cache()
    # a cell (a lag for <dmu^2> and D_pp) is resolved when FP64 itself reproduces it within
    # resolve_tol both under a one-FP32-ulp perturbation and from an independent sample
    resolved = {}
    for key, prod in (("D", "D_mumu"), ("pm", "delta_mu2"), ("Dpp", "D_pp")):
        ok = np.ones(np.shape(ref[key]), bool)
        for f in ("f64_f32ulp", "f64_resample"):
            rr = rel(floors[f][key], ref[key])
            ok &= np.isfinite(rr) & (rr <= resolve_tol)
        resolved[prod] = ok
    results = dict(floors)
    for form in forms:
        results[form] = products(libs[form], st)
        torch.cuda.empty_cache()
    if arrays is not None:
        arrays.update(results, f64=ref, resolved=resolved)
    for form, r in results.items():
        out[form] = {"D_mumu": rel_err(r["D"], ref["D"], cells, resolved["D_mumu"]),
                     "delta_mu2": rel_err(r["pm"], ref["pm"], None, resolved["delta_mu2"]),
                     "D_pp": rel_err(r["Dpp"], ref["Dpp"], None, resolved["D_pp"]),
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
