"""Transport statistics: drop-in mirrors of the reference's CPU kernels.

process_mu_chunk_dmumu      <- process_mu_chunk_dmumu_cpu!   src/compute_delta_mu2_dmumu_full.jl:656
process_momenta_chunk_dpp   <- process_momenta_chunk_dpp_cpu! src/compute_dpp_full.jl:247
fill_energy_snapshots       <- fill_energy_snapshots!          src/compute_dpp_full.jl:290
reconstruct_mu_chunk        <- reconstruct_mu_chunk_gpu        src/compute_delta_mu2_curve.jl:186

Array conventions follow the reference's Julia arrays read as C-ordered
numpy arrays with the axes reversed:
  mu_chunk  Julia (nsave, chunk)         -> numpy (chunk, nsave)
  momenta   Julia (chunk, 3, nsave)      -> numpy (nsave, 3, chunk)
  dmumu_*   Julia (n_bins, n_lags)       -> numpy (n_lags, n_bins)
  energy    Julia (n_snap, n_particles)  -> numpy (n_particles, n_snap)
numpy arguments go through the host entry points; CUDA torch tensors go
through the *_device entry points on torch's current stream.  All
accumulators are add-into, as in the reference.

The derived arrays (compute_dmumu_arrays_full, average_over_tau_full,
build_output_dataframe, compute_dpp_arrays) are a few FP64 divisions per
(bin, lag) and stay host-side numpy, restated from the reference.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib

START = {"sliding": _lib.PT_START_SLIDING, "injection": _lib.PT_START_INJECTION}


def _is_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and x.is_cuda


def _check(arr, shape, dtype, name):
    if tuple(arr.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(arr.shape)}, expected {tuple(shape)}")
    if _is_cuda(arr):
        import torch
        tdt = {np.float32: torch.float32, np.float64: torch.float64, np.int64: torch.int64}[dtype]
        if arr.dtype != tdt or not arr.is_contiguous():
            raise ValueError(f"{name} must be a contiguous {tdt} tensor")
    elif arr.dtype != dtype or not arr.flags.c_contiguous:
        raise ValueError(f"{name} must be a C-contiguous {np.dtype(dtype)} array")


def new_dmumu_accumulators(n_lags: int, n_bins: int, device=None):
    """Zeroed accumulators (pipeline:1674-1681)."""
    if device is not None:
        import torch
        z = lambda s, t: torch.zeros(s, dtype=t, device=device)  # noqa: E731
        i64, f64 = torch.int64, torch.float64
    else:
        z = lambda s, t: np.zeros(s, dtype=t)  # noqa: E731
        i64, f64 = np.int64, np.float64
    return {"particle_counts": z(n_lags, i64), "particle_means": z(n_lags, f64), "particle_m2s": z(n_lags, f64),
            "pair_sum_squares": z(n_lags, f64), "pair_counts": z(n_lags, i64),
            "dmumu_counts": z((n_lags, n_bins), i64), "dmumu_sum_delta": z((n_lags, n_bins), f64),
            "dmumu_sum_delta2": z((n_lags, n_bins), f64)}


def process_mu_chunk_dmumu(mu_chunk, lag_steps, mu_edges, particle_counts, particle_means, particle_m2s,
                           pair_sum_squares, pair_counts, dmumu_counts, dmumu_sum_delta, dmumu_sum_delta2,
                           start_mode="sliding", bin_abs=True, layout="time_fastest", nsave=None):
    """Accumulate one chunk of mu series into the D_mumu / <dmu^2> accumulators.

    mu_chunk: float32, (chunk, pitch) for layout "time_fastest" (the Julia
    mu_chunk, or the time-fastest cache of the FP32 push; the first nsave
    saves of each row are used, all of them by default) or (nsave, chunk) for
    "particle_fastest" (the mu cache as written: one row per save)."""
    start_mode = str(start_mode)
    if start_mode not in START:
        raise ValueError(f"Unknown dmumu_start_mode: {start_mode}")
    if layout == "time_fastest":
        chunk, pitch = mu_chunk.shape
        nsave = pitch if nsave is None else int(nsave)
        if not 1 <= nsave <= pitch:
            raise ValueError("nsave must be in [1, mu_chunk.shape[1]]")
        sp, ss = pitch, 1
    elif layout == "particle_fastest":
        nsave, chunk = mu_chunk.shape
        sp, ss = 1, chunk
    else:
        raise ValueError("layout must be time_fastest or particle_fastest")
    n_lags = len(lag_steps)
    n_bins = len(mu_edges) - 1
    _check(mu_chunk, mu_chunk.shape, np.float32, "mu_chunk")
    for a, nm, dt in ((particle_counts, "particle_counts", np.int64), (particle_means, "particle_means", np.float64),
                      (particle_m2s, "particle_m2s", np.float64), (pair_sum_squares, "pair_sum_squares", np.float64),
                      (pair_counts, "pair_counts", np.int64)):
        _check(a, (n_lags,), dt, nm)
    for a, nm, dt in ((dmumu_counts, "dmumu_counts", np.int64), (dmumu_sum_delta, "dmumu_sum_delta", np.float64),
                      (dmumu_sum_delta2, "dmumu_sum_delta2", np.float64)):
        _check(a, (n_lags, n_bins), dt, nm)
    accs = (dmumu_counts, dmumu_sum_delta, dmumu_sum_delta2, particle_counts, particle_means, particle_m2s,
            pair_sum_squares, pair_counts)
    if _is_cuda(mu_chunk):
        import torch
        lags = torch.as_tensor(np.asarray(lag_steps, dtype=np.int64), device=mu_chunk.device)
        edges = torch.as_tensor(np.asarray(mu_edges, dtype=np.float64), device=mu_chunk.device)
        ctx = _lib.torch_context(mu_chunk)
        _lib.call("pt_dmumu_accumulate_device", ctx.handle, _lib.ptr(mu_chunk), chunk, nsave, sp, ss, _lib.ptr(lags),
                  n_lags, _lib.ptr(edges), n_bins, START[start_mode], int(bool(bin_abs)),
                  *[_lib.ptr(a) for a in accs])
    else:
        lags = np.ascontiguousarray(lag_steps, dtype=np.int64)
        edges = np.ascontiguousarray(mu_edges, dtype=np.float64)
        ctx = _lib.context(0)
        _lib.call("pt_dmumu_accumulate", ctx.handle, _lib.ptr(mu_chunk), chunk, nsave, sp, ss, _lib.ptr(lags), n_lags,
                  _lib.ptr(edges), n_bins, START[start_mode], int(bool(bin_abs)), *[_lib.ptr(a) for a in accs])


def process_phase_space_chunk_dmumu(positions, momenta, Bx, By, Bz, grid, lag_steps, mu_edges, particle_counts,
                                    particle_means, particle_m2s, pair_sum_squares, pair_counts, dmumu_counts,
                                    dmumu_sum_delta, dmumu_sum_delta2, start_mode="sliding", bin_abs=True):
    """Phase-space D_mumu on the device: mu reconstructed from positions and
    momenta inside the binning kernel (reconstruct_mu_chunk_gpu feeding
    process_mu_chunk_dmumu_cpu!, src/compute_delta_mu2_dmumu_full.jl:1137-1164).

    positions, momenta: CUDA tensors shaped (nsave, 3, chunk) -- any row and
    component strides, particles contiguous (e.g. views [:, 0:3] and [:, 3:6]
    of the device phase-space cache (nsave, 6, n)); float32 (the reference's
    default compute precision) or float64.  Bx, By, Bz: CUDA tensors (nz, ny,
    nx) of the same dtype.  Accumulators as for process_mu_chunk_dmumu (CUDA)."""
    import torch

    start_mode = str(start_mode)
    if start_mode not in START:
        raise ValueError(f"Unknown dmumu_start_mode: {start_mode}")
    if not (_is_cuda(positions) and _is_cuda(momenta)):
        raise ValueError("positions and momenta must be CUDA tensors")
    dt = positions.dtype
    if dt not in (torch.float32, torch.float64) or momenta.dtype != dt:
        raise ValueError("positions and momenta must share dtype float32 or float64")
    if positions.dim() != 3 or positions.shape[1] != 3 or tuple(momenta.shape) != tuple(positions.shape):
        raise ValueError("positions and momenta must be shaped (nsave, 3, chunk)")
    if positions.stride() != momenta.stride() or positions.stride(2) != 1:
        raise ValueError("positions and momenta need equal strides and contiguous particles")
    nsave, _, chunk = positions.shape
    bs = [b.contiguous() for b in (Bx, By, Bz)]
    for b in bs:
        if b.dtype != dt or not b.is_cuda or tuple(b.shape) != grid.shape:
            raise ValueError("B components must be CUDA tensors of the positions' dtype shaped (nz, ny, nx)")
    n_lags = len(lag_steps)
    n_bins = len(mu_edges) - 1
    for a, nm, t in ((particle_counts, "particle_counts", np.int64), (particle_means, "particle_means", np.float64),
                     (particle_m2s, "particle_m2s", np.float64), (pair_sum_squares, "pair_sum_squares", np.float64),
                     (pair_counts, "pair_counts", np.int64)):
        _check(a, (n_lags,), t, nm)
    for a, nm, t in ((dmumu_counts, "dmumu_counts", np.int64), (dmumu_sum_delta, "dmumu_sum_delta", np.float64),
                     (dmumu_sum_delta2, "dmumu_sum_delta2", np.float64)):
        _check(a, (n_lags, n_bins), t, nm)
    accs = (dmumu_counts, dmumu_sum_delta, dmumu_sum_delta2, particle_counts, particle_means, particle_m2s,
            pair_sum_squares, pair_counts)
    lags = torch.as_tensor(np.asarray(lag_steps, dtype=np.int64), device=positions.device)
    edges = torch.as_tensor(np.asarray(mu_edges, dtype=np.float64), device=positions.device)
    ctx = _lib.torch_context(positions)
    g = grid.to_c()
    _lib.call("pt_dmumu_accumulate_phase_space_device", ctx.handle, _lib.ptr(positions), _lib.ptr(momenta), chunk,
              nsave, positions.stride(0), positions.stride(1), _lib.ptr_array(bs), _lib.C.byref(g),
              int(dt == torch.float64), _lib.ptr(lags), n_lags, _lib.ptr(edges), n_bins, START[start_mode],
              int(bool(bin_abs)), *[_lib.ptr(a) for a in accs])


def new_dpp_accumulators(n_lags: int, device=None):
    if device is not None:
        import torch
        return {"counts": torch.zeros(n_lags, dtype=torch.int64, device=device),
                **{k: torch.zeros(n_lags, dtype=torch.float64, device=device)
                   for k in ("sum_delta_p", "sum_delta_p2", "sum_delta_p_norm", "sum_delta_p_norm2")}}
    return {"counts": np.zeros(n_lags, dtype=np.int64),
            **{k: np.zeros(n_lags) for k in ("sum_delta_p", "sum_delta_p2", "sum_delta_p_norm", "sum_delta_p_norm2")}}


def process_momenta_chunk_dpp(momenta, lag_steps, p0, counts, sum_delta_p, sum_delta_p2, sum_delta_p_norm,
                              sum_delta_p_norm2):
    """Accumulate D_pp lag sums for one momenta chunk, float32 (nsave, 3, chunk)."""
    nsave, three, chunk = momenta.shape
    if three != 3:
        raise ValueError("momenta dataset must have shape (particles, 3, steps).")
    if not (math.isfinite(p0) and p0 > 0.0):
        raise ValueError("Cannot compute D_pp normalization: invalid p0.")
    n_lags = len(lag_steps)
    _check(momenta, momenta.shape, np.float32, "momenta")
    for a, nm, dt in ((counts, "counts", np.int64), (sum_delta_p, "sum_delta_p", np.float64),
                      (sum_delta_p2, "sum_delta_p2", np.float64), (sum_delta_p_norm, "sum_delta_p_norm", np.float64),
                      (sum_delta_p_norm2, "sum_delta_p_norm2", np.float64)):
        _check(a, (n_lags,), dt, nm)
    accs = (counts, sum_delta_p, sum_delta_p2, sum_delta_p_norm, sum_delta_p_norm2)
    if _is_cuda(momenta):
        import torch
        lags = torch.as_tensor(np.asarray(lag_steps, dtype=np.int64), device=momenta.device)
        ctx = _lib.torch_context(momenta)
        _lib.call("pt_dpp_accumulate_device", ctx.handle, _lib.ptr(momenta), chunk, nsave, _lib.ptr(lags), n_lags,
                  float(p0), *[_lib.ptr(a) for a in accs])
    else:
        lags = np.ascontiguousarray(lag_steps, dtype=np.int64)
        _lib.call("pt_dpp_accumulate", _lib.context(0).handle, _lib.ptr(momenta), chunk, nsave, _lib.ptr(lags), n_lags,
                  float(p0), *[_lib.ptr(a) for a in accs])


def fill_energy_snapshots(energy_snapshots, momenta, snapshot_indices, particle_offset: int = 0):
    """energy_snapshots: float64 (n_particles, n_snap); snapshot_indices are
    0-based save indices; writes rows particle_offset .. + chunk.  With CUDA
    tensors (momenta and energy_snapshots) it runs on the device without a
    host round trip (pt_energy_snapshots_device)."""
    nsave, _, chunk = momenta.shape
    if _is_cuda(momenta):
        import torch

        snaps = torch.as_tensor(np.asarray(snapshot_indices, dtype=np.int64), device=momenta.device)
        if not (_is_cuda(energy_snapshots) and energy_snapshots.dtype == torch.float64
                and energy_snapshots.is_contiguous() and energy_snapshots.shape[1] == len(snaps)
                and energy_snapshots.shape[0] >= particle_offset + chunk):
            raise ValueError("energy_snapshots must be a contiguous CUDA float64 tensor (n_particles, n_snap)")
        _check(momenta, momenta.shape, np.float32, "momenta")
        ctx = _lib.torch_context(momenta)
        _lib.call("pt_energy_snapshots_device", ctx.handle, _lib.ptr(momenta), chunk, nsave, _lib.ptr(snaps),
                  len(snaps), int(particle_offset), _lib.ptr(energy_snapshots))
        return
    snaps = np.ascontiguousarray(snapshot_indices, dtype=np.int64)
    if energy_snapshots.shape[1] != len(snaps) or energy_snapshots.shape[0] < particle_offset + chunk:
        raise ValueError("energy_snapshots has the wrong shape")
    _check(momenta, momenta.shape, np.float32, "momenta")
    if energy_snapshots.dtype != np.float64 or not energy_snapshots.flags.c_contiguous:
        raise ValueError("energy_snapshots must be C-contiguous float64")
    _lib.call("pt_energy_snapshots", _lib.context(0).handle, _lib.ptr(momenta), chunk, nsave, _lib.ptr(snaps),
              len(snaps), int(particle_offset), _lib.ptr(energy_snapshots))


def energy_histogram(momenta, snapshot_indices, e_min_GeV: float, e_max_GeV: float, n_bins: int = 256, counts=None):
    """Log-binned kinetic-energy histograms of the snapshot saves on the device:
    counts (n_snap, n_bins) int64; bin k spans e_min*(e_max/e_min)^(k/n .. (k+1)/n).
    momenta: CUDA float32 tensor (nsave, 3, chunk)."""
    import torch

    nsave, _, chunk = momenta.shape
    snaps = torch.as_tensor(np.asarray(snapshot_indices, dtype=np.int64), device=momenta.device)
    if counts is None:
        counts = torch.zeros((len(snaps), n_bins), dtype=torch.int64, device=momenta.device)
    ctx = _lib.torch_context(momenta)
    _lib.call("pt_energy_histogram_device", ctx.handle, _lib.ptr(momenta), chunk, nsave, _lib.ptr(snaps), len(snaps),
              float(e_min_GeV), float(e_max_GeV), int(n_bins), _lib.ptr(counts))
    return counts


def reconstruct_mu_chunk(positions, momenta, Bx, By, Bz, grid, dtype=np.float32):
    """mu of a phase-space chunk at the compute precision ``dtype``.
    positions/momenta: (nsave, 3, chunk); B: C-ordered (nz, ny, nx);
    returns mu shaped (chunk, nsave) (the Julia (nsave, chunk) array)."""
    dtype = np.dtype(dtype)
    f64 = dtype == np.float64
    pos = np.ascontiguousarray(positions, dtype=dtype)
    mom = np.ascontiguousarray(momenta, dtype=dtype)
    nsave, _, chunk = pos.shape
    bs = [np.ascontiguousarray(b, dtype=dtype) for b in (Bx, By, Bz)]
    out = np.empty((chunk, nsave), dtype=dtype)
    g = grid.to_c()
    _lib.call("pt_reconstruct_mu", _lib.context(0).handle, _lib.ptr(pos), _lib.ptr(mom), chunk, nsave,
              _lib.ptr_array(bs), _lib.C.byref(g), int(f64), _lib.ptr(out))
    return out


# --------------------------------------------------------------------------
# limits of the D_mumu entry points (the launch arithmetic of lagstats.cu)
# --------------------------------------------------------------------------
_DMUMU_SMEM_BUDGET = 200 * 1024  # shared memory a D_mumu CTA may use (B200 opt-in maximum is 227 KiB)
_DMUMU_NOALLOC_BYTES = 16 << 20  # the no-alloc entry's fixed device array
_WELFORD_PART_BYTES = 40


def _a16(v: int) -> int:
    return (v + 15) & ~15


def _dmumu_shape(nsave: int, n_lags: int, n_bins: int):
    nl_cap = min(max(32, ((_DMUMU_SMEM_BUDGET // 2) // (n_bins * 24)) // 32 * 32), 256)
    idx = 2 if nsave <= 65535 else 4
    slot = (_a16((nsave + 1) * 4) + _a16(nsave * idx) + _a16(4 * (8 * (n_bins + 1) + n_bins + 2)) +
            _a16(16 * nl_cap))
    nl = min(nl_cap, n_lags)  # the first lag batch is the widest
    fixed = _a16(8 * (n_bins + 1)) + max(nl * n_bins * 24, _WELFORD_PART_BYTES * 1024)
    return nl, slot, fixed


def dmumu_noalloc_fits(nsave: int, n_lags: int, n_bins: int) -> bool:
    """Whether pt_dmumu_accumulate_device_noalloc takes this shape: every
    series is staged on chip, and one CTA's partials fit the fixed array."""
    if n_lags <= 0:
        return True
    nl, slot, fixed = _dmumu_shape(nsave, n_lags, n_bins)
    per_cta = nl * n_bins * 24 + _WELFORD_PART_BYTES * nl + 64
    return fixed + slot <= _DMUMU_SMEM_BUDGET and (_DMUMU_NOALLOC_BYTES - 1024) // per_cta >= 1


def dmumu_scratch_bound(nsave: int, n_lags: int, n_bins: int, num_sms: int = 148) -> int:
    """Upper bound of the device scratch pt_dmumu_accumulate_device asks its
    context for when the series are staged in global memory (1024-thread
    CTAs, at most two per SM, eight series per CTA)."""
    if n_lags <= 0:
        return 0
    nl, slot, _ = _dmumu_shape(nsave, n_lags, n_bins)
    grid = 2 * num_sms
    return 3 * _a16(grid * nl * n_bins * 8) + _a16(_WELFORD_PART_BYTES * grid * nl) + grid * 8 * slot


# --------------------------------------------------------------------------
# derived arrays (host)
# --------------------------------------------------------------------------
def _jl_max0(x: float) -> float:
    """Julia's max(0.0, x) for Float64: a NaN argument gives NaN (Python's
    max(0.0, nan) gives 0.0)."""
    return x if (x != x or x > 0.0) else 0.0


def compute_dmumu_arrays_full(counts, sum_delta, sum_delta2, tau_s, tau_norm, min_count_per_cell: int):
    """src/compute_delta_mu2_dmumu_full.jl:706-744; arrays are (n_lags, n_bins)."""
    counts = np.asarray(counts)
    shape = counts.shape
    out = {k: np.full(shape, np.nan) for k in ("mean_delta", "mean_delta2", "drift_norm", "dmumu_raw_norm",
                                               "dmumu_centered_norm", "dmumu_raw_per_s", "dmumu_centered_per_s")}
    for li in range(shape[0]):
        tn, tp = float(tau_norm[li]), float(tau_s[li])
        for b in range(shape[1]):
            c = int(counts[li, b])
            if c < min_count_per_cell:
                continue
            dm = sum_delta[li, b] / c
            d2 = sum_delta2[li, b] / c
            cen = _jl_max0(d2 - dm * dm)
            out["mean_delta"][li, b] = dm
            out["mean_delta2"][li, b] = d2
            out["drift_norm"][li, b] = dm / tn
            out["dmumu_raw_norm"][li, b] = d2 / (2.0 * tn)
            out["dmumu_centered_norm"][li, b] = cen / (2.0 * tn)
            out["dmumu_raw_per_s"][li, b] = d2 / (2.0 * tp)
            out["dmumu_centered_per_s"][li, b] = cen / (2.0 * tp)
    return out


def average_over_tau_full(values, counts, min_count_per_cell: int):
    """src/compute_delta_mu2_dmumu_full.jl:746-776; returns (unweighted, count_weighted) per bin."""
    values, counts = np.asarray(values), np.asarray(counts)
    n_lags, n_bins = values.shape
    unw, cw = np.full(n_bins, np.nan), np.full(n_bins, np.nan)
    for b in range(n_bins):
        vs = ws = 0.0
        nv = tw = 0
        for li in range(n_lags):
            v, c = values[li, b], int(counts[li, b])
            if math.isfinite(v) and c >= min_count_per_cell:
                vs += v
                nv += 1
                ws += v * c
                tw += c
        if nv > 0:
            unw[b] = vs / nv
        if tw > 0:
            cw[b] = ws / tw
    return unw, cw


def sem_from_stats(count: int, m2: float) -> float:
    """src/compute_delta_mu2_curve.jl:387-393"""
    if count <= 1:
        return math.nan
    return math.sqrt((m2 / (count - 1)) / count)


def build_output_table(lag_steps, t_s, t_norm, particle_counts, particle_means, particle_m2s, pair_sum_squares,
                       pair_counts):
    """Columns of build_output_dataframe (src/compute_delta_mu2_curve.jl:409-429)."""
    lag_steps = np.asarray(lag_steps)
    tau_s = np.array([t_s[l] - t_s[0] for l in lag_steps])
    tau_norm = np.array([t_norm[l] - t_norm[0] for l in lag_steps])
    std = np.array([math.nan if c <= 1 else math.sqrt(particle_m2s[i] / (c - 1)) for i, c in enumerate(particle_counts)])
    sem = np.array([sem_from_stats(int(c), float(particle_m2s[i])) for i, c in enumerate(particle_counts)])
    pair_mean = np.array([math.nan if pair_counts[i] == 0 else pair_sum_squares[i] / pair_counts[i]
                          for i in range(len(pair_counts))])
    return {"lag_step": lag_steps, "tau_s": tau_s, "tau_norm": tau_norm, "tau_gyroperiods": tau_norm / (2.0 * math.pi),
            "delta_mu2_particle_mean": np.asarray(particle_means), "delta_mu2_particle_std": std,
            "delta_mu2_particle_sem": sem, "delta_mu2_pair_mean": pair_mean,
            "n_particles_used": np.asarray(particle_counts), "n_pairs_used": np.asarray(pair_counts)}


def compute_dpp_arrays(counts, sum_delta_p, sum_delta_p2, sum_delta_p_norm, sum_delta_p_norm2, tau_s, tau_norm):
    """src/compute_dpp_full.jl:301-330"""
    n = len(counts)
    keys = ("mean_delta_p", "mean_delta_p2", "mean_delta_p_norm", "mean_delta_p_norm2", "dpp_raw_per_s",
            "dpp_centered_per_s", "dpp_raw_norm", "dpp_centered_norm")
    out = {k: np.full(n, np.nan) for k in keys}
    for i in range(n):
        c = int(counts[i])
        if c <= 0:
            continue
        dm, d2 = sum_delta_p[i] / c, sum_delta_p2[i] / c
        nm, n2 = sum_delta_p_norm[i] / c, sum_delta_p_norm2[i] / c
        cen, cenn = _jl_max0(d2 - dm * dm), _jl_max0(n2 - nm * nm)
        out["mean_delta_p"][i], out["mean_delta_p2"][i] = dm, d2
        out["mean_delta_p_norm"][i], out["mean_delta_p_norm2"][i] = nm, n2
        out["dpp_raw_per_s"][i] = d2 / (2.0 * float(tau_s[i]))
        out["dpp_centered_per_s"][i] = cen / (2.0 * float(tau_s[i]))
        out["dpp_raw_norm"][i] = n2 / (2.0 * float(tau_norm[i]))
        out["dpp_centered_norm"][i] = cenn / (2.0 * float(tau_norm[i]))
    return out
