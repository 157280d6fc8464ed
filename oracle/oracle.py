"""ctypes binding of the CPU oracle (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; it is the checker, never the product.
Array layouts follow the reference's Julia arrays (see ``pt_oracle.c``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None


class Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
        ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
    ]


def grid_struct(g) -> Grid:
    """Build the C grid struct from any object with the grid attributes."""
    return Grid(g.nx, g.ny, g.nz, g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax, g.dx, g.dy, g.dz)


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = C.CDLL(path)
        P = C.c_void_p
        i64, i32, d = C.c_int64, C.c_int, C.c_double
        L.or_trilinear.restype = d
        L.or_trilinear.argtypes = [P, d, d, d, C.POINTER(Grid)]
        L.or_pitch_mu.restype = d
        L.or_pitch_mu.argtypes = [d] * 6
        L.or_mu_bin_index.restype = i32
        L.or_mu_bin_index.argtypes = [d, P, i32]
        L.or_push_run.restype = None
        L.or_push_run.argtypes = [P, C.POINTER(Grid), P, P, P, P, P, P, P, i64, d, i64, i64, i64, i64, i32, i32,
                                  i32, P, P, P, P, i32]
        L.or_reconstruct_mu_f64.restype = None
        L.or_reconstruct_mu_f64.argtypes = [P, P, i64, i64, P, C.POINTER(Grid), P, i32]
        L.or_reconstruct_mu_f32.restype = None
        L.or_reconstruct_mu_f32.argtypes = [P, P, i64, i64, P, i64, i64, i64, P, P, i32]
        L.or_dmumu_accumulate.restype = None
        L.or_dmumu_accumulate.argtypes = [P, i64, i64, i64, i64, P, i32, P, i32, i32, i32, P, P, P, P, P, P, P, P,
                                          i32]
        L.or_dmumu_accumulate_f64.restype = None
        L.or_dmumu_accumulate_f64.argtypes = L.or_dmumu_accumulate.argtypes
        L.or_dpp_accumulate.restype = None
        L.or_dpp_accumulate.argtypes = [P, i64, i64, P, i32, d, P, P, P, P, P, i32]
        L.or_energy_snapshots.restype = None
        L.or_energy_snapshots.argtypes = [P, i64, i64, P, i32, i64, P]
        L.or_kinetic_energy_gev.restype = d
        L.or_kinetic_energy_gev.argtypes = [d]
        L.or_num_threads.restype = i32
        L.or_init_particles.restype = i64
        L.or_init_particles.argtypes = [i64, C.c_uint64, d, i32, i32, d, P, P, C.POINTER(Grid), P, P, P, P, P, P]
        L.or_dmumu_arrays_full.restype = None
        L.or_dmumu_arrays_full.argtypes = [P, P, P, P, P, i32, i32, i64, P]
        L.or_average_over_tau_full.restype = None
        L.or_average_over_tau_full.argtypes = [P, P, i32, i32, i64, P, P]
        L.or_sem_from_stats.restype = d
        L.or_sem_from_stats.argtypes = [i64, d]
        L.or_output_table.restype = None
        L.or_output_table.argtypes = [P, i32, P, P, P, P, P, P, P]
        L.or_dpp_arrays.restype = None
        L.or_dpp_arrays.argtypes = [P, P, P, P, P, P, P, i32, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _ptr_array(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


def num_threads() -> int:
    return int(lib().or_num_threads())


def trilinear(arr, x, y, z, grid) -> float:
    a = np.asfortranarray(arr, dtype=np.float64)
    g = grid_struct(grid)
    return float(lib().or_trilinear(_p(a), x, y, z, C.byref(g)))


def mu_bin_index(v, edges) -> int:
    e = np.ascontiguousarray(edges, dtype=np.float64)
    return int(lib().or_mu_bin_index(float(v), _p(e), len(e) - 1))


def push_run(fields, grid, state, alive, dt, nsteps, stride, periodic=True, cache_mode=1, out_f64=False,
             step_begin=0, step_count=None, nthreads=0):
    """Advance ``state`` (dict x1..p3 of float64 arrays, modified in place) and
    return (cache, alive_count).  ``fields`` are six Fortran-ordered float64
    arrays Bx, By, Bz, ux, uy, uz in SI units."""
    fl = [np.asfortranarray(f, dtype=np.float64) for f in fields]
    n = state["x1"].shape[0]
    if step_count is None:
        step_count = nsteps - step_begin
    nsave = (nsteps - 1) // stride + 1
    dt_out = np.float64 if out_f64 else np.float32
    mu = pos = mom = None
    if cache_mode == 1:
        mu = np.full((nsave, n), np.nan, dtype=dt_out)
    elif cache_mode == 2:
        pos = np.full((nsave, 3, n), np.nan, dtype=dt_out)
        mom = np.full((nsave, 3, n), np.nan, dtype=dt_out)
    alive_count = np.zeros(nsteps, dtype=np.int64)
    g = grid_struct(grid)
    keys = ["x1", "x2", "x3", "p1", "p2", "p3"]
    for k in keys:
        assert state[k].dtype == np.float64 and state[k].flags.c_contiguous
    assert alive.dtype == np.uint8
    lib().or_push_run(_ptr_array(fl), C.byref(g), *[_p(state[k]) for k in keys], _p(alive), n, dt, nsteps,
                      step_begin, step_count, stride, int(periodic), cache_mode, int(out_f64), _p(mu), _p(pos),
                      _p(mom), _p(alive_count), nthreads)
    if cache_mode == 1:
        return mu, alive_count
    if cache_mode == 2:
        return (pos, mom), alive_count
    return None, alive_count


def reconstruct_mu_f64(pos, mom, bfields, grid, nthreads=0):
    """pos/mom: arrays shaped (nsave, 3, chunk); returns mu shaped (chunk, nsave)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mom = np.ascontiguousarray(mom, dtype=np.float64)
    nsave, _, chunk = pos.shape
    bf = [np.asfortranarray(b, dtype=np.float64) for b in bfields]
    out = np.empty((chunk, nsave), dtype=np.float64)
    g = grid_struct(grid)
    lib().or_reconstruct_mu_f64(_p(pos), _p(mom), chunk, nsave, _ptr_array(bf), C.byref(g), _p(out), nthreads)
    return out


def reconstruct_mu_f32(pos, mom, bfields, grid, nthreads=0):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    mom = np.ascontiguousarray(mom, dtype=np.float32)
    nsave, _, chunk = pos.shape
    bf = [np.asfortranarray(b, dtype=np.float32) for b in bfields]
    lims = np.array([grid.xmin, grid.ymin, grid.zmin, grid.xmax, grid.ymax, grid.zmax, grid.dx, grid.dy, grid.dz],
                    dtype=np.float32)
    out = np.empty((chunk, nsave), dtype=np.float32)
    lib().or_reconstruct_mu_f32(_p(pos), _p(mom), chunk, nsave, _ptr_array(bf), grid.nx, grid.ny, grid.nz, _p(lims),
                                _p(out), nthreads)
    return out


def dmumu_accumulate(mu, lag_steps, edges, acc, injection=False, bin_abs=True, time_fastest=True, nthreads=0):
    """mu: (chunk, nsave) if time_fastest else (nsave, chunk), float32 (or
    float64: a mu chunk at compute precision Float64).
    acc: dict with counts/sum_d/sum_d2 shaped (n_lags, n_bins) and the per-lag
    w_count/w_mean/w_m2/pair_ss/pair_n arrays (add-into)."""
    f64 = np.asarray(mu).dtype == np.float64
    mu = np.ascontiguousarray(mu, dtype=np.float64 if f64 else np.float32)
    if time_fastest:
        chunk, nsave = mu.shape
        sp, ss = nsave, 1
    else:
        nsave, chunk = mu.shape
        sp, ss = 1, chunk
    lags = np.ascontiguousarray(lag_steps, dtype=np.int64)
    e = np.ascontiguousarray(edges, dtype=np.float64)
    fn = lib().or_dmumu_accumulate_f64 if f64 else lib().or_dmumu_accumulate
    fn(_p(mu), chunk, nsave, sp, ss, _p(lags), len(lags), _p(e), len(e) - 1, int(injection), int(bin_abs),
       _p(acc["counts"]), _p(acc["sum_d"]), _p(acc["sum_d2"]), _p(acc["w_count"]), _p(acc["w_mean"]), _p(acc["w_m2"]),
       _p(acc["pair_ss"]), _p(acc["pair_n"]), nthreads)
    return acc


def dpp_accumulate(mom, lag_steps, p0, acc, nthreads=0):
    """mom: (nsave, 3, chunk) float32; acc: dict of per-lag arrays (add-into)."""
    mom = np.ascontiguousarray(mom, dtype=np.float32)
    nsave, _, chunk = mom.shape
    lags = np.ascontiguousarray(lag_steps, dtype=np.int64)
    lib().or_dpp_accumulate(_p(mom), chunk, nsave, _p(lags), len(lags), float(p0), _p(acc["counts"]),
                            _p(acc["sum_dp"]), _p(acc["sum_dp2"]), _p(acc["sum_dpn"]), _p(acc["sum_dpn2"]), nthreads)
    return acc


def energy_snapshots(mom, snap_steps, out, particle_offset=0):
    """mom: (nsave, 3, chunk) float32; out: (n_total, n_snap) float64 (C order,
    i.e. the Julia (n_snap, n_total) array)."""
    mom = np.ascontiguousarray(mom, dtype=np.float32)
    nsave, _, chunk = mom.shape
    snaps = np.ascontiguousarray(snap_steps, dtype=np.int64)
    lib().or_energy_snapshots(_p(mom), chunk, nsave, _p(snaps), len(snaps), particle_offset, _p(out))
    return out


def init_particles(n, seed, energy_GeV, grid, injection="isotropic", mu0=0.0, position_mode="random",
                   position=(0.5, 0.5, 0.5), bfield=None):
    """Counter-stream restatement of the device initialiser; bfield = (Bx, By,
    Bz) C-ordered (nz, ny, nx) FP64 arrays for fixed-mu injection.  Returns
    (state dict, number of particles with zero or non-finite |B|)."""
    out = {k: np.empty(int(n), dtype=np.float64) for k in ("x1", "x2", "x3", "p1", "p2", "p3")}
    pos = np.ascontiguousarray(position, dtype=np.float64)
    fixed_mu = injection.replace("-", "_") == "fixed_mu"
    bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bfield] if fixed_mu else []
    g = grid_struct(grid)
    bad = lib().or_init_particles(int(n), int(seed) & 0xFFFFFFFFFFFFFFFF, float(energy_GeV), int(fixed_mu),
                                  int(position_mode == "random"), float(mu0), _p(pos),
                                  _ptr_array(bs) if bs else None, C.byref(g),
                                  *[_p(out[k]) for k in ("x1", "x2", "x3", "p1", "p2", "p3")])
    return out, int(bad)


DMUMU_ARRAY_KEYS = ("mean_delta", "mean_delta2", "drift_norm", "dmumu_raw_norm", "dmumu_centered_norm",
                    "dmumu_raw_per_s", "dmumu_centered_per_s")
DPP_ARRAY_KEYS = ("mean_delta_p", "mean_delta_p2", "mean_delta_p_norm", "mean_delta_p_norm2", "dpp_raw_per_s",
                  "dpp_centered_per_s", "dpp_raw_norm", "dpp_centered_norm")
TABLE_KEYS = ("tau_s", "tau_norm", "tau_gyroperiods", "delta_mu2_particle_std", "delta_mu2_particle_sem",
              "delta_mu2_pair_mean")


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def dmumu_arrays_full(counts, sum_d, sum_d2, tau_s, tau_norm, min_count_per_cell):
    """compute_dmumu_arrays_full on (n_lags, n_bins) arrays (the Julia
    (n_bins, n_lags) arrays in C order); returns a dict of the seven arrays."""
    counts = _i64(counts)
    n_lags, n_bins = counts.shape
    out = np.empty((7, n_lags, n_bins))
    lib().or_dmumu_arrays_full(_p(counts), _p(_f64(sum_d)), _p(_f64(sum_d2)), _p(_f64(tau_s)), _p(_f64(tau_norm)),
                               n_lags, n_bins, int(min_count_per_cell), _p(out))
    return dict(zip(DMUMU_ARRAY_KEYS, out))


def average_over_tau_full(values, counts, min_count_per_cell):
    counts = _i64(counts)
    n_lags, n_bins = counts.shape
    unw, cw = np.empty(n_bins), np.empty(n_bins)
    lib().or_average_over_tau_full(_p(_f64(values)), _p(counts), n_lags, n_bins, int(min_count_per_cell), _p(unw),
                                   _p(cw))
    return unw, cw


def sem_from_stats(count, m2):
    return float(lib().or_sem_from_stats(int(count), float(m2)))


def output_table(lag_steps, t_s, t_norm, particle_counts, particle_m2s, pair_sum_squares, pair_counts):
    """The computed columns of build_output_dataframe."""
    lags = _i64(lag_steps)
    out = np.empty((6, len(lags)))
    lib().or_output_table(_p(lags), len(lags), _p(_f64(t_s)), _p(_f64(t_norm)), _p(_i64(particle_counts)),
                          _p(_f64(particle_m2s)), _p(_f64(pair_sum_squares)), _p(_i64(pair_counts)), _p(out))
    return dict(zip(TABLE_KEYS, out))


def dpp_arrays(counts, sum_dp, sum_dp2, sum_dpn, sum_dpn2, tau_s, tau_norm):
    counts = _i64(counts)
    out = np.empty((8, len(counts)))
    lib().or_dpp_arrays(_p(counts), _p(_f64(sum_dp)), _p(_f64(sum_dp2)), _p(_f64(sum_dpn)), _p(_f64(sum_dpn2)),
                        _p(_f64(tau_s)), _p(_f64(tau_norm)), len(counts), _p(out))
    return dict(zip(DPP_ARRAY_KEYS, out))
