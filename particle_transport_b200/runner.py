"""Ensemble runners: the Python host's mirror of the reference seams.

run_gpu_ensemble       <- src/phase_space_gpu_runner.jl:476 (phase-space cache)
run_mu_cache_ensemble  <- src/multimode_multienergy_cache_pipeline.jl:1380 (mu cache)

Both keep the reference's host logic (time grid, save stride, initial
state, time axes, alive fraction) and hand the integration loop to
libptb200: pt_push_run with host buffers (the same call the Julia shim
makes), the per-save rows arriving through a callback in place of the
HDF5 hyperslab writer.  DeviceEnsemble / FastEnsemble drive the
device-resident entry points for pipelines that keep everything in HBM.
"""
from __future__ import annotations

import ctypes as C
import math
from types import SimpleNamespace

import numpy as np

from . import _lib
from .fields import F64_STORAGE, FieldLibrary, reference_B0_T
from .particles import energy_to_gamma, energy_to_speed, init_particles
from .time_units import (campaign_time_reference, reference_Omega0, resolve_save_stride,
                         resolve_trajectory_time_grid, sampled_step_indices)

KEYS = ("x1", "x2", "x3", "p1", "p2", "p3")
CACHE = {"none": _lib.PT_CACHE_NONE, "mu": _lib.PT_CACHE_MU, "phase_space": _lib.PT_CACHE_PHASE_SPACE}
PRECISION = {"f64": _lib.PT_PUSH_F64, "f32": _lib.PT_PUSH_F32}


def push_params(dt: float, nsteps: int, stride: int, periodic: bool = True, cache: str = "mu", cache_f64=False,
                precision: str = "f64", steps_per_launch: int = 0, sort_every: int = 0,
                kernel_variant: int = 0, cache_pitch: int = 0) -> _lib.PushParams:
    """pt_push_params.  cache_pitch > 0 selects the time-fastest mu cache of
    the FP32 push: save row r of particle p at p * cache_pitch + (r - row_base)."""
    return _lib.PushParams(float(dt), int(nsteps), int(stride), int(bool(periodic)), CACHE[cache], int(bool(cache_f64)),
                           PRECISION[precision], int(steps_per_launch), int(sort_every), int(kernel_variant),
                           int(cache_pitch))


def n_saves(nsteps: int, stride: int) -> int:
    return (int(nsteps) - 1) // int(stride) + 1


class CacheCollector:
    """In-memory stand-in for the HDF5 cache writers: rows land in
    mu[nsave, n] or positions/momenta[nsave, 3, n] (the on-disk C layouts)."""

    def __init__(self, n: int, nsave: int, cache: str = "mu", f64: bool = False):
        dt = np.float64 if f64 else np.float32
        self.cache = cache
        self.n = n
        if cache == "mu":
            self.mu = np.full((nsave, n), np.nan, dtype=dt)
        else:
            self.positions = np.full((nsave, 3, n), np.nan, dtype=dt)
            self.momenta = np.full((nsave, 3, n), np.nan, dtype=dt)
        self.dtype = dt
        self.rows_seen = 0

    def __call__(self, save_index: int, row: np.ndarray) -> None:
        if self.cache == "mu":
            self.mu[save_index] = row
        else:
            r = row.reshape(6, self.n)
            self.positions[save_index] = r[:3]
            self.momenta[save_index] = r[3:]
        self.rows_seen += 1


def run_push_host(field: FieldLibrary, state: dict, alive: np.ndarray, params: _lib.PushParams, on_save=None):
    """pt_push_run: advance the host state in place over all params.nsteps
    samples; on_save(save_index, row_view) receives every cache row (copy it
    to keep it).  Returns alive_count[nsteps]."""
    n = state["x1"].shape[0]
    for k in KEYS:
        if state[k].dtype != np.float64 or not state[k].flags.c_contiguous or state[k].shape != (n,):
            raise ValueError(f"state[{k}] must be a contiguous float64 array of length {n}")
    if alive.dtype != np.uint8 or alive.shape != (n,):
        raise ValueError("alive must be a uint8 array of length n")
    dtype = np.float64 if params.cache_f64 else np.float32
    err = []

    def _cb(user, save_index, data, nbytes):
        try:
            if on_save is not None:
                row = np.ctypeslib.as_array(C.cast(data, C.POINTER(C.c_double if params.cache_f64 else C.c_float)),
                                            shape=(nbytes // np.dtype(dtype).itemsize,))
                on_save(int(save_index), row)
            return 0
        except Exception as e:  # abort the run, re-raised below
            err.append(e)
            return 1

    cb = _lib.SAVE_FN(_cb)
    alive_count = np.zeros(int(params.nsteps), dtype=np.int64)
    rc = _lib.load().pt_push_run(field.ctx.handle, field.handle, *[_lib.ptr(state[k]) for k in KEYS], _lib.ptr(alive),
                                 n, C.byref(params), cb, None, _lib.ptr(alive_count))
    if err:
        raise err[0]
    _lib.check(rc, "pt_push_run")
    return alive_count


class DeviceEnsemble:
    """FP64 SI state resident on the device (torch tensors) for the FP64 push
    (pt_push_advance_device) over a ref_f64 or brick_f64 field.  CUDA float64
    contiguous state arrays are used as they are, not copied: the push
    advances them in place (over brick_f64 with a sort cadence, through a
    brick-sorted copy that is scattered back after each call)."""

    def __init__(self, field: FieldLibrary, state: dict, alive):
        import torch

        if field.storage not in F64_STORAGE:
            raise ValueError("DeviceEnsemble runs the FP64 push on a ref_f64 or brick_f64 field")
        self.field = field
        self.state = {k: torch.as_tensor(state[k], dtype=torch.float64, device="cuda").contiguous() for k in KEYS}
        self.alive = torch.as_tensor(alive, dtype=torch.uint8, device="cuda").contiguous()
        self.n = int(self.alive.shape[0])

    def advance(self, params, step_begin: int, step_count: int, cache=None, row_base: int = 0, rows: int = 0,
                deaths=None):
        ctx = _lib.torch_context(self.alive)
        _lib.call("pt_push_advance_device", ctx.handle, self.field.handle, *[_lib.ptr(self.state[k]) for k in KEYS],
                  _lib.ptr(self.alive), self.n, C.byref(params), int(step_begin), int(step_count), _lib.ptr(cache),
                  int(row_base), int(rows), _lib.ptr(deaths))


class FastEnsemble:
    """Mixed-precision state (pt_fast_state) for the FP32 push on brick fields."""

    def __init__(self, field: FieldLibrary, state: dict, alive):
        import torch

        if field.storage in F64_STORAGE:
            raise ValueError("FastEnsemble needs an FP32-push brick field (brick_f32 or brick_bf16)")
        self.field = field
        st = {k: torch.as_tensor(state[k], dtype=torch.float64, device="cuda").contiguous() for k in KEYS}
        al = torch.as_tensor(alive, dtype=torch.uint8, device="cuda").contiguous()
        self.n = int(al.shape[0])
        ctx = _lib.torch_context(al)
        out = C.c_void_p()
        _lib.call("pt_fast_state_create", ctx.handle, field.handle, *[_lib.ptr(st[k]) for k in KEYS], _lib.ptr(al),
                  self.n, C.byref(out))
        self.handle = out

    def advance(self, params, step_begin: int, step_count: int, cache=None, row_base: int = 0, rows: int = 0,
                deaths=None):
        ctx = _lib.torch_context(0)
        _lib.call("pt_push_advance_fast", ctx.handle, self.field.handle, self.handle, C.byref(params),
                  int(step_begin), int(step_count), _lib.ptr(cache), int(row_base), int(rows), _lib.ptr(deaths))

    def sort(self):
        """Re-sort the slots by brick (pt_fast_state_sort) on torch's current stream."""
        ctx = _lib.torch_context(0)
        _lib.call("pt_fast_state_sort", ctx.handle, self.handle)

    def export(self):
        import torch

        st = {k: torch.empty(self.n, dtype=torch.float64, device="cuda") for k in KEYS}
        al = torch.empty(self.n, dtype=torch.uint8, device="cuda")
        ctx = _lib.torch_context(al)
        _lib.call("pt_fast_state_export", ctx.handle, self.handle, *[_lib.ptr(st[k]) for k in KEYS], _lib.ptr(al))
        return st, al

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().pt_fast_state_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# reference-shaped drivers
# --------------------------------------------------------------------------
def resolve_total_field_time_reference(fields_si, energy_GeV: float):
    """resolve_total_field_time_reference (src/phase_space_gpu_runner.jl:458-470):
    B0 = mean |B| of the total field, Omega0 = q B0 / (gamma0 m)."""
    B0 = reference_B0_T(fields_si[0], fields_si[1], fields_si[2])
    g0 = energy_to_gamma(energy_GeV)
    from .fields import M_P, Q_E
    return campaign_time_reference(B0, reference_Omega0(B0, g0, Q_E, M_P))


def _time_setup(cfg, field: FieldLibrary, energy_GeV: float, time_reference):
    if time_reference is None:
        raise ValueError("an explicit campaign time reference is required (derived from the total field)")
    Omega0 = float(time_reference.Omega0_reference_s_inv)
    v0 = energy_to_speed(energy_GeV)
    g = field.grid
    min_dx = min(g.dx, g.dy, g.dz)
    tt = resolve_trajectory_time_grid(cfg, Omega0, v0, min_dx)
    st = resolve_save_stride(cfg, tt)
    dt = float(tt.dt_s)
    nsteps = int(tt.n_integration_steps)
    t_s = dt * np.arange(nsteps, dtype=np.float64)
    t_norm = t_s * Omega0
    t_gp = t_norm / (2 * math.pi)
    save_idx = sampled_step_indices(nsteps, st.trajectory_time_stride) - 1
    return SimpleNamespace(Omega0=Omega0, dt=dt, nsteps=nsteps, stride=int(st.trajectory_time_stride),
                           trajectory_time=tt, save_time=st, t_s=t_s, t_norm=t_norm, t_gyroperiods=t_gp,
                           save_indices=save_idx)


def _run(cfg, field, energy_GeV, time_reference, cache, state, fields_host_B):
    ts = _time_setup(cfg, field, energy_GeV, time_reference)
    n = int(cfg["n_particles"])
    if state is None:
        state = init_particles(n, field.grid, energy_GeV, seed=int(cfg.get("seed", 42)),
                               injection_mode=str(cfg.get("injection_mode", "isotropic")),
                               mu0=float(cfg.get("injection_mu0", 0.0)), B=fields_host_B,
                               position_mode=str(cfg.get("injection_position_mode", "random")),
                               position=tuple(cfg.get("injection_position", (0.5, 0.5, 0.5))))
    state = {k: np.ascontiguousarray(state[k], dtype=np.float64).copy() for k in KEYS}
    alive = np.ones(n, dtype=np.uint8)
    boundary = str(cfg.get("boundary", "periodic"))
    if boundary not in ("periodic", "open"):
        raise ValueError(f"Unknown boundary mode: {boundary}. Use open or periodic.")
    precision = str(cfg.get("precision", "f64"))
    f64_out = str(cfg.get("cache_output_precision", "Float32")).lower() in ("float64", "f64")
    params = push_params(ts.dt, ts.nsteps, ts.stride, periodic=boundary == "periodic", cache=cache, cache_f64=f64_out,
                         precision=precision, sort_every=int(cfg.get("sort_every", 0)))
    nsave = n_saves(ts.nsteps, ts.stride)
    col = CacheCollector(n, nsave, cache, f64_out)
    alive_count = run_push_host(field, state, alive, params, col)
    alive_fraction = alive_count.astype(np.float64) / float(n) if n else np.zeros(ts.nsteps)
    return ts, col, state, alive, alive_fraction


def run_mu_cache_ensemble(cfg, field: FieldLibrary, *, energy_GeV: float, time_reference, state=None,
                          fields_host_B=None):
    """Mirror of run_mu_cache_ensemble (pipeline:1380-1535) with the mu cache
    kept in memory (result.mu is the on-disk [nsave][n_particles] array)."""
    ts, col, st, alive, af = _run(cfg, field, energy_GeV, time_reference, "mu", state, fields_host_B)
    si = ts.save_indices
    return SimpleNamespace(mu=col.mu, t_norm=ts.t_norm[si], t_s=ts.t_s[si], t_gyroperiods=ts.t_gyroperiods[si],
                           alive_fraction=af[si], alive_fraction_all=af, nsave=len(si), Omega0=ts.Omega0, dt=ts.dt,
                           trajectory_time=ts.trajectory_time, save_time=ts.save_time,
                           B0=float(time_reference.B0_reference_T), final_state=st, final_alive=alive)


def run_gpu_ensemble(cfg, field: FieldLibrary, *, energy_GeV: float, time_reference, state=None,
                     fields_host_B=None):
    """Mirror of run_gpu_ensemble (src/phase_space_gpu_runner.jl:476-633) with
    the phase-space cache kept in memory (positions/momenta [nsave][3][n])."""
    ts, col, st, alive, af = _run(cfg, field, energy_GeV, time_reference, "phase_space", state, fields_host_B)
    si = ts.save_indices
    return SimpleNamespace(positions=col.positions, momenta=col.momenta, t_norm=ts.t_norm, t_s=ts.t_s,
                           t_gyroperiods=ts.t_gyroperiods, alive_fraction=af, nsave=len(si), Omega0=ts.Omega0,
                           dt=ts.dt, trajectory_time=ts.trajectory_time, save_time=ts.save_time,
                           B0=float(time_reference.B0_reference_T), final_state=st, final_alive=alive)
