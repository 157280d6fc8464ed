"""Time reference, time grid, save stride and lag grid (host logic).

These are the scalar and index inputs that cross the library boundary
(``dt``, ``nsteps``, ``stride``, ``lag_steps``).  In the reference they are
computed on the Julia host by ``src/time_units.jl``; this module restates the
same functions for the Python host so that the parity tests and the bench can
build the kernels' inputs exactly as the reference pipeline would.  The
reference's own test file ``test/runtests.jl`` pins them; the same cases run
in ``tests/test_time_units.py``.

Julia semantics reproduced here: ``round`` is half-to-even, ``argmin`` returns
the first minimum, and float ranges (``range(a, b, length=n)`` and
``a:s:b``) follow Julia's rational-detection rules with correctly rounded
elements (Base ``range_start_stop_length`` / ``(:)(::IEEEFloat...)``).
"""
from __future__ import annotations

import math
from fractions import Fraction
from types import SimpleNamespace

import numpy as np

REFERENCE_GYROPERIOD_NAME = "reference gyroperiod"
TIME_REFERENCE_MODE = "total-field-mean-magnitude"


class TimeUnitsError(ValueError):
    """Raised where the reference calls ``error(...)``."""


# --------------------------------------------------------------------------
# Julia float-range emulation
# --------------------------------------------------------------------------
_M24 = 16777216  # maxintfloat(Float32, Int), used by Base.rat


def _rat(x: float):
    """Base.rat: continued-fraction convergent a/b with Float64(a)/b == x."""
    y = x
    a = d = 1
    b = c = 0
    while abs(y) <= _M24:
        f = int(math.trunc(y))
        y -= f
        a, c = f * a + c, a
        b, d = f * b + d, b
        if max(abs(a), abs(b)) > _M24:
            return c, d
        if b != 0 and float(a) / float(b) == x:
            break
        y = math.inf if y == 0.0 else 1.0 / y
    return a, b


def julia_range_length(start: float, stop: float, length: int) -> np.ndarray:
    """collect(range(start, stop, length=length)) for Float64."""
    start, stop = float(start), float(stop)
    n = int(length)
    if n < 0:
        raise TimeUnitsError("range length must be non-negative")
    if n == 0:
        return np.zeros(0)
    if n == 1:
        return np.array([start])
    if start == stop:
        return np.full(n, start)
    fs, fe = Fraction(start), Fraction(stop)
    sn, sd = _rat(start)
    en, ed = _rat(stop)
    if sd != 0 and ed != 0:
        den = sd * ed // math.gcd(sd, ed)
        m = 2.0 ** 53
        if den != 0 and abs(den * start) <= m and abs(den * stop) <= m:
            sn2 = round(den * start)
            en2 = round(den * stop)
            if sn2 / den == start and en2 / den == stop:
                fs, fe = Fraction(sn2, den), Fraction(en2, den)
    out = np.empty(n)
    for i in range(n):
        out[i] = float((fs * (n - 1 - i) + fe * i) / (n - 1))
    return out


def julia_colon(start: float, step: float, stop: float) -> np.ndarray:
    """collect(start:step:stop) for Float64."""
    start, step, stop = float(start), float(step), float(stop)
    if step == 0.0:
        raise TimeUnitsError("range step cannot be zero")
    stn, std = _rat(step)
    if std != 0 and stn / std == step:
        san, sad = _rat(start)
        son, sod = _rat(stop)
        if sad != 0 and sod != 0 and san / sad == start and son / sod == stop:
            den = sad * std // math.gcd(sad, std)
            m = 2.0 ** 53
            if den != 0 and abs(start * den) <= m and abs(step * den) <= m and den % sad == 0 and den % std == 0:
                start_n = round(start * den)
                step_n = round(step * den)
                length = max(0, (den * son - sod * start_n + step_n * sod) // (step_n * sod))

                def isbetween(a, x, b):
                    return a <= x <= b or b <= x <= a

                if isbetween(start, start + (length - 1) * step, stop + step / 2) and not isbetween(
                        start, start + length * step, stop):
                    return np.array([float(Fraction(start_n + i * step_n, den)) for i in range(length)])
    lf = (stop - start) / step
    if lf < 0:
        length = 0
    elif lf == 0:
        length = 1
    else:
        length = round(lf) + 1
        stop2 = start + (length - 1) * step
        length -= int(start < stop < stop2) + int(start > stop > stop2)
    fs, fst = Fraction(start), Fraction(step)
    return np.array([float(fs + i * fst) for i in range(length)])


def julia_round_int(x: float) -> int:
    """round(Int, x): nearest, ties to even."""
    return int(round(float(x)))


def julia_unique(values):
    seen, out = set(), []
    for v in values:
        if v not in seen:
            seen.add(v)
            out.append(v)
    return out


# --------------------------------------------------------------------------
# src/time_units.jl:6-24
# --------------------------------------------------------------------------
def reference_gyroperiod_s(Omega0: float) -> float:
    return 2.0 * math.pi / float(Omega0)


def gyroperiods_to_tOmega0(n: float) -> float:
    return 2.0 * math.pi * float(n)


def tOmega0_to_gyroperiods(t: float) -> float:
    return float(t) / (2.0 * math.pi)


def gyroperiods_to_seconds(n: float, Omega0: float) -> float:
    return gyroperiods_to_tOmega0(n) / float(Omega0)


def seconds_to_gyroperiods(t_s: float, Omega0: float) -> float:
    return float(t_s) * float(Omega0) / (2.0 * math.pi)


def assert_finite_positive(value, key_name: str) -> float:
    v = float(value)
    if not (math.isfinite(v) and v > 0.0):
        raise TimeUnitsError(key_name + " must be finite and positive.")
    return v


def reference_B0_T(Bx, By, Bz) -> float:
    """mean(sqrt.(Bx.^2 .+ By.^2 .+ Bz.^2)) (src/time_units.jl:18-20)."""
    Bx, By, Bz = (np.asarray(a, dtype=np.float64) for a in (Bx, By, Bz))
    return float(np.mean(np.sqrt(Bx * Bx + By * By + Bz * Bz)))


def reference_Omega0(B0_T: float, gamma0: float, charge_C: float, mass_kg: float) -> float:
    return float(charge_C) * float(B0_T) / (float(gamma0) * float(mass_kg))


def campaign_time_reference(B0_reference_T, Omega0_reference_s_inv, source_mode="total", source_path="",
                            source_identity=None, field_subset="nothing"):
    Om = float(Omega0_reference_s_inv)
    return SimpleNamespace(
        B0_reference_T=float(B0_reference_T), Omega0_reference_s_inv=Om,
        reference_gyroperiod_s=reference_gyroperiod_s(Om), time_reference_mode=TIME_REFERENCE_MODE,
        time_reference_name=REFERENCE_GYROPERIOD_NAME, time_reference_source_mode=str(source_mode),
        time_reference_source_path=str(source_path),
        time_reference_source_identity=str(source_path if source_identity is None else source_identity),
        time_reference_field_subset=str(field_subset))


def require_explicit_campaign_time_reference(trajectory_mode, time_reference, caller="trajectory runner"):
    if time_reference is not None:
        return time_reference
    raise TimeUnitsError("Trajectory mode '" + str(trajectory_mode).lower() +
                         "' requires an explicit campaign time reference derived from the total-field dataset. The "
                         + caller + " must not derive B0_reference from the trajectory field.")


# --------------------------------------------------------------------------
# src/time_units.jl:50-140
# --------------------------------------------------------------------------
def resolve_eta_requested(cfg):
    if cfg.get("integration_steps_per_gyroperiod") is not None:
        spg = assert_finite_positive(cfg["integration_steps_per_gyroperiod"], "integration_steps_per_gyroperiod")
        return 2.0 * math.pi / spg, spg, "gyroperiods"
    eta = assert_finite_positive(cfg["eta"], "eta")
    return eta, 2.0 * math.pi / eta, "legacy_eta"


def requested_duration_gyroperiods(cfg):
    if cfg.get("trajectory_duration_gyroperiods") is not None:
        return assert_finite_positive(cfg["trajectory_duration_gyroperiods"],
                                      "trajectory_duration_gyroperiods"), "gyroperiods"
    t = assert_finite_positive(cfg["tOmega0_max"], "tOmega0_max")
    return tOmega0_to_gyroperiods(t), "legacy_tOmega0"


def resolve_trajectory_time_grid(cfg, Omega0, v0, min_dx):
    eta, req_spg, integration_source = resolve_eta_requested(cfg)
    dt_gyro_s = eta / float(Omega0)
    dt_cfl_s = math.inf
    limited = "gyro"
    dt_s = dt_gyro_s
    if bool(cfg.get("use_cfl", False)):
        cfl = assert_finite_positive(cfg["cfl"], "cfl")
        dt_cfl_s = cfl * float(min_dx) / float(v0)
        if dt_cfl_s < dt_s:
            dt_s = dt_cfl_s
            limited = "cfl"
    req_gp, duration_source = requested_duration_gyroperiods(cfg)
    req_s = gyroperiods_to_seconds(req_gp, Omega0)
    n = int(math.floor(req_s / dt_s)) + 1
    if not n > 1:
        raise TimeUnitsError("Trajectory duration resolves to fewer than two integration samples.")
    actual_s = (n - 1) * dt_s
    actual_t = actual_s * float(Omega0)
    return SimpleNamespace(
        eta_requested=eta, integration_source=integration_source,
        requested_integration_steps_per_gyroperiod=req_spg,
        actual_integration_steps_per_gyroperiod=reference_gyroperiod_s(Omega0) / dt_s,
        dt_s=dt_s, dt_tOmega0=dt_s * float(Omega0), dt_gyroperiods=seconds_to_gyroperiods(dt_s, Omega0),
        dt_gyro_s=dt_gyro_s, dt_cfl_s=dt_cfl_s, timestep_limited_by=limited, duration_source=duration_source,
        requested_trajectory_duration_gyroperiods=req_gp, requested_trajectory_duration_s=req_s,
        actual_trajectory_duration_gyroperiods=tOmega0_to_gyroperiods(actual_t),
        actual_trajectory_duration_tOmega0=actual_t, actual_trajectory_duration_s=actual_s,
        n_integration_steps=n)


def resolve_save_stride(cfg, tt):
    if cfg.get("trajectory_save_interval_gyroperiods") is not None:
        req = assert_finite_positive(cfg["trajectory_save_interval_gyroperiods"],
                                     "trajectory_save_interval_gyroperiods")
        stride = max(1, julia_round_int(req / tt.dt_gyroperiods))
        return SimpleNamespace(trajectory_time_stride=stride, save_interval_source="gyroperiods",
                               requested_trajectory_save_interval_gyroperiods=req,
                               actual_trajectory_save_interval_gyroperiods=stride * tt.dt_gyroperiods,
                               actual_trajectory_save_interval_s=stride * tt.dt_s)
    stride = int(cfg["trajectory_time_stride"])
    if stride < 1:
        raise TimeUnitsError("trajectory_time_stride must be >= 1")
    gp = stride * tt.dt_gyroperiods
    return SimpleNamespace(trajectory_time_stride=stride, save_interval_source="legacy_steps",
                           requested_trajectory_save_interval_gyroperiods=gp,
                           actual_trajectory_save_interval_gyroperiods=gp,
                           actual_trajectory_save_interval_s=stride * tt.dt_s)


def sampled_step_indices(nsteps: int, stride: int) -> np.ndarray:
    """1-based save steps 1:stride:nsteps (src/phase_space_gpu_runner.jl:393-396)."""
    if stride < 1:
        raise TimeUnitsError("trajectory_time_stride must be >= 1")
    return np.arange(1, nsteps + 1, stride, dtype=np.int64)


def t_gyroperiods_from_axes(t_s, t_norm, Omega0=None):
    if t_norm is not None:
        return np.asarray(t_norm, dtype=np.float64) / (2.0 * math.pi)
    if Omega0 is not None:
        return np.asarray(t_s, dtype=np.float64) * float(Omega0) / (2.0 * math.pi)
    raise TimeUnitsError("Cannot resolve t_gyroperiods without t_norm or Omega0.")


def _isapprox(a, b, rtol, atol):
    return np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))


def validate_time_axes_result(t_s, t_norm, t_gp, key_name="time axes", require_uniform=True, rtol=1.0e-10,
                              atol=1.0e-12):
    t_s, t_norm, t_gp = (np.asarray(a, dtype=np.float64) for a in (t_s, t_norm, t_gp))
    n = len(t_s)
    if len(t_norm) != n or len(t_gp) != n or n <= 1:
        return SimpleNamespace(valid=False, reason="time_length_mismatch", message=key_name + ": length mismatch")
    if not (np.all(np.isfinite(t_s)) and np.all(np.isfinite(t_norm)) and np.all(np.isfinite(t_gp))):
        return SimpleNamespace(valid=False, reason="inconsistent_time_units", message=key_name + ": non-finite")
    if not (np.all(np.diff(t_s) > 0) and np.all(np.diff(t_norm) > 0) and np.all(np.diff(t_gp) > 0)):
        return SimpleNamespace(valid=False, reason="inconsistent_time_units",
                               message=key_name + ": time axes must be strictly increasing.")
    if not np.all(_isapprox(t_norm / (2.0 * math.pi), t_gp, rtol, atol)):
        return SimpleNamespace(valid=False, reason="inconsistent_time_units",
                               message=key_name + ": t_norm and t_gyroperiods are inconsistent.")
    if require_uniform:
        iv = np.diff(t_gp)
        if not np.all(np.abs(iv - iv[0]) <= atol + rtol * abs(iv[0])):
            return SimpleNamespace(valid=False, reason="nonuniform_time_axis",
                                   message=key_name + ": nonuniform primary time axis")
    return SimpleNamespace(valid=True, reason="ok", message="ok")


def validate_time_axes(t_s, t_norm, t_gp, key_name="time axes", require_uniform=False, rtol=1.0e-10,
                       atol=1.0e-12) -> int:
    r = validate_time_axes_result(t_s, t_norm, t_gp, key_name, require_uniform, rtol, atol)
    if not r.valid:
        raise TimeUnitsError(r.message)
    return len(t_s)


# --------------------------------------------------------------------------
# src/time_units.jl:212-459 (lag grid)
# --------------------------------------------------------------------------
def _norm_sym(value) -> str:
    return str(value).strip().lower().replace("-", "_")


def normalize_lag_boundary_policy(value) -> str:
    p = _norm_sym(value)
    if p not in ("strict", "nearest"):
        raise TimeUnitsError("lag_boundary_policy must be strict or nearest.")
    return p


def normalize_lag_range_policy(value) -> str:
    p = _norm_sym(value)
    if p not in ("fixed", "first_cache_step", "common_cache_intersection"):
        raise TimeUnitsError("lag_range_policy must be fixed, first-cache-step, or common-cache-intersection.")
    return p


def normalize_lag_common_scope(value) -> str:
    p = _norm_sym(value)
    if p not in ("campaign", "reference_group"):
        raise TimeUnitsError("lag_common_scope must be campaign or reference-group.")
    return p


def lag_cache_summary(t_gp):
    t_gp = np.asarray(t_gp, dtype=np.float64)
    if len(t_gp) <= 1:
        raise TimeUnitsError("Need at least two cached samples to resolve lags.")
    offsets = t_gp[1:] - t_gp[0]
    cmin, cmax = float(offsets[0]), float(offsets[-1])
    interval = cmin if len(offsets) == 1 else float(np.diff(t_gp)[0])
    tol = 1.0e-12 + 1.0e-10 * max(abs(interval), abs(cmax), 1.0)
    return SimpleNamespace(offsets=offsets, cache_min_gp=cmin, cache_max_gp=cmax, cache_save_interval_gp=interval,
                           tolerance=tol)


def nearest_positive_cache_lag(requested_gp, cache):
    r = float(requested_gp)
    if not (math.isfinite(r) and r > 0.0):
        raise TimeUnitsError("Lag boundary values must be finite and positive reference gyroperiods.")
    loc = int(np.argmin(np.abs(cache.offsets - r)))
    step = loc + 1
    actual = float(cache.offsets[loc])
    return step, actual, abs(actual - r)


def resolve_one_lag_boundary(requested_gp, cache, cfg, boundary_name):
    policy = normalize_lag_boundary_policy(cfg.get("lag_boundary_policy", "strict"))
    r = float(requested_gp)
    _, actual, err = nearest_positive_cache_lag(r, cache)
    if policy == "strict":
        if boundary_name == "minimum":
            if not r >= cache.cache_min_gp - cache.tolerance:
                raise TimeUnitsError(f"Requested lag range minimum {r} is outside representable cache range.")
        else:
            if not r <= cache.cache_max_gp + cache.tolerance:
                raise TimeUnitsError(f"Requested lag range maximum {r} is outside representable cache range.")
        return r
    max_rel = float(cfg.get("max_lag_boundary_relative_error", 0.0))
    if not (math.isfinite(max_rel) and max_rel >= 0.0):
        raise TimeUnitsError("max_lag_boundary_relative_error must be finite and nonnegative.")
    if not err <= 0.5 * cache.cache_save_interval_gp + cache.tolerance:
        raise TimeUnitsError(f"Requested lag boundary {r} is too far from the nearest cached lag {actual}.")
    rel = err / max(abs(r), np.finfo(np.float64).eps)
    if not rel <= max_rel + cache.tolerance:
        raise TimeUnitsError(f"Requested lag boundary {r} maps to {actual} with relative error {rel}.")
    return actual


def configured_lag_bounds(cfg, cache):
    cmin = cfg.get("lag_min_gyroperiods")
    cmax = cfg.get("lag_max_gyroperiods")
    policy = normalize_lag_range_policy(cfg.get("lag_range_policy", "fixed"))
    if policy == "first_cache_step":
        if cmin is not None:
            raise TimeUnitsError("lag_range_policy = first-cache-step requires lag_min_gyroperiods to be absent.")
        lo = cache.cache_min_gp
        hi = cache.cache_max_gp if cmax is None else assert_finite_positive(cmax, "lag_max_gyroperiods")
        return cmin, cmax, lo, hi, math.nan, math.nan
    lo = cache.cache_min_gp if cmin is None else assert_finite_positive(cmin, "lag_min_gyroperiods")
    hi = cache.cache_max_gp if cmax is None else assert_finite_positive(cmax, "lag_max_gyroperiods")
    if policy == "common_cache_intersection":
        cm = float(cfg.get("common_cache_lag_min_gyroperiods", math.nan))
        cM = float(cfg.get("common_cache_lag_max_gyroperiods", math.nan))
        if not (math.isfinite(cm) and math.isfinite(cM)):
            raise TimeUnitsError("lag_range_policy = common-cache-intersection requires a preflight common range.")
        if not cM > cm:
            raise TimeUnitsError("Common cache lag intersection is empty.")
        lo, hi = max(lo, cm), min(hi, cM)
        if not hi > lo:
            raise TimeUnitsError("Effective lag range is empty after applying common-cache-intersection.")
        return cmin, cmax, lo, hi, cm, cM
    return cmin, cmax, lo, hi, math.nan, math.nan


def build_requested_lags_from_bounds(cfg, lo, hi):
    mode = _norm_sym(cfg["lag_mode"])
    lo, hi = float(lo), float(hi)
    if not hi >= lo:
        raise TimeUnitsError("lag_max_gyroperiods must be >= lag_min_gyroperiods after policy resolution.")
    if mode == "uniform_samples":
        n = int(cfg["n_lag_samples"])
        if n <= 0:
            raise TimeUnitsError("n_lag_samples must be positive.")
        return julia_range_length(lo, hi, n), "gyroperiods"
    if mode == "stride":
        st = assert_finite_positive(cfg["lag_stride_gyroperiods"], "lag_stride_gyroperiods")
        return julia_colon(lo, st, hi + st * 1.0e-12), "gyroperiods"
    raise TimeUnitsError(f"Unknown lag_mode: {mode}")


def requested_lag_grid_gyroperiods(cfg, max_cache_lag_step, t_gp):
    mode = _norm_sym(cfg["lag_mode"])
    t_gp = np.asarray(t_gp, dtype=np.float64)
    if cfg.get("lag_min_gyroperiods") is not None:
        lo = assert_finite_positive(cfg["lag_min_gyroperiods"], "lag_min_gyroperiods")
        hi = (assert_finite_positive(cfg["lag_max_gyroperiods"], "lag_max_gyroperiods")
              if cfg.get("lag_max_gyroperiods") is not None else float(t_gp[max_cache_lag_step] - t_gp[0]))
        if not hi >= lo:
            raise TimeUnitsError("lag_max_gyroperiods must be >= lag_min_gyroperiods.")
        return build_requested_lags_from_bounds(cfg, lo, hi)
    min_step = max(1, int(cfg.get("min_lag_steps", 1)))
    max_step = (max_cache_lag_step if cfg.get("max_lag_steps") is None
                else min(int(cfg["max_lag_steps"]), max_cache_lag_step))
    if not max_step >= min_step:
        raise TimeUnitsError("No lag steps selected.")
    if mode == "uniform_samples":
        n = min(int(cfg["n_lag_samples"]), max_step - min_step + 1)
        steps = julia_unique([julia_round_int(v) for v in julia_range_length(min_step, max_step, n)])
    elif mode == "stride":
        st = int(cfg["lag_step_stride"])
        if st < 1:
            raise TimeUnitsError("lag_step_stride must be >= 1")
        steps = list(range(min_step, max_step + 1, st))
    else:
        raise TimeUnitsError(f"Unknown lag_mode: {mode}")
    return np.array([float(t_gp[s] - t_gp[0]) for s in steps]), "legacy_steps"


def resolve_lag_grid(cfg, t_gp, min_unique_lags=2):
    t_gp = np.asarray(t_gp, dtype=np.float64)
    nsteps = len(t_gp)
    if nsteps <= 1:
        raise TimeUnitsError("Need at least two cached samples to resolve lags.")
    max_cache_lag_step = nsteps - 1
    cache = lag_cache_summary(t_gp)
    range_policy = normalize_lag_range_policy(cfg.get("lag_range_policy", "fixed"))
    boundary_policy = normalize_lag_boundary_policy(cfg.get("lag_boundary_policy", "strict"))
    rel = float(cfg.get("max_lag_boundary_relative_error", 0.0))
    if not (math.isfinite(rel) and rel >= 0.0):
        raise TimeUnitsError("max_lag_boundary_relative_error must be finite and nonnegative.")
    cmin = cfg.get("lag_min_gyroperiods")
    cmax = cfg.get("lag_max_gyroperiods")
    common_min = common_max = eff_min = eff_max = math.nan
    if range_policy == "fixed" and cmin is None:
        requested, source = requested_lag_grid_gyroperiods(cfg, max_cache_lag_step, t_gp)
    else:
        cmin, cmax, rmin, rmax, common_min, common_max = configured_lag_bounds(cfg, cache)
        if range_policy == "common_cache_intersection":
            eff_min, eff_max = rmin, rmax
        else:
            eff_min = resolve_one_lag_boundary(rmin, cache, cfg, "minimum")
            eff_max = resolve_one_lag_boundary(rmax, cache, cfg, "maximum")
        if not eff_max > eff_min:
            raise TimeUnitsError("Effective lag range resolves to zero width after applying lag boundary policy.")
        requested, source = build_requested_lags_from_bounds(cfg, eff_min, eff_max)
    requested = np.asarray(requested, dtype=np.float64)
    if len(requested) == 0:
        raise TimeUnitsError("No requested lag values were generated.")
    rq_min, rq_max = float(np.min(requested)), float(np.max(requested))
    tol = cache.tolerance
    if boundary_policy == "strict" and (rq_min < cache.cache_min_gp - tol or rq_max > cache.cache_max_gp + tol):
        raise TimeUnitsError(f"Requested lag range [{rq_min}, {rq_max}] is outside representable cache range.")
    lag_steps, req_u, actual, errs, seen = [], [], [], [], set()
    for r in requested:
        if not (math.isfinite(r) and r > 0.0):
            raise TimeUnitsError("Requested lag values must be finite and positive reference gyroperiods.")
        loc = int(np.argmin(np.abs(cache.offsets - r)))
        step = loc + 1
        if not 1 <= step <= max_cache_lag_step:
            raise TimeUnitsError("Resolved lag step is outside the cached trajectory.")
        err = abs(float(cache.offsets[loc]) - float(r))
        if not err <= 0.5 * cache.cache_save_interval_gp + tol:
            raise TimeUnitsError("Internal lag mapping inconsistency.")
        if step not in seen:
            seen.add(step)
            lag_steps.append(step)
            req_u.append(float(r))
            actual.append(float(t_gp[step] - t_gp[0]))
            errs.append(err)
    if len(lag_steps) < min_unique_lags:
        raise TimeUnitsError(f"Lag grid resolved to fewer than {min_unique_lags} unique positive cached-step offsets.")
    order = np.argsort(np.array(lag_steps), kind="stable")
    lag_steps = np.array(lag_steps, dtype=np.int64)[order]
    req_u = np.array(req_u)[order]
    actual = np.array(actual)[order]
    errs = np.array(errs)[order]
    eps = np.finfo(np.float64).eps
    return SimpleNamespace(
        lag_steps=lag_steps, requested_tau_gyroperiods=req_u, common_requested_tau_gyroperiods=requested,
        tau_gyroperiods=actual, tau_norm=np.array([gyroperiods_to_tOmega0(a) for a in actual]),
        lag_mapping_error_gyroperiods=errs,
        max_lag_mapping_error_gyroperiods=float(errs.max()) if len(errs) else 0.0,
        max_lag_mapping_relative_error=float((errs / np.maximum(np.abs(req_u), eps)).max()) if len(errs) else 0.0,
        requested_lag_count=len(requested), unique_lag_count=len(lag_steps),
        duplicate_lag_mapping_count=len(requested) - len(lag_steps),
        duplicate_lag_mapping_fraction=(len(requested) - len(lag_steps)) / len(requested),
        cache_lag_min_gyroperiods=cache.cache_min_gp, cache_lag_max_gyroperiods=cache.cache_max_gp,
        cache_save_interval_gyroperiods=cache.cache_save_interval_gp, lag_range_policy=range_policy,
        lag_boundary_policy=boundary_policy, max_lag_boundary_relative_error=rel,
        configured_lag_min_gyroperiods=math.nan if cmin is None else float(cmin),
        configured_lag_max_gyroperiods=math.nan if cmax is None else float(cmax),
        common_cache_lag_min_gyroperiods=common_min, common_cache_lag_max_gyroperiods=common_max,
        effective_lag_min_gyroperiods=eff_min if math.isfinite(eff_min) else rq_min,
        effective_lag_max_gyroperiods=eff_max if math.isfinite(eff_max) else rq_max,
        lag_comparison_group_identity=str(cfg.get("lag_comparison_group_identity", "not-applicable")),
        lag_common_scope=normalize_lag_common_scope(cfg.get("lag_common_scope", "campaign")),
        lag_source=source)


def log_spaced_lag_steps(max_step: int, n: int, min_step: int = 1) -> np.ndarray:
    """Explicit log-spaced lag list (rounded half-even, de-duplicated, sorted).

    The reference has no log lag mode; runs that want log-spaced lags pass the
    explicit integer list across the boundary (the kernels take any list)."""
    vals = np.exp(np.linspace(math.log(min_step), math.log(max_step), n))
    return np.array(sorted(julia_unique([julia_round_int(v) for v in vals])), dtype=np.int64)


def selected_energy_snapshot_indices(nsteps: int, count: int) -> np.ndarray:
    """unique(round.(Int, range(1, nsteps, length=k))) as 1-based indices
    (src/compute_dpp_full.jl:242-245)."""
    k = min(max(1, int(count)), int(nsteps))
    return np.array(julia_unique([julia_round_int(v) for v in julia_range_length(1.0, float(nsteps), k)]),
                    dtype=np.int64)


def build_mu_edges_full(mu_min: float, mu_max: float, n_bins: int, bin_abs: bool = True):
    """edges = range(mu_min, mu_max, length=n_bins+1); centers = midpoints
    (src/compute_delta_mu2_dmumu_full.jl:289-302)."""
    mu_min, mu_max, n_bins = float(mu_min), float(mu_max), int(n_bins)
    if not mu_min < mu_max:
        raise TimeUnitsError("mu_min must be less than mu_max.")
    if n_bins <= 0:
        raise TimeUnitsError("n_mu_bins must be positive.")
    if bin_abs and (mu_min < 0.0 or mu_max > 1.0):
        raise TimeUnitsError("mu range must lie in [0, 1] when mu_bin_abs is true.")
    edges = julia_range_length(mu_min, mu_max, n_bins + 1)
    centers = 0.5 * (edges[:-1] + edges[1:])
    return edges, centers
