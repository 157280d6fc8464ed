"""The reference's own test cases (test/runtests.jl) against the host restatement
of src/time_units.jl.  These are the only golden values the reference ships;
they pin the dt / nsteps / stride / lag_steps inputs the kernels consume."""
import math

import numpy as np
import pytest

from particle_transport_b200 import time_units as tu


def approx(a, b):
    return np.allclose(a, b, rtol=math.sqrt(np.finfo(float).eps), atol=0)


def test_gyroperiod_conversions():  # runtests.jl:6-13
    Om = 4.0
    assert approx(tu.reference_gyroperiod_s(Om), math.pi / 2)
    assert approx(tu.gyroperiods_to_tOmega0(1.0), 2 * math.pi)
    assert approx(tu.tOmega0_to_gyroperiods(2 * math.pi), 1.0)
    assert approx(tu.gyroperiods_to_seconds(3.0, Om), 3.0 * 2 * math.pi / Om)
    assert approx(tu.seconds_to_gyroperiods(tu.gyroperiods_to_seconds(2.5, Om), Om), 2.5)


def _tcfg(**kw):
    cfg = dict(integration_steps_per_gyroperiod=64.0, eta=0.1, trajectory_duration_gyroperiods=10.0,
               tOmega0_max=100.0, use_cfl=False, cfl=0.2, trajectory_save_interval_gyroperiods=0.25,
               trajectory_time_stride=1)
    cfg.update(kw)
    return cfg


def test_trajectory_time_resolution():  # runtests.jl:15-42
    cfg = _tcfg()
    r = tu.resolve_trajectory_time_grid(cfg, 2.0, 1.0, 1.0)
    assert approx(r.eta_requested, 2 * math.pi / 64)
    assert approx(r.requested_integration_steps_per_gyroperiod, 64.0)
    assert approx(r.actual_integration_steps_per_gyroperiod, 64.0)
    assert r.timestep_limited_by == "gyro"
    assert r.actual_trajectory_duration_gyroperiods <= 10.0
    st = tu.resolve_save_stride(cfg, r)
    assert st.trajectory_time_stride == 16
    assert approx(st.actual_trajectory_save_interval_gyroperiods, 0.25)
    c2 = _tcfg(use_cfl=True)
    r2 = tu.resolve_trajectory_time_grid(c2, 2.0, 100.0, 1.0)
    assert r2.timestep_limited_by == "cfl"
    assert r2.actual_integration_steps_per_gyroperiod > r2.requested_integration_steps_per_gyroperiod


def test_legacy_equivalence():  # runtests.jl:44-61
    cfg = _tcfg(integration_steps_per_gyroperiod=None, trajectory_duration_gyroperiods=None, tOmega0_max=20.0,
                trajectory_save_interval_gyroperiods=None, trajectory_time_stride=3)
    r = tu.resolve_trajectory_time_grid(cfg, 5.0, 1.0, 1.0)
    assert approx(r.eta_requested, 0.1)
    assert approx(r.requested_trajectory_duration_gyroperiods, 20.0 / (2 * math.pi))
    assert r.n_integration_steps == int(math.floor((20.0 / 5.0) / (0.1 / 5.0))) + 1
    assert tu.resolve_save_stride(cfg, r).trajectory_time_stride == 3


def _lcfg(**kw):
    cfg = dict(lag_mode="uniform_samples", lag_range_policy="fixed", lag_boundary_policy="strict",
               max_lag_boundary_relative_error=0.0, lag_min_gyroperiods=0.25, lag_max_gyroperiods=1.1,
               lag_stride_gyroperiods=None, min_lag_steps=1, max_lag_steps=None, lag_step_stride=1, n_lag_samples=5)
    cfg.update(kw)
    return cfg


def test_lag_mapping():  # runtests.jl:63-113
    t_gp = tu.julia_colon(0.0, 0.25, 5.0)
    g = tu.resolve_lag_grid(_lcfg(), t_gp)
    assert np.all(g.lag_steps >= 1)
    assert np.all(np.diff(g.lag_steps) > 0)
    assert np.all(g.tau_gyroperiods > 0)
    assert approx(g.tau_norm, 2 * math.pi * g.tau_gyroperiods)
    sg = tu.resolve_lag_grid(_lcfg(lag_mode="stride", lag_min_gyroperiods=0.25, lag_max_gyroperiods=1.0,
                                   lag_stride_gyroperiods=0.25), t_gp)
    assert list(sg.lag_steps) == [1, 2, 3, 4]
    assert approx(sg.tau_gyroperiods, [0.25, 0.5, 0.75, 1.0])
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(_lcfg(lag_min_gyroperiods=0.01, lag_max_gyroperiods=0.5), t_gp)
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(_lcfg(lag_min_gyroperiods=0.5, lag_max_gyroperiods=8.0), t_gp)
    d = tu.resolve_lag_grid(_lcfg(lag_min_gyroperiods=0.26, lag_max_gyroperiods=0.49, n_lag_samples=4), t_gp,
                            min_unique_lags=1)
    assert d.requested_lag_count == 4
    assert d.unique_lag_count < d.requested_lag_count
    assert d.duplicate_lag_mapping_count > 0
    assert d.duplicate_lag_mapping_fraction > 0.0


def test_lag_boundary_policies():  # runtests.jl:115-157
    step = 0.016087419809019843
    t_gp = tu.julia_colon(0.0, step, 5.984520168955382)
    cfg = _lcfg(max_lag_boundary_relative_error=0.05, lag_min_gyroperiods=0.015625, lag_max_gyroperiods=5.0,
                n_lag_samples=40)
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(cfg, t_gp)
    near = dict(cfg, lag_boundary_policy="nearest")
    g = tu.resolve_lag_grid(near, t_gp)
    assert approx(g.tau_gyroperiods[0], step)
    assert approx(g.requested_tau_gyroperiods[0], step)
    assert approx(g.effective_lag_min_gyroperiods, step)
    assert g.lag_boundary_policy == "nearest"
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(dict(near, max_lag_boundary_relative_error=0.01), t_gp)
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(dict(near, lag_min_gyroperiods=0.001), t_gp)
    mx = dict(near, lag_min_gyroperiods=step, lag_max_gyroperiods=t_gp[-1] + 0.25 * step)
    assert approx(tu.resolve_lag_grid(mx, t_gp).tau_gyroperiods[-1], t_gp[-1])
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(dict(mx, lag_max_gyroperiods=t_gp[-1] + 2.0 * step), t_gp)


def test_lag_range_policies():  # runtests.jl:159-208
    a = tu.julia_colon(0.0, 0.25, 5.0)
    b = tu.julia_colon(0.0, 0.30, 4.8)
    cfg = _lcfg(lag_range_policy="first_cache_step", lag_min_gyroperiods=None, lag_max_gyroperiods=1.0,
                n_lag_samples=4)
    assert approx(tu.resolve_lag_grid(cfg, b).effective_lag_min_gyroperiods, 0.30)
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(dict(cfg, lag_min_gyroperiods=0.25), b)
    common = dict(cfg, lag_range_policy="common_cache_intersection", lag_min_gyroperiods=0.25, lag_max_gyroperiods=5.0,
                  common_cache_lag_min_gyroperiods=max(tu.lag_cache_summary(a).cache_min_gp,
                                                       tu.lag_cache_summary(b).cache_min_gp),
                  common_cache_lag_max_gyroperiods=min(tu.lag_cache_summary(a).cache_max_gp,
                                                       tu.lag_cache_summary(b).cache_max_gp),
                  lag_comparison_group_identity="test-group")
    g = tu.resolve_lag_grid(common, a)
    assert approx(g.effective_lag_min_gyroperiods, 0.30)
    assert approx(g.effective_lag_max_gyroperiods, 4.8)
    assert g.lag_comparison_group_identity == "test-group"
    assert approx(g.common_requested_tau_gyroperiods[0], 0.30)
    assert tu.normalize_lag_common_scope("reference-group") == "reference_group"
    assert tu.normalize_lag_common_scope("campaign") == "campaign"
    with pytest.raises(tu.TimeUnitsError):
        tu.normalize_lag_common_scope("mode")
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(dict(common, common_cache_lag_min_gyroperiods=5.0, common_cache_lag_max_gyroperiods=4.0), a)
    with pytest.raises(tu.TimeUnitsError):
        tu.resolve_lag_grid(dict(common, n_lag_samples=20, lag_min_gyroperiods=0.31, lag_max_gyroperiods=0.37), a)


def test_time_axes():  # runtests.jl:210-219
    t_s = np.array([0.0, 0.5, 1.0])
    t_norm = t_s * 4.0
    t_gp = tu.t_gyroperiods_from_axes(t_s, t_norm)
    assert tu.validate_time_axes(t_s, t_norm, t_gp) == 3
    assert tu.validate_time_axes(t_s, t_norm, t_gp, require_uniform=True) == 3
    with pytest.raises(tu.TimeUnitsError):
        tu.validate_time_axes([0.0, 0.5, 0.4], t_norm, t_gp)
    with pytest.raises(tu.TimeUnitsError):
        tu.validate_time_axes([0.0, 0.5, 1.2], [0.0, 2.0, 4.8], [0.0, 2.0 / (2 * math.pi), 4.8 / (2 * math.pi)],
                              require_uniform=True)


def test_shared_reference_metadata():  # runtests.jl:221-232
    B = [np.full((2, 2, 2), 3.0), np.full((2, 2, 2), 4.0), np.zeros((2, 2, 2))]
    assert approx(tu.reference_B0_T(*B), 5.0)
    ref = tu.campaign_time_reference(5.0, 2.0, source_mode="total", source_path="total.h5")
    assert approx(ref.B0_reference_T, 5.0)
    assert approx(ref.Omega0_reference_s_inv, 2.0)
    assert ref.time_reference_source_mode == "total"
    assert ref.time_reference_source_path == "total.h5"
    assert approx(ref.reference_gyroperiod_s, math.pi)


def test_direct_runner_reference_guard():  # runtests.jl:234-240
    ref = tu.campaign_time_reference(5.0, 2.0, source_mode="total", source_path="total.h5")
    assert tu.require_explicit_campaign_time_reference("total", ref, caller="test") is ref
    for mode in ("alfven", "fast", "slow", "unknown", "total"):
        with pytest.raises(tu.TimeUnitsError):
            tu.require_explicit_campaign_time_reference(mode, None, caller="test")


def test_structured_time_validation():  # runtests.jl:242-259
    t_gp = np.array([0.0, 0.25, 0.5, 0.75, 0.85])
    t_norm = 2.0 * math.pi * t_gp
    t_s = t_norm / 4.0
    r = tu.validate_time_axes_result(t_s, t_norm, t_gp, require_uniform=True)
    assert not r.valid and r.reason == "nonuniform_time_axis"
    bad = t_norm.copy()
    bad[-1] += 0.1
    r = tu.validate_time_axes_result(t_s, bad, t_gp, require_uniform=True)
    assert not r.valid and r.reason == "inconsistent_time_units"
    r = tu.validate_time_axes_result(t_s[:-1], t_norm, t_gp, require_uniform=True)
    assert not r.valid and r.reason == "time_length_mismatch"


def test_julia_ranges():
    # range(0, 1, length=21) edges are i/20 correctly rounded
    e = tu.julia_range_length(0.0, 1.0, 21)
    assert all(e[i] == i / 20 for i in range(21))
    # 0.0:0.25:5.0 -> 21 exact quarters
    r = tu.julia_colon(0.0, 0.25, 5.0)
    assert len(r) == 21 and r[-1] == 5.0
    # half-even rounding of the save stride and snapshot picks
    assert tu.julia_round_int(2.5) == 2 and tu.julia_round_int(3.5) == 4
    assert list(tu.selected_energy_snapshot_indices(801, 5)) == [1, 201, 401, 601, 801]
    assert list(tu.selected_energy_snapshot_indices(4, 4)) == [1, 2, 3, 4]


def test_config1_time_grid():
    """64 steps per T_g0 for 50 T_g0 resolves to 3201 samples, stride 4 -> 801 saves."""
    Om = 0.123456
    r = tu.resolve_trajectory_time_grid(dict(integration_steps_per_gyroperiod=64.0, trajectory_duration_gyroperiods=50.0),
                                        Om, 1.0, 1.0)
    st = tu.resolve_save_stride(dict(trajectory_save_interval_gyroperiods=4 / 64), r)
    assert r.n_integration_steps in (3200, 3201)
    assert st.trajectory_time_stride == 4
