"""The Python mirrors of the reference's push seams -- run_mu_cache_ensemble
(src/multimode_multienergy_cache_pipeline.jl:1380) and run_gpu_ensemble
(src/phase_space_gpu_runner.jl:476) -- driven by a config dict with the
reference's keys: the time grid, the save stride, the initial state and the
push must compose as in the reference, and the caches must equal the oracle's
on the same seeded inputs (FP64, bit for bit)."""
import math

import numpy as np
import pytest

from helpers import copy_state, fortran_fields, small_problem
from particle_transport_b200 import runner as R
from particle_transport_b200.fields import FieldLibrary
from particle_transport_b200.particles import energy_to_speed, init_particles

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    cfg = {"n_particles": 257, "seed": 9, "integration_steps_per_gyroperiod": 64,
           "trajectory_duration_gyroperiods": 3.0, "trajectory_save_interval_gyroperiods": 0.25,
           "boundary": "periodic", "injection_mode": "isotropic"}
    cfg.update(kw)
    return cfg


def test_mu_cache_ensemble_matches_oracle(cuda, oracle):
    pb = small_problem(n=16, n_particles=4, u_over_c=1e-4)
    tref = R.resolve_total_field_time_reference(pb.fields, 2.0)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    cfg = _cfg()
    res = R.run_mu_cache_ensemble(cfg, fl, energy_GeV=2.0, time_reference=tref, fields_host_B=pb.fields[:3])
    # time grid: 3 T_g0 at 64 steps per T_g0 (192 or 193 samples, floor of a
    # rounded ratio); 0.25 T_g0 saves -> stride 16
    Om = tref.Omega0_reference_s_inv
    assert res.dt == pytest.approx((2 * math.pi / 64) / Om, rel=1e-15)
    n = res.trajectory_time.n_integration_steps
    assert n in (192, 193)
    assert res.save_time.trajectory_time_stride == 16 and res.nsave == (n - 1) // 16 + 1
    assert res.t_norm[1] == pytest.approx(16 * res.dt * Om, rel=1e-15)
    assert res.t_gyroperiods[1] == pytest.approx(0.25, rel=1e-12)
    st = init_particles(257, pb.grid, 2.0, seed=9, B=pb.fields[:3])
    mu_o, ac_o = oracle.push_run(fortran_fields(pb.fields), pb.grid, copy_state(st), np.ones(257, np.uint8), res.dt,
                                 n, 16, cache_mode=1)
    assert np.array_equal(res.mu, mu_o, equal_nan=True)
    assert np.array_equal(res.alive_fraction, ac_o[np.arange(0, n, 16)] / 257.0)


def test_gpu_ensemble_phase_space_open_boundary(cuda, oracle):
    pb = small_problem(n=12, n_particles=4, u_over_c=1e-4, energy_GeV=30.0)
    tref = R.resolve_total_field_time_reference(pb.fields, 30.0)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    cfg = _cfg(boundary="open", trajectory_time_stride=4, trajectory_save_interval_gyroperiods=None,
               trajectory_duration_gyroperiods=2.0, n_particles=200, seed=3)
    res = R.run_gpu_ensemble(cfg, fl, energy_GeV=30.0, time_reference=tref)
    n = res.trajectory_time.n_integration_steps
    st = init_particles(200, pb.grid, 30.0, seed=3)
    (pos, mom), ac = oracle.push_run(fortran_fields(pb.fields), pb.grid, copy_state(st), np.ones(200, np.uint8),
                                     res.dt, n, 4, periodic=False, cache_mode=2)
    assert np.array_equal(res.positions, pos, equal_nan=True)
    assert np.array_equal(res.momenta, mom, equal_nan=True)
    assert np.array_equal(res.alive_fraction, ac / 200.0)
    assert res.alive_fraction[-1] < 1.0  # particles left the open box


def test_cfl_limited_time_step(cuda):
    """use_cfl: dt = min(eta / Omega0, cfl * min_dx / v0) (time_units:67-111)."""
    pb = small_problem(n=12, n_particles=4, cells_per_rg=0.05)  # small cells: the CFL bound binds
    tref = R.resolve_total_field_time_reference(pb.fields, 1.0)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    cfg = _cfg(use_cfl=True, cfl=0.5, n_particles=16, trajectory_duration_gyroperiods=0.5)
    res = R.run_mu_cache_ensemble(cfg, fl, energy_GeV=1.0, time_reference=tref, fields_host_B=pb.fields[:3])
    assert res.trajectory_time.timestep_limited_by == "cfl"
    assert res.dt == pytest.approx(0.5 * pb.grid.dx / energy_to_speed(1.0), rel=1e-15)


def test_runner_requires_time_reference_and_known_boundary(cuda):
    pb = small_problem(n=8, n_particles=4)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    with pytest.raises(ValueError, match="time reference"):
        R.run_mu_cache_ensemble(_cfg(), fl, energy_GeV=1.0, time_reference=None)
    tref = R.resolve_total_field_time_reference(pb.fields, 1.0)
    with pytest.raises(ValueError, match="boundary"):
        R.run_mu_cache_ensemble(_cfg(boundary="reflecting"), fl, energy_GeV=1.0, time_reference=tref)
