"""Particle initialisation: the counter-stream restatement in the oracle
(checked here against the reference's formulas) and the device initialiser
(checked against the oracle on a B200).

Reference: init_particles / rand_unit_vector / fixed_mu_unit_vector,
src/phase_space_gpu_runner.jl:51-66, 170-245."""
import math

import numpy as np
import pytest

from helpers import small_problem
from particle_transport_b200 import fields as F
from particle_transport_b200.particles import energy_to_gamma, energy_to_speed

KEYS = ("x1", "x2", "x3", "p1", "p2", "p3")


def _pscale(E):
    return energy_to_gamma(E) * F.M_P * energy_to_speed(E)


def _mu_local(st, pb):
    from oracle import oracle as o
    g = pb.grid
    out = []
    for i in range(len(st["x1"])):
        b = [o.trilinear(f.T, st["x1"][i], st["x2"][i], st["x3"][i], g) for f in pb.fields[:3]]
        p = (st["p1"][i], st["p2"][i], st["p3"][i])
        out.append(sum(a * c for a, c in zip(p, b)) / (math.sqrt(sum(a * a for a in p)) * math.sqrt(sum(c * c for c in b))))
    return np.array(out)


def test_oracle_init_isotropic_formulas(oracle):
    from oracle import oracle as o
    pb = small_problem(n=8, n_particles=4)
    st, bad = o.init_particles(20000, 7, 10.0, pb.grid)
    assert bad == 0
    g = pb.grid
    for k, lo, hi in (("x1", g.xmin, g.xmax), ("x2", g.ymin, g.ymax), ("x3", g.zmin, g.zmax)):
        assert np.all(st[k] >= lo) and np.all(st[k] < hi)
        assert abs(np.mean((st[k] - lo) / (hi - lo)) - 0.5) < 0.01
    pm = np.sqrt(st["p1"] ** 2 + st["p2"] ** 2 + st["p3"] ** 2)
    assert np.max(np.abs(pm / _pscale(10.0) - 1)) < 1e-15
    # isotropic: <u> = 0 and <uz^2> = 1/3
    u = np.stack([st["p1"], st["p2"], st["p3"]]) / pm
    assert np.all(np.abs(u.mean(axis=1)) < 0.02)
    assert abs(np.mean(u[2] ** 2) - 1.0 / 3.0) < 0.01


def test_oracle_init_reproducible_and_seeded(oracle):
    from oracle import oracle as o
    pb = small_problem(n=8, n_particles=4)
    a, _ = o.init_particles(1000, 1, 1.0, pb.grid)
    b, _ = o.init_particles(1000, 1, 1.0, pb.grid)
    c, _ = o.init_particles(1000, 2, 1.0, pb.grid)
    # a prefix of a longer run is the same particles (counter-based stream)
    d, _ = o.init_particles(1500, 1, 1.0, pb.grid)
    for k in KEYS:
        assert np.array_equal(a[k], b[k])
        assert np.array_equal(a[k], d[k][:1000])
        assert not np.array_equal(a[k], c[k])


def test_oracle_init_fixed_mu(oracle):
    from oracle import oracle as o
    pb = small_problem(n=10, n_particles=4)
    st, bad = o.init_particles(300, 5, 3.0, pb.grid, injection="fixed_mu", mu0=-0.35, bfield=pb.fields[:3])
    assert bad == 0
    assert np.max(np.abs(_mu_local(st, pb) + 0.35)) < 1e-13


def test_oracle_init_fixed_position(oracle):
    from oracle import oracle as o
    pb = small_problem(n=8, n_particles=4)
    st, _ = o.init_particles(10, 5, 3.0, pb.grid, position_mode="fixed", position=(0.25, 0.5, 1.0))
    g = pb.grid
    assert np.all(st["x1"] == g.xmin + 0.25 * (g.xmax - g.xmin))
    assert np.all(st["x3"] == g.zmin + 1.0 * (g.zmax - g.zmin))


def test_oracle_init_zero_field_flags(oracle):
    from oracle import oracle as o
    pb = small_problem(n=8, n_particles=4)
    zero = [np.zeros_like(f) for f in pb.fields[:3]]
    st, bad = o.init_particles(50, 5, 3.0, pb.grid, injection="fixed_mu", mu0=0.2, bfield=zero)
    assert bad == 50 and np.all(np.isnan(st["p1"]))


# ------------------------------------------------------------------ device
@pytest.mark.gpu
@pytest.mark.parametrize("injection,position_mode", [("isotropic", "random"), ("fixed_mu", "random"),
                                                     ("fixed_mu", "fixed"), ("isotropic", "fixed")])
def test_device_init_matches_oracle(cuda, injection, position_mode):
    from oracle import oracle as o
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import init_particles_device
    pb = small_problem(n=16, n_particles=4)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    n = 100_003
    kw = dict(injection_mode=injection, mu0=0.6, position_mode=position_mode, position=(0.3, 0.7, 0.1))
    dev = init_particles_device(fl, n, 10.0, seed=12345, **kw)
    ref, bad = o.init_particles(n, 12345, 10.0, pb.grid, injection=injection, mu0=0.6, position_mode=position_mode,
                                position=(0.3, 0.7, 0.1), bfield=pb.fields[:3])
    assert bad == 0
    got = {k: v.cpu().numpy() for k, v in dev.items()}
    for k in ("x1", "x2", "x3"):
        assert np.array_equal(got[k], ref[k]), k
    ps = _pscale(10.0)
    for k in ("p1", "p2", "p3"):
        # cos/sin of CUDA and of the host libm may differ in the last bits
        assert np.max(np.abs(got[k] - ref[k])) <= 4e-16 * ps * 4, k


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["brick_f32", "brick_bf16", "brick_bf16x"])
def test_device_init_fixed_mu_on_bricks(cuda, storage):
    """On a brick field the local direction comes from the stored FP32/BF16
    values: mu about the FP64 field is mu0 to the storage precision."""
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import init_particles_device
    pb = small_problem(n=12, n_particles=4)
    fl = FieldLibrary(pb.fields, pb.grid, storage)
    st = {k: v.cpu().numpy() for k, v in init_particles_device(fl, 400, 1.0, seed=3, injection_mode="fixed_mu",
                                                                mu0=0.5).items()}
    err = np.abs(_mu_local(st, pb) - 0.5)
    assert err.max() < (1e-6 if storage == "brick_f32" else 2e-2), err.max()


@pytest.mark.gpu
def test_device_init_errors(cuda):
    from particle_transport_b200._lib import PtError
    from particle_transport_b200.fields import FieldLibrary
    from particle_transport_b200.particles import init_particles_device
    pb = small_problem(n=8, n_particles=4)
    zero = [np.zeros_like(f) for f in pb.fields[:3]] + list(pb.fields[3:])
    fl0 = FieldLibrary(zero, pb.grid, "ref_f64", B_ref_T=1e-10)
    with pytest.raises(PtError, match="local B is zero or non-finite"):
        init_particles_device(fl0, 64, 1.0, injection_mode="fixed_mu", mu0=0.1)
    fl = FieldLibrary(pb.fields, pb.grid, "ref_f64")
    with pytest.raises(PtError, match="outside the simulation box"):
        init_particles_device(fl, 8, 1.0, position_mode="fixed", position=(0.5, 1.5, 0.5))
    with pytest.raises(PtError, match="mu0 must be in"):
        init_particles_device(fl, 8, 1.0, injection_mode="fixed_mu", mu0=1.5)
    # the context stays usable after the error
    st = init_particles_device(fl, 8, 1.0)
    assert bool(np.all(np.isfinite(st["p1"].cpu().numpy())))
