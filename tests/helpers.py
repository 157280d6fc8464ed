"""Small seeded problems shared by the tests (host arrays only)."""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

from particle_transport_b200 import fields as F
from particle_transport_b200.particles import energy_to_gamma, init_particles
from particle_transport_b200.time_units import reference_Omega0


def small_problem(n=16, n_particles=256, energy_GeV=1.0, dB=0.5, u_over_c=1e-4, seed=3, steps_per_gyro=64,
                  cells_per_rg=1.0, kmax=None, injection="isotropic"):
    """n^3 periodic box whose cell is cells_per_rg gyroradii of a 1 GeV proton
    in B0 = 1 uG (config-1 convention), seeded turbulence and particles."""
    kmax = kmax or n // 2
    f_uG = F.synthetic_mhd_fields(n, 2, kmax, dB, 1.0, u_over_c, seed)
    fields_si = [np.ascontiguousarray(f.numpy()) for f in F.to_si(f_uG)]
    rg = F.gyroradius_m(1.0, 1e-10)
    grid = F.build_uniform_grid((n - 1) * rg * cells_per_rg, n, n, n)
    B0 = F.reference_B0_T(*fields_si[:3])
    g0 = energy_to_gamma(energy_GeV)
    Om = reference_Omega0(B0, g0, F.Q_E, F.M_P)
    dt = (2 * math.pi / steps_per_gyro) / Om
    st = init_particles(n_particles, grid, energy_GeV, seed=seed + 11, injection_mode=injection, mu0=0.5,
                        B=fields_si[:3])
    return SimpleNamespace(fields=fields_si, grid=grid, state=st, dt=dt, Omega0=Om, B0=B0, gamma0=g0)


def fortran_fields(fields):
    """C-ordered (nz, ny, nx) arrays as Fortran-ordered (nx, ny, nz) views for the oracle."""
    return [np.asfortranarray(f.T) for f in fields]


def copy_state(st):
    return {k: np.array(v, dtype=np.float64, copy=True) for k, v in st.items()}


def random_mu_cache(n, nsave, seed=0, nan_frac=0.0, walk=True):
    """float32 mu series shaped (n, nsave) (time fastest), values in [-1, 1]."""
    rng = np.random.default_rng(seed)
    if walk:
        x = np.cumsum(rng.normal(0, 0.08, size=(n, nsave)), axis=1) + rng.uniform(-1, 1, size=(n, 1))
        mu = np.clip(np.sin(x), -1, 1)
    else:
        mu = rng.uniform(-1, 1, size=(n, nsave))
    mu = mu.astype(np.float32)
    if nan_frac > 0:
        mu[rng.random(mu.shape) < nan_frac] = np.nan
    return np.ascontiguousarray(mu)


def zero_dmumu(n_lags, n_bins):
    return {"counts": np.zeros((n_lags, n_bins), np.int64), "sum_d": np.zeros((n_lags, n_bins)),
            "sum_d2": np.zeros((n_lags, n_bins)), "w_count": np.zeros(n_lags, np.int64), "w_mean": np.zeros(n_lags),
            "w_m2": np.zeros(n_lags), "pair_ss": np.zeros(n_lags), "pair_n": np.zeros(n_lags, np.int64)}


def zero_dpp(n_lags):
    return {"counts": np.zeros(n_lags, np.int64), "sum_dp": np.zeros(n_lags), "sum_dp2": np.zeros(n_lags),
            "sum_dpn": np.zeros(n_lags), "sum_dpn2": np.zeros(n_lags)}
