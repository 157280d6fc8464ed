"""Particle initialisation on the host (src/phase_space_gpu_runner.jl:51-245).

The reference seeds a Julia MersenneTwister, whose stream cannot be
reproduced here; this module draws from numpy's PCG64 seeded with the same
integer and otherwise applies the reference's formulas: uniform positions
in [xmin, xmax], isotropic directions (z = 2r - 1, phi = 2 pi r) or a fixed
pitch cosine mu0 about the local field with a random gyrophase, and
|p| = gamma0 m v0.  The kernels are always given the arrays produced here,
so the oracle and the device see identical initial states.
"""
from __future__ import annotations

import math

import numpy as np

from .fields import C_LIGHT, GEV_TO_J, M_P, UniformGrid


def energy_to_gamma(E_GeV: float) -> float:
    """src/phase_space_gpu_runner.jl:51-54 (Float64)."""
    kinetic = float(E_GeV * GEV_TO_J)
    return kinetic / (M_P * (C_LIGHT * C_LIGHT)) + 1.0


def energy_to_speed(E_GeV: float) -> float:
    """src/phase_space_gpu_runner.jl:56-59 (Float64)."""
    g = energy_to_gamma(E_GeV)
    return C_LIGHT * math.sqrt(1.0 - 1.0 / (g * g))


def trilinear_host(arr, x, y, z, grid: UniformGrid):
    """Vectorised trilinear_sample (src/phase_space_gpu_runner.jl:247-276);
    arr is C-ordered (nz, ny, nx).  Same expression order as the reference."""
    fx = (x - grid.xmin) / grid.dx + 1.0
    fy = (y - grid.ymin) / grid.dy + 1.0
    fz = (z - grid.zmin) / grid.dz + 1.0
    i0 = np.clip(np.floor(fx), 1, grid.nx - 1)
    j0 = np.clip(np.floor(fy), 1, grid.ny - 1)
    k0 = np.clip(np.floor(fz), 1, grid.nz - 1)
    tx, ty, tz = fx - i0, fy - j0, fz - k0
    i, j, k = i0.astype(np.int64) - 1, j0.astype(np.int64) - 1, k0.astype(np.int64) - 1
    c000 = arr[k, j, i]; c100 = arr[k, j, i + 1]; c010 = arr[k, j + 1, i]; c110 = arr[k, j + 1, i + 1]
    c001 = arr[k + 1, j, i]; c101 = arr[k + 1, j, i + 1]; c011 = arr[k + 1, j + 1, i]; c111 = arr[k + 1, j + 1, i + 1]
    c00 = c000 * (1 - tx) + c100 * tx
    c10 = c010 * (1 - tx) + c110 * tx
    c01 = c001 * (1 - tx) + c101 * tx
    c11 = c011 * (1 - tx) + c111 * tx
    c0 = c00 * (1 - ty) + c10 * ty
    c1 = c01 * (1 - ty) + c11 * ty
    return c0 * (1 - tz) + c1 * tz


def init_particles(n: int, grid: UniformGrid, energy_GeV: float, seed: int = 42, injection_mode: str = "isotropic",
                   mu0: float = 0.0, B=None, position_mode: str = "random", position=(0.5, 0.5, 0.5)):
    """Initial SI state (x1, x2, x3, p1, p2, p3) as float64 arrays of length n.

    injection_mode "isotropic" or "fixed_mu" (then B = (Bx, By, Bz) in SI,
    C-ordered (nz, ny, nx) host arrays); position_mode "random" or "fixed"
    (position in box fractions)."""
    injection_mode = injection_mode.replace("-", "_")
    if injection_mode not in ("isotropic", "fixed_mu"):
        raise ValueError("injection_mode must be isotropic or fixed-mu")
    rng = np.random.Generator(np.random.PCG64(seed))
    g0 = energy_to_gamma(energy_GeV)
    v0 = energy_to_speed(energy_GeV)
    pscale = g0 * M_P * v0
    if position_mode == "random":
        x1 = rng.random(n) * (grid.xmax - grid.xmin) + grid.xmin
        x2 = rng.random(n) * (grid.ymax - grid.ymin) + grid.ymin
        x3 = rng.random(n) * (grid.zmax - grid.zmin) + grid.zmin
    elif position_mode == "fixed":
        x1 = np.full(n, grid.xmin + position[0] * (grid.xmax - grid.xmin))
        x2 = np.full(n, grid.ymin + position[1] * (grid.ymax - grid.ymin))
        x3 = np.full(n, grid.zmin + position[2] * (grid.zmax - grid.zmin))
    else:
        raise ValueError("position_mode must be random or fixed")
    if injection_mode == "isotropic":
        # rand_unit_vector, src/phase_space_gpu_runner.jl:61-66
        z = 2 * rng.random(n) - 1
        phi = 2 * math.pi * rng.random(n)
        r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
        ux, uy, uz = r * np.cos(phi), r * np.sin(phi), z
    else:
        if not -1.0 <= mu0 <= 1.0:
            raise ValueError("injection_mu0 must be in [-1, 1]")
        if B is None:
            raise ValueError("fixed-mu injection requires magnetic field arrays")
        bx = trilinear_host(np.asarray(B[0]), x1, x2, x3, grid)
        by = trilinear_host(np.asarray(B[1]), x1, x2, x3, grid)
        bz = trilinear_host(np.asarray(B[2]), x1, x2, x3, grid)
        # fixed_mu_unit_vector, src/phase_space_gpu_runner.jl:170-194
        bn = np.sqrt(bx * bx + by * by + bz * bz)
        if not np.all(np.isfinite(bn) & (bn != 0)):
            raise ValueError("cannot use fixed-mu injection where local B is zero or non-finite")
        bhx, bhy, bhz = bx / bn, by / bn, bz / bn
        small = np.abs(bhx) < 0.9
        e1x = np.where(small, 0.0, -bhz)
        e1y = np.where(small, bhz, 0.0)
        e1z = np.where(small, -bhy, bhx)
        e1n = np.sqrt(e1x * e1x + e1y * e1y + e1z * e1z)
        e1x, e1y, e1z = e1x / e1n, e1y / e1n, e1z / e1n
        e2x = bhy * e1z - bhz * e1y
        e2y = bhz * e1x - bhx * e1z
        e2z = bhx * e1y - bhy * e1x
        phi = 2 * math.pi * rng.random(n)
        perp = math.sqrt(max(0.0, 1.0 - mu0 * mu0))
        c, s = np.cos(phi), np.sin(phi)
        ux = mu0 * bhx + perp * (c * e1x + s * e2x)
        uy = mu0 * bhy + perp * (c * e1y + s * e2y)
        uz = mu0 * bhz + perp * (c * e1z + s * e2z)
    return {"x1": np.ascontiguousarray(x1), "x2": np.ascontiguousarray(x2), "x3": np.ascontiguousarray(x3),
            "p1": np.ascontiguousarray(pscale * ux), "p2": np.ascontiguousarray(pscale * uy),
            "p3": np.ascontiguousarray(pscale * uz)}


def init_particles_device(field, n: int, energy_GeV: float, seed: int = 42, injection_mode: str = "isotropic",
                          mu0: float = 0.0, position_mode: str = "random", position=(0.5, 0.5, 0.5)):
    """Initial SI state written on the device (pt_particles_init_device): the
    reference's formulas over a counter-based SplitMix64 stream, so a job's
    state depends only on (seed, n, energy, injection, field) and needs no
    host work.  Fixed-mu injection samples B from the field library's own
    stored values.  Returns a dict of CUDA float64 tensors x1..p3."""
    import torch

    from . import _lib

    injection_mode = injection_mode.replace("-", "_")
    modes = {"isotropic": _lib.PT_INJECT_ISOTROPIC, "fixed_mu": _lib.PT_INJECT_FIXED_MU}
    pmodes = {"random": _lib.PT_POSITION_RANDOM, "fixed": _lib.PT_POSITION_FIXED}
    if injection_mode not in modes:
        raise ValueError("injection_mode must be isotropic or fixed-mu")
    if position_mode not in pmodes:
        raise ValueError("position_mode must be random or fixed")
    dev = torch.device("cuda", field.ctx.device)
    out = {k: torch.empty(int(n), dtype=torch.float64, device=dev) for k in ("x1", "x2", "x3", "p1", "p2", "p3")}
    prm = _lib.InitParams(int(n), int(seed) & 0xFFFFFFFFFFFFFFFF, float(energy_GeV), modes[injection_mode],
                          pmodes[position_mode], float(mu0), (_lib.C.c_double * 3)(*[float(v) for v in position]))
    ctx = _lib.torch_context(out["x1"])
    _lib.call("pt_particles_init_device", ctx.handle, field.handle, _lib.C.byref(prm),
              *[_lib.ptr(out[k]) for k in ("x1", "x2", "x3", "p1", "p2", "p3")])
    return out
