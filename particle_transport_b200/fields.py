"""Static field libraries: node grid, synthetic turbulence and device upload.

Array convention: a field component is a C-ordered array of shape
(nz, ny, nx), i.e. x fastest in memory -- the same bytes as the reference's
Julia arrays of size (nx, ny, nz) (src/phase_space_gpu_runner.jl:260-267).

The reference reads MHD snapshots from HDF5 (load_static_fields,
src/phase_space_gpu_runner.jl:95-123).  No snapshot ships with it, so the
benchmark configurations use seeded synthetic Gaussian turbulence generated
here: random-phase Fourier modes with a power-law spectrum, projected to be
divergence-free, written in microgauss and km/s so that the reference's unit
conversion (x 1e-10, x 1e3) applies unchanged.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .time_units import julia_range_length

C_LIGHT = 2.99792458e8
Q_E = 1.602176634e-19
M_P = 1.67262192369e-27
UGAUSS_TO_T = 1e-10
KMPS_TO_MPS = 1e3
PC_TO_M = 3.085677581e16
GEV_TO_J = 1e9 * 1.602176634e-19

STORAGE = {"ref_f64": _lib.PT_FIELD_REF_F64, "brick_f32": _lib.PT_FIELD_BRICK_F32,
           "brick_bf16": _lib.PT_FIELD_BRICK_BF16, "brick_bf16x": _lib.PT_FIELD_BRICK_BF16_XPAIR,
           "brick_f64": _lib.PT_FIELD_BRICK_F64}
# storages the FP64 (exact) push reads
F64_STORAGE = ("ref_f64", "brick_f64")


@dataclass
class UniformGrid:
    nx: int
    ny: int
    nz: int
    xmin: float
    ymin: float
    zmin: float
    xmax: float
    ymax: float
    zmax: float
    dx: float
    dy: float
    dz: float

    def to_c(self) -> _lib.Grid:
        return _lib.Grid(self.nx, self.ny, self.nz, self.xmin, self.ymin, self.zmin, self.xmax, self.ymax, self.zmax,
                         self.dx, self.dy, self.dz)

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)


def build_uniform_grid(box_length_m: float, nx: int, ny: int, nz: int) -> UniformGrid:
    """build_uniform_coords (src/phase_space_gpu_runner.jl:125-130): nodes
    range(0, L, length=n); xmin = x[1], xmax = x[end], dx = x[2] - x[1]."""
    ax = [julia_range_length(0.0, float(box_length_m), n) for n in (nx, ny, nz)]
    return UniformGrid(nx, ny, nz, ax[0][0], ax[1][0], ax[2][0], ax[0][-1], ax[1][-1], ax[2][-1],
                       ax[0][1] - ax[0][0], ax[1][1] - ax[1][0], ax[2][1] - ax[2][0])


def gyroradius_m(energy_GeV: float, B_T: float) -> float:
    """r_g = p / (q B) of a proton with the given kinetic energy."""
    gamma = energy_GeV * GEV_TO_J / (M_P * C_LIGHT ** 2) + 1.0
    v = C_LIGHT * math.sqrt(1.0 - 1.0 / (gamma * gamma))
    return gamma * M_P * v / (Q_E * B_T)


# --------------------------------------------------------------------------
# synthetic turbulence
# --------------------------------------------------------------------------
def _wavenumbers(n: int, torch, device):
    k = torch.fft.fftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    kh = torch.fft.rfftfreq(n, d=1.0 / n, device=device, dtype=torch.float64)
    kz = k.view(n, 1, 1)
    ky = k.view(1, n, 1)
    kx = kh.view(1, 1, -1)
    return kx, ky, kz


# c_s^2 / v_A^2 of the finite-beta mode decomposition of the synthetic variants
MODE_ALPHA = 1.0


def _mode_basis(kx, ky, kz, alpha, torch):
    """Unit vectors per wave vector (B0 along z; k_perp > 0):
    e_A = k x z / |k x z| (Alfven), e_P = k^ x e_A (the second polarisation
    perpendicular to k, in the k-z plane), and the fast and slow MHD
    displacement directions of Cho & Lazarian (2003, MNRAS 345, 325, eq. 5-6)
    for alpha = c_s^2 / v_A^2:
        xi_f ~ (-1 + alpha + sqrt(D)) k_par z^ + (1 + alpha + sqrt(D)) k_perp k_perp^,
        D = (1 + alpha)^2 - 4 alpha cos^2(theta),
    and xi_s, the direction orthogonal to it in the (k_perp^, z) plane
    (their eq. 6 with the minus sign); with e_A they form an orthonormal basis.  Returns (e_A, e_P, xi_f, xi_s)
    as tuples of three tensors, and each mode's magnetic response
    |xi . k_perp^| (the field a displacement xi bends: k x (xi x z) has
    magnitude k |xi . k_perp^|)."""
    kp = torch.sqrt(kx * kx + ky * ky).clamp_min(1e-30)
    kk = torch.sqrt(kx * kx + ky * ky + kz * kz).clamp_min(1e-30)
    cos, sin = kz / kk, kp / kk
    zero, one = torch.zeros_like(kx), torch.ones_like(kx)
    e_a = (ky / kp, -kx / kp, zero)
    kph = (kx / kp, ky / kp, zero)
    e_p = (cos * kph[0], cos * kph[1], -sin)
    sq = torch.sqrt(((1 + alpha) ** 2 - 4 * alpha * cos * cos).clamp_min(0.0))
    f_par = (-1 + alpha + sq) * cos
    f_perp = (1 + alpha + sq) * sin  # > 0 whenever k_perp > 0
    nrm = torch.sqrt(f_par * f_par + f_perp * f_perp).clamp_min(1e-30)
    f_par, f_perp = f_par / nrm, f_perp / nrm
    # xi_s is xi_f turned by 90 degrees in the (k_perp^, z) plane: the same
    # direction as the formula's slow vector, which vanishes (0/0) at
    # perpendicular propagation, where its limit is z
    s_par, s_perp = f_perp, -f_par
    xi_f = (f_perp * kph[0], f_perp * kph[1], f_par * one)
    xi_s = (s_perp * kph[0], s_perp * kph[1], s_par * one)
    return e_a, e_p, xi_f, xi_s, f_perp.abs(), s_perp.abs()


def solenoidal_field(n: int, kmin: float, kmax: float, rms: float, seed: int, spectrum: str = "isotropic",
                     device="cpu", modes: str = "total", kind: str = "magnetic"):
    """Seeded divergence-free Gaussian random vector field on an n^3 grid.

    spectrum "isotropic": |A(k)|^2 ~ |k|^(-11/3) for kmin <= |k| <= kmax
    (energy spectrum E(k) ~ k^(-5/3)).
    spectrum "gs": Goldreich-Sridhar-like anisotropy about z: |A|^2 ~
    k_perp^(-10/3) for kmin <= k_perp <= kmax and |k_par| <= k_perp^(2/3) kmin^(1/3)
    (E(k_perp) ~ k_perp^(-5/3)).
    modes: "total", or one MHD mode family of the total field, with B0
    along z (the reference reads such variants from an MHD mode
    decomposition; these are their synthetic stand-ins):
      - "alfven": the projection on e_A = k x z / |k x z|, for either kind;
      - kind "velocity": the projection on the fast or slow displacement
        direction xi_f, xi_s of a finite-beta plasma (c_s^2 / v_A^2 =
        MODE_ALPHA); e_A, xi_f, xi_s are orthonormal, so the three variants
        add up to the total velocity field, and fast / slow carry the
        compressive parts;
      - kind "magnetic": the component along e_P, the polarisation
        perpendicular to k in the k-z plane (divergence-free), split between
        fast and slow by their magnetic responses |xi . k_perp^| (power
        preserving: |dB_f|^2 + |dB_s|^2 = |dB . e_P|^2).
    Wave vectors along z (k_perp = 0) go to the Alfven variant.  Every
    variant then bends the field lines and has a motional electric field
    E = -u x B.
    Returns three float64 torch tensors of shape (n, n, n) (z, y, x) scaled to
    sqrt(<|A|^2>) = rms over the grid (before any mode projection).
    """
    import torch

    dev = torch.device(device)
    kx, ky, kz = _wavenumbers(n, torch, dev)
    k2 = kx * kx + ky * ky + kz * kz
    kperp = torch.sqrt(kx * kx + ky * ky)
    if spectrum == "isotropic":
        kk = torch.sqrt(k2)
        mask = (kk >= kmin) & (kk <= kmax)
        power = torch.where(mask, kk.clamp_min(1e-30) ** (-11.0 / 3.0), torch.zeros_like(kk))
    elif spectrum == "gs":
        mask = (kperp >= kmin) & (kperp <= kmax) & (kz.abs() <= kperp.clamp_min(1e-30) ** (2.0 / 3.0) * kmin ** (1.0 / 3.0))
        power = torch.where(mask, kperp.clamp_min(1e-30) ** (-10.0 / 3.0), torch.zeros_like(kperp))
    else:
        raise ValueError("spectrum must be isotropic or gs")
    amp = torch.sqrt(power)
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))
    shape = (n, n, n // 2 + 1)
    comps = []
    for _ in range(3):
        re = torch.randn(shape, generator=g, device=dev, dtype=torch.float64)
        im = torch.randn(shape, generator=g, device=dev, dtype=torch.float64)
        comps.append(torch.complex(re, im) * amp)
    ax, ay, az = comps
    # project out the component along k (div A = 0)
    kdot = (kx * ax + ky * ay + kz * az) / k2.clamp_min(1e-30)
    ax = ax - kx * kdot
    ay = ay - ky * kdot
    az = az - kz * kdot
    fields = [torch.fft.irfftn(c, s=(n, n, n)) for c in (ax, ay, az)]
    scale = rms / math.sqrt(float(sum((f * f).mean() for f in fields)))
    if modes != "total":
        if modes not in ("alfven", "fast", "slow"):
            raise ValueError("modes must be total, alfven, fast or slow")
        if kind not in ("magnetic", "velocity"):
            raise ValueError("kind must be magnetic or velocity")
        spec = [torch.fft.rfftn(f) for f in fields]
        zero = torch.zeros_like(spec[0])
        e_a, e_p, xi_f, xi_s, bf, bs = _mode_basis(kx, ky, kz, MODE_ALPHA, torch)
        weight = torch.ones_like(kx)
        if modes == "alfven":
            e = e_a
            along_z = (spec[0], spec[1], spec[2])
        else:
            along_z = (zero, zero, zero)
            if kind == "velocity":
                e = xi_f if modes == "fast" else xi_s
            else:
                e = e_p
                b = bf if modes == "fast" else bs
                weight = b / torch.sqrt(bf * bf + bs * bs).clamp_min(1e-30)
        dot = (e[0] * spec[0] + e[1] * spec[1] + e[2] * spec[2]) * weight
        par = kperp < 1e-12  # k along z: no k x z direction
        proj = [torch.where(par, az_, dot * ei) for az_, ei in zip(along_z, e)]
        fields = [torch.fft.irfftn(c, s=(n, n, n)) for c in proj]
    return [f * scale for f in fields]


def synthetic_mhd_fields(n: int, kmin: float, kmax: float, dB_over_B0: float, B0_uG: float = 1.0,
                         u_rms_over_c: float = 0.0, seed: int = 1, spectrum: str = "isotropic", modes: str = "total",
                         device="cpu"):
    """(Bx, By, Bz, ux, uy, uz) in microgauss and km/s: B = B0 z + dB with
    dB_rms = dB_over_B0 * B0, u an independent solenoidal field with u_rms =
    u_rms_over_c * c (zero when u_rms_over_c == 0)."""
    import torch

    dB = solenoidal_field(n, kmin, kmax, dB_over_B0 * B0_uG, seed, spectrum, device, modes, kind="magnetic")
    dB[2] = dB[2] + B0_uG
    if u_rms_over_c > 0:
        u = solenoidal_field(n, kmin, kmax, u_rms_over_c * C_LIGHT / KMPS_TO_MPS, seed + 7919, spectrum, device, modes,
                             kind="velocity")
    else:
        u = [torch.zeros((n, n, n), dtype=torch.float64, device=device) for _ in range(3)]
    return dB + u


def to_si(fields_uG_kms, velocity_unit_in_m_per_s: float = KMPS_TO_MPS):
    """The unit conversion of load_static_fields (src/phase_space_gpu_runner.jl:114-119)."""
    out = []
    for i, f in enumerate(fields_uG_kms):
        out.append(f * (UGAUSS_TO_T if i < 3 else velocity_unit_in_m_per_s))
    return out


def reference_B0_T(Bx, By, Bz) -> float:
    """mean(sqrt(Bx^2 + By^2 + Bz^2)) (src/time_units.jl:18-20) for numpy or torch arrays."""
    if hasattr(Bx, "double"):
        return float(((Bx * Bx + By * By + Bz * Bz).sqrt()).mean())
    return float(np.mean(np.sqrt(Bx * Bx + By * By + Bz * Bz)))


# --------------------------------------------------------------------------
# device field library
# --------------------------------------------------------------------------
class FieldLibrary:
    """A static field (B, u) resident on the device (pt_field).

    fields: six SI arrays (Bx, By, Bz, ux, uy, uz), each C-ordered (nz, ny, nx)
    float64 -- numpy (uploaded from the host) or CUDA torch tensors (converted
    on the device).  storage: "ref_f64" (reference layout, FP64 push),
    "brick_f64" (Morton bricks of FP64 SI node records, FP64 push, the same
    results), "brick_f32" or "brick_bf16" (Morton bricks, FP32 push); B_ref_T
    scales the FP32-push brick forms (defaults to the mean |B| of the field)."""

    def __init__(self, fields, grid: UniformGrid, storage: str = "ref_f64", B_ref_T: float | None = None,
                 device: int = 0):
        if storage not in STORAGE:
            raise ValueError(f"storage must be one of {sorted(STORAGE)}")
        self.grid = grid
        self.storage = storage
        on_device = hasattr(fields[0], "is_cuda") and fields[0].is_cuda
        arrs = []
        for f in fields:
            if on_device:
                f = f.contiguous().double()
            else:
                f = np.ascontiguousarray(f, dtype=np.float64)
            if tuple(f.shape) != grid.shape:
                raise ValueError(f"field shape {tuple(f.shape)} != grid (nz, ny, nx) {grid.shape}")
            arrs.append(f)
        if B_ref_T is None:
            B_ref_T = reference_B0_T(arrs[0], arrs[1], arrs[2])
        self.B_ref_T = float(B_ref_T)
        self.ctx = _lib.torch_context(arrs[0]) if on_device else _lib.context(device)
        out = _lib.C.c_void_p()
        g = grid.to_c()
        fn = "pt_field_upload_device" if on_device else "pt_field_upload"
        _lib.call(fn, self.ctx.handle, _lib.ptr_array(arrs), _lib.C.byref(g), STORAGE[storage], self.B_ref_T,
                  _lib.C.byref(out))
        self.handle = out
        self.device_bytes = int(_lib.load().pt_field_device_bytes(out))

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().pt_field_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
