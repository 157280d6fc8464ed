"""B200-native trajectory and transport-statistics path of particle_transport.

libptb200.so (CUDA for sm_100a, C ABI in include/ptb200.h) does the work:
the relativistic Boris push with trilinear B/u interpolation (FP64 parity
form and FP32 form over Morton-bricked FP32/BF16 fields), the mu /
phase-space cache writer, and the lag-pair D_mumu / <dmu^2> and D_pp
statistics.  This package is the Python host: time/lag grids, synthetic
fields, particle initialisation and thin wrappers over the C ABI.
"""
from . import _lib  # noqa: F401
from .fields import FieldLibrary, UniformGrid, build_uniform_grid, synthetic_mhd_fields, to_si  # noqa: F401

__all__ = ["FieldLibrary", "UniformGrid", "build_uniform_grid", "synthetic_mhd_fields", "to_si"]
