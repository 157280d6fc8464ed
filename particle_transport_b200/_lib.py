"""ctypes binding of libptb200.so (the C ABI declared in include/ptb200.h).

The library is built in-tree by ``particle_transport_b200/build.py``.  There
is no fallback: if the shared library is missing or no B200 is visible, the
calls raise instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libptb200.so")

PT_OK = 0
PT_ERR_ARG = -1
PT_ERR = {-1: "PT_ERR_ARG", -2: "PT_ERR_CUDA", -3: "PT_ERR_OOM", -4: "PT_ERR_TIMEOUT", -5: "PT_ERR_CALLBACK",
          -6: "PT_ERR_STATE"}

PT_FIELD_REF_F64, PT_FIELD_BRICK_F32, PT_FIELD_BRICK_BF16, PT_FIELD_BRICK_BF16_XPAIR, PT_FIELD_BRICK_F64 = 0, 1, 2, 3, 4
PT_CACHE_NONE, PT_CACHE_MU, PT_CACHE_PHASE_SPACE = 0, 1, 2
PT_PUSH_F64, PT_PUSH_F32 = 0, 1
PT_START_SLIDING, PT_START_INJECTION = 0, 1
PT_INJECT_ISOTROPIC, PT_INJECT_FIXED_MU = 0, 1
PT_POSITION_RANDOM, PT_POSITION_FIXED = 0, 1
CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy

# every exported entry point of include/ptb200.h
EXPORTS = (
    "pt_last_error", "pt_version", "pt_ctx_create", "pt_ctx_destroy", "pt_ctx_set_stream", "pt_ctx_synchronize",
    "pt_ctx_trim",
    "pt_field_upload", "pt_field_upload_device", "pt_field_destroy", "pt_field_device_bytes", "pt_push_run",
    "pt_push_advance_device", "pt_fast_state_create", "pt_fast_state_export", "pt_fast_state_destroy",
    "pt_fast_state_sort", "pt_push_advance_fast", "pt_batch_create", "pt_batch_add", "pt_batch_remove",
    "pt_batch_run", "pt_batch_set_running", "pt_batch_set_launch", "pt_batch_step", "pt_batch_export", "pt_batch_destroy", "pt_dmumu_accumulate",
    "pt_dmumu_accumulate_device",
    "pt_dmumu_accumulate_device_noalloc", "pt_dmumu_accumulate_phase_space_device", "pt_dpp_accumulate",
    "pt_dpp_accumulate_device", "pt_energy_snapshots", "pt_energy_snapshots_device",
    "pt_energy_histogram_device", "pt_reconstruct_mu",
    "pt_particles_init_device",
)


class PtError(RuntimeError):
    """A libptb200 call returned a non-zero status."""

    def __init__(self, code: int, where: str, message: str):
        super().__init__(f"{where}: {PT_ERR.get(code, code)}: {message}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
        ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
    ]


class PushParams(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("nsteps", C.c_int64), ("stride", C.c_int64),
        ("periodic", C.c_int32), ("cache_mode", C.c_int32), ("cache_f64", C.c_int32), ("precision", C.c_int32),
        ("steps_per_launch", C.c_int32), ("sort_every", C.c_int32), ("kernel_variant", C.c_int32),
        ("cache_pitch", C.c_int32),
    ]


class CampaignDesc(C.Structure):
    _fields_ = [
        ("field", C.c_void_p), ("dt", C.c_double), ("nsteps", C.c_int64), ("stride", C.c_int64),
        ("periodic", C.c_int32), ("cache_f64", C.c_int32), ("n", C.c_int64),
        ("d_x1", C.c_void_p), ("d_x2", C.c_void_p), ("d_x3", C.c_void_p), ("d_p1", C.c_void_p),
        ("d_p2", C.c_void_p), ("d_p3", C.c_void_p), ("d_alive", C.c_void_p),
        ("d_cache", C.c_void_p), ("cache_rows", C.c_int64), ("cache_ring", C.c_int32), ("sort_every", C.c_int32),
        ("d_deaths", C.c_void_p), ("d_mom_cache", C.c_void_p), ("n_mom", C.c_int64), ("cache_pitch", C.c_int64),
    ]


class InitParams(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("seed", C.c_uint64), ("energy_GeV", C.c_double), ("injection", C.c_int32),
        ("position_mode", C.c_int32), ("mu0", C.c_double), ("position", C.c_double * 3),
    ]


SAVE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64)

_lib = None
_lock = threading.Lock()


def load():
    """Load libptb200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libptb200.so is not built ({LIB_PATH}); run particle_transport_b200/build.py")
        L = C.CDLL(LIB_PATH)
        P, i64, i32, d = C.c_void_p, C.c_int64, C.c_int, C.c_double
        PP = C.POINTER(C.c_void_p)
        sig = {
            "pt_last_error": (C.c_char_p, []),
            "pt_version": (i32, []),
            "pt_ctx_create": (i32, [i32, PP]),
            "pt_ctx_destroy": (i32, [P]),
            "pt_ctx_set_stream": (i32, [P, P]),
            "pt_ctx_synchronize": (i32, [P]),
            "pt_ctx_trim": (i32, [P]),
            "pt_field_upload": (i32, [P, P, C.POINTER(Grid), i32, d, PP]),
            "pt_field_upload_device": (i32, [P, P, C.POINTER(Grid), i32, d, PP]),
            "pt_field_destroy": (i32, [P]),
            "pt_field_device_bytes": (i64, [P]),
            "pt_push_run": (i32, [P, P, P, P, P, P, P, P, P, i64, C.POINTER(PushParams), SAVE_FN, P, P]),
            "pt_push_advance_device": (i32, [P, P, P, P, P, P, P, P, P, i64, C.POINTER(PushParams), i64, i64, P, i64,
                                             i64, P]),
            "pt_fast_state_create": (i32, [P, P, P, P, P, P, P, P, P, i64, PP]),
            "pt_fast_state_export": (i32, [P, P, P, P, P, P, P, P, P]),
            "pt_fast_state_destroy": (i32, [P]),
            "pt_fast_state_sort": (i32, [P, P]),
            "pt_push_advance_fast": (i32, [P, P, P, C.POINTER(PushParams), i64, i64, P, i64, i64, P]),
            "pt_batch_create": (i32, [P, i64, i32, i32, i32, i32, i32, PP]),
            "pt_batch_add": (i32, [P, P, C.POINTER(CampaignDesc), C.POINTER(C.c_int)]),
            "pt_batch_remove": (i32, [P, P, i32]),
            "pt_batch_run": (i32, [P, P, i64, i32]),
            "pt_batch_set_running": (i32, [P, P, P, i32]),
            "pt_batch_set_launch": (i32, [P, P, i32, i32]),
            "pt_batch_step": (i32, [P, P, i32, C.POINTER(C.c_int64)]),
            "pt_batch_export": (i32, [P, P, i32, P, P, P, P, P, P, P]),
            "pt_batch_destroy": (i32, [P]),
            "pt_dmumu_accumulate": (i32, [P, P, i64, i64, i64, i64, P, i32, P, i32, i32, i32, P, P, P, P, P, P, P,
                                          P]),
            "pt_dmumu_accumulate_device": (i32, [P, P, i64, i64, i64, i64, P, i32, P, i32, i32, i32, P, P, P, P, P,
                                                 P, P, P]),
            "pt_dmumu_accumulate_device_noalloc": (i32, [P, P, i64, i64, i64, i64, P, i32, P, i32, i32, i32, P, P, P,
                                                         P, P, P, P, P]),
            "pt_dmumu_accumulate_phase_space_device": (i32, [P, P, P, i64, i64, i64, i64, P, C.POINTER(Grid), i32, P,
                                                             i32, P, i32, i32, i32, P, P, P, P, P, P, P, P]),
            "pt_dpp_accumulate": (i32, [P, P, i64, i64, P, i32, d, P, P, P, P, P]),
            "pt_dpp_accumulate_device": (i32, [P, P, i64, i64, P, i32, d, P, P, P, P, P]),
            "pt_energy_snapshots": (i32, [P, P, i64, i64, P, i32, i64, P]),
            "pt_energy_snapshots_device": (i32, [P, P, i64, i64, P, i32, i64, P]),
            "pt_energy_histogram_device": (i32, [P, P, i64, i64, P, i32, d, d, i32, P]),
            "pt_reconstruct_mu": (i32, [P, P, P, i64, i64, P, C.POINTER(Grid), i32, P]),
            "pt_particles_init_device": (i32, [P, P, C.POINTER(InitParams), P, P, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, where: str) -> None:
    if rc != PT_OK:
        msg = load().pt_last_error()
        raise PtError(rc, where, msg.decode() if msg else "")


def call(name: str, *args):
    rc = getattr(load(), name)(*args)
    check(rc, name)
    return rc


def ptr(x) -> C.c_void_p | None:
    """Raw pointer of a numpy array, a torch tensor, an int address or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return C.c_void_p(x)
    if hasattr(x, "data_ptr"):
        return C.c_void_p(x.data_ptr())
    if hasattr(x, "ctypes"):
        return C.c_void_p(x.ctypes.data)
    raise TypeError(f"cannot take a pointer of {type(x)}")


def ptr_array(xs):
    return (C.c_void_p * len(xs))(*[ptr(x).value if ptr(x) is not None else None for x in xs])


_ctx = {}


class Context:
    """One pt_ctx per device (not re-entrant: one per host thread)."""

    def __init__(self, device: int = 0):
        out = C.c_void_p()
        call("pt_ctx_create", device, C.byref(out))
        self.handle = out
        self.device = device

    def use_stream(self, stream) -> None:
        """Enqueue device calls on ``stream`` (a torch.cuda.Stream or an int
        cudaStream_t).  Handle 0 is the legacy default stream and is passed as
        cudaStreamLegacy; None selects the library's own stream."""
        if stream is None:
            call("pt_ctx_set_stream", self.handle, None)
            return
        h = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        call("pt_ctx_set_stream", self.handle, C.c_void_p(h if h else CUDA_STREAM_LEGACY))

    def synchronize(self) -> None:
        call("pt_ctx_synchronize", self.handle)

    def trim(self) -> None:
        """Release the buffers the context keeps between calls (pt_ctx_trim)."""
        call("pt_ctx_trim", self.handle)

    def close(self) -> None:
        if self.handle:
            load().pt_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def context(device: int = 0) -> Context:
    key = (threading.get_ident(), device)
    c = _ctx.get(key)
    if c is None:
        c = Context(device)
        _ctx[key] = c
    return c


def torch_context(tensor_or_device=None) -> Context:
    """Context of the tensor's device, bound to torch's current stream there."""
    import torch

    if tensor_or_device is None:
        dev = torch.cuda.current_device()
    elif hasattr(tensor_or_device, "device"):
        dev = tensor_or_device.device.index or 0
    else:
        dev = int(tensor_or_device)
    c = context(dev)
    c.use_stream(torch.cuda.current_stream(dev))
    return c
