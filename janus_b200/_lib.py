"""ctypes binding of the janus_b200 C ABI (``include/janus_b200.h``).

The native library ``janus_b200/lib/libjanus_b200.so`` is the only compute
path: there is no CPU fallback.  If the library is missing it is built with
nvcc (``janus_b200.build``); if that fails, importing any operator raises.
Status codes map to exceptions like the reference's validation layer:
JB_EINVAL -> ValueError, anything else -> RuntimeError.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

JB_OK = 0
JB_EINVAL = -1
JB_EFAULT = -5
JB_F64 = 0
JB_F32 = 1
JB_TRUNCATED = 0
JB_FILTERED = 1
JB_WILLOT = 2

# per-load-case outcome of a solve (status arrays of the run calls)
SOLVE_STATUS = {0: "converged", 1: "max_iter", 2: "non_finite", 3: "diverging"}

_lock = threading.Lock()
_lib = None

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_int64 = ctypes.c_int64
c_double = ctypes.c_double
P_int64 = ctypes.POINTER(ctypes.c_int64)
P_int32 = ctypes.POINTER(ctypes.c_int32)
P_double = ctypes.POINTER(ctypes.c_double)
P_int = ctypes.POINTER(ctypes.c_int)

_SIGS = {
    "jb_version": ([], c_int),
    "jb_last_error": ([], ctypes.c_char_p),
    "jb_max_axis_length": ([c_int], c_int),
    "jb_device_status": ([ctypes.POINTER(ctypes.c_uint)], c_int),
    "jb_set_wait_limit": ([c_int], c_int),
    "jb_fft_create": ([c_int, P_int64, c_int, ctypes.c_uint, ctypes.POINTER(c_void_p)], c_int),
    "jb_fft_destroy": ([c_void_p], c_int),
    "jb_fft_r2c": ([c_void_p, c_void_p, P_int64, c_void_p, c_void_p], c_int),
    "jb_fft_c2r": ([c_void_p, c_void_p, c_void_p, P_int64, c_void_p], c_int),
    "jb_green_continuous_matrix": ([c_int, c_double, c_double, P_double, P_double], c_int),
    "jb_green_continuous_apply": ([c_int, c_double, c_double, P_double, P_double, P_double],
                                  c_int),
    "jb_isotropic_apply": ([c_int, c_double, c_double, P_double, P_double], c_int),
    "jb_green_create": ([c_int, P_int64, c_double, c_double, c_double, c_int, c_int,
                         ctypes.POINTER(c_void_p)], c_int),
    "jb_green_destroy": ([c_void_p], c_int),
    "jb_green_set_tuning": ([c_void_p, P_int, c_int], c_int),
    "jb_green_get_tuning": ([c_void_p, P_int, c_int], c_int),
    "jb_green_apply": ([c_void_p, c_void_p, c_void_p, c_int64, c_void_p], c_int),
    "jb_green_matrix": ([c_void_p, P_int32, P_double], c_int),
    "jb_green_apply_by_freq": ([c_void_p, P_int32, P_double, P_double], c_int),
    "jb_green_apply_by_freq_device": ([c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                       c_void_p], c_int),
    "jb_local_create": ([c_int, P_int64, c_int, P_double, P_double, c_void_p, c_int, c_int,
                         ctypes.POINTER(c_void_p)], c_int),
    "jb_local_create_matrix": ([c_int, P_int64, c_int, P_double, c_void_p, c_int, c_int,
                                ctypes.POINTER(c_void_p)], c_int),
    "jb_local_destroy": ([c_void_p], c_int),
    "jb_local_apply": ([c_void_p, c_void_p, c_void_p, c_int64, c_void_p], c_int),
    "jb_block_linear_apply": ([c_int, c_int64, c_int, c_int, c_void_p, c_void_p, c_void_p,
                               c_int, c_void_p], c_int),
    "jb_local_gradient": ([c_int, c_int, c_int64, c_int, c_void_p, c_void_p, c_double,
                           c_void_p, c_void_p], c_int),
    "jb_mixed_set_method": ([c_void_p, c_int], c_int),
    "jb_batch_create": ([c_int, ctypes.POINTER(c_void_p), c_int, ctypes.POINTER(c_void_p)],
                        c_int),
    "jb_batch_destroy": ([c_void_p], c_int),
    "jb_batch_set_persistent": ([c_void_p, c_int], c_int),
    "jb_batch_run": ([c_void_p, P_double, ctypes.POINTER(c_void_p), c_int, c_int, c_int,
                      c_double, P_double, P_int, P_int, P_double, P_int, P_int, c_void_p],
                     c_int),
    "jb_solver_create": ([c_void_p, c_void_p, c_int, ctypes.POINTER(c_void_p)], c_int),
    "jb_solver_destroy": ([c_void_p], c_int),
    "jb_solver_run": ([c_void_p, P_double, c_void_p, c_int, c_int, c_double, P_double, P_int,
                       P_double, P_int, c_void_p], c_int),
    "jb_solver_set_load": ([c_void_p, P_double], c_int),
    "jb_solver_step": ([c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "jb_solver_timing_begin": ([c_void_p, c_int], c_int),
    "jb_solver_timing_end": ([c_void_p, P_double, P_int, P_int], c_int),
    "jb_solver_pass_name": ([c_void_p, c_int], ctypes.c_char_p),
    "jb_mixed_create": ([c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                         ctypes.POINTER(c_void_p)], c_int),
    "jb_mixed_destroy": ([c_void_p], c_int),
    "jb_gmres_create": ([c_void_p, c_void_p, c_int, c_int, ctypes.POINTER(c_void_p)], c_int),
    "jb_gmres_destroy": ([c_void_p], c_int),
    "jb_gmres_run": ([c_void_p, P_double, c_void_p, c_int, c_int, c_double, P_double, P_int,
                      P_double, P_double, P_int, c_void_p], c_int),
    "jb_mixed_run": ([c_void_p, P_double, c_void_p, c_int, c_int, c_int, c_double, P_double,
                      P_int, P_int, P_double, P_int, c_void_p], c_int),
}


def library_path() -> str:
    return _build.LIB


def lib():
    """Load (building first if needed) the native library."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            path = _build.LIB
            if not os.path.exists(path):
                _build.build()
            handle = ctypes.CDLL(path)
            for name, (args, res) in _SIGS.items():
                fn = getattr(handle, name)
                fn.argtypes = args
                fn.restype = res
            _lib = handle
    return _lib


def check(status: int) -> None:
    if status == JB_OK:
        return
    msg = lib().jb_last_error().decode(errors="replace")
    if status == JB_EINVAL:
        raise ValueError(msg)
    raise RuntimeError(f"janus_b200 native call failed ({status}): {msg}")


def device_status() -> int:
    """Read and clear the device fault word (bit 0: a bounded wait gave up)."""
    v = ctypes.c_uint(0)
    check(lib().jb_device_status(ctypes.byref(v)))
    return v.value


def check_device(what: str = "janus_b200") -> None:
    """Raise RuntimeError if a kernel gave up a bounded wait since the last
    check (the fault word is read and cleared; synchronises the device)."""
    f = device_status()
    if f & 1:
        raise RuntimeError(f"{what}: a kernel gave up a bounded wait for its asynchronous "
                           f"copies (device fault word {f}); its results are invalid")


def set_wait_limit(polls=None) -> None:
    """Polls of the first bounded wait of every asynchronous copy (None: the
    default; 0: every first wait gives up at once).  For tests of the failure
    path."""
    check(lib().jb_set_wait_limit(-1 if polls is None else int(polls)))


def status_names(status) -> list:
    return [SOLVE_STATUS.get(int(v), str(int(v))) for v in status]


def i64_array(values):
    arr = (c_int64 * len(values))(*[int(v) for v in values])
    return arr


def f64_array(values):
    return (c_double * len(values))(*[float(v) for v in values])
