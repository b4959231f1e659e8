"""ctypes binding of the in-tree C-ABI library (include/cuhelmholtz_b200.h).

There is no fallback: if the shared library is missing or fails to load, every
entry point raises.  Build it with ``python -m cuhelmholtz_b200._build``.
"""
from __future__ import annotations

import ctypes
import os
import threading

from ._build import LIBPATH

_lock = threading.Lock()
_lib = None

c_double = ctypes.c_double
c_int = ctypes.c_int
c_void_p = ctypes.c_void_p
c_size_t = ctypes.c_size_t
c_char_p = ctypes.c_char_p
_dp = ctypes.c_void_p  # device pointers are passed as raw addresses

# name -> (restype, argtypes); every extern "C" symbol of the header
SIGNATURES = {
    "chz_version": (c_int, []),
    "chz_status_string": (c_char_p, [c_int]),
    "chz_last_error": (c_char_p, []),
    "chz_do_transform": (c_int, [_dp, _dp, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p]),
    "chz_do_transform_any": (c_int, [_dp, _dp, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p]),
    "chz_helmholtz_workspace_size": (c_size_t, [c_int, c_int, c_int, c_int]),
    "chz_helmholtz_solve": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp,
                                    c_double, c_double, c_int, c_int, _dp, _dp,
                                    c_double, c_double, c_int, c_int, _dp, _dp,
                                    c_double, _dp, c_void_p]),
    "chz_helmholtz_solve_19pt": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp, c_double, c_double, c_int,
                                         c_int, _dp, _dp, c_double, c_double, c_int, c_int, _dp, _dp, c_double,
                                         _dp, c_void_p]),
    "chz_helmholtz_solve_pertrb": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp, c_double, c_double, c_int,
                                           c_int, _dp, _dp, c_double, c_double, c_int, c_int, _dp, _dp, c_double,
                                           _dp, ctypes.POINTER(c_double), c_void_p]),
    "chz_helmholtz_solve_ws": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp,
                                       c_double, c_double, c_int, c_int, _dp, _dp,
                                       c_double, c_double, c_int, c_int, _dp, _dp,
                                       c_double, _dp, c_void_p, c_size_t, c_void_p]),
    "chz_helmholtz_solve_refined": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp,
                                            c_double, c_double, c_int, c_int, _dp, _dp,
                                            c_double, c_double, c_int, c_int, _dp, _dp,
                                            c_double, _dp, c_int, c_double,
                                            ctypes.POINTER(c_int), ctypes.POINTER(c_double),
                                            c_void_p, c_size_t, c_void_p]),
    "chz_helmholtz_adjoint_workspace_size": (c_size_t, [c_int, c_int, c_int, c_int]),
    "chz_helmholtz_adjoint": (c_int, [c_double, c_double, c_int, c_int, c_double, c_double, c_int, c_int,
                                      c_double, c_double, c_int, c_int, c_double,
                                      _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                      c_int, c_int, c_void_p, c_size_t, c_void_p]),
    "chz_batch_plan_create": (c_int, [c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                      ctypes.POINTER(c_double), ctypes.POINTER(c_double),
                                      ctypes.POINTER(c_void_p)]),
    "chz_batch_solve": (c_int, [c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), c_void_p]),
    "chz_batch_workspace_bytes": (c_size_t, [c_void_p]),
    "chz_batch_plan_destroy": (c_int, [c_void_p]),
    "chz_batch_set_autotune": (c_int, [c_int]),
    "chz_batch_plan_tiles": (c_int, [c_void_p, c_void_p, c_void_p]),
    "chz_batch_plan_radix": (c_int, [c_void_p, c_void_p]),
    "chz_batch_set_radix_schedule": (c_int, [c_int]),
    "chz_batch_plan_launch": (c_int, [c_void_p, c_void_p, c_void_p]),
    "chz_batch_set_launch_mode": (c_int, [c_int]),
    "chz_batch_plan_kernels": (c_int, [c_void_p]),
    "chz_helmholtz_solve_noalloc": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp,
                                            c_double, c_double, c_int, c_int, _dp, _dp,
                                            c_double, c_double, c_int, c_int, _dp, _dp,
                                            c_double, _dp, c_void_p]),
    "chz_release_cached": (c_int, []),
    "chz_trace_enable": (c_int, [c_int]),
    "chz_trace_collect": (c_int, [c_char_p, c_size_t]),
    "chz_launch_count": (ctypes.c_ulonglong, []),
    "chz_set_kernel_family": (c_int, [c_int]),
    "chz_debug_flags": (c_int, [c_int]),
    "chz_stream_status": (c_int, [c_void_p]),
    "chz_slab_forward": (c_int, [c_double, c_double, c_int, c_int, _dp, _dp, c_double, c_double, c_int, c_int,
                                 _dp, _dp, c_double, c_double, c_int, c_int, _dp, _dp, _dp, c_int, c_int, _dp,
                                 c_void_p]),
    "chz_slab_z": (c_int, [c_double, c_double, c_int, c_int, c_double, c_double, c_int, c_int, c_double,
                           c_double, c_int, c_int, c_double, _dp, c_int, c_int, c_void_p]),
    "chz_slab_inverse": (c_int, [c_double, c_double, c_int, c_int, c_double, c_double, c_int, c_int, c_double,
                                 c_double, c_int, c_int, _dp, _dp, c_int, c_int, c_void_p]),
    "chz_slab_work_elems": (c_size_t, [c_int, c_int, c_int]),
    "chz_set_wait_limit": (ctypes.c_longlong, [ctypes.c_longlong]),
    "chz_wait_selftest": (c_int, [ctypes.c_longlong, c_void_p]),
}


class LibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded library (loaded once per process)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIBPATH):
            raise LibraryMissing(
                f"{LIBPATH} is not built; run `python -m cuhelmholtz_b200._build` "
                "(the CUDA path has no CPU fallback)")
        handle = ctypes.CDLL(LIBPATH, mode=ctypes.RTLD_GLOBAL)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def library_path() -> str:
    return LIBPATH


def trace_enable(on: bool = True) -> None:
    lib().chz_trace_enable(1 if on else 0)


def trace_collect() -> dict:
    """{label: (launches, total_ms)} for the launches recorded since tracing
    was enabled (waits for them)."""
    buf = ctypes.create_string_buffer(1 << 16)
    n = lib().chz_trace_collect(buf, len(buf))
    if n < 0:
        raise RuntimeError("chz_trace_collect failed")
    out = {}
    for line in buf.value.decode().splitlines():
        label, cnt, ms = line.split()
        out[label] = (int(cnt), float(ms))
    return out


def launch_count() -> int:
    return int(lib().chz_launch_count())
