"""Loader of the in-tree CUDA library ``libkraken_b200.so`` (the C ABI of
include/kraken_b200.h).  There is no fallback: if the library is missing or
fails to load, every GPU entry point raises."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkraken_b200.so")

KR_OK = 0
KR_ERR_INVALID = 1
KR_ERR_INDEX = 2
KR_ERR_CUDA = 3
KR_ERR_CAPACITY = 4
KR_ERR_STATE = 5
KR_ERR_NODEVICE = 6


class KrError(RuntimeError):
    """A C-ABI call returned a non-zero status; ``code`` is the KR_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class SolverParams(C.Structure):
    _fields_ = [("h", C.c_double), ("substeps", C.c_int32), ("iterations", C.c_int32),
                ("lin_drag", C.c_double), ("ang_drag", C.c_double),
                ("max_speed", C.c_double), ("max_ang_speed", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -c 'import kraken_3_gpu_b200.build as b; b.build()')")
    L = C.CDLL(LIB_PATH)
    vp, i32, u32, fp = C.c_void_p, C.c_int32, C.c_uint32, C.POINTER(C.c_float)
    u32p = C.POINTER(C.c_uint32)
    sigs = {
        "kr_device_count": (C.c_int, []),
        "kr_create": (C.c_int, [C.POINTER(SolverParams), u32, u32, fp, u32, u32p, u32, u32p,
                                C.POINTER(vp)]),
        "kr_upload": (C.c_int, [vp, fp, u32p, fp, u32p]),
        "kr_upload_controls": (C.c_int, [vp, u32p]),
        "kr_step": (C.c_int, [vp, i32]),
        "kr_download": (C.c_int, [vp, fp, u32p]),
        "kr_sync": (C.c_int, [vp]),
        "kr_set_stream": (C.c_int, [vp, vp]),
        "kr_world_islands": (C.c_int, [vp, C.POINTER(i32), C.POINTER(i32)]),
        "kr_destroy": (None, [vp]),
        "kr_last_error": (C.c_char_p, [vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc: int, handle=None):
    if rc != KR_OK:
        msg = lib().kr_last_error(handle)
        raise KrError(rc, msg.decode() if msg else f"status {rc}")
