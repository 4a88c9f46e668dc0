"""ctypes binding of libpalzilla_b200.so (the C ABI in include/palzilla_b200.h).

The library is required: importing the package does not fail without it, but
the first call to ``lib()`` raises if the .so is missing or cannot be loaded,
so no code path silently falls back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpalzilla_b200.so")

PZ_OK = 0

vp = C.c_void_p
u32 = C.c_uint32
i32 = C.c_int
f32 = C.c_float
sz = C.c_size_t
i64 = C.c_int64
u64 = C.c_uint64

# name -> (restype, argtypes); mirrors include/palzilla_b200.h
SIGNATURES = {
    "pz_version": (i32, []),
    "pz_last_error": (C.c_char_p, []),
    "pz_scratch_status": (i32, [vp, C.POINTER(u32), vp]),
    "pz_onesweep_scratch_bytes": (sz, [u32]),
    "pz_onesweep_sort": (i32, [vp, vp, vp, vp, u32, i32, i32, i32, vp, sz, vp]),
    "pz_bvh_scratch_bytes": (sz, [i32]),
    "pz_bvh_build": (i32, [vp, i32, u32, vp, vp, vp, sz, vp]),
    "pz_bvh_debug_views": (i32, [vp, i32, C.POINTER(vp), C.POINTER(vp), vp, vp]),
}

_lib = None


class PzError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"palzilla_b200 CUDA library not built: {LIB_PATH} is missing "
                               "(run `python -m palzilla_b200.build`)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int, where: str) -> None:
    if code != PZ_OK:
        msg = lib().pz_last_error().decode(errors="replace")
        raise PzError(code, where, msg)


def call(name: str, *args):
    r = getattr(lib(), name)(*args)
    check(r, name)
    return r
