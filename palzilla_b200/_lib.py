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

class Float3(C.Structure):
    _fields_ = [("x", f32), ("y", f32), ("z", f32)]


class RayGenerator(C.Structure):
    _fields_ = [("origin", Float3), ("right", Float3), ("up", Float3)]


class LensParams(C.Structure):
    _fields_ = [("distance", f32), ("thickness", f32), ("R", f32)]


class TextureRGBX(C.Structure):
    _fields_ = [("texels_dev", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


class BatchTuning(C.Structure):
    _fields_ = [("p1_blocks_per_sm", C.c_int), ("p2_blocks_per_sm", C.c_int), ("p2_chunk", C.c_int)]


class SubdivParams(C.Structure):
    _fields_ = [("max_depth", C.c_int), ("eps", C.c_float), ("max_iterations", C.c_int),
                ("cost_tolerance", C.c_float), ("early_term_warmup", C.c_int), ("fp64_polish", C.c_int)]


class SubdivStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("boxes_tested", "boxes_culled", "leaves", "bins_excluded", "solves",
                                          "converged", "outside_box", "roots", "polished")]


class SolveDesc(C.Structure):
    _fields_ = [("K", i32), ("events", u32), ("paths", vp), ("n_paths", u64), ("first_diffuse", vp),
                ("internals", vp), ("root", vp), ("triangles", vp), ("attribs", vp), ("cache", vp),
                ("cache_capacity", u32), ("cell_step", f32), ("p_light", Float3), ("light_intensity", f32),
                ("radiance_clamp", f32), ("cauchy_a", f32), ("cauchy_b", f32), ("accum", vp), ("spectral", vp),
                ("etas", vp), ("n_bins", i32), ("max_iterations", i32), ("cost_tolerance", f32),
                ("early_term_warmup", i32), ("stats", vp), ("fma_contraction", i32), ("polish_det", f32),
                ("continuation", i32), ("fold_det", f32), ("graze_cos", f32), ("roots", vp)]


def f3(v) -> Float3:
    return Float3(float(v[0]), float(v[1]), float(v[2]))


# name -> (restype, argtypes); mirrors include/palzilla_b200.h
SIGNATURES = {
    "pz_version": (i32, []),
    "pz_last_error": (C.c_char_p, []),
    "pz_scratch_status": (i32, [vp, C.POINTER(u32), vp]),
    "pz_onesweep_scratch_bytes": (sz, [u32]),
    "pz_onesweep_sort": (i32, [vp, vp, vp, vp, u32, i32, i32, i32, vp, sz, vp]),
    "pz_onesweep_sort_static": (i32, [vp, vp, vp, vp, u32, i32, i32, i32, vp, vp]),
    "pz_bvh_scratch_bytes": (sz, [i32]),
    "pz_bvh_build": (i32, [vp, i32, u32, vp, vp, vp, sz, vp]),
    "pz_bvh_debug_views": (i32, [vp, i32, C.POINTER(vp), C.POINTER(vp), vp, vp]),
    "pz_trace_closest": (i32, [vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
    "pz_trace_any": (i32, [vp, vp, vp, i32, vp, vp, vp, vp, vp]),
    "pz_path_cache_bytes": (sz, [u32]),
    "pz_path_cache_clear": (i32, [vp, u32, vp]),
    "pz_path_cache_views": (i32, [vp, u32, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                  C.POINTER(vp), C.POINTER(vp)]),
    "pz_photon_trace": (i32, [vp, vp, vp, vp, i32, i32, Float3, f32, f32, i32, f32, vp, u32, f32, vp, vp]),
    "pz_ray_generator_lookat": (None, [C.POINTER(RayGenerator), Float3, Float3, Float3, f32, i32, i32]),
    "pz_solve_primary": (i32, [vp, vp, i32, i32, C.POINTER(RayGenerator), C.POINTER(LensParams), vp, vp, vp, vp,
                               Float3, f32, f32, f32, f32, Float3, C.POINTER(TextureRGBX), i32, vp, vp]),
    "pz_lookup_flatten": (i32, [u32, vp, vp, vp, u32, vp, i32, vp, u32, f32, vp]),
    "pz_reorder_specular_paths": (i32, [vp, vp, vp, u32, vp]),
    "pz_solve_specular_plain": (i32, [C.POINTER(SolveDesc), vp]),
    "pz_solve_constraints": (i32, [i32, u32, Float3, vp, vp, vp, u32, vp, vp, u32, i32, f32, i32, vp, vp, vp, vp]),
    "pz_solve_batched_scratch_bytes": (sz, [i32, u64, i32]),
    "pz_solve_specular_batched": (i32, [C.POINTER(SolveDesc), vp, vp, sz, i32, vp]),
    "pz_solve_multi_scratch_bytes": (sz, [i32, i32, u32, u64]),
    "pz_solve_multi_prepare": (i32, [vp, vp, u32, vp, sz, vp]),
    "pz_solve_specular_multi": (i32, [i32, i32, u32, u64, vp, sz, vp, vp, vp]),
    "pz_solve_multi_autotune": (i32, [i32, i32, u32, u64, vp, sz, vp, vp, vp, vp]),
    "pz_normal_bounds": (i32, [vp, i32, vp, vp, vp]),
    "pz_path_cuts_scratch_bytes": (sz, [i32, u32]),
    "pz_path_cuts": (i32, [i32, u32, f32, Float3, vp, u32, vp, vp, vp, vp, vp, i32, vp, u32, C.POINTER(u64),
                           C.POINTER(u64), vp, sz, vp]),
    "pz_subdivide_scratch_bytes": (sz, [u64]),
    "pz_subdivide_solve": (i32, [i32, u32, Float3, vp, vp, u32, vp, i32, C.POINTER(SubdivParams), vp, vp, vp, vp, vp,
                                 vp, u64, C.POINTER(u64), C.POINTER(SubdivStats), vp, sz, vp]),
    "pz_subdivide_contribute": (i32, [i32, u32, Float3, f32, f32, vp, vp, u64, vp, vp, i32, vp, vp, vp, vp]),
    "pz_adjoint_forward": (i32, [C.POINTER(SolveDesc), vp]),
    "pz_adjoint_backward": (i32, [C.POINTER(SolveDesc), vp, vp, vp, vp, vp]),
    "pz_adjoint_scratch_bytes": (sz, [u64]),
    "pz_adjoint_backward_compact": (i32, [C.POINTER(SolveDesc), vp, vp, vp, vp, vp, sz, vp]),
    "pz_resolve": (i32, [vp, vp, i32, vp]),
    "pz_resolve_spectral": (i32, [vp, vp, vp, i32, i32, f32, f32, Float3, vp]),
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
    if SIGNATURES[name][0] is i32:
        check(r, name)
    return r
