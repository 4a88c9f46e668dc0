"""TEST INFRASTRUCTURE ONLY: the reference's own GPU kernels on the device.

``oracle/_ref/libpzref_gpu.so`` (the compiler's default FMA contraction, as the reference's
run-time compile builds its kernels) and ``oracle/_ref/libpzref_gpu_exact.so``
(-fmad=false: the reference's CPU float arithmetic) hold minimum_lbvh.cu and main_gpu.cu
compiled from the reference sources by ``oracle/build_ref_gpu.sh``, with host launchers
that replace Orochi (``oracle/ref_gpu_main.cu``).  Buffers are torch cuda tensors.  Only
tests/ and bench.py's reference-kernel workload use this module; the product path never
does.  The reference's onesweep reorder is not run (it takes its tile index from
blockIdx.x and spins without bound on its predecessors, tinyhiponesweep.h:341-381): the
LBVH build here sorts its keys with a stable sort passed in by the caller.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {"default": os.path.join(HERE, "_ref", "libpzref_gpu.so"),
        "exact": os.path.join(HERE, "_ref", "libpzref_gpu_exact.so")}

vp, i32, u32, f32 = C.c_void_p, C.c_int, C.c_uint32, C.c_float
SIGNATURES = {
    "pzg_path_cache_capacity": (i32, []),
    "pzg_triangle_path_bytes": (i32, []),
    "pzg_stack_buffer_bytes": (C.c_size_t, []),
    "pzg_scene_aabb": (i32, [vp, vp, i32, vp]),
    "pzg_build_mortons": (i32, [vp, vp, i32, vp, u32, vp]),
    "pzg_deltas_and_build": (i32, [vp, vp, vp, vp, i32, vp, vp]),
    "pzg_photon_trace": (i32, [vp, vp, vp, vp, i32, vp, f32, f32, i32, vp, vp, vp, f32, f32, vp, vp]),
    "pzg_lookup_flatten": (i32, [u32, vp, vp, vp, vp, i32, i32, vp, vp, vp, f32, vp]),
    "pzg_reorder": (i32, [vp, vp, vp, i32, vp]),
    "pzg_solve_specular": (i32, [i32, vp, vp, u32, vp, vp, vp, vp, vp, vp, f32, f32, vp, vp, vp, f32, u32, f32, f32,
                                 i32, vp]),
    "pzg_pack": (i32, [vp, vp, i32, vp]),
}


def available(variant: str = "exact") -> bool:
    return os.path.exists(LIBS[variant])


def _p(t):
    return C.c_void_p(None if t is None else t.data_ptr())


class RefGpu:
    """The reference's kernels from one of the two builds ("default" or "exact")."""

    def __init__(self, variant: str = "exact"):
        import torch
        self.torch = torch
        self.lib = C.CDLL(LIBS[variant])
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(self.lib, name)
            fn.restype = res
            fn.argtypes = args
        self.capacity = self.lib.pzg_path_cache_capacity()
        assert self.lib.pzg_triangle_path_bytes() == 56

    def _check(self, rc, where):
        if rc != 0:
            raise RuntimeError(f"{where}: CUDA error {rc}")

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    # ---------------------------------------------------------------- LBVH
    def bvh_build(self, tris, n: int, sort_keys, build_option: int = 0):
        """BVHGPUBuilder::build (minimum_lbvh.h:798-886) on the reference's kernels; the keys
        {morton (low 32 bits), index (high 32)} are sorted by sort_keys(keys, tmp, n) (stable on
        the low 32 bits, as the reference's onesweep sorts them).  Returns (nodes uint8 tensor,
        root int32 tensor of one element, sorted keys, deltas)."""
        torch = self.torch
        dev = tris.device
        aabb = torch.empty(6, dtype=torch.float32, device=dev)
        keys = torch.empty(n, dtype=torch.int64, device=dev)
        tmp = torch.empty_like(keys)
        deltas = torch.empty(max(n - 1, 1), dtype=torch.uint8, device=dev)
        nodes = torch.empty(max(n - 1, 1) * 64, dtype=torch.uint8, device=dev)
        root = torch.zeros(1, dtype=torch.int32, device=dev)
        s = self._stream()
        self._check(self.lib.pzg_scene_aabb(_p(aabb), _p(tris), n, s), "getSceneAABB")
        self._check(self.lib.pzg_build_mortons(_p(keys), _p(tris), n, _p(aabb), build_option, s), "buildMortons")
        sort_keys(keys, tmp, n)
        self._check(self.lib.pzg_deltas_and_build(_p(root), _p(nodes), _p(deltas), _p(tris), n, _p(keys), s),
                    "computeDeltas + build")
        return nodes, root, keys, deltas

    # ---------------------------------------------------------------- PathCache
    def new_cache(self, device="cuda"):
        """The reference's PathCache buffers (pk.h:227-402), cleared: hashes u32[2^22],
        TrianglePath[2^22] (56 bytes: hashOfP, eDescriptor, tris[4], parameters[8]), count."""
        torch = self.torch
        return {"hashes": torch.zeros(self.capacity, dtype=torch.int32, device=device),
                "paths": torch.zeros((self.capacity, 14), dtype=torch.int32, device=device),
                "count": torch.zeros(1, dtype=torch.int32, device=device)}

    def cache_from_ours(self, views):
        """The reference's array-of-structs PathCache image of this library's PathCache
        (pz_path_cache_views of a 2^22-slot cache)."""
        torch = self.torch
        cap = self.capacity
        assert views["hash"].numel() == cap
        paths = torch.cat([views["cell"].view(cap, 1), views["events"].view(cap, 1), views["tris"].view(cap, 4),
                           views["params"].view(torch.int32).view(cap, 8)], 1).contiguous()
        return {"hashes": views["hash"].clone(), "paths": paths, "count": views["count"].clone()}

    def photon_trace(self, cache, nodes, root, tris, attribs, n_tris, p_light, eta_min, eta_max, iteration,
                     step, min_throughput, stack):
        import numpy as np
        pl = np.asarray(p_light, np.float32)
        self._check(self.lib.pzg_photon_trace(_p(root), _p(nodes), _p(tris), _p(attribs), n_tris,
                                              pl.ctypes.data_as(C.c_void_p), eta_min, eta_max, iteration,
                                              _p(cache["hashes"]), _p(cache["paths"]), _p(cache["count"]), step,
                                              min_throughput, _p(stack), self._stream()), "photonTrace")

    def new_stack(self, device="cuda"):
        """StackBufferAllocator's buffer (pk.h:1119-1126): 65536 warps x 32 x 128 NodeIndex, zeroed."""
        return self.torch.zeros(self.lib.pzg_stack_buffer_bytes(), dtype=self.torch.uint8, device=device)

    def lookup_flatten(self, events, paths, indexed, counter, fds, width, height, cache, step):
        self._check(self.lib.pzg_lookup_flatten(events, _p(paths), _p(indexed), _p(counter), _p(fds), width, height,
                                                _p(cache["hashes"]), _p(cache["paths"]), _p(cache["count"]), step,
                                                self._stream()), "lookupFlatten")

    def solve_specular(self, K, accum, paths, n, fds, root, nodes, tris, attribs, p_light, light_intensity,
                       radiance_clamp, cache, step, events, cauchy_a, cauchy_b, iteration=0):
        import numpy as np
        pl = np.asarray(p_light, np.float32)
        self._check(self.lib.pzg_solve_specular(K, _p(accum), _p(paths), n, _p(fds), _p(root), _p(nodes), _p(tris),
                                                _p(attribs), pl.ctypes.data_as(C.c_void_p), light_intensity,
                                                radiance_clamp, _p(cache["hashes"]), _p(cache["paths"]),
                                                _p(cache["count"]), step, events, cauchy_a, cauchy_b, iteration,
                                                self._stream()), f"solveSpecularPath_K{K}")


def build() -> bool:
    """Compile both libraries when the reference sources are present and a library is missing
    or older than the launchers; True if they exist."""
    import subprocess
    from oracle import ref_dir
    srcs = [os.path.join(HERE, f) for f in ("ref_gpu_main.cu", "ref_gpu_lbvh.cu", "build_ref_gpu.sh")]
    stale = any(not os.path.exists(p) or os.path.getmtime(p) < max(map(os.path.getmtime, srcs))
                for p in LIBS.values())
    if stale and os.path.isdir(ref_dir()):
        subprocess.run([os.path.join(HERE, "build_ref_gpu.sh")], check=True, stdout=subprocess.DEVNULL,
                       env=dict(os.environ, REF_DIR=ref_dir()))
    return available("default") and available("exact")
