"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the CPU oracle.

Two libraries expose the same function shapes:

* ``oracle/libpz_oracle.so`` (prefix ``pzo_``) -- this repository's CPU restatement
  of the reference algorithm (``oracle/pz_oracle.hpp``), float and FP64;
* ``oracle/_ref/libpzref.so`` (prefix ``pzr_``) -- the reference's own CPU code,
  compiled from its sources by ``oracle/build_ref.sh`` (only when the reference
  is present at build time).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use this
module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libpz_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpzref.so")

NODE_DTYPE = np.dtype([("children", "<u4", (2,)), ("aabbs", "<f4", (2, 6)), ("parent", "<u4"), ("context", "<u4")])
assert NODE_DTYPE.itemsize == 64
NORMAL_BOUND_DTYPE = np.dtype([("bounds", "<f4", (2, 6)), ("counter", "<u4")])
assert NORMAL_BOUND_DTYPE.itemsize == 52
ROOT_DTYPE = np.dtype([("tuple", "<u4"), ("bin", "<u4"), ("depth", "<u4"), ("path", "<u4"), ("params", "<f4", (8,)),
                       ("throughput", "<f4"), ("pad", "<u4", (3,))])
assert ROOT_DTYPE.itemsize == 64
RECORD_DTYPE = np.dtype([("ev", "<u4"), ("tris", "<i4", (4,)), ("params", "<f4", (8,)), ("p", "<f4", (3,))])
assert RECORD_DTYPE.itemsize == 64
INVALID_NODE = 0x7FFFFFFF


def _light(scene, iteration: int) -> np.ndarray:
    """The scene's light point at this iteration (one sample of an area light)."""
    p = scene.light_point(iteration) if hasattr(scene, "light_point") else scene.p_light
    return np.asarray(p, np.float32)


def build_oracle(force: bool = False) -> None:
    """Compile the restatement library (make in oracle/)."""
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < max(
            os.path.getmtime(os.path.join(HERE, f)) for f in ("pz_oracle.hpp", "pz_oracle_subdiv.hpp", "pz_oracle_capi.cpp")):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)


def ref_dir() -> str:
    """Where the reference sources are looked for: $REF_DIR, else a directory named
    "reference" beside this repository's root."""
    return os.environ.get("REF_DIR", os.path.normpath(os.path.join(HERE, "..", "..", "reference")))


def build_ref() -> bool:
    """Compile the reference's CPU code (and its GPU kernels, oracle/ref_gpu.py) when its
    sources are present; True if the CPU library exists."""
    script = os.path.join(HERE, "build_ref.sh")
    if os.path.isdir(ref_dir()):
        subprocess.run([script], check=True, stdout=subprocess.DEVNULL, env=dict(os.environ, REF_DIR=ref_dir()))
        import ref_gpu
        ref_gpu.build()
    return os.path.exists(REF_SO)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class CpuLib:
    """Numpy-facing wrapper; ``prefix`` is "pzo" (restatement) or "pzr" (reference)."""

    def __init__(self, path: str, prefix: str):
        self.lib = C.CDLL(path)
        self.prefix = prefix
        self.path = path

    def f(self, name, restype=None):
        fn = getattr(self.lib, f"{self.prefix}_{name}")
        fn.restype = restype
        return fn

    def has(self, name) -> bool:
        return hasattr(self.lib, f"{self.prefix}_{name}")

    def set_threads(self, n: int) -> None:
        self.f("set_threads")(C.c_int(n))

    def max_threads(self) -> int:
        return self.f("max_threads", C.c_int)()

    # ------------------------------------------------------------------ LBVH
    def build_bvh(self, tris: np.ndarray, opt: int = 0):
        tris = np.ascontiguousarray(tris, np.float32)
        n = tris.shape[0]
        nodes = np.zeros(max(n - 1, 0), NODE_DTYPE)
        root = np.zeros(1, np.uint32)
        sorted_ = np.zeros(n, np.uint64)
        deltas = np.zeros(max(n - 1, 0), np.uint8)
        aabb = np.zeros(6, np.float32)
        self.f("build_bvh", C.c_int)(_p(tris), C.c_int(n), C.c_uint32(opt), _p(nodes), _p(root), _p(sorted_),
                                     _p(deltas), _p(aabb))
        return dict(nodes=nodes, root=int(root[0]), sorted=sorted_, deltas=deltas, aabb=aabb)

    def cpu_builder(self, tris: np.ndarray, opt: int = 0):
        tris = np.ascontiguousarray(tris, np.float32)
        n = tris.shape[0]
        nodes = np.zeros(max(n - 1, 0), NODE_DTYPE)
        root = np.zeros(1, np.uint32)
        self.f("cpu_builder", C.c_int)(_p(tris), C.c_int(n), C.c_uint32(opt), _p(nodes), _p(root))
        return dict(nodes=nodes, root=int(root[0]))

    def morton_keys(self, tris, aabb, opt=0):
        tris = np.ascontiguousarray(tris, np.float32)
        keys = np.zeros(tris.shape[0], np.uint32)
        self.f("morton_keys")(_p(tris), C.c_int(tris.shape[0]), C.c_uint32(opt), _p(np.asarray(aabb, np.float32)),
                              _p(keys))
        return keys

    def stable_sort_u64(self, keys, start_bit=0, end_bit=32):
        k = np.array(keys, np.uint64)
        self.f("stable_sort_u64")(_p(k), C.c_uint32(k.size), C.c_int(start_bit), C.c_int(end_bit))
        return k

    def stable_sort_u32(self, keys, start_bit=0, end_bit=32):
        k = np.array(keys, np.uint32)
        self.f("stable_sort_u32")(_p(k), C.c_uint32(k.size), C.c_int(start_bit), C.c_int(end_bit))
        return k

    def stable_sort_kv(self, keys, values, start_bit=0, end_bit=32):
        k = np.array(keys)
        v = np.array(values, np.uint32)
        self.f("stable_sort_kv")(_p(k), _p(v), C.c_uint32(k.size), C.c_int(k.itemsize), C.c_int(start_bit),
                                 C.c_int(end_bit))
        return k, v

    def validate_lbvh(self, nodes, root, deltas) -> bool:
        return bool(self.f("validate_lbvh", C.c_int)(_p(nodes), C.c_uint32(root), _p(deltas)))

    # ------------------------------------------------------------------ rays
    def trace_closest(self, nodes, root, tris, ro, rd):
        ro = np.ascontiguousarray(ro, np.float32)
        rd = np.ascontiguousarray(rd, np.float32)
        n = ro.shape[0]
        t = np.zeros(n, np.float32)
        uv = np.zeros((n, 2), np.float32)
        tri = np.zeros(n, np.uint32)
        ng = np.zeros((n, 3), np.float32)
        self.f("trace_closest")(_p(nodes), C.c_uint32(root), _p(np.ascontiguousarray(tris, np.float32)), C.c_int(n),
                                _p(ro), _p(rd), _p(t), _p(uv), _p(tri), _p(ng))
        return dict(t=t, uv=uv, tri=tri, ng=ng)

    def trace_any(self, nodes, root, tris, ro, rd, tmax):
        ro = np.ascontiguousarray(ro, np.float32)
        rd = np.ascontiguousarray(rd, np.float32)
        tmax = np.ascontiguousarray(tmax, np.float32)
        hit = np.zeros(ro.shape[0], np.uint8)
        self.f("trace_any")(_p(nodes), C.c_uint32(root), _p(np.ascontiguousarray(tris, np.float32)),
                            C.c_int(ro.shape[0]), _p(ro), _p(rd), _p(tmax), _p(hit))
        return hit

    # ------------------------------------------------------------------ photons / cache
    def photon_trace(self, bvh, scene, iteration=0, photons_per_tri=None, capacity=None, eta_range=None):
        ppt = photons_per_tri or scene.photons_per_triangle
        cap = capacity or scene.n * ppt
        out = np.zeros(cap, RECORD_DTYPE)
        emin, emax = eta_range or scene.eta_range()
        n = self.f("photon_trace", C.c_int64)(
            _p(bvh["nodes"]), C.c_uint32(bvh["root"]), _p(scene.tris), _p(scene.attribs), C.c_int(scene.n),
            _p(_light(scene, iteration)), C.c_float(emin), C.c_float(emax), C.c_int(iteration),
            C.c_float(scene.min_throughput), C.c_int(ppt), _p(out), C.c_int64(cap))
        if n < 0:
            raise RuntimeError("photon record capacity exceeded")
        return out[:n]

    def cache_build(self, records, capacity=1 << 22, step=0.01):
        recs = np.ascontiguousarray(records, RECORD_DTYPE)
        h = np.zeros(capacity, np.uint32)
        cell = np.zeros(capacity, np.uint32)
        ev = np.zeros(capacity, np.uint32)
        tris = np.zeros((capacity, 4), np.int32)
        prm = np.zeros((capacity, 8), np.float32)
        cnt = self.f("cache_build", C.c_int64)(_p(recs), C.c_int64(recs.size), C.c_uint32(capacity),
                                               C.c_float(step), _p(h), _p(cell), _p(ev), _p(tris), _p(prm))
        return dict(hash=h, cell=cell, events=ev, tris=tris, params=prm, count=int(cnt), capacity=capacity, step=step)

    def lookup_flatten(self, cache, p, valid, ev, pair_cap=None):
        p = np.ascontiguousarray(p, np.float32).reshape(-1, 3)
        valid = np.ascontiguousarray(valid, np.uint8)
        npx = p.shape[0]
        counts = np.zeros(npx, np.int32)
        cap = pair_cap or 1 << 24
        pairs = np.zeros((cap, 2), np.int32)
        n = self.f("lookup_flatten", C.c_int64)(
            _p(cache["hash"]), _p(cache["cell"]), _p(cache["events"]), C.c_uint32(cache["capacity"]),
            C.c_float(cache["step"]), _p(p), _p(valid), C.c_int(npx), C.c_uint32(ev), _p(counts), _p(pairs),
            C.c_int64(cap))
        if n < 0:
            raise RuntimeError("pair capacity exceeded")
        return counts, pairs[:n].copy()

    # ------------------------------------------------------------------ camera / eye pass
    def lookat(self, eye, center, up, fovy, w, h):
        out = np.zeros(9, np.float32)
        self.f("lookat")(_p(np.asarray(eye, np.float32)), _p(np.asarray(center, np.float32)),
                         _p(np.asarray(up, np.float32)), C.c_float(fovy), C.c_int(w), C.c_int(h), _p(out))
        return out

    def solve_primary(self, bvh, scene, ray_gen, iteration=0, lens=(0.6, 0.05, 0.0), texture=None):
        """solvePrimary (main_gpu.cu:213-371); texture: an optional floor texture, uint8 array
        (height, width, 4), sampled as Texture8RGBX (pk.h:1075-1098)."""
        W, H = scene.width, scene.height
        accum = np.zeros((H * W, 4), np.float32)
        fd = np.zeros((H * W, 10), np.float32)
        tex = None if texture is None else np.ascontiguousarray(texture, np.uint8)
        self.f("solve_primary")(_p(accum), _p(fd), C.c_int(W), C.c_int(H), _p(np.asarray(ray_gen, np.float32)),
                                _p(np.asarray(lens, np.float32)), _p(bvh["nodes"]), C.c_uint32(bvh["root"]),
                                _p(scene.tris), _p(scene.attribs), _p(_light(scene, iteration)),
                                C.c_float(scene.light_intensity), C.c_float(scene.radiance_clamp),
                                C.c_float(scene.cauchy_a), C.c_float(scene.cauchy_b),
                                _p(np.asarray(scene.albedo, np.float32)), _p(tex),
                                C.c_int(0 if tex is None else tex.shape[1]), C.c_int(0 if tex is None else tex.shape[0]),
                                C.c_int(iteration))
        return accum, fd

    # ------------------------------------------------------------------ solver primitives
    def count_newton_flops(self, K, params, p_beg, p_end, tris, attribs, eta, ev):
        """Floating-point operations of one Newton iteration of the restated
        solveConstraints<K> (pk.h:466-592), counted with a counting scalar type (oracle
        library only): {"add", "mul", "div", "sqrt", "total"}."""
        out = np.zeros(4, np.uint64)
        r = self.f("count_newton_flops", C.c_int)(
            C.c_int(K), _p(np.ascontiguousarray(params, np.float32)), _p(np.asarray(p_beg, np.float32)),
            _p(np.asarray(p_end, np.float32)), _p(np.ascontiguousarray(tris, np.float32)),
            _p(np.ascontiguousarray(attribs)), C.c_float(eta), C.c_uint32(ev), _p(out))
        if r != 0:
            raise ValueError("K must be 1..4")
        c = dict(zip(("add", "mul", "div", "sqrt"), (int(v) for v in out)))
        c["total"] = sum(c.values())
        return c

    def solve_constraints(self, K, params, p_beg, p_end, tris, attribs, eta, ev, max_iter=32, tol=1e-10, warmup=1,
                          dtype=np.float32):
        prm = np.array(params, dtype)
        tr = np.ascontiguousarray(tris, np.float32)
        at = np.ascontiguousarray(attribs)
        it = C.c_int(0)
        if self.prefix == "pzo":
            ok = self.f("solve_constraints", C.c_int)(
                C.c_int(K), C.c_int(0 if dtype == np.float32 else 1), _p(prm), _p(np.asarray(p_beg, np.float64)),
                _p(np.asarray(p_end, np.float64)), _p(tr), _p(at), C.c_double(eta), C.c_uint32(ev), C.c_int(max_iter),
                C.c_double(tol), C.c_int(warmup), C.byref(it))
        else:
            assert dtype == np.float32
            ok = self.f("solve_constraints", C.c_int)(
                C.c_int(K), _p(prm), _p(np.asarray(p_beg, np.float32)), _p(np.asarray(p_end, np.float32)), _p(tr),
                _p(at), C.c_float(eta), C.c_uint32(ev), C.c_int(max_iter), C.c_float(tol), C.c_int(warmup),
                C.byref(it))
        return bool(ok), prm, it.value

    def contributable_throughput(self, K, params, p_beg, p_end, tris, attribs, ev, bvh, scene_tris, eta,
                                 dtype=np.float32):
        prm = np.array(params, dtype)
        if self.prefix == "pzo":
            return float(self.f("contributable_throughput", C.c_double)(
                C.c_int(K), C.c_int(0 if dtype == np.float32 else 1), _p(prm), _p(np.asarray(p_beg, np.float64)),
                _p(np.asarray(p_end, np.float64)), _p(np.ascontiguousarray(tris, np.float32)),
                _p(np.ascontiguousarray(attribs)), C.c_uint32(ev), _p(bvh["nodes"]), _p(scene_tris),
                C.c_uint32(bvh["root"]), C.c_double(eta)))
        return float(self.f("contributable_throughput", C.c_float)(
            C.c_int(K), _p(prm), _p(np.asarray(p_beg, np.float32)), _p(np.asarray(p_end, np.float32)),
            _p(np.ascontiguousarray(tris, np.float32)), _p(np.ascontiguousarray(attribs)), C.c_uint32(ev),
            _p(bvh["nodes"]), _p(scene_tris), C.c_uint32(bvh["root"]), C.c_float(eta)))

    def dAdw(self, ro, rd, p_end, tris, attribs, ev, eta, dtype=np.float32):
        if self.prefix == "pzo":
            return float(self.f("dAdw", C.c_double)(
                C.c_int(0 if dtype == np.float32 else 1), _p(np.asarray(ro, np.float64)),
                _p(np.asarray(rd, np.float64)), _p(np.asarray(p_end, np.float64)),
                _p(np.ascontiguousarray(tris, np.float32)), _p(np.ascontiguousarray(attribs)), C.c_uint32(ev),
                C.c_double(eta)))
        return float(self.f("dAdw", C.c_float)(
            _p(np.asarray(ro, np.float32)), _p(np.asarray(rd, np.float32)), _p(np.asarray(p_end, np.float32)),
            _p(np.ascontiguousarray(tris, np.float32)), _p(np.ascontiguousarray(attribs)), C.c_uint32(ev),
            C.c_float(eta)))

    def render_pairs(self, K, pairs, cache, first_diffuse, bvh, scene, etas, max_iter=32, tol=1e-10, warmup=1,
                     dtype=np.float32, iteration=0):
        pairs = np.ascontiguousarray(pairs, np.int32)
        etas = np.ascontiguousarray(etas, np.float32)
        nb = etas.size
        npx = first_diffuse.shape[0]
        spectral = np.zeros((npx, nb), np.float32)
        stats = np.zeros(3, np.int64)
        ev = scene.ev if hasattr(scene, "ev") else None
        from palzilla_b200.scenes import event_descriptor
        ev = event_descriptor(scene.events)
        args = [C.c_int(K)]
        if self.prefix == "pzo":
            args.append(C.c_int(0 if dtype == np.float32 else 1))
        args += [_p(pairs), C.c_int64(pairs.shape[0]), _p(cache["tris"]), _p(cache["params"]),
                 _p(np.ascontiguousarray(first_diffuse, np.float32)), _p(bvh["nodes"]), C.c_uint32(bvh["root"]),
                 _p(scene.tris), _p(scene.attribs), _p(_light(scene, iteration)),
                 C.c_float(scene.light_intensity), C.c_float(scene.radiance_clamp), C.c_uint32(ev), _p(etas),
                 C.c_int(nb), C.c_int(max_iter), C.c_float(tol), C.c_int(warmup), _p(spectral), _p(stats)]
        self.f("render_pairs", C.c_int)(*args)
        return spectral, stats

    def render_pairs_rgb(self, K, pairs, cache, first_diffuse, bvh, scene, max_iter=32, tol=1e-10, warmup=1,
                         dtype=np.float32, iteration=0):
        """The reference's own solve mode (solveSpecularPath<K>, main_gpu.cu:418-483): each
        (pixel, tuple) pair at its pixel's sampled wavelength, RGB added to a float4
        accumulator per pixel (w = 0 here).  Returns (accum (npx, 4), stats)."""
        pairs = np.ascontiguousarray(pairs, np.int32)
        fd = np.ascontiguousarray(first_diffuse, np.float32)
        accum = np.zeros((fd.shape[0], 4), np.float32)
        stats = np.zeros(3, np.int64)
        from palzilla_b200.scenes import event_descriptor
        args = [C.c_int(K)]
        if self.prefix == "pzo":
            args.append(C.c_int(0 if dtype == np.float32 else 1))
        args += [_p(pairs), C.c_int64(pairs.shape[0]), _p(cache["tris"]), _p(cache["params"]), _p(fd),
                 _p(bvh["nodes"]), C.c_uint32(bvh["root"]), _p(scene.tris), _p(scene.attribs),
                 _p(_light(scene, iteration)), C.c_float(scene.light_intensity), C.c_float(scene.radiance_clamp),
                 C.c_uint32(event_descriptor(scene.events)), C.c_float(scene.cauchy_a), C.c_float(scene.cauchy_b),
                 C.c_int(max_iter), C.c_float(tol), C.c_int(warmup), _p(accum), _p(stats)]
        self.f("render_pairs_rgb", C.c_int)(*args)
        return accum, stats

    def cmf(self, which: int, nm: np.ndarray) -> np.ndarray:
        """CIE 2015 10-degree functions (pk.h:960-1012): 0 x, 1 y, 2 z, 3 pdf of the sampled
        wavelength, 4 its inverse CDF."""
        fn = self.f("cmf", C.c_float)
        return np.array([fn(C.c_int(which), C.c_float(float(x))) for x in np.asarray(nm, np.float32)], np.float32)

    def pack(self, accum) -> np.ndarray:
        """pack (main_gpu.cu:499-513): RGBA8 of accumulator / count."""
        accum = np.ascontiguousarray(accum, np.float32)
        out = np.zeros(accum.shape[0], np.uint32)
        self.f("pack")(_p(accum), C.c_int(accum.shape[0]), _p(out))
        return out

    def resolve_spectral(self, spectral, lambda_min, lambda_max, albedo):
        """Binned spectral image -> (linear sRGB (n, 4), RGBA8 (n,))."""
        spectral = np.ascontiguousarray(spectral, np.float32)
        n, nb = spectral.shape
        rgb = np.zeros((n, 4), np.float32)
        px = np.zeros(n, np.uint32)
        self.f("resolve_spectral")(_p(spectral), C.c_int(n), C.c_int(nb), C.c_float(lambda_min),
                                   C.c_float(lambda_max), _p(np.asarray(albedo, np.float32)), _p(rgb), _p(px))
        return rgb, px

    def render_each(self, K, pairs, cache, first_diffuse, bvh, scene, etas, max_iter=32, tol=1e-10, warmup=1,
                    dtype=np.float64, iteration=0):
        """Contribution of every (pair, bin) before the clamp (0 = rejected), (n_pairs, n_bins) float64."""
        pairs = np.ascontiguousarray(pairs, np.int32)
        etas = np.ascontiguousarray(etas, np.float32)
        out = np.zeros((pairs.shape[0], etas.size), np.float64)
        from palzilla_b200.scenes import event_descriptor
        self.f("render_each", C.c_int)(
            C.c_int(K), C.c_int(0 if dtype == np.float32 else 1), _p(pairs), C.c_int64(pairs.shape[0]),
            _p(cache["tris"]), _p(cache["params"]), _p(np.ascontiguousarray(first_diffuse, np.float32)),
            _p(bvh["nodes"]), C.c_uint32(bvh["root"]), _p(scene.tris), _p(scene.attribs),
            _p(_light(scene, iteration)), C.c_float(scene.light_intensity),
            C.c_uint32(event_descriptor(scene.events)), _p(etas), C.c_int(etas.size), C.c_int(max_iter),
            C.c_float(tol), C.c_int(warmup), _p(out))
        return out

    # ------------------------------------------------------------------ interval / path cuts
    def interval_square(self, l, u):
        out = np.zeros(2, np.float32)
        self.f("interval_square")(_p(np.array([l, u], np.float32)), _p(out))
        return out

    def interval_normalize(self, box6):
        out = np.zeros(6, np.float32)
        self.f("interval_normalize")(_p(np.asarray(box6, np.float32)), _p(out))
        return out

    def fresnel(self, wi, n, eta):
        return float(self.f("fresnel", C.c_float)(_p(np.asarray(wi, np.float32)), _p(np.asarray(n, np.float32)),
                                                 C.c_float(eta)))

    def refract(self, wi, n, eta):
        wo = np.zeros(3, np.float32)
        ok = self.f("refract", C.c_int)(_p(np.asarray(wi, np.float32)), _p(np.asarray(n, np.float32)),
                                        C.c_float(eta), _p(wo))
        return bool(ok), wo

    def normal_bounds(self, nodes, tris, attribs):
        out = np.zeros(nodes.size, NORMAL_BOUND_DTYPE)
        self.f("normal_bounds")(_p(nodes), C.c_int(nodes.size), _p(tris), _p(attribs), _p(out))
        return out

    def path_cuts(self, K, ev, eta, p_beg, p_end, nodes, nbs, tris, attribs, root, cap=1 << 20):
        out = np.zeros((cap, K), np.int32)
        args = [C.c_int(K), C.c_uint32(ev), C.c_float(eta), _p(np.asarray(p_beg, np.float32)),
                _p(np.asarray(p_end, np.float32)), _p(nodes), _p(nbs), _p(tris), _p(attribs), C.c_uint32(root),
                _p(out), C.c_int64(cap)]
        if self.prefix == "pzo":
            visited = C.c_uint64(0)
            args.append(C.byref(visited))
        n = self.f("path_cuts", C.c_int64)(*args)
        if n < 0:
            raise RuntimeError("tuple capacity exceeded")
        return out[:n].copy()

    # ------------------------------------------------------------------ subdivision solve
    def subdivide_solve(self, K, ev, p_beg, p_end, tuples, etas, tris, attribs, bvh, scene_tris, max_depth=12,
                        eps=1e-4, max_iterations=32, cost_tolerance=1e-10, warm_up=1, cap=1 << 20):
        """Roots of the subdivision solve, sorted by (tuple, bin, depth, path), and the stats
        (tested, culled, leaves, bins excluded, solves, converged, outside, roots).  tuples
        index tris / attribs; visibility runs through bvh over scene_tris."""
        tuples = np.ascontiguousarray(tuples, np.uint32)
        etas = np.ascontiguousarray(etas, np.float32)
        out = np.zeros(cap, ROOT_DTYPE)
        stats = np.zeros(8, np.uint64)
        n = self.f("subdivide_solve", C.c_int64)(
            C.c_int(K), C.c_uint32(ev), _p(np.asarray(p_beg, np.float32)), _p(np.ascontiguousarray(p_end, np.float32)),
            _p(tuples), C.c_uint32(len(tuples)), _p(etas), C.c_int(len(etas)), C.c_int(max_depth), C.c_float(eps),
            C.c_int(max_iterations), C.c_float(cost_tolerance), C.c_int(warm_up),
            _p(np.ascontiguousarray(tris, np.float32)), _p(np.ascontiguousarray(attribs)), _p(bvh["nodes"]),
            _p(np.ascontiguousarray(scene_tris, np.float32)), C.c_uint32(bvh["root"]), _p(out), C.c_int64(cap),
            _p(stats))
        if n < 0:
            raise RuntimeError("root capacity exceeded")
        return out[:n].copy(), stats

    def directed(self, op: int, up: bool, a: float, b: float = 0.0) -> float:
        """One directed-rounding operation of the subdivision oracle (0 add, 1 sub, 2 mul,
        3 div downward, 4 sqrt)."""
        return float(self.f("directed", C.c_float)(C.c_int(op), C.c_int(1 if up else 0), C.c_float(a), C.c_float(b)))

    def subdivide_contribute(self, K, ev, scene, tuples, roots, first_diffuse, etas, tris, attribs, iteration=0):
        """Binned spectral image (pixels x bins) of subdivision roots; rows' query = pixel."""
        etas = np.ascontiguousarray(etas, np.float32)
        fd = np.ascontiguousarray(first_diffuse, np.float32)
        spectral = np.zeros((fd.shape[0], etas.size), np.float32)
        self.f("subdivide_contribute")(
            C.c_int(K), C.c_uint32(ev), _p(_light(scene, iteration)), C.c_float(scene.light_intensity),
            C.c_float(scene.radiance_clamp), _p(np.ascontiguousarray(tuples, np.uint32)),
            _p(np.ascontiguousarray(roots)), C.c_int64(len(roots)), _p(fd), _p(etas), C.c_int(etas.size),
            _p(np.ascontiguousarray(tris, np.float32)), _p(np.ascontiguousarray(attribs)), _p(spectral))
        return spectral


_cache: dict = {}


def oracle() -> CpuLib:
    """The restatement library (built on first use)."""
    if "o" not in _cache:
        build_oracle()
        _cache["o"] = CpuLib(ORACLE_SO, "pzo")
    return _cache["o"]


def reference() -> CpuLib | None:
    """The reference's own CPU code, or None when it was not built here."""
    if "r" not in _cache:
        _cache["r"] = CpuLib(REF_SO, "pzr") if os.path.exists(REF_SO) else None
    return _cache["r"]
