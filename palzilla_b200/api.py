"""Python mirror of the reference's host classes over the C ABI.

``OnesweepSort`` and ``BVHGPUBuilder`` keep the reference's class names, method
names and argument meaning (tinyhiponesweep.h:572-668, minimum_lbvh.h:741-900) so
that tests read like code written against the reference.  Device memory is held
in torch tensors (torch is used only as an allocator and for streams); every
computation runs in libpalzilla_b200.so.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib

NODE_BYTES = 64


def _stream(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


class Scratch:
    """Grow-only device scratch buffer."""

    def __init__(self, device="cuda"):
        self.device = device
        self.buf = None

    def get(self, nbytes: int) -> torch.Tensor:
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self.buf

    def status(self, stream=None) -> int:
        st = C.c_uint32(0)
        _lib.call("pz_scratch_status", C.c_void_p(self.buf.data_ptr()), C.byref(st), C.c_void_p(_stream(stream)))
        return st.value


class OnesweepSort:
    """tinyhiponesweep::OnesweepSort (tinyhiponesweep.h:572-668).

    ``sort(keys, values, tmp_keys, tmp_values, n, start_bit, end_bit, stream)`` sorts
    ``keys`` (uint32 or 64-bit tensor) stably on [start_bit, end_bit); ``values``
    (uint32/int32 tensor or None) follow their keys.  The result ends in
    ``keys``/``values``; the tmp tensors are ping-pong storage of equal size.
    """

    def __init__(self, device="cuda"):
        self.scratch = Scratch(device)

    def sort(self, keys, values, tmp_keys, tmp_values, n: int, start_bit: int, end_bit: int, stream=None):
        kb = keys.element_size()
        nbytes = _lib.lib().pz_onesweep_scratch_bytes(n)
        buf = self.scratch.get(nbytes)
        _lib.call("pz_onesweep_sort", C.c_void_p(keys.data_ptr()), C.c_void_p(_ptr(values)),
                  C.c_void_p(tmp_keys.data_ptr()), C.c_void_p(_ptr(tmp_values)), C.c_uint32(n), C.c_int(kb),
                  C.c_int(start_bit), C.c_int(end_bit), C.c_void_p(buf.data_ptr()), C.c_size_t(buf.numel()),
                  C.c_void_p(_stream(stream)))

    def status(self, stream=None) -> int:
        return self.scratch.status(stream)


class BVHGPUBuilder:
    """minimum_lbvh::BVHGPUBuilder (minimum_lbvh.h:741-900).

    ``build(triangles, n, build_option, sorter, stream)``: ``triangles`` is a float32
    cuda tensor of shape (n, 9) (the 36-byte Triangle layout).  Afterwards
    ``m_internals`` (uint8 tensor of (n-1) * 64 bytes), ``m_rootNode`` (uint32 tensor
    of one element) and ``m_nTriangles`` hold the tree, as in the reference.  The
    ``sorter`` argument is accepted for signature compatibility; the builder runs its
    own fused sort on its own scratch.
    """

    def __init__(self, device="cuda"):
        self.device = device
        self.scratch = Scratch(device)
        self.m_internals = None
        self.m_rootNode = torch.zeros(1, dtype=torch.int32, device=device)
        self.m_nTriangles = 0

    def build(self, triangles, n: int, build_option: int = 0, sorter=None, stream=None):
        self.m_nTriangles = n
        nbytes = max(n - 1, 1) * NODE_BYTES
        if self.m_internals is None or self.m_internals.numel() < nbytes:
            self.m_internals = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        buf = self.scratch.get(_lib.lib().pz_bvh_scratch_bytes(n))
        _lib.call("pz_bvh_build", C.c_void_p(triangles.data_ptr()), C.c_int(n), C.c_uint32(build_option),
                  C.c_void_p(self.m_internals.data_ptr()), C.c_void_p(self.m_rootNode.data_ptr()),
                  C.c_void_p(buf.data_ptr()), C.c_size_t(buf.numel()), C.c_void_p(_stream(stream)))

    def empty(self) -> bool:
        return self.m_nTriangles == 0

    @property
    def root(self) -> int:
        return int(self.m_rootNode.item()) & 0xFFFFFFFF

    def debug_views(self, stream=None):
        """(sorted u64 {morton, index} tensor view, deltas u8 view, scene AABB (6 floats))."""
        n = self.m_nTriangles
        sp, dp = C.c_void_p(), C.c_void_p()
        aabb = (C.c_float * 6)()
        _lib.call("pz_bvh_debug_views", C.c_void_p(self.scratch.buf.data_ptr()), C.c_int(n), C.byref(sp),
                  C.byref(dp), C.cast(aabb, C.c_void_p), C.c_void_p(_stream(stream)))
        base = self.scratch.buf.data_ptr()
        so = sp.value - base
        do = dp.value - base
        sorted_ = self.scratch.buf[so:so + 8 * n].view(torch.int64)
        deltas = self.scratch.buf[do:do + max(n - 1, 0)]
        return sorted_, deltas, list(aabb)


# ---------------------------------------------------------------------------------------
# photon pass, eye pass, work list, specular solve
# ---------------------------------------------------------------------------------------
def _vp(t):
    return C.c_void_p(None if t is None else t.data_ptr())


class DeviceScene:
    """Device copies of a scene (triangles, attributes) and its LBVH."""

    def __init__(self, scene, device="cuda", build_option: int = 0, stream=None):
        import numpy as np
        self.scene = scene
        self.n = scene.n
        self.tris = torch.from_numpy(np.ascontiguousarray(scene.tris)).to(device)
        self.attribs = torch.from_numpy(np.ascontiguousarray(scene.attribs).view(np.uint8)).to(device)
        self.builder = BVHGPUBuilder(device)
        self.builder.build(self.tris, self.n, build_option, None, stream)

    @property
    def internals(self):
        return self.builder.m_internals

    @property
    def root_dev(self):
        return self.builder.m_rootNode


class PathCache:
    """PathCache (pk.h:227-402): one device buffer of pz_path_cache_bytes(capacity)."""

    def __init__(self, capacity: int = 1 << 22, step: float = 0.01, device="cuda"):
        self.capacity = capacity
        self.step = step
        self.buf = torch.empty(_lib.lib().pz_path_cache_bytes(capacity), dtype=torch.uint8, device=device)
        self.clear()

    def clear(self, stream=None):
        _lib.call("pz_path_cache_clear", _vp(self.buf), C.c_uint32(self.capacity), C.c_void_p(_stream(stream)))

    def views(self):
        ptrs = [C.c_void_p() for _ in range(6)]
        _lib.call("pz_path_cache_views", _vp(self.buf), C.c_uint32(self.capacity), *[C.byref(p) for p in ptrs])
        base = self.buf.data_ptr()

        def sl(p, nbytes):
            o = p.value - base
            return self.buf[o:o + nbytes]
        cap = self.capacity
        return dict(hash=sl(ptrs[0], 4 * cap).view(torch.int32), cell=sl(ptrs[1], 4 * cap).view(torch.int32),
                    events=sl(ptrs[2], 4 * cap).view(torch.int32), tris=sl(ptrs[3], 16 * cap).view(torch.int32),
                    params=sl(ptrs[4], 32 * cap).view(torch.float32), count=sl(ptrs[5], 4).view(torch.int32))

    def to_host(self):
        import numpy as np
        v = self.views()
        return dict(hash=v["hash"].cpu().numpy().view(np.uint32), cell=v["cell"].cpu().numpy().view(np.uint32),
                    events=v["events"].cpu().numpy().view(np.uint32),
                    tris=v["tris"].cpu().numpy().reshape(-1, 4), params=v["params"].cpu().numpy().reshape(-1, 8),
                    count=int(v["count"].item()), capacity=self.capacity, step=self.step)

    def status(self, stream=None) -> int:
        st = C.c_uint32(0)
        _lib.call("pz_scratch_status", _vp(self.buf), C.byref(st), C.c_void_p(_stream(stream)))
        return st.value


def photon_trace(ds: DeviceScene, cache: PathCache | None, iteration: int = 0, photons_per_triangle=None,
                 eta_range=None, records: bool = False, stream=None):
    """photonTrace (main_gpu.cu:56-211) from the light point of this iteration
    (Scene.light_point).  Returns the per-photon record tensor when asked."""
    sc = ds.scene
    ppt = photons_per_triangle or sc.photons_per_triangle
    emin, emax = eta_range or sc.eta_range()
    rec = torch.empty(ds.n * ppt * 64, dtype=torch.uint8, device=ds.tris.device) if records else None
    _lib.call("pz_photon_trace", _vp(ds.internals), _vp(ds.root_dev), _vp(ds.tris), _vp(ds.attribs),
              C.c_int(ds.n), C.c_int(ppt), _lib.f3(sc.light_point(iteration)), C.c_float(emin), C.c_float(emax),
              C.c_int(iteration),
              C.c_float(sc.min_throughput), _vp(cache.buf if cache else None),
              C.c_uint32(cache.capacity if cache else 0), C.c_float(cache.step if cache else 0.0), _vp(rec),
              C.c_void_p(_stream(stream)))
    return rec


def ray_generator(scene) -> "_lib.RayGenerator":
    cam = scene.camera
    g = _lib.RayGenerator()
    _lib.lib().pz_ray_generator_lookat(C.byref(g), _lib.f3(cam.eye), _lib.f3(cam.center), _lib.f3(cam.up),
                                       C.c_float(cam.fovy), C.c_int(scene.width), C.c_int(scene.height))
    return g


class Frame:
    """Per-frame device buffers of the reference renderer (pk.h:1368-1391 subset)."""

    def __init__(self, scene, path_capacity: int = 1 << 25, device="cuda"):
        W, H = scene.width, scene.height
        self.npx = W * H
        self.accum = torch.zeros((self.npx, 4), dtype=torch.float32, device=device)
        self.fd = torch.zeros(self.npx * 40, dtype=torch.uint8, device=device)
        self.path_capacity = path_capacity
        self.paths = torch.empty(path_capacity * 8, dtype=torch.uint8, device=device)
        self.paths_tmp = torch.empty(path_capacity * 8, dtype=torch.uint8, device=device)
        self.indexed = torch.empty(path_capacity, dtype=torch.int64, device=device)
        self.indexed_tmp = torch.empty(path_capacity, dtype=torch.int64, device=device)
        self.counter = torch.zeros(1, dtype=torch.int32, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.stats = torch.zeros(3, dtype=torch.int64, device=device)
        self.iteration = 0  # the iteration of the last eye pass (its light point)


def solve_primary(ds: DeviceScene, frame: Frame, iteration: int = 0, lens=(0.6, 0.05, 0.0), texture=None,
                  stream=None):
    """solvePrimary (main_gpu.cu:213-371).  texture: an optional floor texture, a uint8 cuda
    tensor of shape (height, width, 4) (RGBX), sampled at the diffuse hit's (x, z) as
    Texture8RGBX (pk.h:1075-1098); None = the scene's constant albedo."""
    sc = ds.scene
    frame.iteration = iteration
    g = ray_generator(sc)
    l = _lib.LensParams(*[float(x) for x in lens])
    tex = None
    if texture is not None:
        assert texture.dtype == torch.uint8 and texture.dim() == 3 and texture.shape[2] == 4 and texture.is_contiguous()
        tex = _lib.TextureRGBX(texture.data_ptr(), int(texture.shape[1]), int(texture.shape[0]))
    _lib.call("pz_solve_primary", _vp(frame.accum), _vp(frame.fd), C.c_int(sc.width), C.c_int(sc.height), C.byref(g),
              C.byref(l), _vp(ds.internals), _vp(ds.root_dev), _vp(ds.tris), _vp(ds.attribs),
              _lib.f3(sc.light_point(iteration)),
              C.c_float(sc.light_intensity), C.c_float(sc.radiance_clamp), C.c_float(sc.cauchy_a),
              C.c_float(sc.cauchy_b), _lib.f3(sc.albedo), C.byref(tex) if tex is not None else None, C.c_int(iteration),
              _vp(frame.status), C.c_void_p(_stream(stream)))


def lookup_flatten(frame: Frame, cache: PathCache, events: int, stream=None) -> int:
    """lookupFlatten + the count read-back of the reference (pk.h:1486-1510).  Returns n_paths."""
    frame.counter.zero_()
    _lib.call("pz_lookup_flatten", C.c_uint32(events), _vp(frame.paths), _vp(frame.indexed), _vp(frame.counter),
              C.c_uint32(frame.path_capacity), _vp(frame.fd), C.c_int(frame.npx), _vp(cache.buf),
              C.c_uint32(cache.capacity), C.c_float(cache.step), C.c_void_p(_stream(stream)))
    return min(int(frame.counter.item()) & 0xFFFFFFFF, frame.path_capacity)


def sort_and_reorder(frame: Frame, n_paths: int, sorter: OnesweepSort, stream=None):
    """Tuple-coherence sort (pk.h:1526) and reorderSpecularPath; the result is in frame.paths."""
    if n_paths == 0:
        return
    sorter.sort(frame.indexed, None, frame.indexed_tmp, None, n_paths, 0, 32, stream)
    _lib.call("pz_reorder_specular_paths", _vp(frame.indexed), _vp(frame.paths_tmp), _vp(frame.paths),
              C.c_uint32(n_paths), C.c_void_p(_stream(stream)))
    frame.paths, frame.paths_tmp = frame.paths_tmp, frame.paths


def solve_desc(ds: DeviceScene, frame: Frame, cache: PathCache, events_str: str, n_paths: int, spectral=None,
               etas=None, stats=None, max_iterations=32, cost_tolerance=1e-10, early_term_warmup=1, exact=True,
               polish_det=0.0, continuation=False, fold_det=0.0, iteration=None, graze_cos=0.0, roots=None):
    """Solve descriptor of one event string; the light is the point of `iteration`
    (Scene.light_point), by default the iteration of the frame's last eye pass.  The plain
    solve runs without FMA contraction unless exact=False (pz_solve_desc.fma_contraction)."""
    from .scenes import event_descriptor
    sc = ds.scene
    if iteration is None:
        iteration = frame.iteration
    d = _lib.SolveDesc()
    d.K = len(events_str)
    d.events = event_descriptor(events_str)
    d.paths = frame.paths.data_ptr()
    d.n_paths = n_paths
    d.first_diffuse = frame.fd.data_ptr()
    d.internals = ds.internals.data_ptr()
    d.root = ds.root_dev.data_ptr()
    d.triangles = ds.tris.data_ptr()
    d.attribs = ds.attribs.data_ptr()
    d.cache = cache.buf.data_ptr()
    d.cache_capacity = cache.capacity
    d.cell_step = cache.step
    d.p_light = _lib.f3(sc.light_point(iteration))
    d.light_intensity = sc.light_intensity
    d.radiance_clamp = sc.radiance_clamp
    d.cauchy_a = sc.cauchy_a
    d.cauchy_b = sc.cauchy_b
    d.accum = frame.accum.data_ptr()
    d.spectral = spectral.data_ptr() if spectral is not None else None
    d.etas = etas.data_ptr() if etas is not None else None
    d.n_bins = sc.n_bins if spectral is not None else 1
    d.max_iterations = max_iterations
    d.cost_tolerance = cost_tolerance
    d.early_term_warmup = early_term_warmup
    d.stats = stats.data_ptr() if stats is not None else None
    d.fma_contraction = 0 if exact else 1
    d.polish_det = polish_det
    d.continuation = 1 if continuation else 0
    d.fold_det = fold_det
    d.graze_cos = graze_cos
    d.roots = roots.data_ptr() if roots is not None else None
    return d


def solve_specular_plain(desc, stream=None):
    _lib.call("pz_solve_specular_plain", C.byref(desc), C.c_void_p(_stream(stream)))


def solve_specular_batched(desc, scratch: Scratch, n_paths_dev=None, blocks_per_sm: int = 0, stream=None):
    """Batched persistent solve; n_paths_dev (device int32 tensor) supplies the item count
    on the device (desc.n_paths is then the capacity)."""
    nbytes = _lib.lib().pz_solve_batched_scratch_bytes(desc.K, desc.n_paths, desc.n_bins)
    buf = scratch.get(nbytes)
    _lib.call("pz_solve_specular_batched", C.byref(desc), _vp(n_paths_dev), _vp(buf), C.c_size_t(buf.numel()),
              C.c_int(blocks_per_sm), C.c_void_p(_stream(stream)))


BATCH_COUNTERS = ("skipped", "predicted", "fallback", "newton_bins", "fp64_polish", "vis_overflow", "vis_candidates",
                  "vis_queries", "fallback_noconv", "fallback_shift", "fallback_probe", "newton_iterations",
                  "newton_bins_refined", "fallback_fold")


def batched_counters(scratch: Scratch) -> dict:
    v = scratch.buf[64:64 + 8 * len(BATCH_COUNTERS)].view(torch.int64).cpu().tolist()
    return dict(zip(BATCH_COUNTERS, v))


def resolve_spectral(spectral, scene, rgb=None, pixels=None, stream=None):
    _lib.call("pz_resolve_spectral", _vp(rgb), _vp(pixels), _vp(spectral), C.c_int(scene.width * scene.height),
              C.c_int(scene.n_bins), C.c_float(scene.lambda_min), C.c_float(scene.lambda_max), _lib.f3(scene.albedo),
              C.c_void_p(_stream(stream)))


# ---------------------------------------------------------------------------------------
# Path Cuts
# ---------------------------------------------------------------------------------------
NORMAL_BOUND_BYTES = 52


def normal_bounds(builder: BVHGPUBuilder, attribs, stream=None):
    """InternalNormalBound array (pk.h:1705-1709) of a built BVH: uint8 tensor of
    (n - 1) * 52 bytes."""
    n = builder.m_nTriangles
    out = torch.empty(max(n - 1, 1) * NORMAL_BOUND_BYTES, dtype=torch.uint8, device=attribs.device)
    _lib.call("pz_normal_bounds", _vp(builder.m_internals), C.c_int(max(n - 1, 0)), _vp(attribs), _vp(out),
              C.c_void_p(_stream(stream)))
    return out


class PathCuts:
    """traverseAdmissibleNodes<K> (pk.h:1760-2220) for a batch of receiver points.

    ``run(K, events, eta, p_beg, p_end, builder, nbs, triangles, attribs, directed)`` returns
    an int32 tensor (n, 1 + K) of {query, triangle[K]} rows and the number of node tuples
    tested."""

    def __init__(self, device="cuda", frontier_capacity: int = 1 << 22, tuple_capacity: int = 1 << 22):
        self.device = device
        self.frontier_capacity = frontier_capacity
        self.tuple_capacity = tuple_capacity
        self.scratch = Scratch(device)

    def run(self, K: int, events: int, eta: float, p_beg, p_end, builder: BVHGPUBuilder, nbs, triangles, attribs,
            directed: bool = False, stream=None):
        nq = p_end.shape[0]
        cap = max(self.frontier_capacity, nq)
        buf = self.scratch.get(_lib.lib().pz_path_cuts_scratch_bytes(K, cap))
        out = torch.empty((self.tuple_capacity, 1 + K), dtype=torch.int32, device=self.device)
        nt, visited = C.c_uint64(0), C.c_uint64(0)
        _lib.call("pz_path_cuts", C.c_int(K), C.c_uint32(events), C.c_float(eta), _lib.f3(p_beg), _vp(p_end),
                  C.c_uint32(nq), _vp(builder.m_internals), _vp(nbs), _vp(triangles), _vp(attribs),
                  _vp(builder.m_rootNode), C.c_int(1 if directed else 0), _vp(out), C.c_uint32(self.tuple_capacity),
                  C.byref(nt), C.byref(visited), _vp(buf), C.c_size_t(buf.numel()), C.c_void_p(_stream(stream)))
        return out[: nt.value], visited.value


# ---------------------------------------------------------------------------------------
# subdivision solve
# ---------------------------------------------------------------------------------------
ROOT_FIELDS = ("tuple", "bin", "depth", "path")


class SubdivisionSolver:
    """Per-tuple parametric-domain subdivision under affine bounds, then Newton in the
    surviving boxes (pz_subdivide_solve; no reference counterpart).

    ``run(K, events, p_beg, p_end, tuples, etas, triangles, attribs, scene_builder,
    scene_triangles)``: ``tuples`` is an int32 (n, 1 + K) tensor of {query, triangle[K]}
    rows indexing ``triangles`` / ``attribs`` (what PathCuts.run or work_list_rows
    return); visibility runs through the scene's BVH.  Returns (ids, params, throughput,
    stats): ids an int64 (m, 4) tensor of {tuple row, bin, depth, path} per root, params
    float (m, 2K), throughput float (m,), stats a dict of the kernel's counters."""

    def __init__(self, device="cuda", box_capacity: int = 1 << 22, root_capacity: int = 1 << 20, max_depth: int = 12,
                 eps: float = 1e-4, max_iterations: int = 32, cost_tolerance: float = 1e-10,
                 early_term_warmup: int = 1, fp64_polish: bool = False):
        self.device = device
        self.box_capacity = box_capacity
        self.root_capacity = root_capacity
        self.params = _lib.SubdivParams(max_depth, eps, max_iterations, cost_tolerance, early_term_warmup,
                                        1 if fp64_polish else 0)
        self.scratch = Scratch(device)
        self.roots = torch.empty(root_capacity * 64, dtype=torch.uint8, device=device)

    def run(self, K: int, events: int, p_beg, p_end, tuples, etas, triangles, attribs, scene_builder: BVHGPUBuilder,
            scene_triangles, stream=None):
        n = int(tuples.shape[0])
        cap = max(self.box_capacity, n)
        buf = self.scratch.get(_lib.lib().pz_subdivide_scratch_bytes(cap))
        nr = C.c_uint64(0)
        st = _lib.SubdivStats()
        _lib.call("pz_subdivide_solve", C.c_int(K), C.c_uint32(events), _lib.f3(p_beg), _vp(p_end), _vp(tuples),
                  C.c_uint32(n), _vp(etas), C.c_int(int(etas.numel())), C.byref(self.params), _vp(triangles),
                  _vp(attribs), _vp(scene_builder.m_internals), _vp(scene_triangles), _vp(scene_builder.m_rootNode),
                  _vp(self.roots), C.c_uint64(self.root_capacity), C.byref(nr), C.byref(st), _vp(buf),
                  C.c_size_t(buf.numel()), C.c_void_p(_stream(stream)))
        m = nr.value
        rec = self.roots[: m * 64].view(torch.int32).view(m, 16)
        ids = rec[:, :4].to(torch.int64) & 0xFFFFFFFF
        params = rec[:, 4:4 + 2 * K].contiguous().view(torch.float32)
        thr = rec[:, 12].contiguous().view(torch.float32)
        stats = {f: int(getattr(st, f)) for f, _ in _lib.SubdivStats._fields_}
        return ids, params, thr, stats

    def contribute(self, K: int, events: int, scene, tuples, n_roots: int, frame: "Frame", etas, triangles, attribs,
                   spectral, iteration: int = 0, stream=None):
        """Adds the roots of the last run() to `spectral` (pixels x bins); the tuple rows'
        query index is the pixel of frame's FirstDiffuse records (pz_subdivide_contribute)."""
        _lib.call("pz_subdivide_contribute", C.c_int(K), C.c_uint32(events), _lib.f3(scene.light_point(iteration)),
                  C.c_float(scene.light_intensity), C.c_float(scene.radiance_clamp), _vp(tuples), _vp(self.roots),
                  C.c_uint64(n_roots), _vp(frame.fd), _vp(etas), C.c_int(int(etas.numel())), _vp(triangles),
                  _vp(attribs), _vp(spectral), C.c_void_p(_stream(stream)))


def receiver_points(frame: "Frame"):
    """The receiver point of every pixel (FirstDiffuse.p), a contiguous float (npx, 3)."""
    return frame.fd.view(torch.float32).view(frame.npx, 10)[:, :3].contiguous()


def work_list_rows(frame: "Frame", cache: PathCache, n_paths: int, K: int):
    """{pixel, triangle[K]} rows (int32, n_paths x (1 + K)) of a frame's work list -- one
    per (pixel, cached tuple) -- the rows pz_subdivide_solve takes."""
    sp = frame.paths[: n_paths * 8].view(torch.int32).view(n_paths, 2)
    tris = cache.views()["tris"].view(-1, 4)
    return torch.cat([sp[:, :1], tris[sp[:, 1].long(), :K]], 1).contiguous()


# ---------------------------------------------------------------------------------------
# batches of scenes
# ---------------------------------------------------------------------------------------
class SceneBatch:
    """Scenes of one K and bin count solved together by the batched persistent solver
    (pz_solve_multi_prepare / pz_solve_specular_multi / pz_solve_multi_autotune).

    ``descs``: one solve descriptor per scene (binned mode; n_paths = its capacity when
    ``counts`` gives the device item counters, else its item count)."""

    def __init__(self, descs, counts=None, device="cuda", stream=None):
        n = len(descs)
        self.K, self.n_bins, self.n = descs[0].K, descs[0].n_bins, n
        self.total = sum(int(d.n_paths) for d in descs)
        self._descs = (_lib.SolveDesc * n)(*descs)
        self._counts = (C.c_void_p * n)(*[None if c is None else c.data_ptr() for c in (counts or [None] * n)])
        nbytes = _lib.lib().pz_solve_multi_scratch_bytes(self.K, self.n_bins, n, self.total)
        self.scratch = torch.empty(nbytes, dtype=torch.uint8, device=device)
        _lib.call("pz_solve_multi_prepare", C.cast(self._descs, C.c_void_p), C.cast(self._counts, C.c_void_p),
                  C.c_uint32(n), _vp(self.scratch),
                  C.c_size_t(nbytes), C.c_void_p(_stream(stream)))

    def solve(self, tuning=None, stats=None, stream=None):
        t = None if tuning is None else C.byref(_lib.BatchTuning(*tuning))
        _lib.call("pz_solve_specular_multi", C.c_int(self.K), C.c_int(self.n_bins), C.c_uint32(self.n),
                  C.c_uint64(self.total), _vp(self.scratch), C.c_size_t(self.scratch.numel()), t, _vp(stats),
                  C.c_void_p(_stream(stream)))

    def autotune(self, stats=None, stream=None):
        """Renders the batch once per candidate (clear the images afterwards); returns the
        fastest (p1_blocks_per_sm, p2_blocks_per_sm, p2_chunk) and its time in ms."""
        best, ms = _lib.BatchTuning(), C.c_float(0.0)
        _lib.call("pz_solve_multi_autotune", C.c_int(self.K), C.c_int(self.n_bins), C.c_uint32(self.n),
                  C.c_uint64(self.total), _vp(self.scratch), C.c_size_t(self.scratch.numel()), _vp(stats),
                  C.byref(best), C.byref(ms), C.c_void_p(_stream(stream)))
        return (best.p1_blocks_per_sm, best.p2_blocks_per_sm, best.p2_chunk), ms.value

    def counters(self) -> dict:
        v = self.scratch[64:64 + 8 * len(BATCH_COUNTERS)].view(torch.int64).cpu().tolist()
        return dict(zip(BATCH_COUNTERS, v))
