"""Batched persistent solver (pz_solve_specular_batched) against the plain per-tuple solver
and the CPU oracle, on identical solver inputs (one PathCache and one work list).

The batched solver runs the reference's arithmetic without FMA contraction, as the
exact-arithmetic plain build does, so its image equals the float oracle's (the reference's
own CPU code) up to the order of the float atomics: relative RMSE <= 1e-5.  Against the
plain FMA build it differs exactly as much as that build differs from the oracle (FP32
accept / reject flips at triangle edges and caustic folds).  The FP64 error of every image
is printed and bounded.  Scenes: single-refraction heightfield lens (T), two-sheet lens
(TT), the two-sheet lens under a slab of opaque blockers, and 20,000 random pixels of the
dispersive sphere frame (icosphere-5, 64 bins).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from palzilla_b200 import _lib
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return float(np.sqrt(((a - b) ** 2).mean()) / max(np.sqrt((b ** 2).mean()), 1e-30))


def _prepare(sc, iteration=0, capacity=1 << 22, path_capacity=1 << 23):
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=path_capacity)
    A.solve_primary(ds, frame, iteration=iteration)
    cache = A.PathCache(capacity=capacity, step=sc.cell_step)
    A.photon_trace(ds, cache, iteration=iteration)
    n = A.lookup_flatten(frame, cache, S.event_descriptor(sc.events))
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    return ds, frame, cache, n


def _solve(ds, frame, cache, sc, n, mode, scratch=None, stats=None, polish_det=0.0, graze_cos=0.0):
    spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    d = A.solve_desc(ds, frame, cache, sc.events, n, spectral=spectral, etas=etas, stats=stats,
                     exact=(mode == "exact"), polish_det=polish_det, graze_cos=graze_cos)
    if mode == "batched":
        A.solve_specular_batched(d, scratch if scratch is not None else A.Scratch())
    else:
        A.solve_specular_plain(d)
    torch.cuda.synchronize()
    return spectral.cpu().numpy()


def _oracle_images(orc, sc, frame, cache, n, pixels=None):
    pairs = frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2).copy()
    if pixels is not None:
        pairs = pairs[np.isin(pairs[:, 0], pixels)].copy()
    gc = cache.to_host()
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    bvh = orc.build_bvh(sc.tris)
    K = len(sc.events)
    # the light point of the frame's iteration (the sphere's area light moves with it)
    f32, _ = orc.render_pairs(K, pairs, gc, fd, bvh, sc, sc.bin_etas(), iteration=frame.iteration)
    f64, _ = orc.render_pairs(K, pairs, gc, fd, bvh, sc, sc.bin_etas(), dtype=np.float64, iteration=frame.iteration)
    return f32, f64


@pytest.mark.parametrize("events,side", [("T", 64), ("TT", 40)])
def test_batched_lens_matches_plain_and_oracle(orc, events, side):
    sc = S.lens_scene(side=side, seed=21, width=128, height=128, n_bins=16, events=events)
    ds, frame, cache, n = _prepare(sc)
    assert n > 1000
    scratch = A.Scratch()
    st_b = torch.zeros(3, dtype=torch.int64, device="cuda")
    img_b = _solve(ds, frame, cache, sc, n, "batched", scratch, st_b)
    img_p = _solve(ds, frame, cache, sc, n, "plain")
    img_x = _solve(ds, frame, cache, sc, n, "exact")
    f32, f64 = _oracle_images(orc, sc, frame, cache, n)
    cnt = A.batched_counters(scratch)
    assert cnt["skipped"] + cnt["predicted"] + cnt["fallback"] == n
    assert int(st_b[0].item()) == n * sc.n_bins
    assert scratch.status() == 0
    r = {"batched_vs_plain_exact": _rel(img_b, img_x), "batched_vs_oracle": _rel(img_b, f32),
         "plain_exact_vs_oracle": _rel(img_x, f32), "batched_vs_plain": _rel(img_b, img_p),
         "plain_vs_oracle": _rel(img_p, f32), "batched_vs_fp64": _rel(img_b, f64), "oracle_vs_fp64": _rel(f32, f64)}
    print(f"\n[{events}] n={n} " + " ".join(f"{k}={v:.2e}" for k, v in r.items()) + f" counters={cnt}")
    assert r["plain_exact_vs_oracle"] <= 1e-5
    assert r["batched_vs_oracle"] <= 1e-5
    assert r["batched_vs_plain_exact"] <= 1e-5
    assert r["batched_vs_plain"] <= max(1e-3, 1.5 * r["plain_vs_oracle"])
    assert r["batched_vs_fp64"] <= max(1.01 * r["oracle_vs_fp64"], 1e-5)


def test_batched_fp64_polish(orc):
    """With polish_det = 1e-6, roots of near-singular Jacobians are refined in FP64 (and their
    throughput evaluated in FP64); the image moves off the reference's float arithmetic by a
    bounded amount and its FP64 error is reported."""
    sc = S.lens_scene(side=40, seed=21, width=128, height=128, n_bins=16, events="TT")
    ds, frame, cache, n = _prepare(sc)
    scratch = A.Scratch()
    img_b = _solve(ds, frame, cache, sc, n, "batched", scratch, polish_det=1e-6)
    f32, f64 = _oracle_images(orc, sc, frame, cache, n)
    cnt = A.batched_counters(scratch)
    r = {"polished_vs_oracle": _rel(img_b, f32), "polished_vs_fp64": _rel(img_b, f64),
         "oracle_vs_fp64": _rel(f32, f64)}
    print("\n[TT polish] " + " ".join(f"{k}={v:.2e}" for k, v in r.items()) + f" polished={cnt['fp64_polish']}")
    assert cnt["fp64_polish"] > 0
    assert r["polished_vs_oracle"] <= 1e-3
    assert r["polished_vs_fp64"] <= 2.0 * r["oracle_vs_fp64"]


def test_batched_fp64_grazing(orc):
    """Roots where a segment meets a surface at |cos| below graze_cos are polished in FP64
    and admitted by the FP64 throughput test.  The lens's paths cross its sheets at |cos|
    of 0.95 to 1, so a threshold of 0.999 sends most of its roots down the FP64 path.
    FP64 then changes only the decisions of roots at triangle edges, whose FP32 root is off
    by about 1e-4 in the barycentrics (in a CPU replication, 6 of 16,000 decisions flip);
    each flip adds or drops a whole contribution.  So the check is on how many (pixel, bin)
    entries move and on the image's energy, not on an RMSE dominated by a few flips."""
    sc = S.lens_scene(side=40, seed=21, width=128, height=128, n_bins=16, events="TT")
    ds, frame, cache, n = _prepare(sc)
    base = _solve(ds, frame, cache, sc, n, "batched")
    scratch = A.Scratch()
    img_b = _solve(ds, frame, cache, sc, n, "batched", scratch, graze_cos=0.999)
    cnt = A.batched_counters(scratch)
    moved = np.abs(img_b - base) > 0.01 * np.abs(base) + 1e-6
    energy = float(img_b.sum() / base.sum())
    print(f"\n[TT grazing] polished={cnt['fp64_polish']} entries moved by > 1%: {int(moved.sum())} of "
          f"{moved.size} ({moved.mean():.2e}); energy ratio {energy:.6f}")
    assert cnt["fp64_polish"] > 100000
    assert moved.mean() < 1e-2 and abs(energy - 1.0) < 1e-3
    # a threshold no path reaches leaves the image as it is
    img_0 = _solve(ds, frame, cache, sc, n, "batched", graze_cos=0.1)
    assert _rel(img_0, base) < 1e-6


def test_batched_occluded_lens(orc):
    """Opaque blockers between the light and a two-sheet lens: the warp's shared shadow
    queries and each lane's candidate tests must reach the visibility decisions of the
    plain path (one any-hit walk per path segment) and of the oracle.  The blockers come
    after the lens and receiver triangles, so the same (pixel, tuple) pairs rendered by the
    oracle in the open lens show that the blockers take light away."""
    sc = S.occluded_lens_scene(side=40, seed=21, n_blockers=300, events="TT")
    ds, frame, cache, n = _prepare(sc)
    assert n > 1000
    scratch = A.Scratch()
    img_b = _solve(ds, frame, cache, sc, n, "batched", scratch)
    img_x = _solve(ds, frame, cache, sc, n, "exact")
    f32, f64 = _oracle_images(orc, sc, frame, cache, n)
    open_sc = S.lens_scene(side=40, seed=21, events="TT", n_bins=sc.n_bins, width=sc.width, height=sc.height)
    pairs = frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2).copy()
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    f32_open, _ = orc.render_pairs(2, pairs, cache.to_host(), fd, orc.build_bvh(open_sc.tris), open_sc,
                                   sc.bin_etas(), iteration=frame.iteration)
    cnt = A.batched_counters(scratch)
    kept = float(f32.sum() / f32_open.sum())
    r = {"batched_vs_plain_exact": _rel(img_b, img_x), "batched_vs_oracle": _rel(img_b, f32),
         "batched_vs_fp64": _rel(img_b, f64), "oracle_vs_fp64": _rel(f32, f64)}
    print(f"\n[occluded TT] n={n} light kept by the blockers {kept:.4f} " +
          " ".join(f"{k}={v:.2e}" for k, v in r.items()) +
          f" queries={cnt['vis_queries']} candidates={cnt['vis_candidates']} overflow={cnt['vis_overflow']}")
    assert scratch.status() == 0
    assert kept < 1.0  # the blockers occlude some of the solved paths
    assert r["batched_vs_plain_exact"] <= 1e-5
    assert r["batched_vs_oracle"] <= 1e-5
    assert r["batched_vs_fp64"] <= max(1.01 * r["oracle_vs_fp64"], 1e-5)


def test_batched_sphere_sample(orc):
    """Dispersive sphere at full size; the oracle checks 20,000 random pixels (all their
    work items x 64 bins)."""
    sc = S.sphere_scene()
    sc.photons_per_triangle = 205
    ds, frame, cache, n = _prepare(sc, iteration=3, path_capacity=1 << 25)
    img_b = _solve(ds, frame, cache, sc, n, "batched")
    img_x = _solve(ds, frame, cache, sc, n, "exact")
    img_p = _solve(ds, frame, cache, sc, n, "plain")
    pairs = frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2)
    px = np.sort(np.random.default_rng(5).choice(np.unique(pairs[:, 0]), 20000, replace=False))
    f32, f64 = _oracle_images(orc, sc, frame, cache, n, pixels=px)
    r = {"batched_vs_oracle": _rel(img_b[px], f32[px]), "plain_exact_vs_oracle": _rel(img_x[px], f32[px]),
         "batched_vs_fp64": _rel(img_b[px], f64[px]), "oracle_vs_fp64": _rel(f32[px], f64[px]),
         "plain_vs_oracle": _rel(img_p[px], f32[px]), "full_batched_vs_plain_exact": _rel(img_b, img_x),
         "full_batched_vs_plain": _rel(img_b, img_p), "full_plain_vs_plain_exact": _rel(img_p, img_x)}
    print("\n[sphere] " + " ".join(f"{k}={v:.2e}" for k, v in r.items()))
    assert r["plain_exact_vs_oracle"] <= 1e-5
    assert r["batched_vs_oracle"] <= 1e-5
    assert r["full_batched_vs_plain_exact"] <= 1e-5
    assert r["batched_vs_fp64"] <= max(1.01 * r["oracle_vs_fp64"], 1e-5)
    # the plain FMA build flips single (pixel, bin) entries at edges and folds
    assert r["full_batched_vs_plain"] <= max(1e-3, 1.5 * r["full_plain_vs_plain_exact"])


def test_batched_host_checks():
    L = _lib.lib()
    sc = S.lens_scene(side=16, seed=1, width=32, height=32, n_bins=4, events="T")
    ds, frame, cache, n = _prepare(sc, capacity=1 << 20, path_capacity=1 << 18)
    assert n > 16
    spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    need = L.pz_solve_batched_scratch_bytes(1, n, sc.n_bins)
    assert L.pz_solve_batched_scratch_bytes(1, n, 0) == 0 and L.pz_solve_batched_scratch_bytes(1, n, 65) == 0
    small = torch.empty(need - 256, dtype=torch.uint8, device="cuda")
    d = A.solve_desc(ds, frame, cache, sc.events, n, spectral=spectral, etas=etas)
    r = L.pz_solve_specular_batched(C.byref(d), None, C.c_void_p(small.data_ptr()), C.c_size_t(small.numel()), 0, s)
    assert r == 2 and b"scratch" in L.pz_last_error()
    d0 = A.solve_desc(ds, frame, cache, sc.events, 0, spectral=spectral, etas=etas)
    r = L.pz_solve_specular_batched(C.byref(d0), None, C.c_void_p(small.data_ptr()), C.c_size_t(small.numel()), 0, s)
    assert r == 0
    dr = A.solve_desc(ds, frame, cache, sc.events, n)  # no spectral image: binned mode is required
    big = torch.empty(need, dtype=torch.uint8, device="cuda")
    r = L.pz_solve_specular_batched(C.byref(dr), None, C.c_void_p(big.data_ptr()), C.c_size_t(big.numel()), 0, s)
    assert r == 1
    torch.cuda.synchronize()
    assert float(spectral.abs().sum()) == 0.0


def test_batched_device_count():
    """The item count read on the device (the lookup counter) gives the same image as the
    host count."""
    sc = S.lens_scene(side=32, seed=4, width=64, height=64, n_bins=8, events="T")
    ds, frame, cache, n = _prepare(sc, path_capacity=1 << 20)
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    imgs = []
    for dev in (False, True):
        spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")
        d = A.solve_desc(ds, frame, cache, sc.events, frame.path_capacity if dev else n, spectral=spectral, etas=etas)
        A.solve_specular_batched(d, A.Scratch(), n_paths_dev=frame.counter if dev else None)
        torch.cuda.synchronize()
        imgs.append(spectral.cpu().numpy())
    assert _rel(imgs[1], imgs[0]) <= 1e-6
