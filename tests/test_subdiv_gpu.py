"""Per-tuple parametric-domain subdivision under affine bounds (pz_subdivide_solve) and the
roots' image (pz_subdivide_contribute) on the GPU against the CPU oracle
(oracle/pz_oracle_subdiv.hpp).

Parity: the oracle repeats every affine operation with the same directed rounding, so the
surviving boxes, the Newton starts and therefore the roots are identical: the same
(tuple, bin, depth, path) records with bitwise-equal barycentrics and throughputs.  The
roots are also stated against FP64 (the oracle's Newton in double from each root).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from palzilla_b200 import _lib
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _dev(sc):
    t = torch.from_numpy(np.ascontiguousarray(sc.tris, np.float32)).cuda()
    at = torch.from_numpy(np.ascontiguousarray(sc.attribs).view(np.uint8).reshape(-1)).cuda()
    b = A.BVHGPUBuilder()
    b.build(t, t.shape[0], 0)
    return t, at, b


def _ends(n, seed):
    rng = np.random.default_rng(seed)
    e = rng.uniform(-0.4, 0.4, (n, 3)).astype(np.float32)
    e[:, 1] = 0.0
    return e


def _sorted(ids, params, thr):
    ids = ids.cpu().numpy()
    order = np.lexsort((ids[:, 3], ids[:, 2], ids[:, 1], ids[:, 0]))
    return ids[order], params.cpu().numpy()[order], thr.cpu().numpy()[order]


def _check_equal(exp, ids, params, thr, K):
    assert len(exp) == len(ids)
    exp_ids = np.stack([exp[f].astype(np.int64) for f in A.ROOT_FIELDS], 1)
    assert (ids == exp_ids).all()
    assert params.tobytes() == np.ascontiguousarray(exp["params"][:, : 2 * K]).tobytes()
    assert thr.tobytes() == exp["throughput"].tobytes()


STAT_KEYS = ("boxes_tested", "boxes_culled", "leaves", "bins_excluded", "solves", "converged", "outside_box", "roots")


@pytest.mark.parametrize("amplitude,side,bins", [(0.01, 32, 1), (0.03, 16, 1), (0.05, 8, 4)])
def test_single_refraction_all_triangles_matches_oracle(orc, amplitude, side, bins):
    """Every (receiver point, lens triangle) row: most rows die at depth 0, the rest are
    subdivided to their roots.  Several bins share the subdivision."""
    sc = S.lens_scene(side=side, seed=3, amplitude=amplitude, events="T", width=16, height=16)
    t, at, b = _dev(sc)
    ends = _ends(12, 7)
    spec = np.nonzero(sc.attribs["material"] != 0)[0]
    rows = np.array([[q, i] for q in range(len(ends)) for i in spec], np.int32)
    etas = np.array([1.5, 1.52, 1.54, 1.56][:bins], np.float32)
    ev = S.event_descriptor("T")
    solver = A.SubdivisionSolver(box_capacity=1 << 20, root_capacity=1 << 16)
    ids, params, thr, st = solver.run(1, ev, sc.p_light, torch.from_numpy(ends).cuda(), torch.from_numpy(rows).cuda(),
                                      torch.from_numpy(etas).cuda(), t, at, b, t)
    torch.cuda.synchronize()
    ids, params, thr = _sorted(ids, params, thr)
    bo = orc.build_bvh(sc.tris, 0)
    exp, est = orc.subdivide_solve(1, ev, sc.p_light, ends, rows, etas, sc.tris, sc.attribs, bo, sc.tris)
    _check_equal(exp, ids, params, thr, 1)
    assert [st[k] for k in STAT_KEYS] == est.tolist()
    assert st["roots"] > 0 and st["boxes_culled"] > len(rows) // 2
    print(f"\nrows {len(rows)}: boxes {st['boxes_tested']} (culled {st['boxes_culled']}), leaves {st['leaves']}, "
          f"roots {st['roots']}")


@pytest.mark.parametrize("max_depth,eps", [(0, 1e-4), (5, 1e-4), (16, 0.0)])
def test_uneven_depths_in_one_queue_match_oracle(orc, max_depth, eps):
    """Rows of a rough lens (many boxes deep) mixed with rows of a smooth one (most die at
    depth 0) in one persistent launch, with the box queue at its smallest (one entry per
    tuple): the warps' stacks hold the deep tuples' boxes, lending them to the queue as
    other warps run dry.  Roots and statistics equal the oracle's at every depth limit."""
    rough = S.lens_scene(side=8, seed=3, amplitude=0.05, events="T", width=16, height=16)
    smooth = S.lens_scene(side=24, seed=4, amplitude=0.005, events="T", width=16, height=16)
    # one soup: the rough lens's specular triangles, then the smooth lens's
    sr = np.nonzero(rough.attribs["material"] != 0)[0]
    ss = np.nonzero(smooth.attribs["material"] != 0)[0]
    tris = np.concatenate([rough.tris[sr], smooth.tris[ss]])
    attribs = np.concatenate([rough.attribs[sr], smooth.attribs[ss]])
    ends = _ends(8, 13)
    rows = np.array([[q, i] for q in range(len(ends)) for i in range(len(tris))], np.int32)
    t = torch.from_numpy(np.ascontiguousarray(tris, np.float32)).cuda()
    at = torch.from_numpy(np.ascontiguousarray(attribs).view(np.uint8).reshape(-1)).cuda()
    scene_t = torch.from_numpy(np.ascontiguousarray(rough.tris, np.float32)).cuda()
    b = A.BVHGPUBuilder()
    b.build(scene_t, scene_t.shape[0], 0)
    etas = np.array([1.5, 1.55], np.float32)
    ev = S.event_descriptor("T")
    solver = A.SubdivisionSolver(box_capacity=len(rows), root_capacity=1 << 18, max_depth=max_depth, eps=eps)
    ids, params, thr, st = solver.run(1, ev, rough.p_light, torch.from_numpy(ends).cuda(), torch.from_numpy(rows).cuda(),
                                      torch.from_numpy(etas).cuda(), t, at, b, scene_t)
    torch.cuda.synchronize()
    ids, params, thr = _sorted(ids, params, thr)
    bo = orc.build_bvh(rough.tris, 0)
    exp, est = orc.subdivide_solve(1, ev, rough.p_light, ends, rows, etas, tris, attribs, bo, rough.tris,
                                   max_depth=max_depth, eps=eps, cap=1 << 18)
    _check_equal(exp, ids, params, thr, 1)
    assert [st[k] for k in STAT_KEYS] == est.tolist()
    print(f"\nmax depth {max_depth}: rows {len(rows)}, boxes {st['boxes_tested']}, leaves {st['leaves']}, "
          f"roots {st['roots']}")


def test_two_refractions_path_cuts_rows_match_oracle(orc):
    """Rows from Path Cuts (directed rounding) over the lens's specular triangles, K = 2."""
    sc = S.lens_scene(side=12, seed=5, events="TT", width=16, height=16)
    spec = np.nonzero(sc.attribs["material"] != 0)[0]
    t, at, b = _dev(sc)
    st_ = torch.from_numpy(np.ascontiguousarray(sc.tris[spec], np.float32)).cuda()
    sa_ = torch.from_numpy(np.ascontiguousarray(sc.attribs[spec]).view(np.uint8).reshape(-1)).cuda()
    bs = A.BVHGPUBuilder()
    bs.build(st_, st_.shape[0], 1)
    nbs = A.normal_bounds(bs, sa_)
    ends = _ends(16, 11)
    ev = S.event_descriptor("TT")
    rows, _ = A.PathCuts(frontier_capacity=1 << 20, tuple_capacity=1 << 20).run(
        2, ev, 1.5, sc.p_light, torch.from_numpy(ends).cuda(), bs, nbs, st_, sa_, directed=True)
    assert rows.shape[0] > 0
    etas = np.array([1.5, 1.55], np.float32)
    solver = A.SubdivisionSolver(box_capacity=1 << 23, root_capacity=1 << 18)
    ids, params, thr, st = solver.run(2, ev, sc.p_light, torch.from_numpy(ends).cuda(), rows,
                                      torch.from_numpy(etas).cuda(), st_, sa_, b, t)
    torch.cuda.synchronize()
    ids, params, thr = _sorted(ids, params, thr)
    bo = orc.build_bvh(sc.tris, 0)
    exp, est = orc.subdivide_solve(2, ev, sc.p_light, ends, rows.cpu().numpy(), etas, sc.tris[spec], sc.attribs[spec],
                                   bo, sc.tris)
    _check_equal(exp, ids, params, thr, 2)
    assert [st[k] for k in STAT_KEYS] == est.tolist() and st["roots"] > 0
    print(f"\nK=2: {rows.shape[0]} path-cuts rows, boxes {st['boxes_tested']}, leaves {st['leaves']}, "
          f"roots {st['roots']}")


def test_roots_against_fp64_and_polish(orc):
    """Float roots against the oracle's FP64 Newton from the same root; the FP64 polish
    brings them to the FP64 root."""
    sc = S.lens_scene(side=16, seed=3, amplitude=0.03, events="T", width=16, height=16)
    t, at, b = _dev(sc)
    ends = _ends(8, 1)
    spec = np.nonzero(sc.attribs["material"] != 0)[0]
    rows = np.array([[q, i] for q in range(len(ends)) for i in spec], np.int32)
    etas = torch.tensor([1.5], device="cuda")
    ev = S.event_descriptor("T")
    res = {}
    for polish in (False, True):
        solver = A.SubdivisionSolver(box_capacity=1 << 20, root_capacity=1 << 16, fp64_polish=polish)
        ids, params, thr, st = solver.run(1, ev, sc.p_light, torch.from_numpy(ends).cuda(),
                                          torch.from_numpy(rows).cuda(), etas, t, at, b, t)
        res[polish] = _sorted(ids, params, thr) + (st,)
    assert res[True][3]["polished"] >= res[True][3]["roots"] > 0
    errs = {False: [], True: []}
    for polish in (False, True):
        ids, params, _, _ = res[polish]
        for (row, _, _, _), p in zip(ids, params):
            q, tri = rows[row]
            ok, pd, _ = orc.solve_constraints(1, p.astype(np.float64), sc.p_light, ends[q], sc.tris[[tri]],
                                              sc.attribs[[tri]], 1.5, ev, max_iter=8, tol=1e-24, warmup=8,
                                              dtype=np.float64)
            if ok:
                errs[polish].append(np.abs(pd - p).max())
    e0, e1 = np.max(errs[False]), np.max(errs[True])
    m0, m1 = np.median(errs[False]), np.median(errs[True])
    print(f"\n|root - FP64 root| max / median: float {e0:.2e} / {m0:.2e}, after FP64 polish {e1:.2e} / {m1:.2e} "
          f"({len(errs[True])} roots)")
    assert e0 < 1e-3 and e1 <= e0 and m1 <= 1e-6


def test_frame_render_from_work_list_matches_oracle(orc):
    """A single-refraction lens frame: every (pixel, cached tuple) work item of the photon
    pass is solved by subdivision instead of one Newton from the photon's barycentrics,
    and its roots are added to the binned spectral image.  Roots equal the oracle's; the
    image equals the oracle's sum of the same roots (to the order of the float atomics)."""
    sc = S.lens_scene(side=32, seed=1, events="T", width=48, height=48, n_bins=4)
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 20)
    cache = A.PathCache(capacity=1 << 20, step=sc.cell_step)
    A.solve_primary(ds, frame, iteration=0)
    A.photon_trace(ds, cache, iteration=0)
    ev = S.event_descriptor("T")
    n = A.lookup_flatten(frame, cache, ev)
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    rows = A.work_list_rows(frame, cache, n, 1)
    ends = A.receiver_points(frame)
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    solver = A.SubdivisionSolver(box_capacity=1 << 22, root_capacity=1 << 20)
    ids, params, thr, st = solver.run(1, ev, sc.light_point(0), ends, rows, etas, ds.tris, ds.attribs, ds.builder,
                                      ds.tris)
    spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")
    solver.contribute(1, ev, sc, rows, st["roots"], frame, etas, ds.tris, ds.attribs, spectral)
    torch.cuda.synchronize()
    assert n > 0 and st["roots"] > 0
    ids_s, params_s, thr_s = _sorted(ids, params, thr)
    bo = orc.build_bvh(sc.tris, 0)
    rows_h = rows.cpu().numpy()
    exp, est = orc.subdivide_solve(1, ev, sc.light_point(0), ends.cpu().numpy(), rows_h, sc.bin_etas(), sc.tris,
                                   sc.attribs, bo, sc.tris)
    _check_equal(exp, ids_s, params_s, thr_s, 1)
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    img = orc.subdivide_contribute(1, ev, sc, rows_h, exp, fd, sc.bin_etas(), sc.tris, sc.attribs)
    gpu = spectral.cpu().numpy().astype(np.float64)
    rel = float(np.sqrt(((gpu - img) ** 2).mean() / (img.astype(np.float64) ** 2).mean()))
    assert img.sum() > 0 and rel < 1e-6, rel
    # against the single-start solve of the same work list (exact-arithmetic plain build)
    plain = torch.zeros_like(spectral)
    A.solve_specular_plain(A.solve_desc(ds, frame, cache, "T", n, spectral=plain, etas=etas, exact=True))
    torch.cuda.synchronize()
    pl = plain.cpu().numpy().astype(np.float64)
    print(f"\n{n} work items x {sc.n_bins} bins: {st['boxes_tested']} boxes, {st['leaves']} leaves, "
          f"{st['roots']} roots; image vs oracle {rel:.1e}; energy subdivision / single start "
          f"{gpu.sum() / max(pl.sum(), 1e-30):.4f}")


def test_host_checks():
    L = _lib.lib()
    p = _lib.SubdivParams(12, 1e-4, 32, 1e-10, 1, 0)
    n = C.c_uint64(0)
    z = _lib.f3((0, 0, 0))
    assert L.pz_subdivide_solve(5, 1, z, None, None, 1, None, 1, C.byref(p), None, None, None, None, None, None, 0,
                                C.byref(n), None, None, 0, None) == 1
    bad = _lib.SubdivParams(21, 1e-4, 32, 1e-10, 1, 0)
    assert L.pz_subdivide_solve(1, 1, z, None, None, 1, None, 1, C.byref(bad), None, None, None, None, None, None, 0,
                                C.byref(n), None, None, 0, None) == 1
    assert L.pz_subdivide_solve(1, 1, z, None, None, 0, None, 1, C.byref(p), None, None, None, None, None, None, 0,
                                C.byref(n), None, None, 0, None) == 0 and n.value == 0
    assert L.pz_subdivide_contribute(1, 1, z, 1.0, 1.0, None, None, 0, None, None, 1, None, None, None, None) == 0
    assert L.pz_subdivide_scratch_bytes(1000) >= 256 + 3 * 8000


def test_capacity_overflow_is_reported():
    """A root list or leaf list too small for the work is reported as PZ_ERR_DEVICE (the
    kernels drop what does not fit and set the capacity bit), and the counts still say how
    many roots there were.  (The box queue itself needs little room: each warp keeps the
    boxes of its tuples on its own stack, so a box capacity of one entry per tuple holds the
    queue; the leaf list has the same capacity and overflows when the leaves outnumber it.)"""
    sc = S.lens_scene(side=8, seed=5, amplitude=0.05, events="T", width=16, height=16)
    t, at, b = _dev(sc)
    ends = torch.from_numpy(_ends(6, 2)).cuda()
    spec = np.nonzero(sc.attribs["material"] != 0)[0]
    rows = torch.from_numpy(np.array([[q, i] for q in range(6) for i in spec], np.int32)).cuda()
    etas = torch.tensor([1.5, 1.53, 1.56], device="cuda")
    ev = S.event_descriptor("T")
    ok = A.SubdivisionSolver(box_capacity=1 << 16, root_capacity=1 << 12)
    _, _, _, st = ok.run(1, ev, sc.p_light, ends, rows, etas, t, at, b, t)
    assert st["roots"] > 4
    small_roots = A.SubdivisionSolver(box_capacity=1 << 16, root_capacity=4)
    with pytest.raises(RuntimeError, match="capacity"):
        small_roots.run(1, ev, sc.p_light, ends, rows, etas, t, at, b, t)
    # a lens frame's work list has several leaves per tuple: a leaf list with room for one
    # per tuple (the least scratch the solver accepts) overflows
    fs = S.lens_scene(side=32, seed=1, events="T", width=48, height=48, n_bins=4)
    ds = A.DeviceScene(fs)
    frame = A.Frame(fs, path_capacity=1 << 20)
    cache = A.PathCache(capacity=1 << 20, step=fs.cell_step)
    A.solve_primary(ds, frame, iteration=0)
    A.photon_trace(ds, cache, iteration=0)
    nf = A.lookup_flatten(frame, cache, ev)
    frows = A.work_list_rows(frame, cache, nf, 1)
    fends = A.receiver_points(frame)
    fetas = torch.from_numpy(fs.bin_etas()).cuda()
    big = A.SubdivisionSolver(box_capacity=1 << 22, root_capacity=1 << 20)
    _, _, _, stf = big.run(1, ev, fs.light_point(0), fends, frows, fetas, ds.tris, ds.attribs, ds.builder, ds.tris)
    assert stf["leaves"] > 2 * nf
    small_boxes = A.SubdivisionSolver(box_capacity=nf, root_capacity=1 << 20)
    with pytest.raises(RuntimeError, match="capacity"):
        small_boxes.run(1, ev, fs.light_point(0), fends, frows, fetas, ds.tris, ds.attribs, ds.builder, ds.tris)
    # the solver stays usable after an overflow
    _, _, _, st2 = ok.run(1, ev, sc.p_light, ends, rows, etas, t, at, b, t)
    assert st2 == st
