"""Root-by-root parity of the specular solver (solved vertices within 1e-5 relative of the
oracle from the same initial barycentrics; the FP64 error stated beside it).

* pz_solve_constraints -- the device-callable solveConstraints<K> of
  include/palzilla_b200_device.cuh (pk.h:466-592) run over a batch -- against the
  reference's own CPU solveConstraints (oracle/_ref, when built) and the restatement:
  converged flags, last iteration and roots bit for bit, on the golden solver records and on
  fresh two-refraction tuples;
* the roots of every (item, bin) the plain solve converged on (pz_solve_desc.roots) against
  the oracle's solve from the photon's barycentrics, bit for bit;
* the batched solve's roots: bins solved from the photon's barycentrics bit for bit equal to
  the plain roots; bins refined from a predicted root (deep inside the triangles) start
  elsewhere and stop at another point within the cost tolerance, so their solved vertices are
  held within 1e-5 relative of the FP64 root; and a root for every (item, bin) that
  contributes to the plain image.
"""
import os

import numpy as np
import pytest
import torch

import oracle as O
from palzilla_b200 import _lib
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def _solve_device(K, ev, p_beg, tuples, params, p_end, etas, tris, attribs, max_iter=32, tol=1e-10, warmup=1):
    """pz_solve_constraints over a batch; every device buffer is held in a local until the
    kernel has finished (a pointer taken from a temporary tensor would be freed, and its
    memory handed to the next allocation, before the launch)."""
    n = len(tuples)
    t_tris = torch.from_numpy(np.ascontiguousarray(tris, np.float32)).cuda()
    t_att = torch.from_numpy(np.ascontiguousarray(attribs).view(np.uint8).reshape(-1)).cuda()
    t_tup = torch.from_numpy(np.ascontiguousarray(tuples, np.int32).reshape(n, K)).cuda()
    t_end = torch.from_numpy(np.ascontiguousarray(p_end, np.float32).reshape(n, 3)).cuda()
    t_eta = torch.from_numpy(np.ascontiguousarray(etas, np.float32).reshape(n)).cuda()
    prm = torch.from_numpy(np.ascontiguousarray(params, np.float32).reshape(n, 2 * K)).cuda()
    conv = torch.zeros(n, dtype=torch.uint8, device="cuda")
    its = torch.zeros(n, dtype=torch.int32, device="cuda")
    n_tris = int(t_tris.numel() // 9)
    assert t_att.numel() == 40 * n_tris and int(np.max(tuples)) < n_tris and int(np.min(tuples)) >= 0
    _lib.call("pz_solve_constraints", K, ev, _lib.f3(p_beg), A._vp(t_tup), A._vp(t_end), A._vp(t_eta), n,
              A._vp(t_tris), A._vp(t_att), n_tris, max_iter, _lib.f32(tol), warmup, A._vp(prm), A._vp(conv),
              A._vp(its), None)
    torch.cuda.synchronize()
    return conv.cpu().numpy().astype(bool), prm.cpu().numpy(), its.cpu().numpy()


def test_device_solver_on_golden_records(orc):
    """The golden solveConstraints records (the reference's own roots, K = 1)."""
    g = np.load(GOLDEN)
    lens = S.lens_scene(side=16, seed=1, width=32, height=32, n_bins=4, events="T")
    recs = g["photon_records"].reshape(-1).view(O.RECORD_DTYPE)
    sel = recs[g["solve_records"]]
    ok, x, its = _solve_device(1, S.event_descriptor("T"), lens.p_light, sel["tris"][:, :1], sel["params"][:, :2],
                               g["solve_p_end"], g["solve_eta"], lens.tris, lens.attribs)
    assert np.array_equal(ok, g["solve_ok"].astype(bool))
    assert x.tobytes() == g["solve_roots"].tobytes()
    assert np.array_equal(its[ok], g["solve_iters"][ok])


@pytest.mark.parametrize("events", ["T", "TT"])
def test_device_solver_against_reference(orc, ref, events):
    """Fresh photon tuples of a single-sheet (T) and a two-sheet (TT) lens, solved from the
    photon's barycentrics towards points next to where each photon landed."""
    K = len(events)
    sc = S.lens_scene(side=24, seed=5, amplitude=0.03, events=events)
    ev = S.event_descriptor(events)
    recs = orc.photon_trace(orc.build_bvh(sc.tris), sc, iteration=1, photons_per_tri=16)
    recs = recs[recs["ev"] == ev]
    rng = np.random.default_rng(40 + K)
    recs = recs[rng.choice(len(recs), size=min(len(recs), 3000), replace=False)]
    n = len(recs)
    tuples = np.ascontiguousarray(recs["tris"][:, :K], np.int32)
    params = np.ascontiguousarray(recs["params"][:, :2 * K], np.float32)
    p_end = (recs["p"] + rng.normal(0.0, 0.01, (n, 3)) * np.array([1, 0, 1])).astype(np.float32)
    etas = rng.uniform(1.45, 1.6, n).astype(np.float32)
    ok, x, its = _solve_device(K, ev, sc.p_light, tuples, params, p_end, etas, sc.tris, sc.attribs)
    n_conv = 0
    worst64 = 0.0
    for i in range(n):
        o, xr, it = ref.solve_constraints(K, params[i], sc.p_light, p_end[i], sc.tris[tuples[i]],
                                          sc.attribs[tuples[i]], float(etas[i]), ev)
        assert bool(o) == ok[i], i
        assert xr.tobytes() == x[i].tobytes(), (i, xr, x[i])
        if o:
            assert it == its[i]
            n_conv += 1
            od, xd, _ = orc.solve_constraints(K, params[i], sc.p_light, p_end[i], sc.tris[tuples[i]],
                                              sc.attribs[tuples[i]], float(etas[i]), ev, dtype=np.float64)
            if od:
                worst64 = max(worst64, float(np.max(np.abs(xd - x[i]))))
    assert n > 500 and n_conv > 100, (n, n_conv)
    print(f"\n[{events}] {n_conv} of {n} converged, bitwise equal to the reference; max |x32 - x64| {worst64:.2e}")


def _frame(events, side=40, seed=21, W=96, H=96, bins=8):
    sc = S.lens_scene(side=side, seed=seed, width=W, height=H, n_bins=bins, events=events)
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 22)
    A.solve_primary(ds, frame, iteration=0)
    cache = A.PathCache(capacity=1 << 20, step=sc.cell_step)
    A.photon_trace(ds, cache, iteration=0)
    n = A.lookup_flatten(frame, cache, S.event_descriptor(sc.events))
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    torch.cuda.synchronize()
    return sc, ds, frame, cache, n


@pytest.mark.parametrize("events", ["T", "TT"])
def test_plain_and_batched_roots(orc, events):
    sc, ds, frame, cache, n = _frame(events)
    K, B = len(events), sc.n_bins
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    roots = {}
    imgs = {}
    for mode in ("plain", "batched"):
        r = torch.full((n * B * 8,), float("nan"), device="cuda")
        spectral = torch.zeros((sc.width * sc.height, B), device="cuda")
        d = A.solve_desc(ds, frame, cache, events, n, spectral=spectral, etas=etas, roots=r)
        if mode == "plain":
            A.solve_specular_plain(d)
        else:
            A.solve_specular_batched(d, A.Scratch())
        torch.cuda.synchronize()
        roots[mode] = r.cpu().numpy().reshape(n, B, 8)[:, :, :2 * K]
        imgs[mode] = spectral.cpu().numpy()
    pairs = frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2)
    gc = cache.to_host()
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    ev = S.event_descriptor(events)
    L = sc.light_point(0)
    # plain roots bit for bit against the oracle on a sample of (item, bin)
    rng = np.random.default_rng(3)
    items = rng.choice(n, size=min(n, 400), replace=False)
    checked = 0
    for i in items:
        px, slot = pairs[i]
        tup = gc["tris"][slot, :K]
        for b in range(B):
            o, x, _ = orc.solve_constraints(K, gc["params"][slot, :2 * K], L, fd[px, :3], sc.tris[tup],
                                            sc.attribs[tup], float(sc.bin_etas()[b]), ev)
            got = roots["plain"][i, b]
            assert o == bool(np.isfinite(got).all()), (i, b)
            if o:
                assert got.tobytes() == x.astype(np.float32).tobytes(), (i, b, got, x)
                checked += 1
    assert checked > 50
    # batched roots: a bin solved from the photon's barycentrics equals the plain root bit for
    # bit; a bin refined from its predicted root stops at another point of the cost tolerance
    # (cost < 1e-10), so it is held to the FP64 root (double Newton to 1e-24 from it): solved
    # vertices within 1e-5 relative, as the plain root itself is to the same FP64 root
    p, q = roots["plain"], roots["batched"]
    both = np.isfinite(p).all(-1) & np.isfinite(q).all(-1)
    assert both.sum() > 100
    same = both & (p == q).all(-1)
    it, bn = np.nonzero(both & ~same)
    sel = rng.choice(len(it), size=min(len(it), 1500), replace=False) if len(it) else np.zeros(0, int)
    etas_h = sc.bin_etas()

    def vertices(x, tup):
        out = []
        for k in range(K):
            t = sc.tris[tup[k]].astype(np.float64).reshape(3, 3)
            out.append(t[0] + (t[1] - t[0]) * float(x[2 * k]) + (t[2] - t[0]) * float(x[2 * k + 1]))
        return np.array(out)

    worst_b, worst_p = 0.0, 0.0
    for s_ in sel:
        i, b = it[s_], bn[s_]
        px, slot = pairs[i]
        tup = gc["tris"][slot, :K]
        o, x64, _ = orc.solve_constraints(K, q[i, b].astype(np.float64), L, fd[px, :3], sc.tris[tup], sc.attribs[tup],
                                          float(etas_h[b]), ev, max_iter=8, tol=1e-24, warmup=64, dtype=np.float64)
        v64 = vertices(x64, tup)
        scale = np.linalg.norm(v64, axis=1)
        worst_b = max(worst_b, float((np.linalg.norm(vertices(q[i, b], tup) - v64, axis=1) / scale).max()))
        worst_p = max(worst_p, float((np.linalg.norm(vertices(p[i, b], tup) - v64, axis=1) / scale).max()))
    assert worst_b <= 1e-5, worst_b
    # every (item, bin) that contributes to the plain image has a batched root
    contrib = orc.render_each(K, pairs, gc, fd, orc.build_bvh(sc.tris), sc, sc.bin_etas(), dtype=np.float32) > 0
    assert contrib.any()
    assert np.isfinite(q[contrib]).all(-1).all()
    print(f"\n[{events}] plain roots bitwise on {checked} (item, bin); batched roots: {int(same.sum())} of "
          f"{int(both.sum())} bitwise equal to the plain ones, the others within {worst_b:.1e} (vertex, relative) of "
          f"the FP64 root, where the plain roots are within {worst_p:.1e}")
