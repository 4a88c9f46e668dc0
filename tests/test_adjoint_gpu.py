"""Adjoint of the caustic render (pz_adjoint_forward / pz_adjoint_backward) on the
heightfield lens of the gradient workload: 128 x 128 vertex grid (32,258 triangles), 512 x 512
image, 8 wavelength bins, target image rendered from a second seeded heightfield, L2 loss.
Gradients with respect to the vertex heights and the Cauchy coefficients (A, B) are
checked on 64 seeded random vertices:

* against central finite differences of the GPU render itself (step 1e-3 on the heights);
* against an FP64 reference: the vector-Jacobian product g . dI/dh with the same loss
  weights g = dL/dI, from central differences of the CPU oracle's FP64 render at steps
  2^-12 and 2^-13 (heights stay exactly representable) with Richardson extrapolation.

The work list is fixed at the initial geometry; the edge tests, visibility and the clamp
select paths but carry no gradient, so single vertices whose paths cross a triangle edge
within the step are outliers of the finite differences; the bounds below are on the
agreement over the 64 vertices.
"""
import numpy as np
import pytest
import torch

import oracle as O
from palzilla_b200 import scenes as S

from grad_harness import CausticProblem, CausticRender

pytestmark = pytest.mark.gpu

SIDE = 128


@pytest.fixture(scope="module")
def setup():
    sc, corners, h0 = S.adjoint_scene(side=SIDE, seed=1)
    P = CausticProblem(sc, corners)
    sc2, c2, h2 = S.adjoint_scene(side=SIDE, seed=2)
    P2 = CausticProblem(sc2, c2)
    cauchy = torch.tensor([1.5, 4200.0], dtype=torch.float32, device="cuda")
    target = P2.forward(torch.from_numpy(h2).cuda(), cauchy).clone()
    torch.cuda.synchronize()
    del P2
    heights = torch.from_numpy(h0).cuda()
    h = heights.clone().requires_grad_(True)
    c = cauchy.clone().requires_grad_(True)
    I = CausticRender.apply(h, c, P)
    loss = ((I - target) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    g = (2.0 * (I.detach() - target)).cpu().numpy()
    rng = np.random.default_rng(4001)
    interior = [(r, q) for r in range(2, SIDE - 2) for q in range(2, SIDE - 2)]
    pick = rng.choice(len(interior), 64, replace=False)
    verts = np.array([interior[i][0] * SIDE + interior[i][1] for i in pick], np.int64)
    return dict(P=P, sc=sc, corners=corners, heights=heights, cauchy=cauchy, target=target, I=I.detach(),
                grad_h=h.grad.detach().cpu().numpy(), grad_c=c.grad.detach().cpu().numpy(), g=g, verts=verts)


def _touched(st, v):
    """Work items whose tuple triangle has vertex v, and the pixels they write."""
    P = st["P"]
    tris_of_v = np.nonzero((st["corners"] == v).any(1))[0]
    pairs = P.frame.paths[: P.n_paths * 8].cpu().numpy().view(np.int32).reshape(-1, 2)
    if "slot_tri" not in st:
        st["slot_tri"] = P.cache.to_host()["tris"][:, 0]
        st["pairs"] = pairs.copy()
    sel = np.isin(st["slot_tri"][st["pairs"][:, 1]], tris_of_v)
    return st["pairs"][sel], np.unique(st["pairs"][sel][:, 0])


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-12)


def test_gradient_vs_gpu_finite_differences(setup):
    """Central differences of the GPU loss at step 1e-3 on the heights.  Paths that cross
    a triangle edge or the clamp within the step make single differences jump; the bound
    is on the median disagreement, relative to the largest gradient."""
    st = setup
    P, h0, cauchy, target = st["P"], st["heights"], st["cauchy"], st["target"]
    step = 1e-3
    fd, an = [], []
    for v in st["verts"]:
        _, px = _touched(st, v)
        pxt = torch.from_numpy(px).cuda().long()
        Ls = []
        for s in (+1.0, -1.0):
            h = h0.clone()
            h[v] += s * step
            I = P.forward(h, cauchy)
            Ls.append(float(((I[pxt] - target[pxt]).double() ** 2).sum()))
        fd.append((Ls[0] - Ls[1]) / (2.0 * step))
        an.append(st["grad_h"][v])
    P.set_heights(h0)
    fd, an = np.array(fd), np.array(an)
    scale = np.abs(an).max()
    err = np.abs(fd - an) / scale
    print(f"\n[fd 1e-3] max |grad| {scale:.3e}  median err {np.median(err):.2e}  p75 {np.percentile(err, 75):.2e}  "
          f"max {err.max():.2e}")
    assert np.median(err) < 2e-2


def _accepted(c, clamp):
    return (c > 0) & (c < clamp)


def test_gradient_vs_fp64_reference(setup, orc):
    """FP64 reference: central differences of the CPU oracle's FP64 per-path contributions at
    two exactly representable steps with Richardson extrapolation, weighted by the same
    g = dL/dI, over the paths that every render accepts unclamped (the FP32 forward's set
    included), so that no path enters or leaves the set between the perturbed states."""
    st = setup
    P, sc = st["P"], st["sc"]
    cache = P.cache.to_host()
    fd_host = P.frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    base = P.base_tris.cpu().numpy().reshape(-1, 3, 3).copy()
    h0 = st["heights"].cpu().numpy()
    corners = st["corners"]
    etas = sc.bin_etas()
    g = st["g"]
    clamp = sc.radiance_clamp
    m = corners >= 0

    def render(pairs, hh, et, dtype=np.float64):
        tris = base.copy()
        tris[:, :, 1][m] = hh[corners[m]]
        tris = tris.reshape(-1, 9)
        sc.tris = tris
        bvh = orc.build_bvh(tris)
        return orc.render_each(1, pairs, cache, fd_host, bvh, sc, et, dtype=dtype)

    ref, an = [], []
    try:
        for v in st["verts"]:
            pairs, _ = _touched(st, v)
            if len(pairs) == 0:
                continue
            c0 = render(pairs, h0, etas)
            c32 = render(pairs, h0, etas, np.float32)  # the GPU forward's own decisions
            if any(np.float32(h0[v] + sg * h) != h0[v] + sg * h for h in (2.0 ** -12, 2.0 ** -13) for sg in (1, -1)):
                continue  # a height next to a binade edge: no exact step
            states = []
            for h in (2.0 ** -12, 2.0 ** -13):
                for sgn in (+1.0, -1.0):
                    hh = h0.copy()
                    hh[v] = np.float32(h0[v] + sgn * h)
                    states.append(render(pairs, hh, etas))
            ok = _accepted(c32, clamp) & _accepted(c0, clamp)
            for c in states:
                ok &= _accepted(c, clamp)
            w = g[pairs[:, 0]] * ok
            d1 = float((w * (states[0] - states[1])).sum()) / (2.0 * 2.0 ** -12)
            d2 = float((w * (states[2] - states[3])).sum()) / (2.0 * 2.0 ** -13)
            ref.append((4.0 * d2 - d1) / 3.0)
            an.append(st["grad_h"][v])

        # Cauchy coefficients over every work item: d eta_b = h for every bin
        pairs_all = st["pairs"]
        sc.tris = base.reshape(-1, 9)
        bvh = orc.build_bvh(sc.tris)
        c0 = orc.render_each(1, pairs_all, cache, fd_host, bvh, sc, etas)
        ok = _accepted(c0, clamp) & _accepted(orc.render_each(1, pairs_all, cache, fd_host, bvh, sc, etas,
                                                              dtype=np.float32), clamp)
        del c0
        diffs = []
        for h in (2.0 ** -16, 2.0 ** -17):
            cp = orc.render_each(1, pairs_all, cache, fd_host, bvh, sc, (etas + np.float32(h)).astype(np.float32))
            cm = orc.render_each(1, pairs_all, cache, fd_host, bvh, sc, (etas - np.float32(h)).astype(np.float32))
            ok &= _accepted(cp, clamp) & _accepted(cm, clamp)
            diffs.append((cp - cm) / (2.0 * h))
            del cp, cm
        w = g[pairs_all[:, 0]] * ok
        per_bin = [(w * dd).sum(0) for dd in diffs]
        dLdeta = (4.0 * per_bin[1] - per_bin[0]) / 3.0
        print(f"\n[fp64 cauchy] paths in the reference set {int(ok.sum())} of {ok.size}")
        dA = float(dLdeta.sum())
        dB = float((dLdeta * (etas.astype(np.float64) - sc.cauchy_a) / sc.cauchy_b).sum())
    finally:
        sc.tris = base.reshape(-1, 9)
    ref, an = np.array(ref), np.array(an)
    assert len(ref) >= 40
    scale = np.abs(ref).max()
    err = np.abs(ref - an) / scale
    rel = np.abs(ref - an) / np.maximum(np.abs(ref), 1e-30)
    print(f"\n[fp64 heights] n {len(ref)}  max |grad| {scale:.3e}  median err {np.median(err):.2e}  "
          f"p90 {np.percentile(err, 90):.2e}  max {err.max():.2e}  median rel {np.median(rel):.2e}")
    print(f"[fp64 cauchy] dL/dA ref {dA:.6e} adjoint {st['grad_c'][0]:.6e} | dL/dB ref {dB:.6e} "
          f"adjoint {st['grad_c'][1]:.6e}")
    assert np.median(err) < 1e-3
    assert np.percentile(err, 90) < 2e-2
    # a global parameter sums ~5 M path derivatives, some of them near caustic folds where
    # the FP32 derivative of 1 / dAdw loses digits: a few percent
    assert _rel(st["grad_c"][0], dA) < 5e-2 and _rel(st["grad_c"][1], dB) < 5e-2


def test_compact_backward_equals_one_kernel(setup):
    """pz_adjoint_backward_compact (filter the accepted paths into a list, then
    differentiate only those) gives the one-kernel pz_adjoint_backward's gradients, up to
    the order of the float atomics; a list too small for the accepted paths sets the
    capacity bit of the scratch status word."""
    import ctypes as C
    from palzilla_b200 import _lib
    from palzilla_b200 import api as A
    P, h, cauchy = setup["P"], setup["heights"], setup["cauchy"]
    g = (2.0 * (setup["I"] - setup["target"])).contiguous()
    gh1, gc1 = P.backward(h, cauchy, g, compact=True)
    gh0, gc0 = P.backward(h, cauchy, g, compact=False)
    torch.cuda.synchronize()
    a, b = gh1.cpu().numpy().astype(np.float64), gh0.cpu().numpy().astype(np.float64)
    err = np.abs(a - b).max() / np.abs(b).max()
    errc = np.abs(gc1.cpu().numpy() - gc0.cpu().numpy()) / np.abs(gc0.cpu().numpy())
    print(f"\ncompact vs one kernel: heights max err {err:.1e} of the largest, cauchy {errc.max():.1e}")
    # a height gradient sums a few hundred path terms; dL/dA and dL/dB sum millions of terms
    # of both signs in float atomics, whose order alone moves them by about 1e-4 relative
    assert np.abs(b).max() > 0 and err < 1e-4 and errc.max() < 2e-3
    # a list of 1,000 pairs: the gradient misses the rest, and the status word says so
    P.set_heights(h)
    d = P.desc(cauchy, torch.zeros(1, device="cuda"), P.etas(cauchy))
    small = torch.empty(_lib.lib().pz_adjoint_scratch_bytes(1000), dtype=torch.uint8, device="cuda")
    gh2, gc2 = torch.zeros_like(h), torch.zeros(2, device="cuda")
    _lib.call("pz_adjoint_backward_compact", C.byref(d), A._vp(g), A._vp(P.corners), A._vp(gh2), A._vp(gc2),
              A._vp(small), C.c_size_t(small.numel()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    st = C.c_uint32(0)
    _lib.call("pz_scratch_status", C.c_void_p(small.data_ptr()), C.byref(st),
              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st.value & 0x2
