"""This library's kernels against the reference's own GPU kernels on the same device.

The reference's minimum_lbvh.cu and main_gpu.cu are compiled for sm_100a from its sources
(oracle/build_ref_gpu.sh; -fmad=false, its CPU float arithmetic) and launched as its
renderer launches them (oracle/ref_gpu.py):
* LBVH: getSceneAABB, buildMortons, computeDeltas and build, with the keys sorted by this
  library's stable sort (the reference's onesweep reorder is not run: it takes its tile
  index from blockIdx.x and spins without bound on its predecessors) -- nodes, root, sorted
  keys and deltas bit for bit against pz_bvh_build;
* photon pass: photonTrace into the reference's array-of-structs PathCache against
  pz_photon_trace -- the sets of cached paths agree to 0.1% (the reference's GPU build
  normalises with the approximate rsqrtf where its CPU code, which this library follows bit
  for bit, divides by sqrt; which photon claims a slot is racy in both);
* specular solve in the reference's own mode (one wavelength per pixel, RGB into the
  float4 accumulator): solveSpecularPath_K<K> against pz_solve_specular_plain on the same
  work list: pixels lit in both within 1e-5 relative RMSE (the reference's CMF weights use
  __expf, this library's expf), pixels lit in one only bounded, and the images within the
  1e-3 relative RMSE bar.
"""
import numpy as np
import pytest
import torch

import ref_gpu
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available("exact"), reason="reference GPU kernels not built here")]


@pytest.fixture(scope="module")
def rg():
    return ref_gpu.RefGpu("exact")


def _sorter():
    s = A.OnesweepSort()
    return lambda keys, tmp, n: s.sort(keys, None, tmp, None, n, 0, 32)


@pytest.mark.parametrize("which", ["sphere", "lens", "soup"])
def test_lbvh_against_reference_kernels(rg, which):
    if which == "sphere":
        tris = S.sphere_scene().tris
    elif which == "lens":
        tris = S.lens_scene(side=64, seed=3).tris
    else:
        tris = S.random_soup((1 << 20) + 77, seed=9)
    n = tris.shape[0]
    t = torch.from_numpy(np.ascontiguousarray(tris, np.float32)).cuda()
    nodes, root, keys, deltas = rg.bvh_build(t, n, _sorter())
    b = A.BVHGPUBuilder()
    b.build(t, n, 0)
    torch.cuda.synchronize()
    ours_sorted, ours_deltas, _ = b.debug_views()
    assert torch.equal(keys, ours_sorted)
    assert torch.equal(deltas[: n - 1], ours_deltas)
    assert torch.equal(nodes[: (n - 1) * 64], b.m_internals[: (n - 1) * 64])
    assert int(root.item()) & 0xFFFFFFFF == b.root


def _paths(hashes, events, tris):
    used = hashes != 0
    return set(zip(hashes[used].tolist(), events[used].tolist(), map(tuple, tris[used].tolist())))


def test_photon_pass_against_reference_kernel(rg):
    """The reference's GPU build normalises with the device's approximate rsqrtf
    (helper_math.h:1437-1441; e.g. the photon's ray offset, main_gpu.cu:190), where its CPU
    code -- and this library, which is pinned to it bit for bit -- divides by sqrt; so the
    two GPU photon passes may disagree on a marginal photon.  The set of cached paths
    {hash, event string, triangles} must agree to 0.1%."""
    sc = S.lens_scene(side=48, seed=11, width=64, height=64, n_bins=4, events="TT")
    ds = A.DeviceScene(sc)
    cache = A.PathCache(capacity=rg.capacity, step=sc.cell_step)
    A.photon_trace(ds, cache, iteration=4)
    rc = rg.new_cache()
    stack = rg.new_stack()
    emin, emax = sc.eta_range()
    rg.photon_trace(rc, ds.internals, ds.root_dev, ds.tris, ds.attribs, ds.n, sc.light_point(4), emin, emax, 4,
                    sc.cell_step, sc.min_throughput, stack)
    torch.cuda.synchronize()
    g = cache.to_host()
    rp = rc["paths"].cpu().numpy()
    ours = _paths(g["hash"], g["events"], g["tris"])
    ref = _paths(rc["hashes"].cpu().numpy().view(np.uint32), rp[:, 1].view(np.uint32), rp[:, 2:6])
    diff = len(ours ^ ref)
    assert len(ref) > 1000 and diff <= 1e-3 * len(ref), (len(ours), len(ref), diff)
    print(f"\n{len(ours)} cached paths here, {len(ref)} by the reference's kernel, {diff} differ")
    del stack


@pytest.mark.parametrize("events", ["T", "TT"])
def test_reference_mode_solve_against_reference_kernel(rg, events):
    sc = S.lens_scene(side=40, seed=21, width=128, height=128, n_bins=1, events=events)
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 22)
    A.solve_primary(ds, frame, iteration=2)
    cache = A.PathCache(capacity=rg.capacity, step=sc.cell_step)
    A.photon_trace(ds, cache, iteration=2)
    ev = S.event_descriptor(events)
    n = A.lookup_flatten(frame, cache, ev)
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    frame.accum.zero_()
    A.solve_specular_plain(A.solve_desc(ds, frame, cache, events, n))
    acc_ref = torch.zeros_like(frame.accum)
    rc = rg.cache_from_ours(cache.views())
    rg.solve_specular(len(events), acc_ref, frame.paths, n, frame.fd, ds.root_dev, ds.internals, ds.tris, ds.attribs,
                      sc.light_point(2), sc.light_intensity, sc.radiance_clamp, rc, sc.cell_step, ev, sc.cauchy_a,
                      sc.cauchy_b, 2)
    torch.cuda.synchronize()
    ours, ref = frame.accum[:, :3].double(), acc_ref[:, :3].double()
    assert n > 0 and float(ref.abs().sum()) > 0
    # the reference's GPU build normalises with the approximate rsqrtf (shading normals, the
    # shadow rays' offsets, the receiver cosine), so a marginal path may flip: pixels lit in
    # one image only are counted and bounded; where both are lit the values agree to 1e-5
    lit_o, lit_r = (ours != 0).any(1), (ref != 0).any(1)
    both = lit_o & lit_r
    flipped = int((lit_o ^ lit_r).sum())
    assert flipped <= max(2, int(1e-3 * int(lit_r.sum()))), (flipped, int(lit_r.sum()))
    rel_both = float(torch.sqrt(((ours[both] - ref[both]) ** 2).mean() / (ref[both] ** 2).mean()))
    rel = float(torch.sqrt(((ours - ref) ** 2).mean() / (ref ** 2).mean()))
    assert rel_both <= 1e-5, rel_both
    assert rel <= 1e-3, rel
    print(f"\n[{events}] {n} items; against the reference's solveSpecularPath_K{len(events)}: rel RMSE {rel:.1e}, "
          f"{rel_both:.1e} over the {int(both.sum())} pixels both light, {flipped} pixels lit in one image only")
