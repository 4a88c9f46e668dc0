"""LBVH parity: GPU builder output bit-exact with the oracle (the reference's builder
run on the stable sort order): sorted keys, deltas, every InternalNode field and root.
"""
import numpy as np
import pytest
import torch

from palzilla_b200 import scenes as S
from palzilla_b200.api import BVHGPUBuilder

pytestmark = pytest.mark.gpu


def gpu_build(tris, opt=0):
    b = BVHGPUBuilder()
    t = torch.from_numpy(np.ascontiguousarray(tris, np.float32)).cuda()
    n = tris.shape[0]
    b.build(t, n, opt)
    torch.cuda.synchronize()
    assert b.scratch.status() == 0
    sorted_, deltas, aabb = b.debug_views()
    nodes = b.m_internals[: max(n - 1, 0) * 64].cpu().numpy()
    return dict(nodes=nodes, root=b.root, sorted=sorted_.cpu().numpy().view(np.uint64),
                deltas=deltas.cpu().numpy(), aabb=np.array(aabb, np.float32))


def check(orc, tris, opt=0):
    g = gpu_build(tris, opt)
    o = orc.build_bvh(tris, opt)
    n = tris.shape[0]
    assert g["root"] == o["root"]
    if n >= 1:
        assert np.array_equal(g["sorted"], o["sorted"])
        assert np.array_equal(g["aabb"], o["aabb"])
    if n >= 2:
        assert np.array_equal(g["deltas"], o["deltas"])
        assert g["nodes"].tobytes() == o["nodes"].tobytes()
        assert orc.validate_lbvh(o["nodes"], o["root"], o["deltas"])


@pytest.mark.parametrize("n", [1, 2, 3, 257, 513, 4097, 65_537, 300_001])
def test_random_soup(orc, n):
    check(orc, S.random_soup(n, seed=1000 + n))


def test_lens_scene(orc):
    check(orc, S.lens_scene().tris)


def test_sphere_scene(orc):
    check(orc, S.sphere_scene().tris)


def test_use_normal_option(orc):
    check(orc, S.lens_scene(events="TT").tris, opt=1)


def test_duplicate_centroids(orc):
    # many triangles with identical centroids: equal Morton keys, order decided by stability
    base = S.random_soup(64, seed=9)
    tris = np.repeat(base, 50, axis=0)
    check(orc, tris)


def test_empty_scene():
    b = BVHGPUBuilder()
    t = torch.zeros((1, 9), dtype=torch.float32, device="cuda")
    b.build(t, 0)
    torch.cuda.synchronize()
    assert b.root == 0x7FFFFFFF


def test_full_size_build_valid(orc):
    """2^22 random triangles: the GPU tree satisfies the delta-monotonicity invariant
    (validate_lbvh, minimum_lbvh.h:424-435) and every leaf appears exactly once."""
    n = 1 << 22
    tris = S.random_soup(n, seed=2022)
    g = gpu_build(tris)
    nodes = np.frombuffer(g["nodes"].tobytes(), dtype=np.dtype([("c", "<u4", (2,)), ("b", "<f4", (12,)),
                                                                ("p", "<u4"), ("x", "<u4")]))
    assert orc.validate_lbvh(g["nodes"], g["root"], g["deltas"])
    ch = nodes["c"].ravel()
    leaves = ch[(ch >> 31) == 1] & 0x7FFFFFFF
    assert leaves.size == n and np.array_equal(np.sort(leaves), np.arange(n, dtype=np.uint32))
