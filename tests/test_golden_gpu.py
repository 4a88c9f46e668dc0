"""GPU path against the golden vectors of the reference's own CPU code
(tests/golden/golden.npz, made by tests/golden/make_golden.py from oracle/_ref): LBVH
nodes, root, sorted keys and deltas; closest and any hits; photon records; the PathCache
hash set; all bitwise."""
import os

import numpy as np
import pytest
import torch

from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


@pytest.mark.parametrize("name", ["lens", "ico3", "soup"])
def test_lbvh_matches_golden(g, name):
    tris = torch.from_numpy(g[f"{name}_tris"]).cuda()
    b = A.BVHGPUBuilder()
    b.build(tris, tris.shape[0], 0)
    torch.cuda.synchronize()
    n = tris.shape[0]
    assert b.m_internals[: (n - 1) * 64].cpu().numpy().tobytes() == g[f"{name}_nodes"].tobytes()
    assert b.root == int(g[f"{name}_root"][0])
    sorted_, deltas, _ = b.debug_views()
    assert np.array_equal(sorted_.cpu().numpy().view(np.uint64), g[f"{name}_sorted"])
    assert np.array_equal(deltas.cpu().numpy(), g[f"{name}_deltas"])


def test_rays_and_photons_match_golden(g):
    sc = S.lens_scene(side=16, seed=1, width=32, height=32, n_bins=4, events="T")
    assert np.array_equal(sc.tris, g["lens_tris"])
    ds = A.DeviceScene(sc)
    ro, rd = torch.from_numpy(g["ray_o"]).cuda(), torch.from_numpy(g["ray_d"]).cuda()
    n = ro.shape[0]
    t = torch.empty(n, device="cuda")
    uv = torch.empty((n, 2), device="cuda")
    tri = torch.empty(n, dtype=torch.int32, device="cuda")
    ng = torch.empty((n, 3), device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    A._lib.call("pz_trace_closest", A._vp(ds.internals), A._vp(ds.root_dev), A._vp(ds.tris), n, A._vp(ro),
                A._vp(rd), A._vp(t), A._vp(uv), A._vp(tri), A._vp(ng), A._vp(status), None)
    hit = torch.empty(n, dtype=torch.uint8, device="cuda")
    tmax = torch.from_numpy(g["ray_tmax"]).cuda()  # held until the kernel has run
    A._lib.call("pz_trace_any", A._vp(ds.internals), A._vp(ds.root_dev), A._vp(ds.tris), n, A._vp(ro), A._vp(rd),
                A._vp(tmax), A._vp(hit), None)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert t.cpu().numpy().tobytes() == g["hit_t"].tobytes()
    assert uv.cpu().numpy().tobytes() == g["hit_uv"].tobytes()
    assert tri.cpu().numpy().view(np.uint32).tobytes() == g["hit_tri"].tobytes()
    assert ng.cpu().numpy().tobytes() == g["hit_ng"].tobytes()
    assert np.array_equal(hit.cpu().numpy(), g["any_hit"])

    rec = A.photon_trace(ds, None, iteration=3, photons_per_triangle=8, records=True)
    torch.cuda.synchronize()
    got = rec.cpu().numpy().reshape(-1, 64)
    got = got[got[:, :4].copy().view(np.uint32)[:, 0] != 0]
    assert got.tobytes() == g["photon_records"].tobytes()

    cache = A.PathCache(capacity=1 << 22, step=sc.cell_step)
    A.photon_trace(ds, cache, iteration=3, photons_per_triangle=8)
    torch.cuda.synchronize()
    gc = cache.to_host()
    assert set(gc["hash"][gc["hash"] != 0].tolist()) == set(g["cache_hash"].tolist())
