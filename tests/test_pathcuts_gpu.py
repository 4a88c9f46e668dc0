"""Path Cuts on the GPU (pz_normal_bounds, pz_path_cuts) against the reference's
traverseAdmissibleNodes<K> (pk.h:1760-2220): the golden tuple sets of the reference's own
CPU code (tests/golden/golden.npz) and the CPU oracle on fresh queries.

Parity: in round-to-nearest mode the set of admissible tuples of every query equals the
reference's; with directed rounding it contains it.  Normal bounds are bitwise equal.
"""
import os

import numpy as np
import pytest
import torch

import oracle as O
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


def _setup(tris, attribs):
    t = torch.from_numpy(np.ascontiguousarray(tris, np.float32)).cuda()
    at = torch.from_numpy(np.ascontiguousarray(attribs).view(np.uint8).reshape(-1)).cuda()
    b = A.BVHGPUBuilder()
    b.build(t, t.shape[0], 1)  # PZ_BUILD_OPTION_USE_NORMAL, as the reference's specular BVH
    nbs = A.normal_bounds(b, at)
    torch.cuda.synchronize()
    return t, at, b, nbs


def _sets(rows, nq):
    out = [set() for _ in range(nq)]
    for r in rows.tolist():
        out[r[0]].add(tuple(r[1:]))
    return out


def test_normal_bounds_and_tuples_match_golden():
    g = np.load(GOLDEN)
    lens = S.lens_scene(side=16, seed=1, width=32, height=32, n_bins=4, events="T")
    t, at, b, nbs = _setup(lens.tris, lens.attribs)
    n = lens.n
    assert b.m_internals[: (n - 1) * 64].cpu().numpy().tobytes() == g["nb_nodes"].tobytes()
    assert nbs[: (n - 1) * 52].cpu().numpy().tobytes() == g["nb_bounds"].tobytes()
    ends = torch.from_numpy(g["cuts_K1_ends"]).cuda()
    pc = A.PathCuts(frontier_capacity=1 << 16, tuple_capacity=1 << 16)
    rows, visited = pc.run(1, S.event_descriptor("T"), 1.5, lens.p_light, ends, b, nbs, t, at)
    got = _sets(rows.cpu().numpy(), len(ends))
    for i in range(len(ends)):
        assert got[i] == set(map(tuple, g[f"cuts_K1_{i}"].tolist())), i
    assert visited > 0

    tt_tris = g["tt_tris"]
    tt_attribs = g["tt_attribs"].reshape(-1).view(S.ATTRIB_DTYPE)
    t2, at2, b2, nbs2 = _setup(tt_tris, tt_attribs)
    n2 = tt_tris.shape[0]
    assert b2.m_internals[: (n2 - 1) * 64].cpu().numpy().tobytes() == g["tt_nodes"].tobytes()
    assert nbs2[: (n2 - 1) * 52].cpu().numpy().tobytes() == g["tt_bounds"].tobytes()
    pe = torch.tensor([[0.02, 0.0, 0.03]], dtype=torch.float32, device="cuda")
    rows, _ = pc.run(2, S.event_descriptor("TT"), 1.5, (0.0, 3.0, 0.0), pe, b2, nbs2, t2, at2)
    assert _sets(rows.cpu().numpy(), 1)[0] == set(map(tuple, g["cuts_K2"].tolist()))
    assert len(g["cuts_K2"]) > 100


@pytest.mark.parametrize("events", ["T", "TT"])
def test_batch_of_queries_matches_oracle_and_directed_superset(orc, events):
    sc = S.lens_scene(side=12 if events == "TT" else 32, seed=5, width=16, height=16, n_bins=4, events=events)
    K = len(events)
    ev = S.event_descriptor(events)
    t, at, b, nbs = _setup(sc.tris, sc.attribs)
    rng = np.random.default_rng(11)
    nq = 48
    ends = rng.uniform(-0.45, 0.45, (nq, 3)).astype(np.float32)
    ends[:, 1] = 0.0
    pc = A.PathCuts(frontier_capacity=1 << 20, tuple_capacity=1 << 21)
    rows_rn, vis_rn = pc.run(K, ev, 1.52, sc.p_light, torch.from_numpy(ends).cuda(), b, nbs, t, at)
    rows_dr, vis_dr = pc.run(K, ev, 1.52, sc.p_light, torch.from_numpy(ends).cuda(), b, nbs, t, at, directed=True)
    rn = _sets(rows_rn.cpu().numpy(), nq)
    dr = _sets(rows_dr.cpu().numpy(), nq)
    bo = orc.build_bvh(sc.tris, 1)
    nbo = orc.normal_bounds(bo["nodes"], sc.tris, sc.attribs)
    assert nbs[: (sc.n - 1) * 52].cpu().numpy().tobytes() == nbo.tobytes()
    total = 0
    for q in range(nq):
        exp = orc.path_cuts(K, ev, 1.52, sc.p_light, ends[q], bo["nodes"], nbo, sc.tris, sc.attribs, bo["root"])
        assert rn[q] == set(map(tuple, exp.tolist())), q
        assert rn[q] <= dr[q], q
        total += len(rn[q])
    assert total > 0 and vis_dr >= vis_rn
    print(f"\n[{events}] tuples {total} (directed {sum(len(d) for d in dr)}), node tuples {vis_rn} / {vis_dr}")


def test_empty_and_host_checks():
    import ctypes as C
    from palzilla_b200 import _lib
    L = _lib.lib()
    nt = C.c_uint64(7)
    r = L.pz_path_cuts(5, 1, 1.5, _lib.f3((0, 1, 0)), None, 1, None, None, None, None, None, 0, None, 0,
                       C.byref(nt), None, None, 0, None)
    assert r == 1
    r = L.pz_path_cuts(1, 1, 1.5, _lib.f3((0, 1, 0)), None, 0, None, None, None, None, None, 0, None, 0,
                       C.byref(nt), None, None, 0, None)
    assert r == 0 and nt.value == 0
