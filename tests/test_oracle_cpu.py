"""The CPU oracle (oracle/pz_oracle.hpp) pinned against the reference (no GPU needed).

1. Golden vectors: tests/golden/golden.npz holds outputs of the reference's own CPU code
   (oracle/_ref, built from the reference sources by tests/golden/make_golden.py). The
   restatement must reproduce them bit for bit.
2. The reference's property tests (unittest.cpp:54-143: interval square, interval
   normalize, Fresnel reciprocity of refraction), run on the restatement. The upper-bound
   accumulation at unittest.cpp:74 uses fminf where fmaxf is meant; it is fixed here.
3. Live cross-checks against oracle/_ref on fresh seeded inputs, when that library is built
   here.
"""
import os

import numpy as np

from cache_checks import probe_reachability_violations
import pytest

import oracle as O
from palzilla_b200 import scenes as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def lens():
    return S.lens_scene(side=16, seed=1, width=32, height=32, n_bins=4, events="T")


def _bvh(g, name):
    return {"nodes": g[f"{name}_nodes"].reshape(-1).view(O.NODE_DTYPE), "root": int(g[f"{name}_root"][0])}


def _full_cache(g):
    cap = 1 << 22
    tris = np.zeros((cap, 4), np.int32)
    params = np.zeros((cap, 8), np.float32)
    tris[g["cache_slots"]] = g["cache_tris"]
    params[g["cache_slots"]] = g["cache_params"]
    return {"tris": tris, "params": params}


def test_fixture_inputs_match_scene_generators(g, lens):
    assert np.array_equal(g["lens_tris"], lens.tris)
    assert np.array_equal(g["lens_attribs"].reshape(-1), np.ascontiguousarray(lens.attribs).view(np.uint8).reshape(-1))


@pytest.mark.parametrize("name", ["lens", "ico3", "soup"])
def test_lbvh_bitwise(orc, g, name):
    b = orc.build_bvh(g[f"{name}_tris"])
    assert b["nodes"].view(np.uint8).reshape(-1, 64).tobytes() == g[f"{name}_nodes"].tobytes()
    assert b["root"] == int(g[f"{name}_root"][0])
    assert np.array_equal(b["sorted"], g[f"{name}_sorted"])
    assert np.array_equal(b["deltas"], g[f"{name}_deltas"])
    assert orc.validate_lbvh(b["nodes"], b["root"], b["deltas"])


def test_rays_bitwise(orc, g):
    bvh = _bvh(g, "lens")
    h = orc.trace_closest(bvh["nodes"], bvh["root"], g["lens_tris"], g["ray_o"], g["ray_d"])
    for k, gk in (("t", "hit_t"), ("uv", "hit_uv"), ("tri", "hit_tri"), ("ng", "hit_ng")):
        assert h[k].tobytes() == g[gk].tobytes(), k
    hit = orc.trace_any(bvh["nodes"], bvh["root"], g["lens_tris"], g["ray_o"], g["ray_d"], g["ray_tmax"])
    assert np.array_equal(hit, g["any_hit"])
    assert 0 < int(g["any_hit"].sum()) < g["any_hit"].size


def test_photons_and_path_cache_bitwise(orc, g, lens):
    recs = orc.photon_trace(_bvh(g, "lens"), lens, iteration=3, photons_per_tri=8)
    assert recs.view(np.uint8).reshape(recs.size, -1).tobytes() == g["photon_records"].tobytes()
    c = orc.cache_build(recs, capacity=1 << 22, step=lens.cell_step)
    used = np.nonzero(c["hash"])[0]
    assert np.array_equal(used, g["cache_slots"])
    for k in ("hash", "cell", "events", "tris", "params"):
        assert c[k][used].tobytes() == g[f"cache_{k}"].tobytes(), k
    assert probe_reachability_violations(c["hash"], c["cell"], 1 << 22) == 0
    # a crowded table (load about 0.5, chains of tens of slots) keeps the
    # invariant, and the check catches an entry left behind an emptied slot of its chain
    cap = 1 << 15
    c = orc.cache_build(recs, capacity=cap, step=lens.cell_step)
    used = np.nonzero(c["hash"])[0]
    assert 0.3 < used.size / cap < 0.7
    dist = (used - (c["cell"][used] & (cap - 1))) & (cap - 1)
    assert dist.max() > 16
    assert probe_reachability_violations(c["hash"], c["cell"], cap) == 0
    h = c["hash"].copy()
    h[int(c["cell"][used[np.argmax(dist)]]) & (cap - 1)] = 0
    assert probe_reachability_violations(h, c["cell"], cap) >= 1


def test_solver_primitives_bitwise(orc, g, lens):
    recs = g["photon_records"].reshape(-1).view(O.RECORD_DTYPE)
    bvh = _bvh(g, "lens")
    ev = S.event_descriptor("T")
    for i, r in enumerate(g["solve_records"]):
        tri = lens.tris[recs["tris"][r, :1]]
        at = lens.attribs[recs["tris"][r, :1]]
        eta = float(g["solve_eta"][i])
        ok, x, it = orc.solve_constraints(1, recs["params"][r, :2], lens.p_light, g["solve_p_end"][i], tri, at, eta, ev)
        assert ok == bool(g["solve_ok"][i])
        assert x.tobytes() == g["solve_roots"][i].tobytes()
        if ok:  # the reference reports no iteration count for an early rejection
            assert it == g["solve_iters"][i]
            t = orc.contributable_throughput(1, x, lens.p_light, g["solve_p_end"][i], tri, at, ev, bvh, lens.tris, eta)
            assert np.float32(t) == g["solve_throughput"][i]
            v0 = (1 - x[0] - x[1]) * tri[0, 0:3] + x[0] * tri[0, 3:6] + x[1] * tri[0, 6:9]
            d = orc.dAdw(lens.p_light, (v0 - np.asarray(lens.p_light, np.float32)).astype(np.float32),
                         g["solve_p_end"][i], tri, at, ev, eta)
            assert np.float32(d) == g["solve_dadw"][i]
    assert g["solve_ok"].sum() > 64 and (g["solve_throughput"] > 0).sum() > 32


def test_binned_render_bitwise(orc, g, lens):
    img, st = orc.render_pairs(1, g["render_pairs"], _full_cache(g), g["render_fd"], _bvh(g, "lens"), lens,
                               g["render_etas"])
    assert img.tobytes() == g["render_spectral"].tobytes()
    assert np.array_equal(st, g["render_stats"])
    assert (img > 0).sum() > 100


def test_reference_mode_render(orc, g, lens):
    """The reference's own per-pixel-wavelength solve (main_gpu.cu:418-483) on the golden work
    list: the same accepted paths, and RGB accumulators equal up to the order of the float adds
    of a pixel's paths."""
    acc, st = orc.render_pairs_rgb(1, g["render_pairs"], _full_cache(g), g["render_fd"], _bvh(g, "lens"), lens)
    assert np.array_equal(st, g["render_rgb_stats"]) and st[2] > 0
    exp = g["render_rgb_accum"]
    assert np.allclose(acc, exp, rtol=2e-6, atol=1e-7 * float(np.abs(exp).max()))


def test_spectral_model_and_pack_bitwise(orc, g):
    """CIE 2015 10-degree CMFs, the wavelength pdf and its sampling (pk.h:960-1012) and pack
    (main_gpu.cu:499-513) equal the reference's bit for bit."""
    got = np.stack([orc.cmf(w, g["cmf_nm"]) for w in range(4)], 0)
    assert got.tobytes() == g["cmf_out"].tobytes()
    assert orc.cmf(4, g["cmf_u"]).tobytes() == g["cmf_sample"].tobytes()
    assert np.array_equal(orc.pack(g["pack_in"]), g["pack_out"])


def test_interval_fresnel_refract_bitwise(orc, g):
    out = np.array([orc.interval_square(l, u) for l, u in g["isq_in"]], np.float32)
    assert out.tobytes() == g["isq_out"].tobytes()
    out = np.array([orc.interval_normalize(b) for b in g["inorm_in"]], np.float32)
    assert out.tobytes() == g["inorm_out"].tobytes()
    R = np.array([orc.fresnel(g["fr_wi"][i], g["fr_n"][i], float(g["fr_eta"][i])) for i in range(128)], np.float32)
    assert R.tobytes() == g["fr_R"].tobytes()
    for i in range(128):
        ok, wo = orc.refract(g["fr_wi"][i], g["fr_n"][i], float(g["fr_eta"][i]))
        assert ok == bool(g["rf_ok"][i])
        if ok:
            assert wo.tobytes() == g["rf_wo"][i].tobytes()


def test_normal_bounds_and_path_cuts(orc, g, lens):
    nodes = g["nb_nodes"].reshape(-1).view(O.NODE_DTYPE)
    nbs = orc.normal_bounds(nodes, lens.tris, lens.attribs)
    assert nbs.view(np.uint8).reshape(nbs.size, -1).tobytes() == g["nb_bounds"].tobytes()
    ev = S.event_descriptor("T")
    for i, pe in enumerate(g["cuts_K1_ends"]):
        got = orc.path_cuts(1, ev, 1.5, lens.p_light, pe, nodes, nbs, lens.tris, lens.attribs, int(g["nb_root"][0]))
        assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, g[f"cuts_K1_{i}"].tolist()))
    tt_nodes = g["tt_nodes"].reshape(-1).view(O.NODE_DTYPE)
    tt_attribs = g["tt_attribs"].reshape(-1).view(S.ATTRIB_DTYPE)
    nbt = orc.normal_bounds(tt_nodes, g["tt_tris"], tt_attribs)
    assert nbt.view(np.uint8).reshape(nbt.size, -1).tobytes() == g["tt_bounds"].tobytes()
    got = orc.path_cuts(2, S.event_descriptor("TT"), 1.5, (0.0, 3.0, 0.0), np.array([0.02, 0.0, 0.03], np.float32),
                        tt_nodes, nbt, g["tt_tris"], tt_attribs, int(g["tt_root"][0]))
    assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, g["cuts_K2"].tolist()))
    assert len(g["cuts_K2"]) > 100


# ---------------------------------------------------------------- unittest.cpp properties
def test_interval_square_property(orc):
    """unittest.cpp:54-84 (upper bound with fmaxf; the reference accumulates with fminf)."""
    rng = np.random.default_rng(103)
    for _ in range(1000):
        x = np.float32(-16.0 + 32.0 * rng.random())
        lo, hi = orc.interval_square(x, x + np.float32(1.0))
        s = np.linspace(x, x + np.float32(1.0), 1000, dtype=np.float32)
        sq = s * s
        lower, upper = sq.min(), sq.max()
        assert lo <= lower and upper <= hi
        assert lower < lo + 0.01 and hi - 0.01 < upper


def test_interval_normalize_property(orc):
    """unittest.cpp:86-116: the normalised box contains every normalised sample."""
    rng = np.random.default_rng(178)
    for _ in range(300):
        size = np.float32(0.05 + 0.35 * rng.random())
        p = (rng.random(3) * 4.0 - 2.0).astype(np.float32)
        box = np.stack([p, p + size], 1).reshape(-1).astype(np.float32)  # (xl, xu, yl, yu, zl, zu)
        out = orc.interval_normalize(box).reshape(3, 2)
        smp = (p + size * rng.random((1000, 3))).astype(np.float32)
        smp /= np.sqrt((smp * smp).sum(1, keepdims=True)).astype(np.float32)
        eps = 1e-5
        assert np.all(smp >= out[:, 0] - eps) and np.all(smp <= out[:, 1] + eps)


def test_refraction_fresnel_reciprocity(orc):
    """unittest.cpp:118-143: R(wi, n, eta) == R(wo, -n, 1/eta) for the refracted wo."""
    rng = np.random.default_rng(3)
    for _ in range(40):
        eta = float(1.0 + rng.random())
        for i in range(100):
            theta = np.pi * 0.5 * i / 100
            n = np.array([0.0, 0.1 + rng.random() * 3.0, 0.0], np.float32)
            wi = np.array([-np.sin(theta) * n[1], np.cos(theta) * n[1], 0.0], np.float32)
            R = orc.fresnel(wi, n, eta)
            ok, wo = orc.refract(wi, n, eta)
            assert ok
            assert abs(R - orc.fresnel(wo, -n, 1.0 / eta)) < 1e-3


# ---------------------------------------------------------------- live cross-checks
def test_live_bvh_and_photons_vs_reference(orc, ref):
    tris = S.random_soup(5000, seed=77)
    a, b = orc.build_bvh(tris), ref.build_bvh(tris)
    assert a["nodes"].tobytes() == b["nodes"].tobytes() and a["root"] == b["root"]
    sc = S.lens_scene(side=24, seed=9, width=32, height=32, n_bins=4, events="TT")
    bo, br = orc.build_bvh(sc.tris), ref.build_bvh(sc.tris)
    po = orc.photon_trace(bo, sc, iteration=1, photons_per_tri=16)
    pr = ref.photon_trace(br, sc, iteration=1, photons_per_tri=16)
    assert po.tobytes() == pr.tobytes()


def test_live_render_vs_reference(orc, ref):
    sc = S.lens_scene(side=24, seed=9, width=48, height=48, n_bins=4, events="TT")
    bvh = orc.build_bvh(sc.tris)
    recs = orc.photon_trace(bvh, sc, iteration=2, photons_per_tri=32)
    cache = orc.cache_build(recs, capacity=1 << 22, step=sc.cell_step)
    cam = sc.camera
    gen = orc.lookat(cam.eye, cam.center, cam.up, cam.fovy, sc.width, sc.height)
    _, fd = orc.solve_primary(bvh, sc, gen, iteration=2)
    valid = (fd[:, 6:9] != 0).any(1).astype(np.uint8)
    _, pairs = orc.lookup_flatten(cache, fd[:, 0:3], valid, S.event_descriptor("TT"))
    io, so = orc.render_pairs(2, pairs, cache, fd, bvh, sc, sc.bin_etas())
    ir, sr = ref.render_pairs(2, pairs, cache, fd, bvh, sc, sc.bin_etas())
    assert io.tobytes() == ir.tobytes() and np.array_equal(so, sr)
    assert so[2] > 0


def test_subdivision_finds_every_root_of_dense_starts(orc):
    """The subdivision solve (pz_oracle_subdiv.hpp, the checker of pz_subdivide_solve) has no
    reference counterpart; it is pinned by a property: for every wavelength bin, every
    contributing root that the reference's Newton solve (solveConstraints<K>,
    pk.h:466-592) reaches from a dense grid of starts in any (receiver point, lens
    triangle) domain is among its roots, and it reports no root the grid does not find
    (within 1e-3 in the barycentrics: roots of ill-conditioned tuples stop anywhere in a
    1e-4-wide basin).  Three bins share the subdivision, so the per-bin leaf test is
    covered too."""
    sc = S.lens_scene(side=8, seed=5, amplitude=0.05, events="T", width=16, height=16)
    ev = S.event_descriptor("T")
    bvh = orc.build_bvh(sc.tris, 0)
    rng = np.random.default_rng(2)
    ends = rng.uniform(-0.4, 0.4, (6, 3)).astype(np.float32)
    ends[:, 1] = 0.0
    spec = np.nonzero(sc.attribs["material"] != 0)[0]
    rows = np.array([[q, i] for q in range(len(ends)) for i in spec], np.uint32)
    etas = np.array([1.5, 1.53, 1.56], np.float32)
    roots, stats = orc.subdivide_solve(1, ev, sc.p_light, ends, rows, etas, sc.tris, sc.attribs, bvh, sc.tris)
    assert stats[1] > len(rows) // 2 and stats[3] > 0 and len(roots) > 30
    sub = {}
    for r in roots:
        sub.setdefault((int(r["tuple"]), int(r["bin"])), []).append(r["params"][:2])
    grid = [(u, v) for u in np.linspace(0.02, 0.98, 9) for v in np.linspace(0.02, 0.98, 9) if u + v <= 1.0]
    brute = {}
    for ri, (q, tri) in enumerate(rows):
        T, At = sc.tris[[tri]], sc.attribs[[tri]]
        for b, eta in enumerate(etas):
            for u, v in grid:
                ok, p, _ = orc.solve_constraints(1, np.array([u, v], np.float32), sc.p_light, ends[q], T, At, eta, ev)
                if ok and orc.contributable_throughput(1, p, sc.p_light, ends[q], T, At, ev, bvh, sc.tris, eta) > 0:
                    lst = brute.setdefault((ri, b), [])
                    if not any(np.abs(p - x).max() < 1e-4 for x in lst):
                        lst.append(p)
    for key in set(sub) | set(brute):
        a, b = sub.get(key, []), brute.get(key, [])
        assert all(any(np.abs(p - x).max() < 1e-3 for x in a) for p in b), key
        assert all(any(np.abs(p - x).max() < 1e-3 for p in b) for x in a), key


def _f32_neighbours(x):
    """The float32 values just below and above the exact rational x (equal when x is one)."""
    from fractions import Fraction
    f = np.float32(float(x))  # round to nearest double, then to float: within one float step
    lo, hi = f, f
    while Fraction(float(lo)) > x:
        lo = np.nextafter(lo, np.float32(-np.inf))
    while Fraction(float(hi)) < x:
        hi = np.nextafter(hi, np.float32(np.inf))
    while Fraction(float(np.nextafter(lo, np.float32(np.inf)))) <= x:
        lo = np.nextafter(lo, np.float32(np.inf))
    while Fraction(float(np.nextafter(hi, np.float32(-np.inf)))) >= x:
        hi = np.nextafter(hi, np.float32(-np.inf))
    return float(lo), float(hi)


def test_subdivision_directed_rounding_is_exact(orc):
    """The oracle's directed rounding (error-free transformations, no FPU mode switch) gives
    the IEEE round-down / round-up results the GPU intrinsics give: checked against exact
    rational arithmetic on random floats of mixed magnitudes (results within the float
    range), subnormals included."""
    from fractions import Fraction
    rng = np.random.default_rng(9)
    vals = np.concatenate([rng.standard_normal(300) * 10.0 ** rng.integers(-18, 18, 300),
                           rng.standard_normal(50) * 1e-40, [0.0, 1.0, -1.0, 2.0 ** -149, 3.0, 0.1]])
    vals = vals.astype(np.float32)
    pairs = rng.choice(vals, (1500, 2))
    for a, b in pairs:
        a, b = float(a), float(b)
        for op, exact in ((0, Fraction(a) + Fraction(b)), (1, Fraction(a) - Fraction(b)), (2, Fraction(a) * Fraction(b))):
            lo, hi = _f32_neighbours(exact)
            assert orc.directed(op, False, a, b) == lo and orc.directed(op, True, a, b) == hi, (op, a, b)
        if b != 0.0 and abs(a / b) < 1e37:
            lo, _ = _f32_neighbours(Fraction(a) / Fraction(b))
            assert orc.directed(3, False, a, b) == lo, (a, b)
        x = abs(a)
        d, u = orc.directed(4, False, x), orc.directed(4, True, x)
        assert Fraction(d) ** 2 <= Fraction(x) <= Fraction(u) ** 2
        assert u == d or u == float(np.nextafter(np.float32(d), np.float32(np.inf)))
        assert (u == d) == (Fraction(d) ** 2 == Fraction(x))


def test_newton_flop_count(orc):
    """The operation count of one Newton iteration of the restated solver (a counting scalar
    type; used by the bench line's FP32 figure) is positive, the same on every call, and grows
    with the chain: 2K dual evaluations of K vertices, then a 3K x 2K least-squares step."""
    sc = S.lens_scene(side=16, seed=1, events="TT")
    spec = np.nonzero(sc.attribs["material"] != 0)[0]
    tup = [spec[0], spec[len(spec) // 2 + 3]]
    counts = {}
    for K, ev in ((1, "T"), (2, "TT")):
        args = (K, np.full(2 * K, 0.3, np.float32), sc.p_light, (0.0, 0.0, 0.0), sc.tris[tup[:K]],
                sc.attribs[tup[:K]], 1.5, S.event_descriptor(ev))
        c = orc.count_newton_flops(*args)
        assert c == orc.count_newton_flops(*args)
        assert c["add"] > 0 and c["mul"] > 0 and c["div"] > 0 and c["sqrt"] > 0
        assert c["total"] == c["add"] + c["mul"] + c["div"] + c["sqrt"]
        counts[K] = c["total"]
    assert 3 * counts[1] < counts[2] < 5 * counts[1], counts
