"""Generates tests/golden/golden.npz from the reference's own CPU code.

The outputs come from oracle/_ref/libpzref.so: the reference's sources compiled by
oracle/build_ref.sh. That library exists only where the reference sources are present, so
this script runs there:

    python tests/golden/make_golden.py

The fixture stores its inputs next to the reference's outputs, so the tests never have to
rebuild a scene to check the oracle:
- heightfield-lens BVH, icosphere-3 BVH and random-soup BVH (nodes, root, sorted keys, deltas);
- closest and any hits of seeded rays;
- photon records and PathCache slots;
- solveConstraints, contributableThroughput and dAdw on photon tuples;
- a binned render of a small lens frame, and the same work list in the reference's own
  per-pixel-wavelength mode (RGB accumulator);
- CIE 2015 CMF samples, the wavelength pdf and sampling, and pack (RGBA8);
- interval square / normalize, Fresnel and refraction samples;
- normal bounds and path-cuts tuple sets (K = 1 lens, K = 2 two-sheet lens).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from palzilla_b200 import scenes as S  # noqa: E402

OUT = os.path.join(HERE, "golden.npz")


def main():
    if not O.build_ref():
        sys.exit("the reference CPU library could not be built (reference sources absent)")
    ref = O.reference()
    orc = O.oracle()  # used only for inputs the reference has no standalone entry for (eye pass, lookup)
    g = {}

    # ---- LBVH of three scenes
    lens = S.lens_scene(side=16, seed=1, width=32, height=32, n_bins=4, events="T")
    ico = S.icosphere(3)
    soup_tris = S.random_soup(1000, seed=1001)
    for name, tris in (("lens", lens.tris), ("ico3", ico[0]), ("soup", soup_tris)):
        b = ref.build_bvh(tris)
        g[f"{name}_tris"] = np.ascontiguousarray(tris, np.float32)
        g[f"{name}_nodes"] = b["nodes"].view(np.uint8).reshape(-1, 64)
        g[f"{name}_root"] = np.array([b["root"]], np.uint32)
        g[f"{name}_sorted"] = b["sorted"]
        g[f"{name}_deltas"] = b["deltas"]
    lens_bvh = ref.build_bvh(lens.tris)
    g["lens_attribs"] = np.ascontiguousarray(lens.attribs).view(np.uint8).reshape(lens.n, -1)

    # ---- rays against the lens scene
    rng = np.random.default_rng(7)
    ro = rng.uniform(-0.7, 0.7, (512, 3)).astype(np.float32)
    ro[:, 1] = 2.0
    rd = rng.normal(size=(512, 3)).astype(np.float32)
    rd[:, 1] = -np.abs(rd[:, 1]) * 4.0
    tmax = rng.uniform(0.2, 3.0, 512).astype(np.float32)
    h = ref.trace_closest(lens_bvh["nodes"], lens_bvh["root"], lens.tris, ro, rd)
    g.update(ray_o=ro, ray_d=rd, ray_tmax=tmax, hit_t=h["t"], hit_uv=h["uv"], hit_tri=h["tri"], hit_ng=h["ng"],
             any_hit=ref.trace_any(lens_bvh["nodes"], lens_bvh["root"], lens.tris, ro, rd, tmax))

    # ---- photons and the PathCache (K = 1 lens, 8 photons per triangle, iteration 3)
    recs = ref.photon_trace(lens_bvh, lens, iteration=3, photons_per_tri=8)
    g["photon_records"] = recs.view(np.uint8).reshape(recs.size, -1)
    cache = ref.cache_build(recs, capacity=1 << 22, step=lens.cell_step)
    used = np.nonzero(cache["hash"])[0].astype(np.uint32)
    g.update(cache_slots=used, cache_hash=cache["hash"][used], cache_cell=cache["cell"][used],
             cache_events=cache["events"][used], cache_tris=cache["tris"][used], cache_params=cache["params"][used])

    # ---- solver primitives: photon tuples solved towards a point next to where the photon landed
    ev = S.event_descriptor("T")
    lit = np.nonzero(recs["ev"] != 0)[0]
    sel = lit[:: max(1, lit.size // 96)][:96]
    p_end = (recs["p"][sel] + rng.normal(0.0, 0.004, (sel.size, 3)) * np.array([1, 0, 1])).astype(np.float32)
    etas = rng.uniform(1.45, 1.6, sel.size).astype(np.float32)
    ok, roots, iters, thr, dadw = [], [], [], [], []
    for i, s in enumerate(sel):
        tri = lens.tris[recs["tris"][s, :1]]
        at = lens.attribs[recs["tris"][s, :1]]
        o, x, it = ref.solve_constraints(1, recs["params"][s, :2], lens.p_light, p_end[i], tri, at, float(etas[i]), ev)
        ok.append(o)
        roots.append(x)
        iters.append(it)
        thr.append(ref.contributable_throughput(1, x, lens.p_light, p_end[i], tri, at, ev, lens_bvh, lens.tris,
                                                float(etas[i])) if o else 0.0)
        v0 = (1 - x[0] - x[1]) * tri[0, 0:3] + x[0] * tri[0, 3:6] + x[1] * tri[0, 6:9]
        dadw.append(ref.dAdw(lens.p_light, (v0 - np.asarray(lens.p_light, np.float32)).astype(np.float32), p_end[i],
                             tri, at, ev, float(etas[i])) if o else 0.0)
    g.update(solve_records=sel.astype(np.uint32), solve_p_end=p_end, solve_eta=etas, solve_ok=np.array(ok, np.uint8),
             solve_roots=np.array(roots, np.float32), solve_iters=np.array(iters, np.int32),
             solve_throughput=np.array(thr, np.float32), solve_dadw=np.array(dadw, np.float32))

    # ---- a binned render of the small lens frame (eye pass and lookup by the restatement)
    cam = lens.camera
    gen = orc.lookat(cam.eye, cam.center, cam.up, cam.fovy, lens.width, lens.height)
    _, fd = orc.solve_primary(lens_bvh, lens, gen, iteration=3)
    valid = (fd[:, 6:9] != 0).any(1).astype(np.uint8)
    _, pairs = orc.lookup_flatten(cache, fd[:, 0:3], valid, ev)
    img, st = ref.render_pairs(1, pairs, cache, fd, lens_bvh, lens, lens.bin_etas())
    g.update(render_fd=fd, render_pairs=pairs, render_etas=lens.bin_etas(), render_spectral=img,
             render_stats=st)
    # the same work list in the reference's own mode: each pixel's sampled wavelength, RGB into
    # a float4 accumulator (solveSpecularPath<K>, main_gpu.cu:418-483)
    acc, st_rgb = ref.render_pairs_rgb(1, pairs, cache, fd, lens_bvh, lens)
    g.update(render_rgb_accum=acc, render_rgb_stats=st_rgb)

    # ---- spectral model (CIE 2015 10-degree CMFs, wavelength pdf and sampling) and pack
    nm = np.linspace(360.0, 830.0, 941).astype(np.float32)
    u = np.linspace(0.0, 1.0, 257).astype(np.float32)
    g["cmf_nm"] = nm
    g["cmf_u"] = u
    g["cmf_out"] = np.stack([ref.cmf(w, nm) for w in range(4)], 0)
    g["cmf_sample"] = ref.cmf(4, u)
    rng_pack = np.random.default_rng(23)
    acc_in = rng_pack.uniform(0.0, 4.0, (512, 4)).astype(np.float32)
    acc_in[:, 3] = rng_pack.integers(1, 33, 512).astype(np.float32)
    acc_in[:8, :3] = np.array([0.0, 1e-4, 3.13e-3, 1.0, 2.0, 100.0, 0.5, 0.25], np.float32)[:, None]
    g["pack_in"] = acc_in
    g["pack_out"] = ref.pack(acc_in)

    # ---- interval arithmetic, Fresnel, refraction
    xs = np.linspace(-16, 16, 257).astype(np.float32)
    g["isq_in"] = np.stack([xs, xs + 1.0], 1).astype(np.float32)
    g["isq_out"] = np.array([ref.interval_square(l, u) for l, u in g["isq_in"]], np.float32)
    boxes = rng.uniform(-2, 2, (128, 3)).astype(np.float32)
    size = rng.uniform(0.05, 0.4, (128, 1)).astype(np.float32)
    box6 = np.stack([boxes, boxes + size], 2).reshape(-1, 6).astype(np.float32)  # (xl, xu, yl, yu, zl, zu)
    g["inorm_in"] = box6
    g["inorm_out"] = np.array([ref.interval_normalize(b) for b in box6], np.float32)
    wi = rng.normal(size=(128, 3)).astype(np.float32)
    n = rng.normal(size=(128, 3)).astype(np.float32)
    eta = rng.uniform(1.0, 2.0, 128).astype(np.float32)
    g.update(fr_wi=wi, fr_n=n, fr_eta=eta,
             fr_R=np.array([ref.fresnel(wi[i], n[i], float(eta[i])) for i in range(128)], np.float32))
    rr = [ref.refract(wi[i], n[i], float(eta[i])) for i in range(128)]
    g.update(rf_ok=np.array([r[0] for r in rr], np.uint8), rf_wo=np.array([r[1] for r in rr], np.float32))

    # ---- normal bounds and path cuts on BVHs built with USE_NORMAL
    bn = ref.build_bvh(lens.tris, 1)
    nbs = ref.normal_bounds(bn["nodes"], lens.tris, lens.attribs)
    g["nb_nodes"] = bn["nodes"].view(np.uint8).reshape(-1, 64)
    g["nb_root"] = np.array([bn["root"]], np.uint32)
    g["nb_bounds"] = nbs.view(np.uint8).reshape(nbs.size, -1)
    ends = np.array([[0.05, 0.0, -0.1], [0.0, 0.0, 0.0], [-0.2, 0.0, 0.15], [0.3, 0.0, 0.3]], np.float32)
    g["cuts_K1_ends"] = ends
    for i, pe in enumerate(ends):
        g[f"cuts_K1_{i}"] = ref.path_cuts(1, ev, 1.5, lens.p_light, pe, bn["nodes"], nbs, lens.tris, lens.attribs,
                                          bn["root"])
    tt = S.lens_scene(side=8, seed=2, width=16, height=16, n_bins=4, events="TT")
    bt = ref.build_bvh(tt.tris, 1)
    nbt = ref.normal_bounds(bt["nodes"], tt.tris, tt.attribs)
    g["tt_tris"] = np.ascontiguousarray(tt.tris, np.float32)
    g["tt_attribs"] = np.ascontiguousarray(tt.attribs).view(np.uint8).reshape(tt.n, -1)
    g["tt_nodes"] = bt["nodes"].view(np.uint8).reshape(-1, 64)
    g["tt_root"] = np.array([bt["root"]], np.uint32)
    g["tt_bounds"] = nbt.view(np.uint8).reshape(nbt.size, -1)
    g["cuts_K2"] = ref.path_cuts(2, S.event_descriptor("TT"), 1.5, tt.p_light, np.array([0.02, 0.0, 0.03], np.float32),
                                 bt["nodes"], nbt, tt.tris, tt.attribs, bt["root"])

    np.savez_compressed(OUT, **g)
    print(OUT, os.path.getsize(OUT), "bytes,", len(g), "arrays")


if __name__ == "__main__":
    main()
