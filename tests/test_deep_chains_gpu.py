"""Chains of three and four refractions (K = 3, 4: events TTT and TTTT) through two
stacked heightfield lenses: photon pass, work list, and the plain (exact-arithmetic build)
and batched solves, each against the CPU oracle's render of the same work list
(solveSpecularPath<K>, main_gpu.cu:418-497, restated in the oracle for K up to 4)."""
import numpy as np
import pytest
import torch

from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).mean()) / max(np.sqrt((b ** 2).mean()), 1e-30))


@pytest.mark.parametrize("K", [3, 4])
def test_deep_chain_images_match_oracle(orc, K):
    sc = S.stacked_lens_scene(K)
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 22)
    cache = A.PathCache(capacity=1 << 20, step=sc.cell_step)
    A.solve_primary(ds, frame, iteration=0)
    A.photon_trace(ds, cache, iteration=0)
    n = A.lookup_flatten(frame, cache, S.event_descriptor(sc.events))
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    assert n > 0
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    imgs = {}
    for mode in ("plain", "batched"):
        spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")
        stats = torch.zeros(3, dtype=torch.int64, device="cuda")
        d = A.solve_desc(ds, frame, cache, sc.events, n, spectral=spectral, etas=etas, stats=stats,
                         exact=mode == "plain")
        if mode == "plain":
            A.solve_specular_plain(d)
        else:
            A.solve_specular_batched(d, A.Scratch())
        torch.cuda.synchronize()
        imgs[mode] = (spectral.cpu().numpy().astype(np.float64), stats.cpu().numpy())
    pairs = frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2).copy()
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    bvh = orc.build_bvh(sc.tris)
    img_f, st_f = orc.render_pairs(K, pairs, cache.to_host(), fd, bvh, sc, sc.bin_etas())
    img_d, _ = orc.render_pairs(K, pairs, cache.to_host(), fd, bvh, sc, sc.bin_etas(), dtype=np.float64)
    assert st_f[2] > 0 and img_f.sum() > 0
    assert np.array_equal(imgs["plain"][1], st_f), (imgs["plain"][1], st_f)
    r_plain, r_batched = _rel(imgs["plain"][0], img_f), _rel(imgs["batched"][0], img_f)
    assert r_plain <= 1e-5 and r_batched <= 1e-5, (r_plain, r_batched)
    print(f"\nK={K}: {n} work items x {sc.n_bins} bins, {st_f[2]} contributing; rel RMSE plain exact "
          f"{r_plain:.1e}, batched {r_batched:.1e} vs the oracle; FP32 vs FP64 {_rel(img_f, img_d):.1e}")
