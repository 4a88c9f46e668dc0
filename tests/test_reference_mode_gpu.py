"""The reference's own solve mode and the resolve kernels against the CPU oracle.

* reference mode of the plain solve (solveSpecularPath<K>, main_gpu.cu:418-483): each
  (pixel, tuple) at its pixel's sampled wavelength from the eye pass, RGB into the float4
  accumulator -- the mode PKRenderer::step runs.  Same solve counts as the oracle, and the
  accumulator within 1e-5 relative RMSE (the CMF weights use the device's expf, the oracle
  the host's: an ulp or two apart);
* pz_resolve (pack, main_gpu.cu:499-513) and pz_resolve_spectral (the binned image's
  quadrature) against the oracle: linear sRGB within 1e-5, RGBA8 within one step of 255
  (powf differs by an ulp between device and host at a quantisation boundary).
"""
import numpy as np
import pytest
import torch

from palzilla_b200 import _lib
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.sqrt(((a - b) ** 2).mean()) / max(np.sqrt((b ** 2).mean()), 1e-30))


@pytest.mark.parametrize("events", ["T", "TT"])
def test_reference_mode_plain_solve(orc, events):
    sc = S.lens_scene(side=40, seed=21, width=128, height=128, n_bins=1, events=events)
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 22)
    A.solve_primary(ds, frame, iteration=2)
    cache = A.PathCache(capacity=1 << 20, step=sc.cell_step)
    A.photon_trace(ds, cache, iteration=2)
    n = A.lookup_flatten(frame, cache, S.event_descriptor(events))
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    frame.accum.zero_()  # the eye pass's direct light is not part of the solve
    stats = torch.zeros(3, dtype=torch.int64, device="cuda")
    A.solve_specular_plain(A.solve_desc(ds, frame, cache, events, n, stats=stats))
    torch.cuda.synchronize()
    assert n > 0
    pairs = frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2).copy()
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    gc = cache.to_host()
    bvh = orc.build_bvh(sc.tris)
    acc_o, st_o = orc.render_pairs_rgb(len(events), pairs, gc, fd, bvh, sc, iteration=2)
    acc_d, _ = orc.render_pairs_rgb(len(events), pairs, gc, fd, bvh, sc, iteration=2, dtype=np.float64)
    acc = frame.accum.cpu().numpy()
    assert np.array_equal(stats.cpu().numpy(), st_o), (stats, st_o)
    assert st_o[2] > 0
    assert np.all(acc[:, 3] == 0.0)
    rel = _rel(acc[:, :3], acc_o[:, :3])
    assert rel <= 1e-5, rel
    print(f"\n[{events}] reference mode: {n} items, {int(st_o[2])} contributing; rel RMSE vs oracle {rel:.1e}, "
          f"FP32 vs FP64 {_rel(acc[:, :3], acc_d[:, :3]):.1e}")


def test_pack_against_oracle(orc):
    rng = np.random.default_rng(5)
    n = 1 << 16
    acc = rng.uniform(0.0, 3.0, (n, 4)).astype(np.float32)
    acc[:, 3] = rng.integers(1, 65, n).astype(np.float32)
    acc[: n // 8, :3] *= 1e-3  # the linear segment of the OETF
    pixels = torch.zeros(n, dtype=torch.int32, device="cuda")
    acc_d = torch.from_numpy(acc).cuda()  # held until the kernel has run
    _lib.call("pz_resolve", A._vp(pixels), A._vp(acc_d), n, None)
    torch.cuda.synchronize()
    got = pixels.cpu().numpy().view(np.uint32)
    exp = orc.pack(acc)
    gb = np.stack([(got >> s) & 0xFF for s in (0, 8, 16, 24)], 1).astype(np.int32)
    eb = np.stack([(exp >> s) & 0xFF for s in (0, 8, 16, 24)], 1).astype(np.int32)
    diff = np.abs(gb - eb)
    assert diff.max() <= 1 and (diff != 0).mean() < 1e-3, (diff.max(), (diff != 0).mean())


def test_resolve_spectral_against_oracle(orc):
    rng = np.random.default_rng(6)
    n, nb = 1 << 14, 64
    spectral = (rng.exponential(0.02, (n, nb)) * (rng.uniform(0, 1, (n, nb)) < 0.3)).astype(np.float32)
    rgb = torch.zeros((n, 4), device="cuda")
    pixels = torch.zeros(n, dtype=torch.int32, device="cuda")
    albedo = (0.75, 0.7, 0.65)
    spectral_d = torch.from_numpy(spectral).cuda()  # held until the kernel has run
    _lib.call("pz_resolve_spectral", A._vp(rgb), A._vp(pixels), A._vp(spectral_d), n, nb,
              _lib.f32(380.0), _lib.f32(780.0), _lib.f3(albedo), None)
    torch.cuda.synchronize()
    rgb_o, px_o = orc.resolve_spectral(spectral, 380.0, 780.0, albedo)
    r = rgb.cpu().numpy()
    assert np.allclose(r, rgb_o, rtol=1e-5, atol=1e-6 * float(np.abs(rgb_o).max())), float(np.abs(r - rgb_o).max())
    got = pixels.cpu().numpy().view(np.uint32)
    gb = np.stack([(got >> s) & 0xFF for s in (0, 8, 16)], 1).astype(np.int32)
    eb = np.stack([(px_o >> s) & 0xFF for s in (0, 8, 16)], 1).astype(np.int32)
    diff = np.abs(gb - eb)
    assert diff.max() <= 1 and (diff != 0).mean() < 1e-3
