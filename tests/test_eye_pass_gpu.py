"""The eye pass (solvePrimary, main_gpu.cu:213-371) with the reference's two camera-side
features that the frame benchmark leaves off, against the CPU oracle:
* the floor texture (Texture8RGBX::samplePoint, pk.h:1083-1095; main_gpu.cu:343): the
  diffuse hit's albedo is the nearest texel at its (x, z), repeat-wrapped, decoded as
  (c / 255)^2.2;
* the thick lens in front of the camera (solveLens, pk.h:1042-1073): two spherical
  refractions of every camera ray.
FirstDiffuse p and n bit for bit, R within an ulp or two (powf on the device and on the
host), lambda to 1e-5 (expf / logf), the accumulated direct light to 1e-4."""
import numpy as np
import pytest
import torch

from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _compare(orc, sc, ds, iteration, lens=(0.6, 0.05, 0.0), texture=None):
    frame = A.Frame(sc, path_capacity=1 << 16)
    tex_d = None if texture is None else torch.from_numpy(texture).cuda()
    A.solve_primary(ds, frame, iteration=iteration, lens=lens, texture=tex_d)
    torch.cuda.synchronize()
    assert int(frame.status.item()) == 0
    fd = frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    bvh = orc.build_bvh(sc.tris)
    gen = orc.lookat(sc.camera.eye, sc.camera.center, sc.camera.up, sc.camera.fovy, sc.width, sc.height)
    acc_o, fd_o = orc.solve_primary(bvh, sc, gen, iteration=iteration, lens=lens, texture=texture)
    assert np.array_equal(fd[:, :6], fd_o[:, :6])
    assert np.allclose(fd[:, 6:9], fd_o[:, 6:9], rtol=1e-6, atol=0)
    assert np.allclose(fd[:, 9], fd_o[:, 9], rtol=1e-5, atol=0)
    assert np.allclose(frame.accum.cpu().numpy(), acc_o, rtol=1e-4, atol=1e-6)
    return fd


def test_floor_texture(orc):
    sc = S.lens_scene(side=32, seed=4, width=96, height=96)
    ds = A.DeviceScene(sc)
    rng = np.random.default_rng(12)
    tex = rng.integers(1, 256, (7, 13, 4), dtype=np.uint8)  # odd sizes: wrapping and the last texel
    tex[..., 3] = 255
    fd = _compare(orc, sc, ds, 3, texture=tex)
    lit = (fd[:, 6:9] != 0).any(1)
    assert lit.sum() > 1000
    # the albedo varies with the texel, and equals the decoded texel under the hit
    assert len(np.unique(fd[lit, 6])) > 20
    p = fd[lit, :3]
    u, v = p[:, 0] - np.floor(p[:, 0]), p[:, 2] - np.floor(p[:, 2])
    ix = np.minimum(u * np.float32(13), np.float32(12)).astype(np.int32)
    iy = np.minimum(v * np.float32(7), np.float32(6)).astype(np.int32)
    want = (tex[iy, ix, :3].astype(np.float64) / 255.0) ** 2.2
    assert np.allclose(fd[lit, 6:9], want, rtol=1e-5)


def test_thick_lens(orc):
    sc = S.lens_scene(side=32, seed=4, width=96, height=96)
    ds = A.DeviceScene(sc)
    no_lens = _compare(orc, sc, ds, 1)
    lens = (0.3, 0.02, 2.0)  # distance, thickness, sphere radius: a weak lens between camera and receiver
    with_lens = _compare(orc, sc, ds, 1, lens=lens)
    lit = (with_lens[:, 6:9] != 0).any(1) & (no_lens[:, 6:9] != 0).any(1)
    assert lit.sum() > 1000
    # the lens bends the camera rays: the receiver points move
    assert np.abs(with_lens[lit, :3] - no_lens[lit, :3]).max() > 1e-3
