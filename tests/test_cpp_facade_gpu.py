"""The C++ facade (include/palzilla_b200.hpp: PKRenderer, BVHGPUBuilder, OnesweepSort,
RayGenerator) driven by a C++ program (palzilla_b200/pk_render) renders the same image as
the same sequence of C-ABI calls made from Python: two iterations of the reference's
step() (eye pass, photon pass, and lookup / sort / reorder / plain solve for the event
strings T, R, TT, TTTT, TRT, TTT) on a two-sheet heightfield lens under a square area
light, sampled at one point per iteration on both sides."""
import os
import struct
import subprocess

import numpy as np
import pytest
import torch

from palzilla_b200 import api as A
from palzilla_b200 import build as B
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu

EVENTS = ["T", "R", "TT", "TTTT", "TRT", "TTT"]


def _python_render(sc, iterations):
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 25)
    cache = A.PathCache(capacity=1 << 22, step=sc.cell_step)
    sorter = A.OnesweepSort()
    solved = 0
    for it in range(iterations):
        A.solve_primary(ds, frame, iteration=it)
        cache.clear()
        A.photon_trace(ds, cache, iteration=it)
        for ev in EVENTS:
            n = A.lookup_flatten(frame, cache, S.event_descriptor(ev))
            if n == 0:
                continue
            A.sort_and_reorder(frame, n, sorter)
            A.solve_specular_plain(A.solve_desc(ds, frame, cache, ev, n, iteration=it))
            solved += n
    pixels = torch.empty(sc.width * sc.height, dtype=torch.int32, device="cuda")
    A._lib.call("pz_resolve", A._vp(pixels), A._vp(frame.accum), sc.width * sc.height, None)
    torch.cuda.synchronize()
    return frame.accum.cpu().numpy().reshape(-1), pixels.cpu().numpy().view(np.uint32), solved


def test_pk_renderer_matches_c_abi_sequence(tmp_path):
    exe = B.build_pk_render()
    sc = S.lens_scene(side=32, seed=3, width=96, height=96, n_bins=1, events="TT")
    sc.light_size = (0.1, 0.1)  # an area light: each iteration samples another point of it
    iterations = 2
    cam = sc.camera
    path_in, path_out = tmp_path / "scene.bin", tmp_path / "out.bin"
    with open(path_in, "wb") as f:
        f.write(struct.pack("<4i", sc.n, sc.width, sc.height, iterations))
        f.write(struct.pack("<10f", *cam.eye, *cam.center, *cam.up, cam.fovy))
        f.write(struct.pack("<5f", *sc.p_light, *sc.light_size))
        f.write(struct.pack("<5f", sc.light_intensity, sc.radiance_clamp, sc.min_throughput, sc.cauchy_a, sc.cauchy_b))
        f.write(np.ascontiguousarray(sc.tris, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.attribs).tobytes())
    r = subprocess.run([exe, str(path_in), str(path_out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    npx = sc.width * sc.height
    raw = open(path_out, "rb").read()
    accum_cpp = np.frombuffer(raw[: 16 * npx], np.float32)
    pixels_cpp = np.frombuffer(raw[16 * npx: 20 * npx], np.uint32)
    solved_cpp = struct.unpack("<Q", raw[20 * npx:])[0]
    accum_py, pixels_py, solved_py = _python_render(sc, iterations)
    print("\n" + r.stdout.strip())
    # The photon pass is racy by design (the first photon to claim a PathCache slot gives
    # the tuple its Newton start, pk.h:309-346), so two renders differ in a few paths;
    # the work lists (and so the number of solved paths) and the image statistics agree.
    assert solved_cpp == solved_py > 0
    rel = np.sqrt(((accum_cpp.astype(np.float64) - accum_py) ** 2).mean() / (accum_py.astype(np.float64) ** 2).mean())
    same = np.isclose(accum_cpp, accum_py, rtol=1e-4, atol=1e-5).mean()
    diff = np.abs(pixels_cpp.view(np.uint8).astype(int) - pixels_py.view(np.uint8).astype(int))
    print(f"accum rel RMSE {rel:.2e}, equal entries {same:.4f}, RGBA8 max diff {diff.max()}, "
          f"within 1: {(diff <= 1).mean():.4f}")
    assert rel < 5e-2 and same > 0.98 and (diff <= 1).mean() > 0.98
    assert abs(accum_cpp.sum() / accum_py.sum() - 1.0) < 1e-2
    assert (accum_py[3::4] > 0).all()  # every pixel got its eye-path samples
