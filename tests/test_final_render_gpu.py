"""The headless final render of the pk_render driver (main_gpu.cpp:60-85 through the C++
facade): per frame loadFrame from an OBJ of an OBJ sequence, clear, N steps, resolve, and
the frame written as an uncompressed PNG and a PFM.  The PNG must be a valid PNG (CRCs,
zlib stream) whose RGBA8 pixels are the pack (main_gpu.cu:499-513) of the PFM's linear
image; frames of different geometry differ; a floor texture changes the image."""
import struct
import subprocess
import zlib

import numpy as np
import pytest

from palzilla_b200 import build as B
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(kind + body) == crc, kind
        if kind == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 6
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 4 * w)
    assert (raw[:, 0] == 0).all()
    return raw[:, 1:].reshape(h, w, 4)


def read_pfm(path):
    data = open(path, "rb").read()
    head, rest = data.split(b"\n", 3)[:3], data.split(b"\n", 3)[3]
    assert head[0] == b"PF" and float(head[2]) < 0
    w, h = map(int, head[1].split())
    return np.frombuffer(rest, "<f4").reshape(h, w, 3)[::-1]


def test_multi_frame_render(tmp_path, orc):
    for i, seed in enumerate((3, 4)):
        sc = S.lens_scene(side=24, seed=seed, amplitude=0.03)
        S.write_obj(str(tmp_path / f"{i:03d}.obj"), sc.tris, sc.attribs)
    rng = np.random.default_rng(5)
    tex = rng.integers(0, 256, (16, 16, 3), dtype=np.uint8)
    (tmp_path / "floor.ppm").write_bytes(b"P6\n16 16\n255\n" + tex.tobytes())
    cam = sc.camera
    exe = B.build_pk_render()
    common = [exe, "--obj", str(tmp_path / "%03d.obj"), "--frames", "2", "--spp", "2", "--size", "64", "48",
              "--eye", *map(str, cam.eye), "--center", *map(str, cam.center), "--up", *map(str, cam.up),
              "--fovy", str(cam.fovy), "--light", "0", "3", "0", "--pfm"]
    out_tex, out_plain = tmp_path / "tex", tmp_path / "plain"
    out_tex.mkdir()
    out_plain.mkdir()
    r = subprocess.run(common + ["--floor", str(tmp_path / "floor.ppm"), "--out", str(out_tex)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "frame 001" in r.stdout
    r = subprocess.run(common + ["--out", str(out_plain)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    imgs = {}
    for d in (out_tex, out_plain):
        for i in range(2):
            png = read_png(d / f"{i:03d}.png")
            pfm = read_pfm(d / f"{i:03d}.pfm")
            assert png.shape == (48, 64, 4) and pfm.shape == (48, 64, 3)
            acc = np.concatenate([pfm.reshape(-1, 3), np.ones((48 * 64, 1), np.float32)], 1)
            want = orc.pack(acc).view(np.uint8).reshape(48, 64, 4)
            assert np.abs(png.astype(int) - want.astype(int)).max() <= 1
            assert pfm.max() > 0
            imgs[(d.name, i)] = pfm
    assert not np.array_equal(imgs[("tex", 0)], imgs[("tex", 1)])
    assert not np.array_equal(imgs[("tex", 0)], imgs[("plain", 0)])
