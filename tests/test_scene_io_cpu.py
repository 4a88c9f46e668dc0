"""Scene ingestion on the host (no GPU): the OBJ triangle-soup loaders -- the C++ one of
include/palzilla_b200_scene.hpp, run through the pk_render driver, and scenes.load_obj --
read the same triangles, shading normals and material tags (the reference's "mirror" and
"dielectric", pk.h:1306-1318) bit for bit; polygons become fans, negative indices and the
v, v/vt, v//vn, v/vt/vn corner forms are read, corners without a normal take the unit
geometric normal; a scene written with scenes.write_obj reads back unchanged; malformed
files are refused."""
import os
import subprocess

import numpy as np
import pytest

from palzilla_b200 import build as B
from palzilla_b200 import scenes as S

OBJ = """# four-sided glass face, a tagless face, a mirror face
v 0 0 0
v 1 0 0
v 1 0 1
v 0 0 1
v 0.5 1 0.5
vn 0 1 0
vn 0 0.70710678 0.70710678
vt 0 0
usemtl dielectric
f 1//1 2//1 3//1 4//1
usemtl glass
f -5 -4 -1
usemtl mirror
f 2/1/2 3/1/2 5/1/2
"""


def _cxx_parse(path, tmp_path):
    exe = B.build_pk_render()
    out = tmp_path / "parsed.bin"
    subprocess.run([exe, "--parse-obj", str(path), str(out)], check=True, capture_output=True)
    raw = out.read_bytes()
    n = int(np.frombuffer(raw[:4], np.int32)[0])
    tris = np.frombuffer(raw[4:4 + 36 * n], np.float32).reshape(n, 9)
    attribs = np.frombuffer(raw[4 + 36 * n:], S.ATTRIB_DTYPE)
    return tris, attribs


def test_obj_loaders_agree(tmp_path):
    p = tmp_path / "a.obj"
    p.write_text(OBJ)
    t, a = S.load_obj(str(p))
    # the quad is a fan of two triangles; the tagless face is diffuse; the mirror face has the
    # second normal at every corner
    assert t.shape == (4, 9)
    assert a["material"].tolist() == [S.MATERIAL_DIELECTRIC, S.MATERIAL_DIELECTRIC, S.MATERIAL_DIFFUSE,
                                      S.MATERIAL_MIRROR]
    assert np.array_equal(t[1], np.array([0, 0, 0, 1, 0, 1, 0, 0, 1], np.float32))
    assert np.array_equal(t[2], np.array([0, 0, 0, 1, 0, 0, 0.5, 1, 0.5], np.float32))
    g = np.cross(np.array([1, 0, 0], np.float32), np.array([0.5, 1, 0.5], np.float32))
    assert np.allclose(a["ns"][2].reshape(3, 3), g / np.linalg.norm(g), atol=1e-7)
    assert np.array_equal(a["ns"][3].reshape(3, 3), np.tile(np.array([0, 0.70710678, 0.70710678], np.float32), (3, 1)))
    tc, ac = _cxx_parse(p, tmp_path)
    assert tc.tobytes() == t.tobytes() and ac.tobytes() == a.tobytes()


def test_obj_round_trip(tmp_path):
    sc = S.sphere_scene(subdivisions=3)
    p = tmp_path / "sphere.obj"
    S.write_obj(str(p), sc.tris, sc.attribs)
    t, a = S.load_obj(str(p))
    assert t.tobytes() == np.ascontiguousarray(sc.tris, np.float32).tobytes()
    assert a.tobytes() == np.ascontiguousarray(sc.attribs).tobytes()
    tc, ac = _cxx_parse(p, tmp_path)
    assert tc.tobytes() == t.tobytes() and ac.tobytes() == a.tobytes()


@pytest.mark.parametrize("bad", ["v 0 0 0\nf 1 2 3\n", "v 0 0 0\nv 1 0 0\nf 1 2\n", "f x y z\n"])
def test_obj_malformed(tmp_path, bad):
    p = tmp_path / "bad.obj"
    p.write_text(bad)
    with pytest.raises(ValueError):
        S.load_obj(str(p))
    exe = B.build_pk_render()
    r = subprocess.run([exe, "--parse-obj", str(p), str(tmp_path / "o.bin")], capture_output=True)
    assert r.returncode != 0 and b"loadObj" in r.stderr
