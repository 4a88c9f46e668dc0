"""Scene builders used by the GPU tests (host code, no GPU)."""
import numpy as np

from palzilla_b200 import scenes as S


def test_occluded_lens_keeps_the_open_lens_first():
    """The occluded lens is the open two-sheet lens followed by the blockers, so triangle
    indices of the open lens mean the same triangles in both scenes (the occlusion test
    renders one work list in both).  The blockers are diffuse, sit in the slab between the
    light and the lens, and are not degenerate."""
    occ = S.occluded_lens_scene(side=40, seed=21, n_blockers=300, events="TT")
    base = S.lens_scene(side=40, seed=21, events="TT", n_bins=occ.n_bins, width=occ.width, height=occ.height)
    nb = base.tris.shape[0]
    assert occ.tris.shape[0] == nb + 300
    assert np.array_equal(occ.tris[:nb], base.tris)
    assert np.array_equal(occ.attribs[:nb], base.attribs)
    blk = occ.tris[nb:].reshape(-1, 3, 3).astype(np.float64)
    assert (occ.attribs["material"][nb:] == S.MATERIAL_DIFFUSE).all()
    assert blk[:, :, 1].min() > 1.05 and blk[:, :, 1].max() < occ.p_light[1]  # above the lens, below the light
    area = 0.5 * np.linalg.norm(np.cross(blk[:, 1] - blk[:, 0], blk[:, 2] - blk[:, 0]), axis=1)
    assert area.min() > 0.0
    assert np.array_equal(occ.tris, S.occluded_lens_scene(side=40, seed=21, n_blockers=300, events="TT").tris)
