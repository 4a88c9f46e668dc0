"""Seeded synthetic scenes for the caustics hot path.

The reference renders an Alembic scene that is not part of its sources, so every
workload here is generated: heightfield glass lenses over a receiver plane, a
dispersive icosphere, random triangle soups for the sort/build benchmark and an
uneven batch of lenses.  Each generator is deterministic for a given seed.

Binary layouts match the reference's structs (minimum_lbvh.h:207-210,
pk.h:74-78): a triangle is 9 float32 (36 B), an attribute record is one int32
material followed by 9 float32 shading normals (40 B).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MATERIAL_DIFFUSE = 0     # pk.h:67-72
MATERIAL_MIRROR = 1
MATERIAL_DIELECTRIC = 2

ATTRIB_DTYPE = np.dtype([("material", "<i4"), ("ns", "<f4", (9,))])
assert ATTRIB_DTYPE.itemsize == 40

EV_T = 1  # event bit set = transmission (pk.h:117-121)


def event_descriptor(events: str) -> int:
    """EventDescriptor::asU32 (pk.h:122-162) of an event string such as "TT"."""
    bits = 0
    for i, c in enumerate(events):
        if c == "T":
            bits |= 1 << i
        elif c != "R":
            raise ValueError(f"bad event {c!r}")
    return bits | (len(events) << 24)


_R2_G = 1.32471795724474602596  # plastic number, x^3 = x + 1


def light_point(center, size, iteration: int) -> tuple:
    """Sample `iteration` of a square light (Scene.light_point); the same arithmetic as
    palzilla_b200::light_point in include/palzilla_b200.hpp (double, rounded to float)."""
    c = [float(np.float32(x)) for x in center]
    sx, sz = float(np.float32(size[0])), float(np.float32(size[1]))
    if sx == 0.0 and sz == 0.0:
        return tuple(c)
    u = math.fmod(0.5 + iteration / _R2_G, 1.0)
    v = math.fmod(0.5 + iteration / (_R2_G * _R2_G), 1.0)
    return (float(np.float32(c[0] + (u - 0.5) * sx)), c[1], float(np.float32(c[2] + (v - 0.5) * sz)))


@dataclasses.dataclass
class Camera:
    eye: tuple
    center: tuple
    up: tuple
    fovy: float  # radians


@dataclasses.dataclass
class Scene:
    name: str
    tris: np.ndarray      # (n, 9) float32
    attribs: np.ndarray   # (n,) ATTRIB_DTYPE
    p_light: tuple = (0.0, 3.0, 0.0)
    light_size: tuple = (0.0, 0.0)   # extent along x and z of a downward-facing square light
    camera: Camera | None = None
    width: int = 256
    height: int = 256
    cauchy_a: float = 1.5
    cauchy_b: float = 4200.0      # nm^2  (0.0042 um^2)
    lambda_min: float = 380.0
    lambda_max: float = 780.0
    n_bins: int = 16
    events: str = "T"
    light_intensity: float = 16.0    # pk.h:1686
    radiance_clamp: float = 12.0     # pk.h:1688
    min_throughput: float = 0.05     # pk.h:1687
    cell_step: float = 0.01          # pk.h:1376
    photons_per_triangle: int = 256  # PHOTON_BLOCK_SIZE, pk.h:32
    albedo: tuple = (0.75, 0.75, 0.75)

    @property
    def n(self) -> int:
        return int(self.tris.shape[0])

    def light_point(self, iteration: int) -> tuple:
        """The point light that stands for the area light at this iteration: the square
        light_size centred on p_light, sampled by the R2 sequence (Roberts 2018:
        x_i = frac(1/2 + i / g), y_i = frac(1/2 + i / g^2), g the plastic number), one
        sample per iteration.  Iteration 0 is the centre; a light of size zero is the
        point p_light."""
        return light_point(self.p_light, self.light_size, iteration)

    def bin_lambdas(self) -> np.ndarray:
        w = (self.lambda_max - self.lambda_min) / self.n_bins
        return (self.lambda_min + (np.arange(self.n_bins, dtype=np.float64) + 0.5) * w).astype(np.float32)

    def bin_etas(self) -> np.ndarray:
        lam = self.bin_lambdas()
        return (np.float32(self.cauchy_a) + np.float32(self.cauchy_b) / (lam * lam)).astype(np.float32)

    def eta_range(self) -> tuple:
        """(eta_min, eta_max) as the photon pass gets them: Cauchy at the short and
        long ends of the band (pk.h:1448-1449)."""
        a, b = np.float32(self.cauchy_a), np.float32(self.cauchy_b)
        lo, hi = np.float32(self.lambda_min), np.float32(self.lambda_max)
        return float(a + b / (lo * lo)), float(a + b / (hi * hi))


def _attribs(normals: np.ndarray, material: int) -> np.ndarray:
    a = np.zeros(normals.shape[0], dtype=ATTRIB_DTYPE)
    a["material"] = material
    a["ns"] = normals.reshape(-1, 9).astype(np.float32)
    return a


def receiver_plane(size: float, y: float = 0.0):
    """Two diffuse triangles spanning [-size/2, size/2]^2 at height y, facing +y."""
    h = size * 0.5
    p = np.array([[-h, y, -h], [h, y, -h], [h, y, h], [-h, y, h]], dtype=np.float32)
    # winding so that cross(v1 - v0, v2 - v0) points to +y
    tris = np.stack([np.concatenate([p[0], p[2], p[1]]), np.concatenate([p[0], p[3], p[2]])]).astype(np.float32)
    n = np.tile(np.array([0, 1, 0], np.float32), (2, 3, 1))
    return tris, _attribs(n, MATERIAL_DIFFUSE)


def heightfield_lens(side: int = 64, seed: int = 1, amplitude: float = 0.01, n_terms: int = 4,
                     extent: float = 1.0, y: float = 1.0, material: int = MATERIAL_DIELECTRIC):
    """Glass sheet over a side x side vertex grid spanning [-extent/2, extent/2]^2 at
    height y; height is a sum of n_terms sinusoids with seeded frequency in [1, 6],
    phase in [0, 2pi) and direction; shading normals are the analytic gradient normals."""
    rng = np.random.Generator(np.random.PCG64(seed))
    freq = rng.uniform(1.0, 6.0, n_terms)
    phase = rng.uniform(0.0, 2.0 * math.pi, n_terms)
    ang = rng.uniform(0.0, 2.0 * math.pi, n_terms)
    amp = np.full(n_terms, amplitude) if np.isscalar(amplitude) else np.asarray(amplitude)
    dx, dz = np.cos(ang), np.sin(ang)
    g = np.linspace(-extent * 0.5, extent * 0.5, side, dtype=np.float64)
    X, Z = np.meshgrid(g, g, indexing="xy")  # X varies along columns
    arg = 2.0 * math.pi * freq[None, None, :] * (X[..., None] * dx + Z[..., None] * dz) + phase
    H = y + (amp * np.sin(arg)).sum(-1)
    dHdx = (amp * np.cos(arg) * 2.0 * math.pi * freq * dx).sum(-1)
    dHdz = (amp * np.cos(arg) * 2.0 * math.pi * freq * dz).sum(-1)
    P = np.stack([X, H, Z], -1)
    N = np.stack([-dHdx, np.ones_like(H), -dHdz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    i, j = np.meshgrid(np.arange(side - 1), np.arange(side - 1), indexing="xy")
    i, j = i.ravel(), j.ravel()
    a = (j, i); b = (j, i + 1); c = (j + 1, i + 1); d = (j + 1, i)
    # quad a(x0,z0) b(x1,z0) c(x1,z1) d(x0,z1); winding a,d,b and b,d,c gives +y normals
    t0 = np.stack([P[a], P[d], P[b]], 1)
    t1 = np.stack([P[b], P[d], P[c]], 1)
    n0 = np.stack([N[a], N[d], N[b]], 1)
    n1 = np.stack([N[b], N[d], N[c]], 1)
    tris = np.stack([t0, t1], 1).reshape(-1, 3, 3)
    norms = np.stack([n0, n1], 1).reshape(-1, 3, 3)
    return tris.reshape(-1, 9).astype(np.float32), _attribs(norms, material)


def heightfield_corners(side: int) -> np.ndarray:
    """Grid vertex (row * side + column) of every corner of heightfield_lens' triangles,
    (n_triangles, 3) int32 in the same order as its triangles."""
    i, j = np.meshgrid(np.arange(side - 1), np.arange(side - 1), indexing="xy")
    i, j = i.ravel(), j.ravel()
    a, b, c, d = j * side + i, j * side + i + 1, (j + 1) * side + i + 1, (j + 1) * side + i
    t0 = np.stack([a, d, b], 1)
    t1 = np.stack([b, d, c], 1)
    return np.stack([t0, t1], 1).reshape(-1, 3).astype(np.int32)


def icosphere(subdivisions: int = 5, radius: float = 0.5, center=(0.0, 1.0, 0.0), material: int = MATERIAL_DIELECTRIC):
    """Icosphere with 20 * 4^subdivisions triangles, outward winding, smooth normals."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    F = list(faces)
    for _ in range(subdivisions):
        cache = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = V[i] + V[j]
                V.append(m / np.linalg.norm(m))
                cache[key] = len(V) - 1
            return cache[key]

        nf = []
        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = nf
    Vn = np.array(V)
    Fa = np.array(F)
    P = Vn[Fa] * radius + np.asarray(center)
    N = Vn[Fa]
    # make every face wind outward
    ng = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    flip = (ng * (P.mean(1) - np.asarray(center))).sum(-1) < 0
    P[flip] = P[flip][:, [0, 2, 1]]
    N[flip] = N[flip][:, [0, 2, 1]]
    return P.reshape(-1, 9).astype(np.float32), _attribs(N, material)


def random_soup(n: int, seed: int = 1001):
    """n triangles: one vertex uniform in [0,1]^3 plus two edges of length U[1e-3, 1e-2]
    in random directions (the sort + build workload)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    v0 = rng.random((n, 3), dtype=np.float32)
    out = np.empty((n, 9), np.float32)
    out[:, 0:3] = v0
    for k in (1, 2):
        d = rng.standard_normal((n, 3), dtype=np.float32)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        ln = rng.uniform(1e-3, 1e-2, (n, 1)).astype(np.float32)
        out[:, 3 * k:3 * k + 3] = v0 + d * ln
    return out


def _combine(parts):
    tris = np.concatenate([p[0] for p in parts]).astype(np.float32)
    att = np.concatenate([p[1] for p in parts])
    return np.ascontiguousarray(tris), att


def flat_sheet(side: int, y: float, extent: float = 1.0, facing: float = -1.0, material: int = MATERIAL_DIELECTRIC):
    """Flat glass sheet (the bottom face of a two-surface lens), normals along facing*y."""
    g = np.linspace(-extent * 0.5, extent * 0.5, side, dtype=np.float64)
    X, Z = np.meshgrid(g, g, indexing="xy")
    P = np.stack([X, np.full_like(X, y), Z], -1)
    i, j = np.meshgrid(np.arange(side - 1), np.arange(side - 1), indexing="xy")
    i, j = i.ravel(), j.ravel()
    a = (j, i); b = (j, i + 1); c = (j + 1, i + 1); d = (j + 1, i)
    if facing > 0:
        t = np.stack([np.stack([P[a], P[d], P[b]], 1), np.stack([P[b], P[d], P[c]], 1)], 1)
    else:
        t = np.stack([np.stack([P[a], P[b], P[d]], 1), np.stack([P[b], P[c], P[d]], 1)], 1)
    t = t.reshape(-1, 3, 3)
    n = np.zeros_like(t)
    n[..., 1] = facing
    return t.reshape(-1, 9).astype(np.float32), _attribs(n, material)


def lens_scene(side: int = 64, seed: int = 1, amplitude: float = 0.01, events: str = "T", n_bins: int = 16,
               width: int = 256, height: int = 256, name: str | None = None) -> Scene:
    """Heightfield-lens caustic: heightfield glass surface at y=1 over a 1x1 diffuse
    receiver at y=0, point light at (0,3,0).  For "TT" the lens gets a flat bottom face
    at y=0.92 (2 x 15 x 15 triangles), so paths refract twice.  The pinhole camera sits
    between lens and receiver looking straight down, so eye paths reach the receiver
    without crossing glass."""
    parts = [heightfield_lens(side, seed, amplitude)]
    eye_y = 0.9
    if len(events) >= 2:
        parts.append(flat_sheet(16, 0.92))
        eye_y = 0.85
    parts.append(receiver_plane(1.0, 0.0))
    tris, att = _combine(parts)
    fovy = 2.0 * math.atan(0.5 / eye_y)
    cam = Camera(eye=(0.0, eye_y, 0.0), center=(0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0), fovy=fovy)
    return Scene(name=name or f"lens{side}", tris=tris, attribs=att, camera=cam, events=events, n_bins=n_bins,
                 width=width, height=height)


def blocker_slab(n: int, seed: int, y0: float, y1: float, extent: float, size=(0.03, 0.08)):
    """n diffuse triangles with a vertex uniform in [-extent/2, extent/2] x [y0, y1] x
    [-extent/2, extent/2] and two edges of length U[size] in random directions: opaque
    occluders for the visibility tests."""
    rng = np.random.Generator(np.random.PCG64(seed))
    v0 = np.stack([rng.uniform(-extent / 2, extent / 2, n), rng.uniform(y0, y1, n),
                   rng.uniform(-extent / 2, extent / 2, n)], -1)
    t = np.empty((n, 3, 3), np.float64)
    t[:, 0] = v0
    for k in (1, 2):
        d = rng.standard_normal((n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        t[:, k] = v0 + d * rng.uniform(size[0], size[1], (n, 1))
    ng = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    ng /= np.maximum(np.linalg.norm(ng, axis=1, keepdims=True), 1e-30)
    return t.reshape(-1, 9).astype(np.float32), _attribs(np.repeat(ng[:, None, :], 3, 1), MATERIAL_DIFFUSE)


def occluded_lens_scene(side: int = 40, seed: int = 21, n_blockers: int = 300, events: str = "TT", n_bins: int = 16,
                        width: int = 128, height: int = 128) -> Scene:
    """lens_scene with a slab of small opaque triangles between the light and the lens
    (y in [1.2, 2.0] over the central 0.8 x 0.8), so that part of the light segments of
    the specular paths are occluded.  The camera below the lens does not see the slab, so
    the eye pass is the one of the open lens.  The blockers come after the lens and
    receiver triangles: triangle indices of the open lens keep their meaning."""
    base = lens_scene(side=side, seed=seed, events=events, n_bins=n_bins, width=width, height=height)
    bt, ba = blocker_slab(n_blockers, seed + 7, 1.2, 2.0, 0.8)
    tris, att = _combine([(base.tris, base.attribs), (bt, ba)])
    return Scene(name=f"occluded{side}", tris=tris, attribs=att, camera=base.camera, events=events, n_bins=n_bins,
                 width=width, height=height)


def stacked_lens_scene(sheets: int = 4, side: int = 24, seed: int = 1, amplitude: float = 0.01, n_bins: int = 8,
                       width: int = 96, height: int = 96) -> Scene:
    """Two heightfield lenses stacked over the receiver, for chains of 3 and 4 refractions:
    a heightfield sheet at y=1 with a flat bottom at y=0.92, then a second heightfield
    sheet (seed + 1) at y=0.80 with a flat bottom at y=0.72; `sheets` of these four
    surfaces, from the top, are kept (events "T" * sheets).  The camera looks down from
    y=0.6, below the glass."""
    surf = [heightfield_lens(side, seed, amplitude), flat_sheet(16, 0.92),
            heightfield_lens(side, seed + 1, amplitude, y=0.80), flat_sheet(16, 0.72)][:sheets]
    tris, att = _combine(surf + [receiver_plane(1.0, 0.0)])
    eye_y = 0.6
    cam = Camera(eye=(0.0, eye_y, 0.0), center=(0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0),
                 fovy=2.0 * math.atan(0.5 / eye_y))
    return Scene(name=f"stacked{sheets}", tris=tris, attribs=att, camera=cam, events="T" * sheets, n_bins=n_bins,
                 width=width, height=height)


def adjoint_scene(side: int = 128, seed: int = 1, width: int = 512, height: int = 512, n_bins: int = 8,
                  amplitude: float = 0.01):
    """Heightfield lens for gradient checks: the lens_scene with a side x side grid (the
    heightfield's triangles first) and the corner -> grid vertex map of every triangle
    (-1 for the receiver).  Returns (scene, corners, initial heights per grid vertex)."""
    sc = lens_scene(side=side, seed=seed, amplitude=amplitude, events="T", n_bins=n_bins, width=width, height=height,
                    name=f"adjoint{side}")
    hf = heightfield_corners(side)
    corners = np.full((sc.n, 3), -1, np.int32)
    corners[: hf.shape[0]] = hf
    heights = np.zeros(side * side, np.float32)
    ys = sc.tris[: hf.shape[0]].reshape(-1, 3, 3)[:, :, 1]
    heights[hf.ravel()] = ys.ravel()
    return sc, corners, heights


def sphere_scene(subdivisions: int = 5, n_bins: int = 64, width: int = 1024, height: int = 1024,
                 light_size=(0.2, 0.2)) -> Scene:
    """Two-refraction dispersive sphere: icosphere r=0.5 at (0,1,0) over a 4x4 receiver at
    y=0, lit by a 0.2 x 0.2 area light centred at (0,4,0), one point sample of it per
    iteration (Scene.light_point).  The camera at y=0.45, below the sphere, looks down on
    the central 0.9 x 0.9 of the receiver where the caustic falls."""
    sph = icosphere(subdivisions)
    tris, att = _combine([sph, receiver_plane(4.0, 0.0)])
    cam = Camera(eye=(0.0, 0.45, 0.0), center=(0.0, 0.0, 0.0), up=(0.0, 0.0, -1.0), fovy=math.pi / 2)
    return Scene(name=f"sphere{subdivisions}", tris=tris, attribs=att, p_light=(0.0, 4.0, 0.0), light_size=light_size,
                 camera=cam, events="TT", n_bins=n_bins, width=width, height=height)


def uneven_batch(n_scenes: int = 256, seed: int = 3001, side_min: int = 16, side_max: int = 256, width: int = 256,
                 height: int = 256, n_bins: int = 16, photons_per_triangle: int = 256):
    """Uneven batch: grid side log-uniform in [side_min, side_max], 1-2 refractions,
    amplitude U[0.005, 0.03]; width x height receiver image and n_bins bins each."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sides = np.exp(rng.uniform(math.log(side_min), math.log(side_max), n_scenes)).astype(int)
    amps = rng.uniform(0.005, 0.03, n_scenes)
    ks = rng.integers(1, 3, n_scenes)
    scenes = []
    for i in range(n_scenes):
        s = lens_scene(int(sides[i]), seed=seed + 1 + i, amplitude=float(amps[i]), events="T" * int(ks[i]),
                       n_bins=n_bins, width=width, height=height, name=f"batch{i}")
        s.photons_per_triangle = photons_per_triangle
        scenes.append(s)
    return scenes


# ---------------------------------------------------------------------------------------
# scene files
# ---------------------------------------------------------------------------------------
OBJ_MATERIALS = {"mirror": MATERIAL_MIRROR, "dielectric": MATERIAL_DIELECTRIC}


def load_obj(path: str, materials: dict | None = None):
    """A Wavefront OBJ triangle soup as (tris (n, 9) float32, attribs ATTRIB_DTYPE): the
    same reading as palzilla_b200::loadObj (include/palzilla_b200_scene.hpp), triangle for
    triangle.  The material of a face is the one its last `usemtl` names: "mirror" or
    "dielectric", the reference's two tags (pk.h:1306-1318), else diffuse; `materials` maps
    other names.  Polygons become fans (0, i, i + 1); a corner's normal index gives its
    shading normal, and a triangle whose corners have none takes its unit geometric normal at
    all three."""
    mats = dict(OBJ_MATERIALS if materials is None else materials)
    pos, nrm, tris, norms, mat = [], [], [], [], []
    material = MATERIAL_DIFFUSE
    f32 = np.float32

    def resolve(i, n):
        return i - 1 if i > 0 else n + i

    with open(path) as fh:
        for line_no, line in enumerate(fh, 1):
            s = line.strip()
            if s.startswith("v ") or s.startswith("v\t"):
                x = s.split()[1:4]
                pos.append([f32(t) for t in x])
            elif s.startswith("vn ") or s.startswith("vn\t"):
                x = s.split()[1:4]
                nrm.append([f32(t) for t in x])
            elif s.startswith("usemtl ") or s.startswith("usemtl\t"):
                material = mats.get(s[7:].strip(), MATERIAL_DIFFUSE)
            elif s.startswith("f ") or s.startswith("f\t"):
                vi, ni = [], []
                for tok in s.split()[1:]:
                    parts = tok.split("/")
                    v = int(parts[0])
                    n = int(parts[2]) if len(parts) >= 3 and parts[2] else 0
                    rv = resolve(v, len(pos))
                    if v == 0 or not 0 <= rv < len(pos):
                        raise ValueError(f"{path}:{line_no}: vertex index out of range")
                    rn = -1
                    if n != 0:
                        rn = resolve(n, len(nrm))
                        if not 0 <= rn < len(nrm):
                            raise ValueError(f"{path}:{line_no}: normal index out of range")
                    vi.append(rv)
                    ni.append(rn)
                if len(vi) < 3:
                    raise ValueError(f"{path}:{line_no}: face with fewer than three corners")
                for k in range(1, len(vi) - 1):
                    c3 = (0, k, k + 1)
                    t = np.array([pos[vi[c]] for c in c3], np.float32)
                    if all(ni[c] >= 0 for c in c3):
                        ns = np.array([nrm[ni[c]] for c in c3], np.float32)
                    else:
                        e0, e1 = t[1] - t[0], t[2] - t[0]
                        g = np.array([e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2],
                                      e0[0] * e1[1] - e0[1] * e1[0]], np.float32)
                        inv = f32(1.0) / np.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
                        ns = np.tile(g * inv, (3, 1))
                    tris.append(t.reshape(9))
                    norms.append(ns.reshape(9))
                    mat.append(material)
    t = np.array(tris, np.float32).reshape(-1, 9)
    a = np.zeros(len(mat), ATTRIB_DTYPE)
    a["material"] = mat
    a["ns"] = np.array(norms, np.float32).reshape(-1, 9)
    return t, a


def write_obj(path: str, tris: np.ndarray, attribs: np.ndarray, names=None):
    """Writes a triangle soup as OBJ (one `v`, one `vn` per corner; `usemtl` by material:
    names maps a material to its tag, by default the reference's "mirror" and "dielectric",
    "diffuse" otherwise), with 9 significant digits so load_obj reads back the same float32."""
    names = names or {MATERIAL_DIFFUSE: "diffuse", MATERIAL_MIRROR: "mirror", MATERIAL_DIELECTRIC: "dielectric"}
    with open(path, "w") as f:
        cur = None
        for i in range(tris.shape[0]):
            m = int(attribs["material"][i])
            if m != cur:
                f.write(f"usemtl {names[m]}\n")
                cur = m
            for j in range(3):
                f.write("v %.9g %.9g %.9g\n" % tuple(float(x) for x in tris[i, 3 * j:3 * j + 3]))
                f.write("vn %.9g %.9g %.9g\n" % tuple(float(x) for x in attribs["ns"][i, 3 * j:3 * j + 3]))
            b = 3 * i + 1
            f.write(f"f {b}//{b} {b + 1}//{b + 1} {b + 2}//{b + 2}\n")
