"""Seeded synthetic scenes and cameras for the five benchmark workloads.

The reference renders hand-built scenes of ``Triangle`` surfaces (src/main.cpp:340-420,
src/Scene.cpp:47-106).  No dataset is involved: every scene here is generated from a
seeded ``numpy.random.Generator(Philox(seed))`` so the GPU path, the oracle and the
compiled reference all see the same float32 arrays.

Flat scene format (shared by the C ABI, the oracle and the reference harness):

* ``verts``    float32 [V, 3]  world-space vertex positions
* ``normals``  float32 [V, 3]  per-vertex shading normals
* ``tris``     uint32  [M, 3]  vertex indices (v1, v2, v3 in reference order)
* ``tri_obj``  uint32  [M]     object (material) index per triangle
* ``materials`` float32 [K, 8] kd.rgb, ks.rgb, shininess, reflectivity
* ``lights``   float32 [L, 6]  position.xyz, colour.rgb (w of the position is 1)

A camera is the reference's ``Camera`` POD (src/Camera.h:30-64): position, viewing
direction, right and up vectors (their lengths set the field of view) and the image size.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MAT_STRIDE = 10  # kd rgb, ks rgb, shininess, reflectivity, transparency, refractive index
LIGHT_STRIDE = 6


def pad_materials(mats) -> np.ndarray:
    """Material rows as float32 [K, 10]; rows of 8 (no transparency columns) get
    transparency 0 and refractive index 1."""
    m = np.asarray(mats, dtype=np.float32)
    m = m.reshape(-1, m.shape[-1]) if m.ndim > 1 else m.reshape(1, -1) if m.size else m.reshape(0, MAT_STRIDE)
    if m.shape[1] == 8:
        m = np.concatenate([m, np.zeros((m.shape[0], 1), np.float32), np.ones((m.shape[0], 1), np.float32)], 1)
    if m.shape[1] != MAT_STRIDE:
        raise ValueError(f"material rows have {m.shape[1]} values, expected 8 or {MAT_STRIDE}")
    return np.ascontiguousarray(m)


def rng_for(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


@dataclass
class SceneData:
    verts: np.ndarray
    normals: np.ndarray
    tris: np.ndarray
    tri_obj: np.ndarray
    materials: np.ndarray
    lights: np.ndarray
    name: str = "scene"
    ambient_index: float = 1.0  # refractive index outside transparent objects

    def __post_init__(self):
        self.verts = np.ascontiguousarray(self.verts, dtype=np.float32).reshape(-1, 3)
        self.normals = np.ascontiguousarray(self.normals, dtype=np.float32).reshape(-1, 3)
        self.tris = np.ascontiguousarray(self.tris, dtype=np.uint32).reshape(-1, 3)
        self.tri_obj = np.ascontiguousarray(self.tri_obj, dtype=np.uint32).reshape(-1)
        self.materials = pad_materials(self.materials)
        self.lights = np.ascontiguousarray(self.lights, dtype=np.float32).reshape(-1, LIGHT_STRIDE)

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])

    @property
    def n_objects(self) -> int:
        return int(self.materials.shape[0])

    @property
    def n_lights(self) -> int:
        return int(self.lights.shape[0])


@dataclass
class CameraData:
    position: np.ndarray
    view: np.ndarray
    right: np.ndarray
    up: np.ndarray
    width: int
    height: int

    def as_array(self) -> np.ndarray:
        """12 floats: position, viewing direction, right, up (reference field order)."""
        return np.concatenate([self.position, self.view, self.right, self.up]).astype(np.float32)


@dataclass
class Job:
    """One view of one scene: the unit of work of the batched renderer."""
    scene: SceneData
    camera: CameraData
    trace_depth: int = 1
    pixel_offset: float = 0.5
    spp: int = 1
    jitter_seed: int = 0
    extra: dict = field(default_factory=dict)


def look_at(position, target, fov_deg: float, width: int, height: int,
            world_up=(0.0, 1.0, 0.0)) -> CameraData:
    """Pinhole camera in the reference's convention.

    The reference has no field of view (src/Camera.h:30-64): the primary direction is
    ``normalize(aa*right + bb*up + view)`` with aa, bb in [-1, 1] (src/RayTracer.cpp:135-142),
    so |up| = tan(fov/2) and |right| = tan(fov/2) * width/height give a vertical fov.
    """
    p = np.asarray(position, np.float64)
    v = np.asarray(target, np.float64) - p
    v /= np.linalg.norm(v)
    r = np.cross(v, np.asarray(world_up, np.float64))
    if np.linalg.norm(r) < 1e-9:
        r = np.cross(v, np.array([0.0, 0.0, 1.0]))
    r /= np.linalg.norm(r)
    u = np.cross(r, v)
    u /= np.linalg.norm(u)
    th = math.tan(math.radians(fov_deg) * 0.5)
    aspect = width / height
    return CameraData(p.astype(np.float32), v.astype(np.float32),
                      (r * th * aspect).astype(np.float32), (u * th).astype(np.float32),
                      int(width), int(height))


# ----------------------------------------------------------------------------- geometry
_ICO_CACHE: dict[int, tuple[np.ndarray, np.ndarray]] = {}


def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: 20 * 4**level faces, vertices on the unit sphere (float64)."""
    if level in _ICO_CACHE:
        v, f = _ICO_CACHE[level]
        return v.copy(), f.copy()
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
             (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
             (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
             (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
             (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    vl = [np.array(p, np.float64) / np.linalg.norm(p) for p in verts]
    for _ in range(level):
        cache: dict[tuple[int, int], int] = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            idx = cache.get(key)
            if idx is None:
                m = vl[a] + vl[b]
                vl.append(m / np.linalg.norm(m))
                idx = len(vl) - 1
                cache[key] = idx
            return idx

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    v = np.array(vl, np.float64)
    f = np.array(faces, np.int64)
    _ICO_CACHE[level] = (v, f)
    return v.copy(), f.copy()


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def heightfield(cells: int, extent: float, rng: np.random.Generator, amplitude: float = 2.0,
                n_waves: int = 4, y0: float = 0.0):
    """Grid of cells x cells quads over [-extent, extent]^2; heights = sum of seeded sinusoids.

    Normals come from central differences of the height samples (one-sided at the border).
    """
    n = cells + 1
    xs = np.linspace(-extent, extent, n)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    H = np.zeros_like(X)
    for _ in range(n_waves):
        k = rng.uniform(0.02, 0.15, size=2) * rng.choice([-1.0, 1.0], size=2)
        ph = rng.uniform(0, 2 * math.pi)
        H += amplitude * np.sin(k[0] * X + k[1] * Z + ph)
    H += y0
    dx = xs[1] - xs[0]
    gx = np.gradient(H, dx, axis=1)
    gz = np.gradient(H, dx, axis=0)
    N = np.stack([-gx, np.ones_like(H), -gz], axis=-1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    V = np.stack([X, H, Z], axis=-1).reshape(-1, 3)
    idx = np.arange(n * n).reshape(n, n)
    a = idx[:-1, :-1].ravel()
    b = idx[:-1, 1:].ravel()
    c = idx[1:, :-1].ravel()
    d = idx[1:, 1:].ravel()
    F = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], axis=0)
    # interleave the two triangles of a cell so neighbouring ids are spatially close
    F = F.reshape(2, -1, 3).transpose(1, 0, 2).reshape(-1, 3)
    return V, N.reshape(-1, 3), F


def ground_quad(extent: float, y: float):
    V = np.array([[-extent, y, -extent], [extent, y, -extent],
                  [extent, y, extent], [-extent, y, extent]], np.float64)
    N = np.tile(np.array([[0.0, 1.0, 0.0]]), (4, 1))
    F = np.array([[0, 2, 1], [0, 3, 2]], np.int64)
    return V, N, F


def foliage_cluster(n: int, rng: np.random.Generator, radius: float = 2.0):
    """n thin triangles: edge log-U(0.01, 1), aspect ratio log-U(1, 100), random orientation."""
    centers = rng.normal(size=(n, 3))
    centers /= np.linalg.norm(centers, axis=1, keepdims=True)
    centers *= radius * rng.uniform(0, 1, size=(n, 1)) ** (1 / 3)
    edge = np.exp(rng.uniform(math.log(0.01), math.log(1.0), size=n))
    aspect = np.exp(rng.uniform(0.0, math.log(100.0), size=n))
    a = rng.normal(size=(n, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = rng.normal(size=(n, 3))
    b -= (b * a).sum(1, keepdims=True) * a
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    p0 = centers - 0.5 * edge[:, None] * a
    p1 = centers + 0.5 * edge[:, None] * a
    p2 = centers + (edge / aspect)[:, None] * b
    V = np.stack([p0, p1, p2], 1).reshape(-1, 3)
    fn = np.cross(p1 - p0, p2 - p0)
    fn /= np.linalg.norm(fn, axis=1, keepdims=True)
    N = np.repeat(fn, 3, axis=0)
    F = np.arange(3 * n).reshape(n, 3)
    return V, N, F


class _Builder:
    def __init__(self):
        self.V, self.N, self.F, self.O = [], [], [], []
        self.nv = 0
        self.mats = []

    def add(self, V, N, F, material):
        obj = len(self.mats)
        self.mats.append(material)
        self.V.append(np.asarray(V, np.float64))
        self.N.append(np.asarray(N, np.float64))
        self.F.append(np.asarray(F, np.int64) + self.nv)
        self.O.append(np.full(len(F), obj, np.int64))
        self.nv += len(V)
        return obj

    def build(self, lights, name):
        return SceneData(np.concatenate(self.V), np.concatenate(self.N), np.concatenate(self.F),
                         np.concatenate(self.O), np.array(self.mats, np.float64),
                         np.asarray(lights, np.float64), name)


def material(kd, ks, shininess, reflectivity, transparency=0.0, refractive_index=1.0):
    ks = np.broadcast_to(np.asarray(ks, np.float64), (3,))
    return [*kd, *ks, float(shininess), float(reflectivity), float(transparency), float(refractive_index)]


def add_sphere(b: _Builder, level: int, center, radius: float, rot, mat):
    v, f = icosphere(level)
    n = v @ rot.T if rot is not None else v
    return b.add(np.asarray(center, np.float64) + radius * n, n, f, mat)


def _random_material(rng, refl_hi, int_shininess=True, log_shininess_range=None):
    kd = rng.uniform(0, 1, 3)
    ks = rng.uniform(0, 0.5)
    if log_shininess_range is not None:
        sh = math.exp(rng.uniform(*log_shininess_range))
    else:
        sh = math.exp(rng.uniform(math.log(4), math.log(256)))
        if int_shininess:
            sh = float(round(sh))
    return material(kd, ks, sh, rng.uniform(0, refl_hi))


# ----------------------------------------------------------------------------- configs
def config1_scene() -> SceneData:
    """Level-5 icosphere (20,480 tris, r=1) on a 2-triangle ground quad at y=-1; 1 light."""
    b = _Builder()
    add_sphere(b, 5, (0, 0, 0), 1.0, None, material((0.7, 0.3, 0.3), 0.3, 32, 0.2))
    b.add(*ground_quad(10.0, -1.0), material((0.7, 0.3, 0.3), 0.3, 32, 0.0))
    return b.build([[5, 5, 5, 1, 1, 1]], "icosphere5+quad")


def config1_camera(width=512, height=512) -> CameraData:
    return look_at((0, 1.5, 4), (0, 0, 0), 60.0, width, height)


def config2_scene(seed: int = 1002, n_spheres: int = 200, cells: int = 128) -> SceneData:
    """128x128-cell height field over [-100,100]^2 plus 200 level-4 icospheres; 4 lights."""
    rng = rng_for(seed)
    b = _Builder()
    V, N, F = heightfield(cells, 100.0, rng)
    b.add(V, N, F, _random_material(rng, 0.5))
    for _ in range(n_spheres):
        c = rng.uniform(-50, 50, 3)
        r = math.exp(rng.uniform(math.log(0.5), math.log(3.0)))
        add_sphere(b, 4, c, r, random_rotation(rng), _random_material(rng, 0.5))
    lights = []
    for _ in range(4):
        p = rng.uniform(-60, 60, 3)
        i = rng.uniform(0.5, 1.5)
        lights.append([*p, i, i, i])
    return b.build(lights, "heightfield128+200xico4")


def config2_camera(width=1920, height=1080) -> CameraData:
    return look_at((0, 60, 160), (0, 0, 0), 60.0, width, height)


CONFIG3_RES = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]


def config3_jobs(seed: int = 1003, n_views: int = 64, n_scenes: int = 16,
                 res_choices=CONFIG3_RES, tri_range=(10_000, 500_000)) -> list[Job]:
    """64 random views of the config-1 scene plus 16 mixed scenes at 512^2, depth 3."""
    rng = rng_for(seed)
    base = config1_scene()
    jobs = []
    for i in range(n_views):
        d = rng.normal(size=3)
        d[1] = abs(d[1])
        d /= np.linalg.norm(d)
        w, h = res_choices[rng.integers(len(res_choices))]
        cam = look_at(120.0 * d, (0, 0, 0), 60.0, w, h)
        jobs.append(Job(base, cam, trace_depth=2, pixel_offset=0.5))
    for s in range(n_scenes):
        target = math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))
        sc = mixed_scene(rng, int(target), name=f"mixed{s}")
        cam = look_at((0, 25, 60), (0, 0, 0), 60.0, 512, 512)
        jobs.append(Job(sc, cam, trace_depth=2, pixel_offset=0.5))
    return jobs


def mixed_scene(rng: np.random.Generator, target_tris: int, name="mixed") -> SceneData:
    b = _Builder()
    total = 0
    # one height field takes roughly a third of the budget
    cells = max(8, int(math.sqrt(max(target_tris // 3, 128) / 2)))
    V, N, F = heightfield(cells, 40.0, rng, y0=-6.0)
    b.add(V, N, F, _random_material(rng, 0.5))
    total += len(F)
    while total < target_tris:
        lvl = int(rng.integers(2, 6))
        c = rng.uniform(-30, 30, 3) * np.array([1.0, 0.3, 1.0])
        r = math.exp(rng.uniform(math.log(0.5), math.log(4.0)))
        add_sphere(b, lvl, c, r, random_rotation(rng), _random_material(rng, 0.5))
        total += 20 * 4 ** lvl
    lights = [[*rng.uniform(-40, 40, 3) * np.array([1, 0, 1]) + np.array([0, 40, 0]), 1, 1, 1]
              for _ in range(2)]
    return b.build(lights, name)


def config4_scene(seed: int = 1004, hidden: bool = True) -> SceneData:
    """50 level-3 icospheres in [-10,10]^3 on a ground quad, 3 lights, continuous shininess."""
    rng = rng_for(seed)
    b = _Builder()
    geo = []
    for _ in range(50):
        geo.append((rng.uniform(-10, 10, 3), rng.uniform(0.5, 1.5), random_rotation(rng)))
    mats = [_random_material(rng, 0.0, log_shininess_range=(1.0, 5.0)) for _ in range(51)]
    for (c, r, R), m in zip(geo, mats[:50]):
        add_sphere(b, 3, c, r, R, m)
    b.add(*ground_quad(40.0, -11.5), mats[50])
    lights = []
    for _ in range(3):
        p = rng.uniform(-20, 20, 3) * np.array([1, 0, 1]) + np.array([0, 25, 0])
        i = rng.uniform(0.5, 2.0)
        lights.append([*p, i, i, i])
    sc = b.build(lights, "50xico3+quad")
    if not hidden:
        sc = perturb_params(sc, rng_for(seed + 7), 0.3)
    return sc


def integer_shininess(sc: SceneData) -> SceneData:
    """The same scene with every shininess rounded down to an integer (at least 1).  The
    reference's Material holds its shininess as an int (src/Material.h:47,72), so this is
    the scene its renderer draws when given config 4's continuous shininess."""
    m = sc.materials.copy()
    m[:, 6] = np.maximum(np.floor(m[:, 6]), 1.0)
    return SceneData(sc.verts, sc.normals, sc.tris, sc.tri_obj, m, sc.lights, sc.name + "-intshin",
                     sc.ambient_index)


def perturb_params(sc: SceneData, rng: np.random.Generator, frac: float) -> SceneData:
    m = sc.materials.astype(np.float64).copy()
    l = sc.lights.astype(np.float64).copy()
    m[:, 0:6] *= rng.uniform(1 - frac, 1 + frac, size=(m.shape[0], 6))
    m[:, 6] = np.exp(np.log(m[:, 6]) * rng.uniform(1 - frac, 1 + frac, size=m.shape[0]))
    l[:, 3:6] *= rng.uniform(1 - frac, 1 + frac, size=(l.shape[0], 1))
    return SceneData(sc.verts, sc.normals, sc.tris, sc.tri_obj, m, l, sc.name + "-perturbed")


def config4_cameras(n_views: int = 8, size: int = 256) -> list[CameraData]:
    cams = []
    for i in range(n_views):
        a = 2 * math.pi * i / n_views
        cams.append(look_at((30 * math.cos(a), 18.0, 30 * math.sin(a)), (0, -2, 0), 60.0, size, size))
    return cams


def config5_scene(seed: int = 1005, instances: int = 800, cluster_tris: int = 5000,
                  cells: int = 512) -> SceneData:
    """800 instances of a 5,000-thin-triangle cluster over a 512x512-cell height field."""
    rng = rng_for(seed)
    b = _Builder()
    V, N, F = heightfield(cells, 200.0, rng)
    b.add(V, N, F, _random_material(rng, 0.9))
    cV, cN, cF = foliage_cluster(cluster_tris, rng)
    for _ in range(instances):
        R = random_rotation(rng)
        t = rng.uniform([-200, 0, -200], [200, 50, 200])
        b.add(cV @ R.T + t, cN @ R.T, cF, _random_material(rng, 0.9))
    lights = []
    for _ in range(8):
        p = rng.uniform([-200, 60, -200], [200, 150, 200])
        i = rng.uniform(0.3, 0.8)
        lights.append([*p, i, i, i])
    return b.build(lights, "foliage800x5000+heightfield512")


def config5_camera(width=3840, height=2160) -> CameraData:
    return look_at((0, 90, 260), (0, 10, 0), 60.0, width, height)


def small_random_scene(seed: int, n_spheres: int = 4, level: int = 2, lights: int = 2,
                       refl: float = 0.5, transparent: int = 0, ambient_index: float = 1.0,
                       both: int = 0) -> SceneData:
    """A few icospheres over a quad: quick scenes for parity edge cases.  The first
    `transparent` spheres get non-reflective transparent materials (refractive index
    1.333, 1.52 or 2.42 in turn); the next `both` spheres get materials that are both
    reflective (0.35) and transparent (index 1.45, 1.6 or 1.333 in turn), whose hits spawn
    two secondary rays."""
    rng = rng_for(seed)
    b = _Builder()
    for k in range(n_spheres):
        center, radius, rot = rng.uniform(-2, 2, 3), rng.uniform(0.3, 1.2), random_rotation(rng)
        m = _random_material(rng, refl)
        if k < transparent:
            m[7], m[8], m[9] = 0.0, 1.0, (1.333, 1.52, 2.42)[k % 3]
        elif k < transparent + both:
            m[7], m[8], m[9] = 0.35, 1.0, (1.45, 1.6, 1.333)[k % 3]
        add_sphere(b, level, center, radius, rot, m)
    b.add(*ground_quad(6.0, -2.5), _random_material(rng, refl))
    ls = [[*rng.uniform([-5, 3, -5], [5, 8, 5]), 1, 1, 1] for _ in range(lights)]
    sc = b.build(ls, f"small{seed}")
    sc.ambient_index = float(ambient_index)
    return sc


def mirror_hall_scene(seed: int = 71) -> SceneData:
    """Two parallel mirrors with four spheres between them over a reflective floor, under
    eight lights: paths down to the deepest trace depth (7: eight hits) and eight shadow
    bits per hit."""
    rng = rng_for(seed)
    V, N, F, O = [], [], [], []

    def add(v, n, f, obj):
        F.append(np.asarray(f) + sum(len(x) for x in V))
        V.append(np.asarray(v, np.float64))
        N.append(np.asarray(n, np.float64))
        O.append(np.full(len(f), obj))

    for obj, x in ((0, -2.0), (1, 2.0)):  # mirrors facing each other
        v = [[x, -2, -6], [x, -2, 6], [x, 3, 6], [x, 3, -6]]
        add(v, [[-np.sign(x), 0, 0]] * 4, [[0, 1, 2], [0, 2, 3]] if x > 0 else [[0, 2, 1], [0, 3, 2]], obj)
    add([[-2, -2, -6], [2, -2, -6], [2, -2, 6], [-2, -2, 6]], [[0, 1, 0]] * 4, [[0, 2, 1], [0, 3, 2]], 2)
    iv, ifc = icosphere(2)
    for k, c in enumerate(([-0.8, -1.2, -1.0], [0.9, -0.9, -2.5], [0.0, -0.4, -4.0], [-1.0, 0.2, -3.2])):
        add(iv * 0.6 + c, iv, ifc, 3 + k)
    mats = [material((0.05, 0.05, 0.05), 0.3, 64, 0.95), material((0.05, 0.05, 0.05), 0.3, 64, 0.9),
            material((0.4, 0.4, 0.4), 0.2, 16, 0.3)]
    mats += [material(rng.uniform(0, 1, 3), 0.4, 32, 0.7) for _ in range(4)]
    lights = [[*rng.uniform([-1.8, 1.0, -5.0], [1.8, 2.8, 3.0]), 0.3, 0.3, 0.3] for _ in range(8)]
    return SceneData(np.concatenate(V), np.concatenate(N), np.concatenate(F), np.concatenate(O), mats,
                     np.array(lights), f"mirrors{seed}")


# ----------------------------------------------------------------------------- instancing
@dataclass
class InstancedData:
    """A two-level scene: meshes (each a SceneData whose own materials are unused), and
    instances (mesh index, 3x4 world-from-object transform, material base)."""
    meshes: list
    instances: list
    materials: np.ndarray
    lights: np.ndarray
    name: str = "instances"
    ambient_index: float = 1.0

    def __post_init__(self):
        self.materials = pad_materials(self.materials)
        self.lights = np.ascontiguousarray(self.lights, dtype=np.float32).reshape(-1, LIGHT_STRIDE)

    @property
    def n_tris(self) -> int:
        return sum(self.meshes[m].n_tris for m, _, _ in self.instances)

    def flatten(self) -> SceneData:
        """The same triangles transformed into world space (float64, then float32)."""
        V, N, F, O = [], [], [], []
        nv = 0
        for m, M, base in self.instances:
            sc = self.meshes[m]
            A, t = np.asarray(M, np.float64)[:, :3], np.asarray(M, np.float64)[:, 3]
            V.append(sc.verts.astype(np.float64) @ A.T + t)
            n = sc.normals.astype(np.float64) @ np.linalg.inv(A)
            N.append(n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30))
            F.append(sc.tris.astype(np.int64) + nv)
            O.append(sc.tri_obj.astype(np.int64) + base)
            nv += sc.verts.shape[0]
        return SceneData(np.concatenate(V), np.concatenate(N), np.concatenate(F), np.concatenate(O), self.materials,
                         self.lights, self.name + " (flattened)", self.ambient_index)


def _affine(R, t, scale=1.0):
    M = np.zeros((3, 4))
    M[:, :3] = np.asarray(R, np.float64) * scale
    M[:, 3] = t
    return M


def instanced_test_scene(seed: int, n_instances: int = 12, lights: int = 2, transparent: int = 0) -> InstancedData:
    """Three meshes (a level-2 icosphere, a ground quad, a 300-triangle foliage cluster) placed
    n_instances times: instance 0 is the identity, the others rotated, scaled (one of them
    non-uniformly, one mirrored) and moved; one material per instance."""
    rng = rng_for(seed)
    meshes = []
    v, f = icosphere(2)
    meshes.append(SceneData(v, v, f, np.zeros(len(f)), [material((0.5, 0.5, 0.5), 0.2, 16, 0.0)], np.zeros((0, 6))))
    qv, qn, qf = ground_quad(4.0, 0.0)
    meshes.append(SceneData(qv, qn, qf, np.zeros(len(qf)), [material((0.5, 0.5, 0.5), 0.2, 16, 0.0)], np.zeros((0, 6))))
    cv, cn, cf = foliage_cluster(300, rng, radius=1.0)
    meshes.append(SceneData(cv, cn, cf, np.zeros(len(cf)), [material((0.5, 0.5, 0.5), 0.2, 16, 0.0)], np.zeros((0, 6))))
    instances = [(1, _affine(np.eye(3), (0.0, -2.5, 0.0)), 0)]
    mats = [_random_material(rng, 0.5)]
    for k in range(1, n_instances):
        R = random_rotation(rng)
        t = rng.uniform([-3, -1.5, -3], [3, 1.5, 3])
        s = rng.uniform(0.4, 1.2)
        M = _affine(R, t, s)
        if k == 1:
            M[:, :3] = np.eye(3)  # identity placement of the sphere
            M[:, 3] = 0.0
        if k == 2:
            M[:, :3] = M[:, :3] @ np.diag([1.0, 0.5, 1.5])  # non-uniform scale
        if k == 3:
            M[:, :3] = M[:, :3] @ np.diag([-1.0, 1.0, 1.0])  # mirrored
        instances.append((0 if k % 2 else 2, M, k))
        m = _random_material(rng, 0.5)
        if k <= transparent:
            m[7], m[8], m[9] = 0.0, 1.0, 1.52
        mats.append(m)
    ls = [[*rng.uniform([-5, 3, -5], [5, 8, 5]), 1, 1, 1] for _ in range(lights)]
    return InstancedData(meshes, instances, np.array(mats), np.array(ls), f"instanced{seed}")


def config5_instanced(seed: int = 1005, instances: int = 800, cluster_tris: int = 5000,
                      cells: int = 512) -> InstancedData:
    """Config 5 as instances: the height field once and the foliage cluster stored once and
    placed 800 times (the same rotations, offsets and materials as config5_scene)."""
    rng = rng_for(seed)
    V, N, F = heightfield(cells, 200.0, rng)
    mats = [_random_material(rng, 0.9)]
    unused = [material((0.5, 0.5, 0.5), 0.2, 16, 0.0)]
    hf = SceneData(V, N, F, np.zeros(len(F)), unused, np.zeros((0, 6)), "heightfield")
    cV, cN, cF = foliage_cluster(cluster_tris, rng)
    cl = SceneData(cV, cN, cF, np.zeros(len(cF)), unused, np.zeros((0, 6)), "foliage cluster")
    inst = [(0, _affine(np.eye(3), (0.0, 0.0, 0.0)), 0)]
    for k in range(instances):
        R = random_rotation(rng)
        t = rng.uniform([-200, 0, -200], [200, 50, 200])
        inst.append((1, _affine(R, t), k + 1))
        mats.append(_random_material(rng, 0.9))
    lights = []
    for _ in range(8):
        p = rng.uniform([-200, 60, -200], [200, 150, 200])
        i = rng.uniform(0.3, 0.8)
        lights.append([*p, i, i, i])
    return InstancedData([hf, cl], inst, np.array(mats), np.array(lights), "foliage800x5000+heightfield512, instanced")
