"""Seeded synthetic scenes of the benchmark configurations.

No public dataset is involved: every scene is drawn from numpy's PCG64 with
base seed 0x2545F491 (the reference tests' xorshift seed) plus the
configuration index, in float32.

Scene arrays (the layout the tracer reads, phiray's scene contract in
src/trace/scene.rs and layout.wgsl):
  verts  (V, 4) float32   position xyz, w = 1
  faces  (F, 4) uint32    v0, v1, v2, material id
  mats   (M, 32) float32  trace::Mat's first 32 words (src/trace/mat.rs:9-40):
                          color rgba, rough, metal, trans, ior, emit rgb,
                          bump, tex, nmap, maps[3], sss, sss_radius[3],
                          sheen, sheen_rough, sheen_tint[3], coat,
                          coat_rough, aniso, aniso_rot, second, mix (the
                          procedural slots after them are not used)
  lights (L, 20) float32  camera.wgsl `Light` records (80 bytes each)
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SEED = 0x2545F491
MAT_WORDS = 32
NO_TEX = 0xFFFFFFFF
LIGHT_WORDS = 20


def mat(color, rough=0.5, metal=0.0, trans=0.0, ior=1.5, emit=(0.0, 0.0, 0.0)) -> np.ndarray:
    """One material row; defaults are Tri::new's (src/trace/kernel.rs:55-57):
    no textures, sss radius (0.05, 0.01, 0.005), sheen rough 0.5 and tint 1,
    coat rough 0.03, no second lobe."""
    m = np.zeros(MAT_WORDS, dtype=np.float32)
    w = m.view(np.uint32)
    m[0:4] = color
    m[4], m[5], m[6], m[7] = rough, metal, trans, ior
    m[8:11] = emit
    w[12:17] = NO_TEX
    m[18:21] = (0.05, 0.01, 0.005)
    m[22] = 0.5
    m[23:26] = 1.0
    m[27] = 0.03
    w[30] = NO_TEX
    return m


def lambert(albedo) -> np.ndarray:
    """phiray's "Lambertian": Tri::with_pbr(1.0, 0.0) (tests/power/mod.rs:15-18)."""
    return mat([albedo[0], albedo[1], albedo[2], 1.0], rough=1.0, metal=0.0)


def mirror(albedo) -> np.ndarray:
    """A mirror: with_pbr(0.02, 1.0) (metal; the shader floors rough at 0.04)."""
    return mat([albedo[0], albedo[1], albedo[2], 1.0], rough=0.02, metal=1.0)


def light_area(pos, direction, right, size, size_y, power, shape=0) -> np.ndarray:
    """camera.wgsl Light, kind 3 (area): colour x power, shining along `direction`."""
    l = np.zeros(LIGHT_WORDS, dtype=np.float32)
    l[0:3] = pos
    l.view(np.uint32)[3] = 3
    l[4:7] = power
    l[7] = size
    l[8:11] = direction
    l[12:15] = right
    l[15] = size_y
    l.view(np.uint32)[16] = shape
    return l


# trace::Instance as the C ABI takes it (phx_instance): object -> world in
# Blender's layout (m[col][row] at world[4 col + row]), the mesh, whether it
# casts shadows.
INSTANCE = np.dtype([("world", "<f4", 16), ("mesh", "<u4"), ("casts_shadow", "<u4"), ("pad", "<u4", 6)])


def instance(world_rows, mesh: int, casts_shadow: bool = True) -> np.ndarray:
    """One instance record from a 4 x 4 row-major object -> world matrix."""
    r = np.zeros(1, INSTANCE)
    m = np.asarray(world_rows, np.float64).reshape(4, 4)
    r["world"][0] = m.T.reshape(16).astype(np.float32)  # column-major: m[col][row]
    r["mesh"] = mesh
    r["casts_shadow"] = 1 if casts_shadow else 0
    return r


def placement(t=(0.0, 0.0, 0.0), rot_axis=(0.0, 1.0, 0.0), rot_deg=0.0, scale=(1.0, 1.0, 1.0)) -> np.ndarray:
    """A 4 x 4 row-major matrix: scale, then turn, then move."""
    m = np.eye(4)
    m[:3, :3] = _rot(np.asarray(rot_axis, np.float64), math.radians(rot_deg)) @ np.diag(scale)
    m[:3, 3] = t
    return m


def light_sun(direction, power, angle=0.0) -> np.ndarray:
    """camera.wgsl Light, kind 0 (sun): colour x power arriving along
    `direction`, spread over a cone of `angle` radians (Light.size)."""
    l = np.zeros(LIGHT_WORDS, dtype=np.float32)
    l.view(np.uint32)[3] = 0
    l[4:7] = power
    l[7] = angle
    l[8:11] = direction
    return l


def light_point(pos, power, size=0.0) -> np.ndarray:
    """camera.wgsl Light, kind 1 (point): colour x power from `pos`, a ball of
    diameter `size`."""
    l = np.zeros(LIGHT_WORDS, dtype=np.float32)
    l[0:3] = pos
    l.view(np.uint32)[3] = 1
    l[4:7] = power
    l[7] = size
    return l


def light_spot(pos, direction, power, cone, blend, size=0.0, right=(0.0, 0.0, 0.0), scale=(0.0, 0.0)) -> np.ndarray:
    """camera.wgsl Light, kind 2 (spot): a point lamp masked to the cone
    whose cosine is `cone`, softened over `blend`; a non-zero `right` and
    `scale` make the cone elliptical (light.wgsl spot_mask)."""
    l = light_point(pos, power, size)
    l.view(np.uint32)[3] = 2
    l[8:11] = direction
    l[11] = cone
    l[12:15] = right
    l[17] = blend
    l[18:20] = scale
    return l


def light_off() -> np.ndarray:
    """A zero-power point lamp: keeps Camera.count at 1 so the studio rig
    (light.wgsl:87-90, used only when count == 0 and the world is black)
    stays off."""
    l = np.zeros(LIGHT_WORDS, dtype=np.float32)
    l.view(np.uint32)[3] = 1
    return l


@dataclass
class View:
    """phiray's Camera basis (src/trace/camera.rs:5-60): eye at
    pivot + back * dist / units; tan(fov/2) = 0.5 / (scale * dist)."""

    right: tuple
    up: tuple
    back: tuple
    pivot: tuple
    dist: float
    scale: float
    units: float = 1.0

    @staticmethod
    def look(eye, forward, up, fov_deg: float) -> "View":
        f = np.array(forward, np.float64)
        f /= np.linalg.norm(f)
        u = np.array(up, np.float64)
        r = np.cross(f, u)
        r /= np.linalg.norm(r)
        u = np.cross(r, f)
        back = -f
        dist = 1.0
        pivot = np.array(eye, np.float64) - back * dist
        scale = 0.5 / math.tan(math.radians(fov_deg) / 2.0) / dist
        return View(tuple(r), tuple(u), tuple(back), tuple(pivot), dist, scale)


@dataclass
class Scene:
    name: str
    verts: np.ndarray
    faces: np.ndarray
    mats: np.ndarray
    lights: np.ndarray
    view: View
    width: int
    height: int
    spp: int
    bounces: int
    env: tuple = (0.0, 0.0, 0.0)
    meta: dict = field(default_factory=dict)
    normals: np.ndarray | None = None  # (V, 4) float32 vertex normals, or None: flat faces
    sun: tuple = (0.0, 1.0, 0.0)  # Camera.sun: the studio rig's key light direction
    meshes: np.ndarray | None = None  # (M, 2) uint32 face ranges [lo, hi), or None: one identity instance
    insts: np.ndarray | None = None  # INSTANCE records placing the meshes

    @property
    def ntris(self) -> int:
        return len(self.faces)

    def face_boxes(self) -> np.ndarray:
        """(F, 8) Aabb rows (Aabb::of_tri of each face)."""
        p = self.verts[:, :3]
        a, b, c = p[self.faces[:, 0]], p[self.faces[:, 1]], p[self.faces[:, 2]]
        out = np.zeros((len(self.faces), 8), dtype=np.float32)
        out[:, 0:3] = np.minimum(np.minimum(a, b), c)
        out[:, 4:7] = np.maximum(np.maximum(a, b), c)
        return out


def _unit(rng, n):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _quad(p0, p1, p2, p3, m):
    """Two faces over the diagonal p0-p2 (tests/denoise.rs' quad)."""
    v = np.array([p0, p1, p2, p3], dtype=np.float32)
    f = np.array([[0, 1, 2, m], [0, 2, 3, m]], dtype=np.uint32)
    return v, f


def _assemble(parts):
    verts, faces, base = [], [], 0
    for v, f in parts:
        f = f.copy()
        f[:, :3] += base
        verts.append(v)
        faces.append(f)
        base += len(v)
    v = np.concatenate(verts).astype(np.float32)
    vv = np.ones((len(v), 4), dtype=np.float32)
    vv[:, :3] = v
    return vv, np.concatenate(faces).astype(np.uint32)


def c1_plain(ntris: int = 65536, width: int = 256, height: int = 256, spp: int = 16, bounces: int = 4) -> Scene:
    """Config 1 (CPU-runnable): `ntris` small triangles with centroids
    uniform in the unit cube, two edges of length U(0.005, 0.02) in uniform
    random directions, Lambertian albedo U(0.2, 0.8) per face; a 0.3 x 0.3
    emissive quad (radiance 10) at y = 1.2 facing down; a ground quad at
    y = 0; pinhole camera at (0.5, 0.5, -1.5) looking +z, 45 deg fov."""
    rng = np.random.Generator(np.random.PCG64(SEED + 0))
    c = rng.random((ntris, 3))
    e1 = _unit(rng, ntris) * rng.uniform(0.005, 0.02, (ntris, 1))
    e2 = _unit(rng, ntris) * rng.uniform(0.005, 0.02, (ntris, 1))
    a = c - (e1 + e2) / 3.0
    tri_v = np.stack([a, a + e1, a + e2], axis=1).reshape(-1, 3).astype(np.float32)
    tri_f = np.zeros((ntris, 4), dtype=np.uint32)
    tri_f[:, 0] = np.arange(ntris) * 3
    tri_f[:, 1] = tri_f[:, 0] + 1
    tri_f[:, 2] = tri_f[:, 0] + 2
    tri_f[:, 3] = np.arange(ntris)
    albedo = rng.uniform(0.2, 0.8, (ntris, 3)).astype(np.float32)
    mats = [lambert(a) for a in albedo]
    ground_m = len(mats)
    mats.append(lambert((0.5, 0.5, 0.5)))
    light_m = len(mats)
    mats.append(mat([0.0, 0.0, 0.0, 1.0], rough=1.0, emit=(10.0, 10.0, 10.0)))
    g = _quad((-1.5, 0.0, -1.5), (-1.5, 0.0, 2.5), (2.5, 0.0, 2.5), (2.5, 0.0, -1.5), ground_m)
    h = 0.15
    lq = _quad((0.5 - h, 1.2, 0.5 - h), (0.5 + h, 1.2, 0.5 - h), (0.5 + h, 1.2, 0.5 + h), (0.5 - h, 1.2, 0.5 + h), light_m)
    verts, faces = _assemble([(tri_v, tri_f), g, lq])
    view = View.look((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0)
    return Scene("c1_plain", verts, faces, np.stack(mats), np.stack([light_off()]), view, width, height, spp, bounces)


def _icosphere(levels: int):
    """Unit icosphere: 20 * 4**levels faces, shared vertices."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array(
        [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(
        [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6],
         [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
         [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(levels):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        m01, m12, m20 = (inv[0:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base)
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        f = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1), np.stack([c, m20, m12], 1),
                            np.stack([m01, m12, m20], 1)])
    return v, f


def value_noise(p: np.ndarray, seed: int, octaves: int = 4) -> np.ndarray:
    """Seeded 3D value noise (hashed lattice values, smoothstep-trilinear),
    `octaves` octaves of doubling frequency and halving amplitude, in [-1, 1]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    table = rng.uniform(-1.0, 1.0, 1 << 16)
    perm = rng.permutation(1 << 16)

    def lattice(ix, iy, iz):
        h = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791)
        return table[perm[h & 0xFFFF]]

    out = np.zeros(len(p))
    amp, freq, norm = 1.0, 4.0, 0.0
    for _ in range(octaves):
        q = p * freq
        i = np.floor(q).astype(np.int64)
        fr = q - i
        s = fr * fr * (3.0 - 2.0 * fr)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    w = ((s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) *
                         (s[:, 2] if dz else 1 - s[:, 2]))
                    acc += w * lattice(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
        out += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return out / norm


def c2_mesh(levels: int = 8, width: int = 1920, height: int = 1080, spp: int = 64, bounces: int = 8,
            env: float = 0.05) -> Scene:
    """Config 2: an icosphere subdivided `levels` times (8: 1,310,720 faces),
    radius 0.5 at the origin, displaced radially by seeded 4-octave value
    noise of amplitude 0.05; a 2-face ground plane at y = -0.6; four 0.4 x
    0.4 area lights (kind 3) above, facing down; albedo U(0.1, 0.9) per face,
    30% of faces mirrors. The world is a dim uniform grey (`env`), so the
    diffuse path runs its full `bounces` (with a black world and no emissive
    faces the reference's `indirect` returns nothing, integrate.wgsl:111-121)."""
    rng = np.random.Generator(np.random.PCG64(SEED + 1))
    v, f = _icosphere(levels)
    r = 0.5 * (1.0 + 0.05 * value_noise(v, SEED + 1))
    pos = (v * r[:, None]).astype(np.float32)
    nf = len(f)
    tri_f = np.zeros((nf, 4), np.uint32)
    tri_f[:, :3] = f
    tri_f[:, 3] = np.arange(nf)
    albedo = rng.uniform(0.1, 0.9, (nf, 3)).astype(np.float32)
    is_mirror = rng.random(nf) < 0.3
    mats = np.zeros((nf + 1, MAT_WORDS), np.float32)
    lam = mat([0.5, 0.5, 0.5, 1.0], rough=1.0)
    mir = mat([0.5, 0.5, 0.5, 1.0], rough=0.02, metal=1.0)
    mats[:nf] = np.where(is_mirror[:, None], mir, lam)
    mats[:nf, 0:3] = albedo
    mats[nf] = lambert((0.6, 0.6, 0.6))
    g = _quad((-3.0, -0.6, -3.0), (-3.0, -0.6, 3.0), (3.0, -0.6, 3.0), (3.0, -0.6, -3.0), nf)
    verts, faces = _assemble([(pos, tri_f), g])
    lights = [
        light_area((x, 1.5, z), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.4, 0.4, (p, p, p))
        for (x, z, p) in [(-0.8, -0.8, 30.0), (0.8, -0.8, 20.0), (-0.8, 0.8, 20.0), (0.8, 0.8, 15.0)]
    ]
    view = View.look((0.0, 0.3, -2.2), (0.0, -0.1, 1.0), (0.0, 1.0, 0.0), 40.0)
    return Scene("c2_mesh", verts, faces, mats, np.stack(lights), view, width, height, spp, bounces,
                 env=(env, env, env), meta={"levels": levels})


def _rot(axis, ang):
    axis = axis / np.linalg.norm(axis)
    x, y, z = axis
    c, s = math.cos(ang), math.sin(ang)
    C_ = 1 - c
    return np.array([[c + x * x * C_, x * y * C_ - z * s, x * z * C_ + y * s],
                     [y * x * C_ + z * s, c + y * y * C_, y * z * C_ - x * s],
                     [z * x * C_ - y * s, z * y * C_ + x * s, c + z * z * C_]])


@dataclass
class Rig:
    """CSR linear-blend influences (kernel::Pair rows: bone, weight, next,
    blend) over `rest` (V, 4), and the bone chain's joints."""

    rest: np.ndarray
    offsets: np.ndarray
    pairs: np.ndarray
    joints: np.ndarray
    nbones: int

    def bones(self, frame: int, max_deg: float = 15.0) -> np.ndarray:
        """Column-major world matrices (nbones, 16) float32 for `frame`: each
        bone turns at most `max_deg` degrees about its parent joint (seeded
        per frame), composed down the chain."""
        rng = np.random.Generator(np.random.PCG64(SEED + 2 + 7919 * frame))
        world = np.eye(4)
        out = np.zeros((self.nbones, 16), np.float32)
        for b in range(self.nbones):
            axis = rng.standard_normal(3)
            ang = math.radians(max_deg) * rng.uniform(-1.0, 1.0)
            j = self.joints[b]
            local = np.eye(4)
            local[:3, :3] = _rot(axis, ang)
            local[:3, 3] = j - local[:3, :3] @ j
            world = world @ local
            out[b] = world.T.reshape(16).astype(np.float32)  # column-major
        return out


PAIR = np.dtype([("bone", "<u4"), ("weight", "<f4"), ("next", "<u4"), ("blend", "<f4")])


def c3_skinned(rings: int = 1000, segments: int = 500, nbones: int = 64, width: int = 1920, height: int = 1080,
               spp: int = 16, bounces: int = 4):
    """Config 3: a `rings` x `segments` cylinder grid (500k vertices, ~1M
    faces by default), radius 0.3, height 2, rigged with a chain of `nbones`
    bones along its axis; each vertex takes 1-4 influences (uniform count)
    from the bones nearest its height, weights Dirichlet(1). Returns the rest
    Scene and its Rig. Lights: two area lights; a ground plane; a dim world."""
    rng = np.random.Generator(np.random.PCG64(SEED + 2))
    ys = np.linspace(0.0, 2.0, rings)
    th = np.linspace(0.0, 2.0 * math.pi, segments, endpoint=False)
    Y, T = np.meshgrid(ys, th, indexing="ij")
    pos = np.stack([0.3 * np.cos(T), Y, 0.3 * np.sin(T)], -1).reshape(-1, 3).astype(np.float32)
    r = np.arange(rings - 1)[:, None]
    sgm = np.arange(segments)[None, :]
    a = r * segments + sgm
    b = r * segments + (sgm + 1) % segments
    c = (r + 1) * segments + (sgm + 1) % segments
    d = (r + 1) * segments + sgm
    f1 = np.stack([a, b, c], -1).reshape(-1, 3)
    f2 = np.stack([a, c, d], -1).reshape(-1, 3)
    tri = np.concatenate([f1, f2])
    nf = len(tri)
    tri_f = np.zeros((nf, 4), np.uint32)
    tri_f[:, :3] = tri
    tri_f[:, 3] = (np.arange(nf) % 7).astype(np.uint32)
    mats = [lambert(rng.uniform(0.2, 0.8, 3)) for _ in range(7)]
    mats.append(lambert((0.6, 0.6, 0.6)))
    g = _quad((-3.0, 0.0, -3.0), (-3.0, 0.0, 3.0), (3.0, 0.0, 3.0), (3.0, 0.0, -3.0), 7)
    verts, faces = _assemble([(pos, tri_f), g])
    # Rig: bone b spans heights [b, b + 1) * 2 / nbones, joint at its base.
    nv = len(verts)
    seg_h = 2.0 / nbones
    vb = np.clip((verts[:, 1] / seg_h).astype(np.int64), 0, nbones - 1)
    counts = rng.integers(1, 5, nv)
    counts[len(pos):] = 0  # the ground is not skinned
    offsets = np.zeros(nv + 1, np.uint32)
    offsets[1:] = np.cumsum(counts)
    k = int(offsets[-1])
    pairs = np.zeros(k, PAIR)
    rep = np.repeat(np.arange(nv), counts)
    slot = np.arange(k) - np.repeat(offsets[:-1].astype(np.int64), counts)
    bone = np.clip(vb[rep] + (slot + 1) // 2 * np.where(slot % 2 == 1, 1, -1), 0, nbones - 1)
    pairs["bone"] = bone
    pairs["next"] = bone
    # Dirichlet(1) over each vertex's influences: normalised Exp(1) draws.
    e = rng.exponential(1.0, k)
    sums = np.add.reduceat(e, offsets[:-1][counts > 0].astype(np.int64))
    pairs["weight"] = (e / np.repeat(sums, counts[counts > 0])).astype(np.float32)
    joints = np.stack([np.zeros(nbones), np.arange(nbones) * seg_h, np.zeros(nbones)], -1)
    lights = [light_area((-0.8, 2.8, -0.8), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.6, 0.6, (60.0, 60.0, 60.0)),
              light_area((0.9, 2.5, -0.5), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.4, 0.4, (30.0, 30.0, 30.0))]
    view = View.look((0.0, 1.0, -3.2), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0)
    scene = Scene("c3_skinned", verts, faces, np.stack(mats), np.stack(lights), view, width, height, spp, bounces,
                  env=(0.05, 0.05, 0.05))
    return scene, Rig(verts.copy(), offsets, pairs, joints, nbones)


def _box(center, size, n):
    """An axis-aligned box, each face an n x n grid of quads (12 n^2 faces)."""
    t = np.linspace(-0.5, 0.5, n + 1)
    U, V = np.meshgrid(t, t, indexing="ij")
    verts, faces, base = [], [], 0
    for axis in range(3):
        for side in (-0.5, 0.5):
            p = np.zeros((n + 1, n + 1, 3))
            a1, a2 = (axis + 1) % 3, (axis + 2) % 3
            p[..., axis] = side
            p[..., a1] = U
            p[..., a2] = V if side > 0 else -V
            verts.append(p.reshape(-1, 3))
            i = np.arange(n)[:, None] * (n + 1) + np.arange(n)[None, :]
            q = np.stack([i, i + n + 1, i + n + 2, i + 1], -1).reshape(-1, 4) + base
            faces.append(np.concatenate([q[:, [0, 1, 2]], q[:, [0, 2, 3]]]))
            base += (n + 1) * (n + 1)
    v = np.concatenate(verts) * np.asarray(size) + np.asarray(center)
    return v, np.concatenate(faces)


def procedural(index: int, width: int = 256, height: int = 256, spp: int = 4, bounces: int | None = None,
               target: int | None = None) -> Scene:
    """One seeded procedural scene of the learned denoiser's training set:
    random boxes, spheres and noise-displaced spheres (plus a cloud of small
    triangles; in about half of the scenes a finely tessellated displaced
    sphere with per-face albedo and mirror faces fills much of the view) on a
    ground plane, 10k-500k faces in total (log-uniform
    target), per-object or per-face albedo, some mirror objects, 1-4 area
    lights and sometimes an emissive panel, a dim uniform world, and a camera
    on a random orbit around the objects. `target` overrides the drawn face
    budget (the cloud of small triangles fills up to it)."""
    rng = np.random.Generator(np.random.PCG64(SEED + 4 + 104729 * index))
    drawn = int(math.exp(rng.uniform(math.log(1e4), math.log(5e5))))
    target = drawn if target is None else int(target)
    parts, mats = [], []

    def add(v, f, kind):
        m0 = len(mats)
        nf = len(f)
        if kind == "mirror":
            mats.append(mirror(rng.uniform(0.5, 1.0, 3)))
            mid = np.full(nf, m0)
        elif kind == "faces":  # per-face albedo, like a texture at triangle scale
            k = min(nf, 4096)
            for a in rng.uniform(0.05, 0.95, (k, 3)):
                mats.append(lambert(a))
            mid = m0 + rng.integers(0, k, nf)
        elif kind == "mixed":  # per-face albedo with a share of mirror faces
            k = min(nf, 2048)
            share = rng.uniform(0.1, 0.4)
            for a in rng.uniform(0.1, 0.9, (k, 3)):
                mats.append(mirror(a) if rng.random() < share else lambert(a))
            mid = m0 + rng.integers(0, k, nf)
        else:
            mats.append(lambert(rng.uniform(0.05, 0.95, 3)))
            mid = np.full(nf, m0)
        ff = np.zeros((nf, 4), np.uint32)
        ff[:, :3] = f
        ff[:, 3] = mid
        parts.append((v.astype(np.float32), ff))

    def kind():
        return rng.choice(["plain", "faces", "mirror", "mixed"], p=[0.45, 0.25, 0.15, 0.15])

    ground_y = -0.6
    g = _quad((-4.0, ground_y, -4.0), (-4.0, ground_y, 4.0), (4.0, ground_y, 4.0), (4.0, ground_y, -4.0), 0)
    mats.append(lambert(rng.uniform(0.2, 0.8, 3)))
    parts.append((np.asarray(g[0], np.float32), g[1]))
    if rng.random() < 0.5:  # a back wall
        z = rng.uniform(1.2, 2.5)
        w = _quad((-4.0, ground_y, z), (4.0, ground_y, z), (4.0, 3.0, z), (-4.0, 3.0, z), len(mats))
        mats.append(lambert(rng.uniform(0.2, 0.8, 3)))
        parts.append((np.asarray(w[0], np.float32), w[1]))
    used = 0
    hero = rng.random() < 0.5
    if hero:  # a finely tessellated, noise-displaced sphere filling much of the view
        v, f = _icosphere(6 if rng.random() < 0.6 else 7)
        r = 1.0 + rng.uniform(0.03, 0.1) * value_noise(v, int(rng.integers(1 << 30)))
        s_h = rng.uniform(0.4, 0.65)
        v = v * (r * s_h)[:, None] + np.array([0.0, ground_y + s_h * 1.05, 0.0])
        add(v, f, "mixed" if rng.random() < 0.7 else "faces")
        used += len(f)
    for _ in range(int(rng.integers(2, 8) if not hero else rng.integers(0, 4))):
        c = np.array([rng.uniform(-0.9, 0.9), 0.0, rng.uniform(-0.9, 0.9)])
        s = rng.uniform(0.15, 0.5)
        t = rng.random()
        if t < 0.35:
            n = int(rng.integers(2, 24))
            size = s * rng.uniform(0.5, 1.5, 3)
            c[1] = ground_y + size[1] / 2
            v, f = _box(c, size, n)
        else:
            lv = int(rng.integers(2, 6))
            v, f = _icosphere(lv)
            if t > 0.65:  # displaced
                r = 1.0 + rng.uniform(0.05, 0.25) * value_noise(v, int(rng.integers(1 << 30)))
                v = v * r[:, None]
            c[1] = ground_y + s * rng.uniform(0.7, 1.3)
            v = v * s + c
        add(v, f, kind())
        used += len(f)
    if used < target:  # fill the budget with a cloud of small triangles
        nt = target - used
        cen = np.array([0.0, ground_y + 0.5, 0.0]) + rng.uniform(-0.6, 0.6, (nt, 3)) * np.array([1.5, 0.8, 1.5])
        e1 = _unit(rng, nt) * rng.uniform(0.01, 0.04, (nt, 1))
        e2 = _unit(rng, nt) * rng.uniform(0.01, 0.04, (nt, 1))
        a = cen - (e1 + e2) / 3.0
        v = np.stack([a, a + e1, a + e2], 1).reshape(-1, 3)
        f = np.arange(3 * nt).reshape(nt, 3)
        add(v, f, rng.choice(["plain", "faces"]))
    lights = []
    for _ in range(int(rng.integers(1, 5))):
        pos = (rng.uniform(-1.5, 1.5), rng.uniform(1.0, 2.5), rng.uniform(-1.5, 1.5))
        sz = rng.uniform(0.15, 0.6)
        p = rng.uniform(5.0, 40.0) * rng.uniform(0.7, 1.0, 3)
        lights.append(light_area(pos, (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), sz, sz * rng.uniform(0.5, 1.5), tuple(p)))
    if rng.random() < 0.3:  # an emissive panel seen by the camera and the paths
        h_ = rng.uniform(0.1, 0.3)
        y = rng.uniform(0.5, 1.5)
        x0, z0 = rng.uniform(-1.0, 1.0, 2)
        q = _quad((x0 - h_, y, z0 - h_), (x0 + h_, y, z0 - h_), (x0 + h_, y, z0 + h_), (x0 - h_, y, z0 + h_), len(mats))
        mats.append(mat([0.0, 0.0, 0.0, 1.0], rough=1.0, emit=tuple(rng.uniform(3.0, 15.0) * np.ones(3))))
        parts.append((np.asarray(q[0], np.float32), q[1]))
    verts, faces = _assemble(parts)
    az = rng.uniform(0.0, 2.0 * math.pi)
    el = math.radians(rng.uniform(5.0, 40.0))
    dist = rng.uniform(1.4, 2.2) if hero else rng.uniform(1.8, 3.2)
    look = np.array([0.0, ground_y + 0.4, 0.0])
    eye = look + dist * np.array([math.cos(el) * math.sin(az), math.sin(el), -math.cos(el) * math.cos(az)])
    view = View.look(tuple(eye), tuple(look - eye), (0.0, 1.0, 0.0), rng.uniform(35.0, 55.0))
    env = rng.uniform(0.0, 0.2)
    b = int(rng.integers(4, 9)) if bounces is None else bounces
    return Scene(f"procedural_{index}", verts, faces, np.stack(mats).astype(np.float32), np.stack(lights), view,
                 width, height, spp, b, env=(env, env, env), meta={"index": index, "target": target, "hero": hero})


RESOLUTIONS = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]


def c5_batch(count: int = 64):
    """Config 5's scenes: `count` procedural scenes with face counts
    log-uniform over 10k-2M, resolutions drawn from 256^2, 512^2, 720p and
    1080p, 1, 4 or 16 samples per pixel, 6 bounces (seeded)."""
    rng = np.random.Generator(np.random.PCG64(SEED + 5))
    out = []
    for k in range(count):
        tris = int(math.exp(rng.uniform(math.log(1e4), math.log(2e6))))
        w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
        spp = int(rng.choice([1, 4, 16]))
        out.append(procedural(200000 + k, width=w, height=h, spp=spp, bounces=6, target=tris))
    return out


def _smooth_normals(verts: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals (V, 4), w = 0."""
    p = verts[:, :3].astype(np.float64)
    a, b, c = p[faces[:, 0]], p[faces[:, 1]], p[faces[:, 2]]
    fn = np.cross(b - a, c - a)
    acc = np.zeros_like(p)
    for k in range(3):
        np.add.at(acc, faces[:, k], fn)
    ln = np.linalg.norm(acc, axis=1, keepdims=True)
    out = np.zeros((len(p), 4), np.float32)
    out[:, :3] = np.where(ln > 0, acc / np.where(ln > 0, ln, 1.0), 0.0)
    return out


def features(kind: str, width: int = 64, height: int = 48, spp: int = 4, bounces: int = 4) -> Scene:
    """Small scenes that reach the Rendered shader's paths the benchmark
    configurations leave unused, each a seeded arrangement of a ground
    quad, a back wall, a smooth (vertex-normal) icosphere, a box and a
    small triangle cloud:

      "lamps"   a sun with an angular size, a point lamp with a radius, an
                elliptical spot lamp and a round area lamp (light.wgsl
                lamp_query, spot_mask, area_query's disc branch);
      "rig"     no lamps and a black world: the studio rig lights the scene
                (light.wgsl uses_rig, rig_query, rig_fill);
      "glass"   a glass sphere, a tinted glass panel, a half-transmissive
                box, an alpha cut-out card and an emissive quad seen through
                them (shade.wgsl's see-through and through loop, refraction
                and total internal reflection; bvh.wgsl's shadow rays
                passing glass and cut-outs; integrate.wgsl's through step);
      "layers"  coat, sheen, subsurface and part-metal materials on the
                smooth sphere and the box (brdf.wgsl brdf_w's coat, sheen
                and bleed terms, fresnel_of's dielectric term).
    """
    rng = np.random.Generator(np.random.PCG64(SEED + 6 + {"lamps": 0, "rig": 1, "glass": 2, "layers": 3}[kind]))
    parts, mats, nparts = [], [], []

    def add(v, f, m, normals=None):
        ff = np.zeros((len(f), 4), np.uint32)
        ff[:, :3] = f
        ff[:, 3] = m
        parts.append((np.asarray(v, np.float32), ff))
        nparts.append(normals)

    def material(row):
        mats.append(row)
        return len(mats) - 1

    g = _quad((-2.0, 0.0, -2.0), (-2.0, 0.0, 2.0), (2.0, 0.0, 2.0), (2.0, 0.0, -2.0), 0)
    add(g[0], g[1][:, :3], material(lambert((0.6, 0.6, 0.55))))
    w = _quad((-2.0, 0.0, 1.2), (2.0, 0.0, 1.2), (2.0, 2.0, 1.2), (-2.0, 2.0, 1.2), 0)
    add(w[0], w[1][:, :3], material(lambert((0.5, 0.55, 0.6))))
    sv, sf = _icosphere(3)
    sphere_c = np.array([-0.35, 0.32, 0.3])
    sv = sv * 0.3 + sphere_c
    bv, bf = _box((0.4, 0.25, 0.45), (0.35, 0.5, 0.35), 3)
    cl_n = 300
    cen = rng.uniform(-0.6, 0.6, (cl_n, 3)) * np.array([1.0, 0.3, 0.4]) + np.array([0.0, 0.9, 0.2])
    e1 = _unit(rng, cl_n) * rng.uniform(0.02, 0.05, (cl_n, 1))
    e2 = _unit(rng, cl_n) * rng.uniform(0.02, 0.05, (cl_n, 1))
    a0 = cen - (e1 + e2) / 3.0
    cv = np.stack([a0, a0 + e1, a0 + e2], 1).reshape(-1, 3)
    cf = np.arange(3 * cl_n).reshape(cl_n, 3)
    lights = [light_off()]
    env = (0.0, 0.0, 0.0)
    sun = (0.0, 1.0, 0.0)
    smooth_sphere = True
    if kind == "lamps":
        add(sv, sf, material(mat([0.7, 0.3, 0.2, 1.0], rough=0.35)), "smooth")
        add(bv, bf, material(mat([0.3, 0.6, 0.3, 1.0], rough=0.6, metal=0.2)))
        add(cv, cf, material(lambert((0.8, 0.8, 0.3))))
        lights = [
            light_sun((-0.3, -1.0, 0.4), (1.5, 1.4, 1.2), angle=0.08),
            light_point((0.8, 1.4, -0.6), (18.0, 16.0, 14.0), size=0.15),
            light_spot((-0.9, 1.6, -0.5), (0.45, -0.85, 0.3), (40.0, 40.0, 45.0), cone=0.85, blend=0.08, size=0.05,
                       right=(1.0, 0.0, 0.0), scale=(1.0, 1.6)),
            light_area((0.0, 1.9, 0.2), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.5, 0.3, (8.0, 8.0, 8.0), shape=4),
        ]
        env = (0.02, 0.02, 0.03)
    elif kind == "rig":
        add(sv, sf, material(mat([0.6, 0.6, 0.65, 1.0], rough=0.3)), "smooth")
        add(bv, bf, material(mat([0.8, 0.3, 0.3, 1.0], rough=0.7)))
        add(cv, cf, material(mirror((0.9, 0.9, 0.9))))
        lights = np.zeros((0, LIGHT_WORDS), np.float32)
        sun = tuple(np.array([0.4, 0.8, -0.45]) / np.linalg.norm([0.4, 0.8, -0.45]))
    elif kind == "glass":
        add(sv, sf, material(mat([0.95, 0.95, 1.0, 1.0], rough=0.02, trans=1.0, ior=1.5)), "smooth")
        add(bv, bf, material(mat([0.8, 0.5, 0.2, 1.0], rough=0.4, trans=0.5, ior=1.33)))
        add(cv, cf, material(mat([0.3, 0.7, 0.9, 0.4], rough=0.8)))  # alpha 0.4: a cut-out
        pv, pf = _quad((-0.9, 0.05, -0.45), (0.1, 0.05, -0.45), (0.1, 0.75, -0.55), (-0.9, 0.75, -0.55), 0)
        add(pv, pf[:, :3], material(mat([0.6, 0.9, 0.7, 1.0], rough=0.15, trans=0.9, ior=1.7)))
        ev, ef = _quad((0.5, 1.5, 0.0), (0.9, 1.5, 0.0), (0.9, 1.5, 0.4), (0.5, 1.5, 0.4), 0)
        add(ev, ef[:, :3], material(mat([0.0, 0.0, 0.0, 1.0], rough=1.0, emit=(12.0, 11.0, 9.0))))
        lights = [light_area((-0.5, 1.8, -0.3), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.6, 0.6, (14.0, 14.0, 14.0))]
        env = (0.05, 0.06, 0.08)
    elif kind == "layers":
        coat = mat([0.7, 0.15, 0.1, 1.0], rough=0.5)
        coat[26], coat[27] = 0.8, 0.08
        add(sv, sf, material(coat), "smooth")
        sheen = mat([0.2, 0.25, 0.6, 1.0], rough=0.9)
        sheen[21], sheen[22], sheen[23:26] = 0.8, 0.3, (1.0, 0.9, 0.8)
        sheen[17], sheen[18:21] = 0.6, (0.2, 0.08, 0.04)  # subsurface weight and radius
        add(bv, bf, material(sheen))
        part = mat([0.9, 0.8, 0.5, 1.0], rough=0.25, metal=0.5)
        part[26], part[27] = 0.3, 0.2
        add(cv, cf, material(part))
        lights = [light_area((-0.6, 1.8, -0.6), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.5, 0.5, (16.0, 15.0, 14.0)),
                  light_point((0.9, 1.2, -0.8), (6.0, 6.0, 7.0), size=0.1)]
        env = (0.04, 0.04, 0.05)
    else:
        raise ValueError(kind)
    verts, faces = _assemble(parts)
    normals = np.zeros((len(verts), 4), np.float32)
    at = 0
    for (v, f), nrm in zip(parts, nparts):
        if nrm == "smooth" and smooth_sphere:
            normals[at:at + len(v)] = _smooth_normals(np.c_[v, np.ones(len(v))], f[:, :3].astype(np.int64))
        at += len(v)
    view = View.look((0.1, 0.75, -1.9), (-0.05, -0.25, 1.0), (0.0, 1.0, 0.0), 50.0)
    lights = np.asarray(lights, np.float32).reshape(-1, LIGHT_WORDS)
    return Scene(f"features_{kind}", verts, faces, np.stack(mats).astype(np.float32), lights, view, width, height,
                 spp, bounces, env=env, normals=normals, sun=sun)


def instanced(width: int = 64, height: int = 48, spp: int = 4, bounces: int = 4) -> Scene:
    """Meshes placed by instances (forest.rs, instance.rs): a smooth
    icosphere mesh shown three times — moved, turned with a non-uniform
    scale, and mirrored (a scale of -1, world_ng's case) — one copy casting
    no shadow; a box mesh twice; a glowing panel mesh twice (an emitter
    entry per instance, lamp.rs table_of); the ground as its own mesh at the
    identity; an empty mesh with an instance (never placed in the top
    tree). Two area lamps."""
    parts, mats, normals = [], [], []

    def material(row):
        mats.append(row)
        return len(mats) - 1

    ranges = []

    def mesh(v, f, m, smooth=False):
        lo = sum(len(p[1]) for p in parts)
        ff = np.zeros((len(f), 4), np.uint32)
        ff[:, :3] = f
        ff[:, 3] = m
        v = np.asarray(v, np.float32)
        parts.append((v, ff))
        normals.append(_smooth_normals(np.c_[v, np.ones(len(v))], ff[:, :3].astype(np.int64)) if smooth
                       else np.zeros((len(v), 4), np.float32))
        ranges.append((lo, lo + len(f)))
        return len(ranges) - 1

    g = _quad((-2.5, 0.0, -2.5), (-2.5, 0.0, 2.5), (2.5, 0.0, 2.5), (2.5, 0.0, -2.5), 0)
    ground = mesh(g[0], g[1][:, :3], material(lambert((0.55, 0.55, 0.5))))
    sv, sf = _icosphere(3)
    sphere = mesh(sv * 0.3, sf, material(mat([0.7, 0.35, 0.2, 1.0], rough=0.3)), smooth=True)
    bv, bf = _box((0.0, 0.0, 0.0), (0.3, 0.4, 0.3), 2)
    box = mesh(bv, bf, material(mat([0.3, 0.5, 0.8, 1.0], rough=0.6, metal=0.3)))
    pv, pf = _quad((-0.2, 0.0, -0.2), (0.2, 0.0, -0.2), (0.2, 0.0, 0.2), (-0.2, 0.0, 0.2), 0)
    panel = mesh(pv, pf[:, :3], material(mat([0.0, 0.0, 0.0, 1.0], rough=1.0, emit=(9.0, 8.0, 7.0))))
    empty = len(ranges)
    at = sum(len(p[1]) for p in parts)
    ranges.append((at, at))
    verts, faces = _assemble(parts)
    insts = [
        instance(placement(), ground),
        instance(placement((-0.6, 0.32, 0.2)), sphere),
        instance(placement((0.1, 0.45, 0.5), (1.0, 1.0, 0.0), 35.0, (1.2, 0.7, 1.0)), sphere, casts_shadow=False),
        instance(placement((0.75, 0.3, -0.1), scale=(-1.0, 1.0, 1.0)), sphere),
        instance(placement((-0.2, 0.2, -0.5), (0.0, 1.0, 0.0), 30.0), box),
        instance(placement((0.6, 0.2, 0.7), (0.0, 1.0, 0.0), -20.0, (1.0, 1.5, 1.0)), box),
        instance(placement((-0.5, 1.4, 0.0), (1.0, 0.0, 0.0), 180.0), panel),
        instance(placement((0.7, 1.2, 0.4), (1.0, 0.0, 0.2), 160.0, (1.5, 1.0, 0.8)), panel),
        instance(placement((5.0, 0.0, 0.0)), empty),
    ]
    lights = [light_area((-0.3, 1.9, -0.6), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.5, 0.5, (10.0, 10.0, 10.0)),
              light_area((0.9, 1.7, 0.3), (0.0, -1.0, 0.0), (1.0, 0.0, 0.0), 0.3, 0.4, (6.0, 6.0, 6.0))]
    view = View.look((0.0, 1.0, -2.2), (0.0, -0.35, 1.0), (0.0, 1.0, 0.0), 50.0)
    return Scene("instanced", verts, faces, np.stack(mats).astype(np.float32), np.stack(lights), view, width, height,
                 spp, bounces, env=(0.03, 0.03, 0.04), normals=np.concatenate(normals),
                 meshes=np.asarray(ranges, np.uint32).reshape(-1, 2), insts=np.concatenate(insts))


def flatten(scene: Scene) -> Scene:
    """The same world as one identity instance: every instance's faces
    placed in world space (float64, then float32), normals turned by the
    inverse-transpose. For sanity checks of the instanced path against the
    flat one (close, not bit-equal: the rounding and the trees differ)."""
    vs, fs, ns, base = [], [], [], 0
    for r in scene.insts:
        lo, hi = scene.meshes[r["mesh"]]
        if hi <= lo:
            continue
        f = scene.faces[lo:hi]
        used = np.unique(f[:, :3])
        remap = np.zeros(len(scene.verts), np.int64)
        remap[used] = np.arange(len(used)) + base
        m = r["world"].reshape(4, 4).T.astype(np.float64)  # rows
        p = scene.verts[used, :3].astype(np.float64) @ m[:3, :3].T + m[:3, 3]
        nrm = scene.normals[used, :3].astype(np.float64) @ np.linalg.inv(m[:3, :3])
        ln = np.linalg.norm(nrm, axis=1, keepdims=True)
        nrm = np.where(ln > 1e-12, nrm / np.where(ln > 1e-12, ln, 1.0), 0.0)
        vv = np.ones((len(used), 4), np.float32)
        vv[:, :3] = p
        nn = np.zeros((len(used), 4), np.float32)
        nn[:, :3] = nrm
        ff = f.copy()
        ff[:, :3] = remap[f[:, :3]]
        if np.linalg.det(m[:3, :3]) < 0:  # keep the outward winding a mirror turns over
            ff[:, [1, 2]] = ff[:, [2, 1]]
        vs.append(vv)
        ns.append(nn)
        fs.append(ff)
        base += len(used)
    return Scene(scene.name + "_flat", np.concatenate(vs), np.concatenate(fs).astype(np.uint32), scene.mats,
                 scene.lights, scene.view, scene.width, scene.height, scene.spp, scene.bounces, env=scene.env,
                 normals=np.concatenate(ns))
