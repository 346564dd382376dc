"""Seeded synthetic scenes of the benchmark configurations.

No public dataset is involved: every scene is drawn from numpy's PCG64 with
base seed 0x2545F491 (the reference tests' xorshift seed) plus the
configuration index, in float32.

Scene arrays (the layout the tracer reads, phiray's scene contract in
src/trace/scene.rs and layout.wgsl):
  verts  (V, 4) float32   position xyz, w = 1
  faces  (F, 4) uint32    v0, v1, v2, material id
  mats   (M, 16) float32  Mat (src/trace/mat.rs) reduced to the inputs the
                          Rendered path reads: color rgba, rough, metal,
                          trans, ior, emit rgb, 0, 0, 0, 0, 0
  lights (L, 20) float32  camera.wgsl `Light` records (80 bytes each)
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SEED = 0x2545F491
MAT_WORDS = 16
LIGHT_WORDS = 20


def mat(color, rough=0.5, metal=0.0, trans=0.0, ior=1.5, emit=(0.0, 0.0, 0.0)) -> np.ndarray:
    """One material row; defaults are Tri::new's (src/trace/kernel.rs)."""
    m = np.zeros(MAT_WORDS, dtype=np.float32)
    m[0:4] = color
    m[4], m[5], m[6], m[7] = rough, metal, trans, ior
    m[8:11] = emit
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
