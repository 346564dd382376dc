"""Scenes and inputs of the reference's own Rendered-path tests, restated
for the oracle and the CUDA tracer (test infrastructure).

  src/trace/tri.rs:117-251   the card, the preview camera's rays, the
                             xorshift edge rays and the Möller-Trumbore
                             witness (in float32, operation for operation)
  tests/emitter.rs:1-57      the grey wall under glowing panels
  tests/trace.rs:1-81        the red box on a floor, front view pitched 30 deg
  tests/denoise.rs:1-106     dark and pale quads under a bright patch

Where a reference scene needs something the device path does not take,
the stand-in is named beside it.
"""

from __future__ import annotations

import math

import numpy as np

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib

F32 = np.float32
SAMPLE_COUNT = 32  # Tracer::SAMPLE_COUNT, src/trace/mod.rs:129
W = 48  # tri.rs's preview frame


# ---- src/trace/tri.rs ----

def card():
    """tests/preview.rs's card(3.0, 2.0): a quad at y = 2, two triangles over
    the diagonal q0-q2."""
    half, y = F32(3.0), F32(2.0)
    q = [np.array(v, F32) for v in ([-half, y, -half], [half, y, -half], [half, y, half], [-half, y, half])]
    return [(q[0], q[1], q[2]), (q[0], q[2], q[3])]


def diagonal():
    return [(x, W - 1 - x) for x in range(W)]


def preview_ray(x, y):
    """preview.wgsl's primary ray for pixel (x, y): eye (0, -4, 0)."""
    sx = (F32(x) + F32(0.5)) / F32(W) - F32(0.5)
    sy = (F32(y) + F32(0.5)) / F32(W) - F32(0.5)
    d = np.array([sx, F32(4.0), -sy], F32)
    l = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    return np.array([0.0, -4.0, 0.0], F32), np.array([d[0] / l, d[1] / l, d[2] / l], F32)


def xorshift(seed=0x2545F491):
    x = seed

    def rand():
        nonlocal x
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        return F32(x % 1_000_003) / F32(1_000_003.0)

    return rand


def edge_rays(n):
    """tri.rs:201-227: rays at points along the shared edge, from either
    side and well off the axis (d unnormalised)."""
    (p0, _, p2), _ = card()
    rand = xorshift()
    out = []
    for _ in range(n):
        f = F32(0.02) + F32(0.96) * rand()
        aim = np.array([p0[0] + f * (p2[0] - p0[0]), p0[1], p0[2] + f * (p2[2] - p0[2])], F32)
        side = F32(-1.0) if rand() < F32(0.5) else F32(1.0)
        ox = F32(8.0) * (rand() - F32(0.5))
        oy = p0[1] + side * (F32(0.5) + F32(9.0) * rand())
        oz = F32(8.0) * (rand() - F32(0.5))
        o = np.array([ox, oy, oz], F32)
        out.append((o, (aim - o).astype(F32)))
    return out


def moller_trumbore(ta, tb, tc, o, d):
    """The test tri.rs replaced, kept as its witness (tri.rs:121-136)."""
    def sub(p, q):
        return np.array([p[0] - q[0], p[1] - q[1], p[2] - q[2]], F32)

    def dot(p, q):
        return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]

    def cross(p, q):
        return np.array([p[1] * q[2] - p[2] * q[1], p[2] * q[0] - p[0] * q[2], p[0] * q[1] - p[1] * q[0]], F32)

    e1, e2 = sub(tb, ta), sub(tc, ta)
    pv = cross(d, e2)
    det = dot(e1, pv)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = F32(1.0) / det
        tv = sub(o, ta)
        u = dot(tv, pv) * inv
        q = cross(tv, e1)
        v = dot(d, q) * inv
        t = dot(e2, q) * inv
    if abs(det) < 1e-12 or u < 0.0 or u > 1.0 or v < 0.0 or u + v > 1.0:
        return None
    return (float(t), float(u), float(v)) if t > 0.0 else None


def single_triangle_scene(tri):
    """A one-face scene holding `tri` (for walks of that triangle alone)."""
    v = np.ones((3, 4), F32)
    v[:, :3] = np.stack(tri)
    f = np.array([[0, 1, 2, 0]], np.uint32)
    return scenes.Scene("triangle", v, f, np.stack([scenes.lambert((0.5, 0.5, 0.5))]),
                        np.stack([scenes.light_off()]), None, W, W, 1, 1)


# ---- cameras built field by field (phiray's Camera, zero by default) ----

def camera(**fields) -> np.ndarray:
    c = np.zeros(1, dtype=px.tracer.CAMERA)
    for k, v in fields.items():
        c[k] = v
    return c


# ---- tests/emitter.rs ----

def _panel(y, s):
    q = np.array([[-s, y, -s], [s, y, -s], [s, y, s], [-s, y, s]], F32)
    return q, np.array([[0, 1, 2], [0, 2, 3]])


def emitter_case(case):
    """(scene, camera, expected red radiance, tolerance) of emitter.rs's
    near, far or middle panel over the grey wall (albedo 0.5, rough 1)."""
    y, s, power = {"near": (0.2, 40.0, 0.4), "far": (2.0, 0.1, 50.0), "middle": (1.0, 0.5, 2.0)}[case]
    parts = [_panel(0.0, 40.0), _panel(y, s)]
    verts, faces = scenes._assemble([(v, np.c_[f, np.full(2, m)].astype(np.uint32)) for m, (v, f) in enumerate(parts)])
    wall = scenes.mat([0.5, 0.5, 0.5, 1.0], rough=1.0, metal=0.0)
    glow = scenes.mat([0.0, 0.0, 0.0, 0.0], rough=0.5, trans=0.0, ior=1.5, emit=(power, power, power))
    normals = np.zeros((len(verts), 4), F32)
    normals[:, 1] = 1.0  # Tri::new(.., [n; 3], ..) with n = (0, 1, 0)
    scene = scenes.Scene(f"emitter_{case}", verts, faces, np.stack([wall, glow]), np.zeros((1, 20), F32), None,
                         16, 16, SAMPLE_COUNT, 0, normals=normals)
    cam = camera(w=16, h=16, right=(1, 0, 0), up=(0, 0, 1), back=(0, 1, 0), units=1.0, scale=4.0, aspect=1.0,
                 persp=1, dist=0.1, count=1, ao=1e-3)
    pi = F32(math.pi)
    if case == "near":
        want, tol = 0.5 * 0.4, 0.1
    elif case == "far":
        want, tol = 0.5 / pi * 50.0 * 0.04 / 4.0, 0.1
    else:
        sm = F32(0.5) / np.sqrt(F32(1.25))
        want, tol = 0.5 / pi * 4.0 * 2.0 * sm * math.atan(sm), 0.08
    return scene, cam, float(want), tol


def centre_red(radiance):
    """Mean red radiance of the centre 8 x 8 pixels of the 16 x 16 frame."""
    return float(radiance[4:12, 4:12, 0].astype(np.float64).sum() / 64.0)


def wall_view_oracle(orc, scene, cam):
    """(after all 32 samples, after the first) on the oracle."""
    T = oracle_lib.TraceOracle(orc, scene)
    img, _ = T.trace(cam, 0, 1)
    first = centre_red(px.tracer.radiance_of(img, 16, 16))
    T.trace(cam, 1, SAMPLE_COUNT - 1, px=img)
    return first, centre_red(px.tracer.radiance_of(img, 16, 16))


# ---- tests/trace.rs ----

def _quad4(p, n, m):
    v = np.array(p, F32)
    return v, np.array([[0, 1, 2, m], [0, 2, 3, m]], np.uint32), np.tile(np.r_[n, 0.0], (4, 1)).astype(F32)


def box_scene(persp: bool):
    """A red box on a grey floor (trace.rs:5-25), Blender's front view
    pitched down 30 deg (trace.rs:27-49), 160 x 120, the floor grid on."""
    grey = scenes.mat([0.7, 0.7, 0.7, 1.0])
    red = scenes.mat([0.8, 0.2, 0.2, 1.0])
    parts = [_quad4([[-5, -5, 0], [5, -5, 0], [5, 5, 0], [-5, 5, 0]], [0, 0, 1], 0)]
    l, h = -1.0, 1.0

    def z(a):
        return a + 1.0

    faces = [
        ([[l, l, z(h)], [h, l, z(h)], [h, h, z(h)], [l, h, z(h)]], [0, 0, 1]),
        ([[l, l, z(l)], [h, l, z(l)], [h, l, z(h)], [l, l, z(h)]], [0, -1, 0]),
        ([[h, l, z(l)], [h, h, z(l)], [h, h, z(h)], [h, l, z(h)]], [1, 0, 0]),
        ([[l, h, z(l)], [l, l, z(l)], [l, l, z(h)], [l, h, z(h)]], [-1, 0, 0]),
        ([[h, h, z(l)], [l, h, z(l)], [l, h, z(h)], [h, h, z(h)]], [0, 1, 0]),
    ]
    parts += [_quad4(p, n, 1) for p, n in faces]
    verts, fcs = scenes._assemble([(v, f) for v, f, _ in parts])
    normals = np.concatenate([n for _, _, n in parts])
    scene = scenes.Scene("trace_box", verts, fcs, np.stack([grey, red]), np.zeros((0, 20), F32), None, 160, 120,
                         SAMPLE_COUNT, 0, normals=normals)
    sp, cp = np.sin(F32(30.0) * F32(math.pi / 180.0)), np.cos(F32(30.0) * F32(math.pi / 180.0))
    sun = np.array([0.4, -0.5, 0.77], F32)
    sun = sun / np.sqrt((sun * sun).sum())
    cam = camera(w=160, h=120, right=(1, 0, 0), up=(0, sp, cp), back=(0, -cp, sp), pivot=(0, 0, 1), units=1.0,
                 scale=0.08, aspect=1.0, persp=int(persp), dist=1.0 / (0.08 * 1.44), sun=sun,
                 sky=(0.25, 0.27, 0.3, 1.0), env=(0.3, 0.32, 0.36, 1.0), grid=1.0, grid_color=(0.5, 0.5, 0.5, 0.4))
    return scene, cam


def render_oracle(orc, scene, cam, samples):
    """Tracer::render until done: `samples` frames; the packed pixels as
    RGBA bytes (h, w, 4) and the frame count."""
    w, h = int(cam["w"][0]), int(cam["h"][0])
    img, _ = oracle_lib.TraceOracle(orc, scene).trace(cam, 0, samples)
    return img[: w * h].view(np.uint8).reshape(h, w, 4), samples


def box_checks(rgba, cam):
    w, h = int(cam["w"][0]), int(cam["h"][0])
    return rgba[h // 2, w // 2, :3].astype(int), rgba[2, 2, :3].astype(int)


# ---- tests/denoise.rs ----

SIDE = 48


def denoise_scene():
    """Two quads side by side (denoise.rs:32-58): the left dark (0.05), the
    right pale (0.8), Lambert, facing the orthographic camera; one bounce.
    Stand-in for the reference's sky image (environment images are not
    taken by the device path): a sky of two glowing panels the camera sees
    through (alpha 0, as emitter.rs's panels), a wide dim one (radiance 0.3,
    80 x 80 at 30 above the quads) and a small bright patch (radiance 60)
    high to one side. The emitter table picks a panel by its power, as the
    reference's environment table picks a texel by its luminance, so the
    patch takes about four light samples in ten and the diffuse bounce
    rarely finds it: most samples miss the bright part, which is what makes
    the noise."""
    dark = scenes.mat([0.05, 0.05, 0.05, 1.0], rough=1.0)
    pale = scenes.mat([0.8, 0.8, 0.8, 1.0], rough=1.0)
    dome = scenes.mat([0.0, 0.0, 0.0, 0.0], rough=1.0, emit=(0.3, 0.3, 0.3))
    patch_m = scenes.mat([0.0, 0.0, 0.0, 0.0], rough=1.0, emit=(60.0, 60.0, 60.0))
    n = [0, 0, 1]
    parts = [_quad4([[-4, -4, 0], [0, -4, 0], [0, 4, 0], [-4, 4, 0]], n, 0),
             _quad4([[0, -4, 0], [4, -4, 0], [4, 4, 0], [0, 4, 0]], n, 1)]
    big = 40.0
    parts.append(_quad4([[-big, -big, 30], [-big, big, 30], [big, big, 30], [big, -big, 30]], [0, 0, -1], 2))
    c = np.array([7.0, 8.0, 14.0])
    to = -c / np.linalg.norm(c)
    u = np.cross(to, [0.0, 1.0, 0.0])
    u /= np.linalg.norm(u)
    v = np.cross(u, to)
    s = 2.4
    patch = [c - s * u - s * v, c + s * u - s * v, c + s * u + s * v, c - s * u + s * v]
    parts.append(_quad4(patch, to, 3))
    verts, faces = scenes._assemble([(vv, f) for vv, f, _ in parts])
    normals = np.concatenate([nn for _, _, nn in parts])
    scene = scenes.Scene("denoise_quads", verts, faces, np.stack([dark, pale, dome, patch_m]), np.zeros((1, 20), F32),
                         None, SIDE, SIDE, 12, 1, normals=normals)
    cam = camera(w=SIDE, h=SIDE, right=(1, 0, 0), up=(0, 1, 0), back=(0, 0, 1), units=1.0, scale=0.12, aspect=1.0,
                 bounces=1, count=1)
    return scene, cam


def denoise_render_oracle(orc, samples, denoise):
    scene, cam = denoise_scene()
    img, _ = oracle_lib.TraceOracle(orc, scene).trace(cam, 0, samples)
    if denoise:  # Tracer::denoise: strength 64/8/40/7, the camera's view
        img = orc.denoise(img, SIDE, SIDE, view=tuple(float(x) for x in cam["view"][0]))
    return img[: SIDE * SIDE].view(np.uint8).reshape(SIDE * SIDE * 4)


def byte_diff(a, b):
    """Mean absolute difference per colour byte (denoise.rs diff)."""
    return float(np.abs(a.astype(np.float64) - b.astype(np.float64)).mean())


def edge_numbers(cleaned):
    row = (SIDE // 2) * SIDE

    def at(x):
        return float(cleaned[(row + x) * 4])

    left = sum(at(x) for x in range(4, SIDE // 2 - 4)) / (SIDE // 2 - 8)
    right = sum(at(x) for x in range(SIDE // 2 + 4, SIDE - 4)) / (SIDE // 2 - 8)
    step = at(SIDE // 2 + 1) - at(SIDE // 2 - 2)
    return left, right, step
