"""Direct calls of the Skin and Denoise kernels over device arrays.

Reference: kernel::Skin (src/kernel/skin.rs), kernel::Denoise with
Tracer::denoise_with (src/kernel/denoise.rs, src/trace/read.rs:85-119). The
recordable forms are ``gpu.Skin`` / ``gpu.Denoise`` in a ``Pass``.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .gpu import Gpu, devptr

# Tracer::denoise_with's tuning (read.rs:101-107): normal, albedo, depth, light.
DENOISE_STRENGTH = (64.0, 8.0, 40.0, 7.0)
# Standard view transform, no exposure, gamma 1.
VIEW_STANDARD = (0.0, 0.0, 1.0, 0.0)
PX_LEN = 34  # Tracer::PX_LEN (read.rs:56): words per pixel of the image buffer


def skin(gpu: Gpu, rest, offsets, pairs, bones, nbones: int, out, n: int, min_weight: float = 1e-4) -> None:
    """``Skin`` over device arrays: rest/out vec4 x n, offsets n+1, pairs
    (bone, weight, next, blend) x k, bones column-major mat4 x nbones."""
    N.check(
        N.lib().phx_skin(
            gpu.handle, devptr(rest), devptr(offsets), devptr(pairs), devptr(bones), nbones, devptr(out), n,
            C.c_float(min_weight),
        )
    )


def face_boxes(gpu: Gpu, verts, faces, nfaces: int, boxes) -> None:
    """Face boxes (Aabb::of_tri) of device vec4 vertices and uvec4 faces."""
    N.check(N.lib().phx_face_boxes(gpu.handle, devptr(verts), devptr(faces), nfaces, devptr(boxes)))


def denoise(gpu: Gpu, px, w: int, h: int, strength=DENOISE_STRENGTH, view=VIEW_STANDARD, keep: bool = False) -> None:
    """The four a-trous rounds over a device px image (34 w h + 1 words)."""
    s = (C.c_float * 4)(*strength)
    v = (C.c_float * 4)(*view)
    N.check(N.lib().phx_denoise(gpu.handle, devptr(px), w, h, s, v, 1 if keep else 0))
