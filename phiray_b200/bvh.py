"""``GpuBvh`` and ``Bvh``: phiray's LBVH types over the C ABI.

Reference: src/bvh/gpu.rs (GpuBvh: build, refit, update, download),
src/bvh/build.rs (Bvh), src/bvh/node.rs (Node, Aabb layouts).

Arrays: prims are ``(n, 8) float32`` rows ``[lo.x, lo.y, lo.z, pad, hi.x,
hi.y, hi.z, pad]`` (bvh::Aabb); nodes are ``(m, 8)`` rows of 32 bytes
(bvh::Node): words 3 and 7 are the indices (uint32, leaf bit 31 in word 3).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .gpu import Gpu, GpuArray, devptr

LEAF = N.LEAF
STACK = N.STACK


def aabbs(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    """(n, 8) float32 Aabb rows from (n, 3) corners."""
    n = len(lo)
    out = np.zeros((n, 8), dtype=np.float32)
    out[:, 0:3] = lo
    out[:, 4:7] = hi
    return out


def of_tri(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """``Aabb::of_tri`` for (n, 3) corner arrays."""
    return aabbs(np.minimum(np.minimum(a, b), c), np.maximum(np.maximum(a, b), c))


@dataclass
class Bvh:
    """A downloaded tree (phiray ``Bvh``): nodes (m, 8) float32 with index
    words, order (n,) uint32, depth."""

    nodes: np.ndarray
    order: np.ndarray
    depth: int

    def index(self, k: int) -> tuple[int, int]:
        w = self.nodes[k].view(np.uint32)
        return int(w[3]), int(w[7])

    def is_leaf(self, k: int) -> bool:
        return bool(self.nodes[k].view(np.uint32)[3] & LEAF)

    def bounds(self, k: int) -> tuple[np.ndarray, np.ndarray]:
        return self.nodes[k, 0:3], self.nodes[k, 4:7]

    def reachable(self) -> list[int]:
        """Reachable node indices, root first (``Bvh::reachable``, shape.rs:40-51)."""
        if len(self.nodes) == 0:
            return []
        words = self.nodes.view(np.uint32)
        out, stack = [], [0]
        while stack:
            i = stack.pop()
            out.append(i)
            lo, hi = int(words[i, 3]), int(words[i, 7])
            if not lo & LEAF:
                stack.extend([lo, hi])
        return out


def build_sah(gpu: Gpu, prims: np.ndarray, leaf: int = 4, timeout_ms: int = 0) -> "Bvh":
    """``Bvh::build_sah`` (src/bvh/sah.rs) on the device from host prims:
    the binned SAH tree phiray's tracer walks, read back as a ``Bvh``."""
    prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 8)
    n = len(prims)
    if n == 0:
        return Bvh(np.zeros((0, 8), np.float32), np.zeros(0, np.uint32), 0)
    src = GpuArray.from_(gpu, prims)
    nodes = GpuArray(gpu, (2 * n - 1) * 32)
    order = GpuArray(gpu, n * 4)
    count, depth = C.c_uint32(), C.c_uint32()
    N.check(N.lib().phx_bvh_build_sah(gpu.handle, devptr(src), n, leaf, devptr(nodes), devptr(order),
                                      C.byref(count), C.byref(depth)))
    m = count.value
    out = Bvh(nodes.read(np.float32, timeout_ms=timeout_ms).reshape(-1, 8)[:m].copy(),
              order.read(np.uint32, timeout_ms=timeout_ms), depth.value)
    for a in (src, nodes, order):
        a.free()
    return out


class GpuBvh:
    """An LBVH built and refit on the device (phiray ``GpuBvh``)."""

    def __init__(self, gpu: Gpu, handle: C.c_void_p, leaf: int):
        self.gpu, self.handle, self.leaf = gpu, handle, leaf
        gpu.adopt(self)

    @classmethod
    def build(cls, gpu: Gpu, prims: np.ndarray, leaf: int = 4) -> "GpuBvh":
        """``GpuBvh::build``: host prims in, every stage on the device."""
        prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 8)
        h = C.c_void_p()
        N.check(N.lib().phx_bvh_build(gpu.handle, prims.ctypes.data, len(prims), leaf, C.byref(h)))
        return cls(gpu, h, leaf)

    @classmethod
    def build_device(cls, gpu: Gpu, prims, n: int, leaf: int = 4) -> "GpuBvh":
        h = C.c_void_p()
        N.check(N.lib().phx_bvh_build_device(gpu.handle, devptr(prims), n, leaf, C.byref(h)))
        return cls(gpu, h, leaf)

    def rebuild_device(self, prims, n: int) -> None:
        N.check(N.lib().phx_bvh_rebuild_device(self.handle, devptr(prims), n))

    def refit(self) -> None:
        N.check(N.lib().phx_bvh_refit(self.handle))

    def update(self, prims: np.ndarray) -> bool:
        """``GpuBvh::update``: False (nothing done) when the count changed."""
        prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 8)
        rc = N.check(N.lib().phx_bvh_update(self.handle, prims.ctypes.data, len(prims)))
        return rc != N.PHX_REBUILD

    def update_device(self, prims, n: int) -> bool:
        rc = N.check(N.lib().phx_bvh_update_device(self.handle, devptr(prims), n))
        return rc != N.PHX_REBUILD

    def info(self) -> dict:
        n, m, leaf, depth = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        N.check(N.lib().phx_bvh_info(self.handle, C.byref(n), C.byref(m), C.byref(leaf), C.byref(depth)))
        return {"n": n.value, "nodes": m.value, "leaf": leaf.value, "depth": depth.value}

    def download(self, timeout_ms: int = 0) -> Bvh:
        """``GpuBvh::download``."""
        n = self.info()["n"]
        nodes = np.zeros((max(0, 2 * n - 1), 8), dtype=np.float32)
        order = np.zeros(n, dtype=np.uint32)
        depth = C.c_uint32()
        N.check(
            N.lib().phx_bvh_download(
                self.handle, nodes.ctypes.data if n else None, order.ctypes.data if n else None, C.byref(depth), timeout_ms
            )
        )
        return Bvh(nodes, order, depth.value)

    def device(self) -> dict:
        p, o, nd, c = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        N.check(N.lib().phx_bvh_device(self.handle, C.byref(p), C.byref(o), C.byref(nd), C.byref(c)))
        return {"prims": p.value or 0, "order": o.value or 0, "nodes": nd.value or 0, "codes": c.value or 0}

    def close(self) -> None:
        if self.handle:
            N.lib().phx_bvh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def morton(gpu: Gpu, prims, n: int, codes, scene=None) -> None:
    """Morton codes of device prims into device codes (stage entry point)."""
    N.check(N.lib().phx_morton(gpu.handle, devptr(prims), n, devptr(codes), devptr(scene) or None))


def sort_codes(gpu: Gpu, codes, n: int, order, sorted_codes) -> None:
    """Stable radix sort of device codes (``Bvh::sort_codes``)."""
    N.check(N.lib().phx_sort_codes(gpu.handle, devptr(codes), n, devptr(order), devptr(sorted_codes)))


def karras(gpu: Gpu, sorted_codes, n: int, links) -> None:
    """Karras links (``Link::of``) of device sorted codes."""
    N.check(N.lib().phx_karras(gpu.handle, devptr(sorted_codes), n, devptr(links)))
