"""ctypes loader of the oracle (oracle/liboracle.so): the C++ restatement of
phiray's CPU twins and WGSL that the CUDA kernels are checked against. Test
infrastructure only; builds the library from oracle/Makefile if missing."""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent.parent / "oracle"
LIB = ORACLE_DIR / "liboracle.so"

vp, u32, i32, u64, f32 = C.c_void_p, C.c_uint32, C.c_int32, C.c_uint64, C.c_float

SIGS = {
    "orc_threads": (C.c_int, []),
    "orc_set_threads": (None, [C.c_int]),
    "orc_morton": (u64, [vp, u32]),
    "orc_scene": (None, [vp, u32, vp]),
    "orc_codes": (None, [vp, u32, vp]),
    "orc_sort_codes": (None, [vp, u32, vp, vp]),
    "orc_radix_model": (None, [vp, u32, vp, vp]),
    "orc_delta": (i32, [vp, u32, C.c_int64, C.c_int64]),
    "orc_links": (None, [vp, u32, vp]),
    "orc_assemble": (None, [u32, vp, u32, vp, C.POINTER(u32)]),
    "orc_refit": (None, [vp, u32, vp, vp]),
    "orc_build": (None, [vp, u32, u32, vp, vp, C.POINTER(u32)]),
    "orc_build_sah": (u32, [vp, u32, u32, vp, vp, C.POINTER(u32)]),
    "orc_build_compact": (u32, [vp, u32, u32, vp, vp, C.POINTER(u32)]),
    "orc_compact": (u32, [vp, u32]),
    "orc_reachable": (u32, [vp, u32, vp]),
    "orc_skin": (None, [vp, vp, vp, vp, f32, u32, vp]),
    "orc_denoise": (None, [vp, u32, u32, C.POINTER(f32), C.POINTER(f32), C.c_int]),
    "orc_trace": (None, [vp, vp, u32, vp, vp, u32, vp, u32, u32, vp, C.POINTER(u64), u32, u32]),
    "orc_scene_new": (vp, [vp, vp, u32, vp, vp, u32]),
    "orc_scene_new_sah": (vp, [vp, vp, u32, vp, vp, u32]),
    "orc_scene_trace_walk": (None, [vp, vp, u32, u32, vp, C.POINTER(u64), u32, u32, vp]),
    "orc_scene_free": (None, [vp]),
    "orc_scene_trace": (None, [vp, vp, u32, u32, vp, C.POINTER(u64), u32, u32]),
    "orc_primary": (None, [vp, vp, u32, vp, u32, vp, u32, vp, vp]),
    "orc_show": (None, [vp, vp]),
    "orc_trace_rays": (None, [vp, vp, u32, vp, u32, vp, u32, vp, C.c_int]),
    "orc_tri_hit": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "orc_scene_new_instanced": (vp, [vp, vp, u32, vp, vp, u32, vp, u32, vp, u32]),
    "orc_scene_reinstance": (None, [vp, vp, u32]),
    "orc_scene_primary": (None, [vp, vp, u32, vp, vp, vp]),
    "orc_scene_trace_rays": (None, [vp, vp, u32, vp, C.c_int]),
    "orc_math": (None, [C.c_int, vp, vp, vp, u32]),
}


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(ORACLE_DIR.glob("*.cpp")) + list(ORACLE_DIR.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


class Oracle:
    def __init__(self, lib: C.CDLL):
        self.lib = lib

    # --- BVH (src/bvh/*.rs) ---
    def morton(self, p, group=0) -> int:
        a = np.ascontiguousarray(p, dtype=np.float32)
        return self.lib.orc_morton(a.ctypes.data, group)

    def scene(self, prims):
        prims = np.ascontiguousarray(prims, dtype=np.float32)
        out = np.zeros(8, dtype=np.float32)
        self.lib.orc_scene(prims.ctypes.data, len(prims), out.ctypes.data)
        return out

    def codes(self, prims):
        prims = np.ascontiguousarray(prims, dtype=np.float32)
        out = np.zeros(len(prims), dtype=np.uint32)
        self.lib.orc_codes(prims.ctypes.data, len(prims), out.ctypes.data)
        return out

    def sort_codes(self, codes):
        codes = np.ascontiguousarray(codes, dtype=np.uint32)
        order = np.zeros(len(codes), dtype=np.uint32)
        sorted_ = np.zeros(len(codes), dtype=np.uint32)
        self.lib.orc_sort_codes(codes.ctypes.data, len(codes), order.ctypes.data, sorted_.ctypes.data)
        return order, sorted_

    def radix_model(self, codes):
        codes = np.ascontiguousarray(codes, dtype=np.uint32)
        order = np.zeros(len(codes), dtype=np.uint32)
        sorted_ = np.zeros(len(codes), dtype=np.uint32)
        self.lib.orc_radix_model(codes.ctypes.data, len(codes), order.ctypes.data, sorted_.ctypes.data)
        return order, sorted_

    def links(self, sorted_codes):
        s = np.ascontiguousarray(sorted_codes, dtype=np.uint32)
        out = np.zeros((max(0, len(s) - 1), 4), dtype=np.uint32)
        self.lib.orc_links(s.ctypes.data, len(s), out.ctypes.data)
        return out

    def build(self, prims, leaf=4):
        prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 8)
        n = len(prims)
        nodes = np.zeros((max(0, 2 * n - 1), 8), dtype=np.float32)
        order = np.zeros(n, dtype=np.uint32)
        depth = u32()
        self.lib.orc_build(prims.ctypes.data, n, leaf, nodes.ctypes.data, order.ctypes.data, C.byref(depth))
        return nodes, order, depth.value

    def build_compact(self, prims, leaf=4):
        prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 8)
        n = len(prims)
        nodes = np.zeros((max(1, 2 * n - 1), 8), dtype=np.float32)
        order = np.zeros(n, dtype=np.uint32)
        depth = u32()
        m = self.lib.orc_build_compact(prims.ctypes.data, n, leaf, nodes.ctypes.data, order.ctypes.data, C.byref(depth))
        return nodes[:m].copy(), order, depth.value

    def build_sah(self, prims, leaf=4):
        """src/bvh/sah.rs Bvh::build_sah: (nodes, order, depth)."""
        prims = np.ascontiguousarray(prims, dtype=np.float32).reshape(-1, 8)
        n = len(prims)
        nodes = np.zeros((max(1, 2 * n - 1), 8), dtype=np.float32)
        order = np.zeros(n, dtype=np.uint32)
        depth = u32()
        m = self.lib.orc_build_sah(prims.ctypes.data, n, leaf, nodes.ctypes.data, order.ctypes.data, C.byref(depth))
        return nodes[:m].copy(), order, depth.value

    def refit(self, nodes, order, prims):
        nodes = np.ascontiguousarray(nodes, dtype=np.float32).copy()
        order = np.ascontiguousarray(order, dtype=np.uint32)
        prims = np.ascontiguousarray(prims, dtype=np.float32)
        self.lib.orc_refit(nodes.ctypes.data, len(nodes), order.ctypes.data, prims.ctypes.data)
        return nodes

    def compact(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.float32).copy()
        m = self.lib.orc_compact(nodes.ctypes.data, len(nodes))
        return nodes[:m].copy()

    def reachable(self, nodes):
        nodes = np.ascontiguousarray(nodes, dtype=np.float32)
        out = np.zeros(len(nodes), dtype=np.uint32)
        m = self.lib.orc_reachable(nodes.ctypes.data, len(nodes), out.ctypes.data)
        return out[:m].copy()

    # --- Skin (src/kernel/skin.rs:70-90) ---
    def skin(self, rest, offsets, pairs, bones, min_weight=1e-4):
        rest = np.ascontiguousarray(rest, dtype=np.float32)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        pairs = np.ascontiguousarray(pairs)
        bones = np.ascontiguousarray(bones, dtype=np.float32)
        out = np.zeros_like(rest)
        self.lib.orc_skin(rest.ctypes.data, offsets.ctypes.data, pairs.ctypes.data, bones.ctypes.data,
                          f32(min_weight), len(rest), out.ctypes.data)
        return out

    # --- the watertight triangle test (tri.rs:51-114) and the shared math ---
    def tri_hit(self, a, b, c, o, d):
        """(t, u, v) of the watertight test, or None for a miss."""
        args = [np.ascontiguousarray(v, dtype=np.float32) for v in (a, b, c, o, d)]
        out = np.zeros(3, np.float32)
        hit = self.lib.orc_tri_hit(*[v.ctypes.data for v in args], out.ctypes.data)
        return (float(out[0]), float(out[1]), float(out[2])) if hit else None

    MATH = {"exp2": 0, "log2": 1, "sin": 2, "cos": 3, "pow": 4, "exp": 5}

    def math(self, fn: str, x, y=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, dtype=np.float32)
        out = np.zeros_like(x)
        self.lib.orc_math(self.MATH[fn], x.ctypes.data, y.ctypes.data, out.ctypes.data, len(x))
        return out

    # --- Denoise (denoise.wgsl) ---
    def denoise(self, px, w, h, strength=(64.0, 8.0, 40.0, 7.0), view=(0.0, 0.0, 1.0, 0.0), keep=False):
        px = np.ascontiguousarray(px, dtype=np.uint32).copy()
        s = (f32 * 4)(*strength)
        v = (f32 * 4)(*view)
        self.lib.orc_denoise(px.ctypes.data, w, h, s, v, 1 if keep else 0)
        return px


def _scene_args(scene):
    v = np.ascontiguousarray(scene.verts, dtype=np.float32)
    f = np.ascontiguousarray(scene.faces, dtype=np.uint32)
    m = np.ascontiguousarray(scene.mats, dtype=np.float32)
    return v, f, m


class TraceOracle:
    """The tracer restatement (oracle/trace.cpp) for a `scenes.Scene`."""

    def __init__(self, orc: "Oracle", scene, leaf: int = 4, sah: bool = False):
        self.lib = orc.lib
        self.v, self.f, self.m = _scene_args(scene)
        nrm = getattr(scene, "normals", None)
        self.nrm = None if nrm is None else np.ascontiguousarray(nrm, dtype=np.float32)
        self.leaf = leaf
        meshes = getattr(scene, "meshes", None)
        nptr = None if self.nrm is None else self.nrm.ctypes.data
        if meshes is not None:
            self.meshes = np.ascontiguousarray(meshes, dtype=np.uint32)
            self.insts = np.ascontiguousarray(scene.insts)
            self.handle = self.lib.orc_scene_new_instanced(
                self.v.ctypes.data, self.f.ctypes.data, len(self.f), self.m.ctypes.data, nptr, leaf,
                self.meshes.ctypes.data, len(self.meshes), self.insts.ctypes.data, len(self.insts))
        else:
            new = self.lib.orc_scene_new_sah if sah else self.lib.orc_scene_new
            self.handle = new(self.v.ctypes.data, self.f.ctypes.data, len(self.f), self.m.ctypes.data, nptr, leaf)

    def reinstance(self, insts):
        """Tracer::reinstance: new matrices for the same instances."""
        self.insts = np.ascontiguousarray(insts)
        self.lib.orc_scene_reinstance(self.handle, self.insts.ctypes.data, len(self.insts))

    def __del__(self):
        try:
            self.lib.orc_scene_free(self.handle)
        except Exception:
            pass

    def trace(self, cam, first: int, spp: int, px=None, rows=None):
        w, h = int(cam["w"][0]), int(cam["h"][0])
        if px is None:
            px = np.zeros(34 * w * h + 1, dtype=np.uint32)
        rays = u64()
        r0, nr = (0, 0) if rows is None else rows
        self.lib.orc_scene_trace(self.handle, cam.ctypes.data, first, spp, px.ctypes.data, C.byref(rays), r0, nr)
        return px, rays.value

    def trace_walk(self, cam, first: int, spp: int, rows=None):
        """trace, also returning the walks' (inner-node visits, triangle tests)."""
        w, h = int(cam["w"][0]), int(cam["h"][0])
        px = np.zeros(34 * w * h + 1, dtype=np.uint32)
        rays = u64()
        walk = np.zeros(2, np.uint64)
        r0, nr = (0, 0) if rows is None else rows
        self.lib.orc_scene_trace_walk(self.handle, cam.ctypes.data, first, spp, px.ctypes.data, C.byref(rays), r0, nr,
                                      walk.ctypes.data)
        return px, rays.value, int(walk[0]), int(walk[1])

    def primary(self, cam, frame: int, with_inst: bool = False):
        """Primary hit (face id, t) per pixel; with_inst: also the instance."""
        n = int(cam["w"][0]) * int(cam["h"][0])
        ids = np.zeros(n, np.uint32)
        ts = np.zeros(n, np.float32)
        inst = np.zeros(n, np.uint32)
        self.lib.orc_scene_primary(self.handle, cam.ctypes.data, frame, ids.ctypes.data, ts.ctypes.data,
                                   inst.ctypes.data)
        return (ids, ts, inst) if with_inst else (ids, ts)

    def trace_rays(self, rays, any_hit=False):
        rays = np.ascontiguousarray(rays, dtype=np.float32)
        n = len(rays)
        hits = np.zeros((n, 4), np.float32)
        self.lib.orc_scene_trace_rays(self.handle, rays.ctypes.data, n, hits.ctypes.data, 1 if any_hit else 0)
        return hits


def build() -> Path:
    if _stale():
        subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIB


_cached = None


def load() -> Oracle:
    global _cached
    if _cached is None:
        build()
        lib = C.CDLL(str(LIB))
        for name, (res, args) in SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _cached = Oracle(lib)
    return _cached


def nn():
    """The FP64 network oracle (oracle/nn.py) as a module."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("oracle_nn", ORACLE_DIR / "nn.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod
