"""``Tracer`` and ``Camera``: phiray's Rendered-mode tracer over the C ABI.

Reference: src/trace/mod.rs (Tracer), build.rs (Tracer::new), sample.rs
(sample, sample_in, time), read.rs (readbacks, denoise), pose.rs (repose),
camera.rs (Camera). ``Camera`` is the reference's uniform byte for byte
(5,776 bytes) as a numpy record, so the same bytes a Rust caller holds go
through the ABI unchanged.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .gpu import Gpu, devptr

PX_LEN = 34

LIGHT = np.dtype(
    [
        ("pos", "<f4", 3),
        ("kind", "<u4"),
        ("color", "<f4", 3),
        ("size", "<f4"),
        ("dir", "<f4", 3),
        ("cone", "<f4"),
        ("right", "<f4", 3),
        ("size_y", "<f4"),
        ("shape", "<u4"),
        ("blend", "<f4"),
        ("spot_scale", "<f4", 2),
    ]
)

CAMERA = np.dtype(
    [
        ("n", "<u4"), ("groups_x", "<u4"), ("w", "<u4"), ("h", "<u4"),
        ("right", "<f4", 3), ("persp", "<u4"),
        ("up", "<f4", 3), ("scale", "<f4"),
        ("back", "<f4", 3), ("units", "<f4"),
        ("pivot", "<f4", 3), ("aspect", "<f4"),
        ("sun", "<f4", 3), ("dist", "<f4"),
        ("sky", "<f4", 4),
        ("pan", "<f4", 2), ("ao", "<f4"), ("eps", "<f4"),
        ("frame", "<u4"), ("grid", "<f4"), ("count", "<u4"), ("glow", "<u4"),
        ("grid_color", "<f4", 4), ("env", "<f4", 4), ("split", "<u4", 4), ("view", "<f4", 4),
        ("envmap", "<u4"), ("env_rot", "<f4"), ("bounces", "<u4"), ("env_cdf", "<u4"),
        ("aperture", "<f4"), ("focus", "<f4"), ("blades", "<u4"), ("blade_spin", "<f4"),
        ("aperture_ratio", "<f4"), ("env_hidden", "<u4"), ("see_through", "<f4"), ("grid_hide", "<u4"),
        ("tile", "<u4", 4), ("film", "<u4", 4), ("preview", "<u4", 4), ("slice", "<u4", 4),
        ("insts", "<u4", 4), ("vis", "<u4", 4), ("taa", "<f4", 4), ("fx", "<f4", 4), ("outline", "<f4", 4),
        ("shade", "<u4", 4), ("single", "<f4", 4), ("cavity", "<f4", 4), ("ssao", "<u4", 4),
        ("shadow", "<f4", 4), ("shadow_fade", "<f4", 4), ("matcap", "<u4", 4), ("dof", "<f4", 4),
        ("outline_fx", "<f4", 4), ("outline_pick", "<f4", 4), ("outline_active", "<f4", 4),
        ("outline_move", "<f4", 4), ("adapt", "<f4", 4), ("limit", "<f4", 4), ("depth", "<u4", 4),
        ("integrator", "<f4", 4),
        ("lights", LIGHT, 64),
    ]
)
assert CAMERA.itemsize == 5776


def camera(scene) -> np.ndarray:
    """A Camera record for a `scenes.Scene`: its view, lights, world colour,
    diffuse bounces; Standard view transform, pinhole, no clamp."""
    c = np.zeros(1, dtype=CAMERA)
    v = scene.view
    c["right"], c["up"], c["back"], c["pivot"] = v.right, v.up, v.back, v.pivot
    c["persp"] = 1
    c["dist"], c["scale"], c["units"] = v.dist, v.scale, v.units
    c["aspect"] = scene.width / scene.height
    c["env"][0, :3] = scene.env
    c["view"] = (0.0, 0.0, 1.0, 0.0)
    c["bounces"] = scene.bounces
    c["sun"] = getattr(scene, "sun", (0.0, 1.0, 0.0))
    L = len(scene.lights)
    c["count"] = L
    raw = c["lights"].view(np.float32).reshape(1, 64, 20)
    raw[0, :L] = scene.lights
    return c


class _Scene(C.Structure):
    _fields_ = [
        ("verts", C.c_void_p),
        ("normals", C.c_void_p),
        ("faces", C.c_void_p),
        ("mats", C.c_void_p),
        ("nverts", C.c_uint32),
        ("nfaces", C.c_uint32),
        ("nmats", C.c_uint32),
        ("leaf", C.c_uint32),
    ]


def _counts(px: np.ndarray, n: int) -> np.ndarray:
    """Samples each pixel took (read.rs `counts`: the count plane, at least 1)."""
    return np.maximum(px[31 * n:32 * n], 1).astype(np.float32)


def radiance_of(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """``Tracer::radiance`` of a host px image: sums / samples taken."""
    n = w * h
    lin = px.view(np.float32)[n:4 * n].reshape(n, 3)
    return (lin / _counts(px, n)[:, None]).reshape(h, w, 3)


def lit_of(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """The linear mean over the samples that met something (util.wgsl's emit:
    l / max(k - gone, 1)), the value the view transform is applied to."""
    n = w * h
    f = px.view(np.float32)
    k = px[31 * n:32 * n].astype(np.float32)
    return (f[n:4 * n].reshape(n, 3) / np.maximum(k - f[33 * n:34 * n], 1.0)[:, None]).reshape(h, w, 3)


def display_of(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """``Tracer::display``: the shown plane (no division: it is a mean)."""
    n = w * h
    return px.view(np.float32)[4 * n:7 * n].reshape(h, w, 3).copy()


def albedo_of(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """``Tracer::albedo``: the albedo guide sums / samples taken."""
    n = w * h
    return (px.view(np.float32)[7 * n:10 * n].reshape(n, 3) / _counts(px, n)[:, None]).reshape(h, w, 3)


def normal_of(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """``Tracer::normal``: the normal guide mean, re-normalised (0 where its
    length is 1e-9 or less)."""
    n = w * h
    v = px.view(np.float32)[10 * n:13 * n].reshape(n, 3) / _counts(px, n)[:, None]
    ln = np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])
    out = np.where((ln > 1e-9)[:, None], v / np.where(ln > 1e-9, ln, 1.0)[:, None], 0.0)
    return out.astype(np.float32).reshape(h, w, 3)


def depth_of(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """``Tracer::depth``: the depth guide mean, 1e10 where it is <= 0 (a
    miss records -1 a sample)."""
    n = w * h
    mean = px.view(np.float32)[13 * n:14 * n] / _counts(px, n)
    return np.where(mean <= 0.0, np.float32(1.0e10), mean).astype(np.float32).reshape(h, w)


class Tracer:
    """The Rendered-mode path tracer (phiray ``Tracer``)."""

    def __init__(self, gpu: Gpu, verts: np.ndarray, faces: np.ndarray, mats: np.ndarray, normals=None, leaf: int = 4,
                 meshes=None, insts=None):
        """Tracer::new. With `meshes` ((M, 2) face ranges) and `insts`
        (scenes.INSTANCE records): a scene of meshes placed by instances."""
        self.gpu = gpu
        self._host = [
            np.ascontiguousarray(verts, dtype=np.float32),
            np.ascontiguousarray(faces, dtype=np.uint32),
            np.ascontiguousarray(mats, dtype=np.float32),
            None if normals is None else np.ascontiguousarray(normals, dtype=np.float32),
        ]
        v, f, m, nrm = self._host
        sc = _Scene(
            v.ctypes.data, nrm.ctypes.data if nrm is not None else None, f.ctypes.data, m.ctypes.data,
            len(v), len(f), len(m), leaf,
        )
        h = C.c_void_p()
        if meshes is None:
            N.check(N.lib().phx_tracer_create(gpu.handle, C.byref(sc), C.byref(h)))
        else:
            ms = np.ascontiguousarray(meshes, dtype=np.uint32).reshape(-1, 2)
            ins = np.ascontiguousarray(insts)
            N.check(N.lib().phx_tracer_create_instanced(gpu.handle, C.byref(sc), ms.ctypes.data, len(ms),
                                                        ins.ctypes.data, len(ins), C.byref(h)))
        self.handle = h
        self.w = self.h = 0
        gpu.adopt(self)

    @classmethod
    def of(cls, gpu: Gpu, scene, **kw) -> "Tracer":
        kw.setdefault("normals", getattr(scene, "normals", None))
        if getattr(scene, "meshes", None) is not None:
            kw.setdefault("meshes", scene.meshes)
            kw.setdefault("insts", scene.insts)
        return cls(gpu, scene.verts, scene.faces, scene.mats, **kw)

    TREE_LBVH = 0
    TREE_SAH = 1

    def set_tree(self, tree: int) -> None:
        """Walk the device LBVH (Tracer.TREE_LBVH) or the binned SAH tree
        phiray's tracer builds (Tracer.TREE_SAH); rebuilds now."""
        N.check(N.lib().phx_tracer_set_tree(self.handle, tree))

    def autotune_tree(self, cam: np.ndarray, w: int, h: int, spp: int, frames: int) -> tuple[int, list[float]]:
        """Times each tree's build and an spp-sample trace; keeps the tree with
        the lower build + frames x trace. (chosen, [lbvh build, lbvh trace,
        sah build, sah trace] ms)."""
        chosen = C.c_uint32()
        ms = (C.c_float * 4)()
        N.check(N.lib().phx_tracer_autotune_tree(self.handle, cam.ctypes.data, w, h, spp, frames, C.byref(chosen), ms))
        self.w, self.h = w, h
        return chosen.value, list(ms)

    def reinstance(self, insts) -> None:
        """``Tracer::reinstance``: the same instances placed anew (the top
        tree is rebuilt on the device)."""
        ins = np.ascontiguousarray(insts)
        N.check(N.lib().phx_tracer_reinstance(self.handle, ins.ctypes.data, len(ins)))

    MEGAKERNEL = 0
    STATE_MACHINE = 1
    STATE_MACHINE_6 = 2
    STATE_MACHINE_8 = 3
    MEGAKERNEL_3 = 4
    MEGAKERNEL_2 = 5
    MEGAKERNEL_SYNC = 6
    MEGAKERNEL_2_SYNC = 7
    MEGAKERNEL_5 = 8
    MEGAKERNEL_6 = 9
    MEGAKERNEL_6_SYNC = 10
    MEGAKERNEL_8 = 11
    MEGAKERNEL_8_SYNC = 12
    MEGAKERNEL_10_SYNC = 13
    MEGAKERNEL_12_SYNC = 14
    MEGAKERNEL_16_SYNC = 15
    WAVEFRONT = 16
    MEGAKERNEL_REG = 17
    MEGAKERNEL_8_SYNC_REG = 18
    MEGAKERNEL_16_SYNC_REG = 19
    KERNELS = 20

    def autotune(self, cam: np.ndarray, w: int, h: int, spp: int = 1) -> tuple[int, list[float]]:
        """Times every render kernel on this scene; keeps and returns the fastest."""
        chosen = C.c_uint32()
        ms = (C.c_float * self.KERNELS)()
        N.check(N.lib().phx_tracer_autotune(self.handle, cam.ctypes.data, w, h, spp, C.byref(chosen), ms))
        self.w, self.h = w, h
        return chosen.value, list(ms)

    def set_kernel(self, kind: int) -> None:
        """Render kernel: Tracer.MEGAKERNEL or Tracer.STATE_MACHINE (same image)."""
        N.check(N.lib().phx_tracer_set_kernel(self.handle, kind))

    STACK_LOCAL = 0
    STACK_SHARED = 1
    STACK_REGISTER = 2

    def set_stack(self, place: int) -> None:
        """Where thread-per-ray walks keep their stack: STACK_LOCAL,
        STACK_SHARED (True also means shared) or STACK_REGISTER."""
        N.check(N.lib().phx_tracer_set_stack(self.handle, int(place)))

    WALK_THREAD = 0
    WALK_FETCH = 1
    WALK_SORTED = 2
    WALK_WIDE = 3
    WALK_WIDE_THREAD = 4

    def set_walk(self, mode: int) -> None:
        """Ray-buffer walks: Tracer.WALK_THREAD (a thread per ray),
        Tracer.WALK_FETCH (persistent warps refilling idle lanes),
        Tracer.WALK_SORTED (the same over rays sorted by direction octant and
        origin), all with the same hits; or Tracer.WALK_WIDE (persistent
        warps over a 4-wide tree collapsed from the binary one: the same
        closest t, the face at a tie may differ) and Tracer.WALK_WIDE_THREAD
        (the same walk, a thread per ray)."""
        N.check(N.lib().phx_tracer_set_walk(self.handle, mode))

    def set_samples(self, n: int) -> None:
        N.check(N.lib().phx_tracer_set_samples(self.handle, n))

    def set_adaptive(self, adapt) -> None:
        """``Tracer::set_adaptive``: [threshold, min samples, step, on]."""
        a = (C.c_float * 4)(*[float(v) for v in adapt])
        N.check(N.lib().phx_tracer_set_adaptive(self.handle, a))

    def unconverged(self, timeout_ms: int = 0) -> int | None:
        """``Tracer::unconverged``: pixels not settled after the last sample,
        or None when adaptive sampling is off."""
        c = C.c_uint32()
        rc = N.lib().phx_tracer_unconverged(self.handle, C.byref(c), timeout_ms)
        if rc == N.PHX_ERR_INVALID:
            return None
        N.check(rc)
        return c.value

    def sample(self, cam: np.ndarray, w: int, h: int, slices: int = 1, cancel=None) -> tuple[int, bool]:
        """``Tracer::sample`` / ``sample_in``: (frame, done)."""
        frame, done = C.c_uint32(), C.c_int32()
        N.check(N.lib().phx_tracer_sample(self.handle, cam.ctypes.data, w, h, slices, cancel, C.byref(frame), C.byref(done)))
        self.w, self.h = w, h
        return frame.value, bool(done.value)

    def trace(self, cam: np.ndarray, w: int, h: int, first: int, spp: int) -> None:
        """Frames [first, first + spp) in one launch (stream-ordered)."""
        N.check(N.lib().phx_tracer_trace(self.handle, cam.ctypes.data, w, h, first, spp))
        self.w, self.h = w, h

    def read(self, offset: int, count: int, timeout_ms: int = 0) -> np.ndarray:
        out = np.empty(count, dtype=np.uint32)
        N.check(N.lib().phx_tracer_read(self.handle, offset, out.ctypes.data, count, timeout_ms))
        return out

    def image(self) -> np.ndarray:
        """The whole px buffer (34 w h + 1 words)."""
        return self.read(0, PX_LEN * self.w * self.h + 1)

    def pixels(self) -> np.ndarray:
        """``Tracer::pixels``: packed RGBA8 (n,) uint32."""
        return self.read(0, self.w * self.h)

    def radiance(self) -> np.ndarray:
        """``Tracer::radiance`` (read.rs:240-251): the linear sums over the
        samples each pixel took, (h, w, 3)."""
        return radiance_of(self.image(), self.w, self.h)

    def lit(self) -> np.ndarray:
        """The linear mean over the samples that met something (what emit
        hands the view transform), (h, w, 3)."""
        return lit_of(self.image(), self.w, self.h)

    def display(self) -> np.ndarray:
        """``Tracer::display`` (read.rs:253-262): the shown values, (h, w, 3)."""
        return display_of(self.image(), self.w, self.h)

    def albedo(self) -> np.ndarray:
        """``Tracer::albedo`` (read.rs:264-271): the diffuse-colour guide, (h, w, 3)."""
        return albedo_of(self.image(), self.w, self.h)

    def normal(self) -> np.ndarray:
        """``Tracer::normal`` (read.rs:273-285): the normal guide made unit, (h, w, 3)."""
        return normal_of(self.image(), self.w, self.h)

    def depth(self) -> np.ndarray:
        """``Tracer::depth`` (read.rs:287-309): distance to the first hit, 1e10
        where nothing was met, (h, w)."""
        return depth_of(self.image(), self.w, self.h)

    def show(self, linear) -> None:
        """``Tracer::show`` (read.rs:182-216): a composited linear image shown
        through the tracer's view transform (phx_tracer_show)."""
        lin = np.ascontiguousarray(np.asarray(linear, dtype=np.float32).reshape(-1, 3))
        N.check(N.lib().phx_tracer_show(self.handle, lin.ctypes.data, lin.shape[0]))

    def device_verts(self) -> tuple[int, int]:
        """Device pointer and count of the tracer's own vertex array."""
        p, nv = C.c_void_p(), C.c_uint32()
        N.check(N.lib().phx_tracer_verts(self.handle, C.byref(p), C.byref(nv)))
        return p.value or 0, nv.value

    def device_image(self) -> tuple[int, int]:
        p, words = C.c_void_p(), C.c_uint64()
        N.check(N.lib().phx_tracer_image(self.handle, C.byref(p), C.byref(words)))
        return p.value or 0, words.value

    def snapshot(self, snap) -> None:
        """The image's sums and met-sample counts now, into a device array of
        w h x 4 floats (the learned denoiser's `half` input)."""
        N.check(N.lib().phx_tracer_snapshot(self.handle, devptr(snap)))

    def denoise(self, keep: bool = False) -> None:
        N.check(N.lib().phx_tracer_denoise(self.handle, 1 if keep else 0))

    def time(self) -> tuple[float, int]:
        """``Tracer::time``: (GPU ms of the last call, rays traced)."""
        ms, rays = C.c_float(), C.c_uint64()
        N.check(N.lib().phx_tracer_time(self.handle, C.byref(ms), C.byref(rays)))
        return ms.value, rays.value

    def repose_device(self, verts, rebuild: bool = False) -> None:
        N.check(N.lib().phx_tracer_repose_device(self.handle, devptr(verts), 1 if rebuild else 0))

    def primary(self, cam: np.ndarray, w: int, h: int, frame: int, ids, ts) -> None:
        N.check(N.lib().phx_tracer_primary(self.handle, cam.ctypes.data, w, h, frame, devptr(ids), devptr(ts)))

    def secondary_rays(self, cam: np.ndarray, w: int, h: int, frame: int, rays) -> None:
        N.check(N.lib().phx_tracer_secondary_rays(self.handle, cam.ctypes.data, w, h, frame, devptr(rays)))

    def trace_rays(self, rays, n: int, hits, any_hit: bool = False) -> None:
        N.check(N.lib().phx_trace_rays(self.handle, devptr(rays), n, devptr(hits), 1 if any_hit else 0))

    def trace_rays_stats(self, rays, n: int, hits, any_hit: bool = False) -> tuple[int, int, int]:
        """(rays, inner-node steps, triangle tests) of the same walks."""
        c = (C.c_uint64 * 3)()
        N.check(N.lib().phx_trace_rays_stats(self.handle, devptr(rays), n, devptr(hits), 1 if any_hit else 0, c))
        return c[0], c[1], c[2]

    def trace_stats(self, cam: np.ndarray, w: int, h: int, first: int, spp: int) -> tuple[int, int, int]:
        """``trace`` counted: (rays, inner-node steps, triangle tests)."""
        c = (C.c_uint64 * 3)()
        N.check(N.lib().phx_tracer_trace_stats(self.handle, cam.ctypes.data, w, h, first, spp, c))
        self.w, self.h = w, h
        return c[0], c[1], c[2]

    def close(self) -> None:
        if self.handle:
            N.lib().phx_tracer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
