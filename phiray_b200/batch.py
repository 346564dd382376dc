"""Batched serving over the C ABI (phx_batch_*): many tracers' frames in one
persistent launch, the autotuner over launch forms, and a whole serving
frame (rebuild or refit per scene, trace, learned denoise with the a-trous
fallback) captured once as a CUDA graph and replayed."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .gpu import Gpu

PERSISTENT = 0
PER_SCENE = 1
PERSISTENT_DENSE = 2
STACK_LOCAL = 0
STACK_SHARED = 1

CONFIG_NAMES = [f"persistent/{t}/{'shared' if s else 'local'}" for t in (64, 128, 256) for s in (0, 1)] + [
    "per-scene/megakernel", "per-scene/state-machine", "persistent-dense/128/local", "persistent-dense/256/local",
    "per-scene/megakernel-16-sync"]


class Batch:
    def __init__(self, gpu: Gpu):
        self.gpu = gpu
        h = C.c_void_p()
        N.check(N.lib().phx_batch_create(gpu.handle, C.byref(h)))
        self.handle = h
        self.jobs = []
        gpu.adopt(self)

    def add(self, tracer, cam: np.ndarray, w: int, h: int, first: int, spp: int) -> int:
        idx = C.c_uint32()
        N.check(N.lib().phx_batch_add(self.handle, tracer.handle, cam.ctypes.data, w, h, first, spp, C.byref(idx)))
        tracer.w, tracer.h = w, h
        self.jobs.append(tracer)
        return idx.value

    def clear(self) -> None:
        N.check(N.lib().phx_batch_clear(self.handle))
        self.jobs = []

    def set_config(self, kind: int = PERSISTENT, threads: int = 128, stack: int = STACK_LOCAL) -> None:
        N.check(N.lib().phx_batch_set_config(self.handle, kind, threads, stack))

    def trace(self) -> None:
        N.check(N.lib().phx_batch_trace(self.handle))

    def autotune(self) -> tuple[tuple[int, int, int], dict]:
        kind, threads, stack, n = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        ms = (C.c_float * 16)()
        N.check(N.lib().phx_batch_autotune(self.handle, C.byref(kind), C.byref(threads), C.byref(stack), ms,
                                           C.byref(n)))
        return (kind.value, threads.value, stack.value), {CONFIG_NAMES[i]: ms[i] for i in range(n.value)}

    def capture(self, net=None, threshold: float = 0.1) -> None:
        N.check(N.lib().phx_batch_capture(self.handle, net.handle if net is not None else None, threshold))

    def replay(self, modes) -> None:
        m = np.ascontiguousarray(modes, dtype=np.uint32)
        N.check(N.lib().phx_batch_replay(self.handle, m.ctypes.data))

    def results(self) -> tuple[np.ndarray, np.ndarray]:
        """(latency ns per job after the frame start, rays per job)."""
        n = len(self.jobs)
        lat = np.zeros(n, np.uint64)
        rays = np.zeros(n, np.uint64)
        N.check(N.lib().phx_batch_results(self.handle, lat.ctypes.data, rays.ctypes.data))
        return lat, rays

    def close(self) -> None:
        if self.handle:
            N.lib().phx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
