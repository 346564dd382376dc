"""Host-side mirror of phiray's runtime types over the C ABI.

``Gpu`` (src/gpu/mod.rs:84-331), ``GpuArray`` (src/gpu/array.rs) and
``Pass`` (src/gpu/pass.rs) keep the reference's method names and meanings:
``GpuArray.write`` returns True when it reallocated (rebind needed),
``read`` is a bounded wait, ``Pass.add`` fills the params' leading
``[n, groups_x]`` words, ``Pass.run`` replays every step (here as one CUDA
graph launch).
"""

from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _native as N


def devptr(x) -> int:
    """Device address of a GpuArray, a torch CUDA tensor, or an int."""
    if isinstance(x, GpuArray):
        return x.ptr
    if isinstance(x, int):
        return x
    if x is None:
        return 0
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise ValueError("expected device memory, got a CPU tensor")
        return int(x.data_ptr())
    raise TypeError(f"not a device array: {type(x)}")


def _host(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    return a


class Gpu:
    """One CUDA device and its stream (phiray ``Gpu``)."""

    def __init__(self, ordinal: int = 0):
        h = C.c_void_p()
        N.check(N.lib().phx_ctx_create(ordinal, C.byref(h)))
        self.handle = h
        self.ordinal = ordinal
        self._children = weakref.WeakSet()

    def adopt(self, obj) -> None:
        """Track an object made on this context; close() releases it first."""
        self._children.add(obj)

    @staticmethod
    def count() -> int:
        return N.lib().phx_device_count()

    def wait(self, timeout_ms: int = 0) -> None:
        """``Gpu::wait_for``: bounded drain; raises PhxError(TIMEOUT)."""
        N.check(N.lib().phx_ctx_wait(self.handle, timeout_ms))

    @property
    def stream(self) -> int:
        return N.lib().phx_ctx_stream(self.handle) or 0

    def set_stream(self, stream: int | None) -> None:
        N.check(N.lib().phx_ctx_set_stream(self.handle, stream or None))

    def close(self) -> None:
        if self.handle:
            for child in list(self._children):
                child.close()
            N.lib().phx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuArray:
    """One device buffer (phiray ``GpuArray<T>``)."""

    def __init__(self, gpu: Gpu, nbytes: int, _wrap: int | None = None):
        h = C.c_void_p()
        if _wrap is None:
            N.check(N.lib().phx_buf_alloc(gpu.handle, int(nbytes), C.byref(h)))
        else:
            N.check(N.lib().phx_buf_wrap(gpu.handle, _wrap, int(nbytes), C.byref(h)))
        self.gpu = gpu
        self.handle = h
        gpu.adopt(self)

    @classmethod
    def zeroed(cls, gpu: Gpu, nbytes: int) -> "GpuArray":
        return cls(gpu, nbytes)

    @classmethod
    def from_(cls, gpu: Gpu, data: np.ndarray) -> "GpuArray":
        data = _host(data)
        a = cls(gpu, data.nbytes)
        a.write_at(0, data)
        return a

    @classmethod
    def wrap(cls, gpu: Gpu, tensor) -> "GpuArray":
        """Borrow a torch CUDA tensor's memory (not freed here)."""
        return cls(gpu, tensor.numel() * tensor.element_size(), _wrap=devptr(tensor))

    @property
    def ptr(self) -> int:
        return N.lib().phx_buf_ptr(self.handle) or 0

    @property
    def nbytes(self) -> int:
        return N.lib().phx_buf_size(self.handle)

    def write_at(self, offset: int, data: np.ndarray) -> None:
        data = _host(data)
        N.check(N.lib().phx_buf_write(self.handle, offset, data.ctypes.data, data.nbytes))

    def write(self, data: np.ndarray) -> bool:
        """Replace the contents; True when the buffer was reallocated."""
        data = _host(data)
        re = C.c_int32(0)
        N.check(N.lib().phx_buf_assign(self.handle, data.ctypes.data, data.nbytes, C.byref(re)))
        return bool(re.value)

    def read(self, dtype=np.uint8, count: int | None = None, offset: int = 0, timeout_ms: int = 0) -> np.ndarray:
        dtype = np.dtype(dtype)
        if count is None:
            count = (self.nbytes - offset) // dtype.itemsize
        out = np.empty(count, dtype=dtype)
        N.check(N.lib().phx_buf_read(self.handle, offset, out.ctypes.data, out.nbytes, timeout_ms))
        return out

    def free(self) -> None:
        if self.handle:
            N.lib().phx_buf_free(self.handle)
            self.handle = None

    close = free

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# Param blobs of the kernels a Pass can record (include/phiray_cuda.h).
SKIN_PARAM = np.dtype([("n", "<u4"), ("groups_x", "<u4"), ("min", "<f4"), ("pad", "<u4")])
DENOISE_PARAM = np.dtype(
    [
        ("n", "<u4"),
        ("groups_x", "<u4"),
        ("w", "<u4"),
        ("h", "<u4"),
        ("step", "<u4"),
        ("round", "<u4"),
        ("last", "<u4"),
        ("keep", "<u4"),
        ("strength", "<f4", 4),
        ("view", "<f4", 4),
    ]
)
MORTON_PARAM = np.dtype(
    [("n", "<u4"), ("groups_x", "<u4"), ("pad0", "<u4", 2), ("lo", "<f4", 3), ("pad1", "<f4"), ("inv", "<f4", 3), ("pad2", "<f4")]
)
KARRAS_PARAM = np.dtype([("n", "<u4"), ("groups_x", "<u4"), ("leaves", "<u4"), ("pad", "<u4")])
REFIT_PARAM = np.dtype([("n", "<u4"), ("groups_x", "<u4"), ("pad", "<u4", 2)])


class Kernel:
    """A recordable kernel: its id, param layout and binding count
    (phiray ``Kernel``: NAME, Param, BIND_LIST)."""

    def __init__(self, name: str, kid: int, param: np.dtype, nbufs: int):
        self.NAME, self.id, self.Param, self.nbufs = name, kid, param, nbufs

    def params(self, **fields) -> np.ndarray:
        p = np.zeros(1, dtype=self.Param)
        for k, v in fields.items():
            p[k] = v
        return p


Skin = Kernel("skin", N.KERNEL_SKIN, SKIN_PARAM, 5)
Denoise = Kernel("denoise", N.KERNEL_DENOISE, DENOISE_PARAM, 1)
Morton = Kernel("bvh.morton", N.KERNEL_MORTON, MORTON_PARAM, 2)
Karras = Kernel("bvh.karras", N.KERNEL_KARRAS, KARRAS_PARAM, 2)
Refit = Kernel("bvh.refit", N.KERNEL_REFIT, REFIT_PARAM, 4)


class Pass:
    """Recorded launches replayed together (phiray ``Pass``)."""

    def __init__(self, gpu: Gpu):
        h = C.c_void_p()
        N.check(N.lib().phx_pass_create(gpu.handle, C.byref(h)))
        self.gpu = gpu
        self.handle = h
        self._keep: list = []
        gpu.adopt(self)

    def add(self, kernel: Kernel, n: int, params: np.ndarray, buffers: list[GpuArray]) -> int:
        return self.add_over(kernel, n, n, params, buffers)

    def add_over(self, kernel: Kernel, n: int, items: int, params: np.ndarray, buffers: list[GpuArray]) -> int:
        params = np.ascontiguousarray(params)
        arr = (C.c_void_p * max(1, len(buffers)))(*[b.handle.value for b in buffers])
        step = C.c_uint32(0)
        N.check(
            N.lib().phx_pass_add(
                self.handle, kernel.id, n, items, params.ctypes.data, params.nbytes, arr, len(buffers), C.byref(step)
            )
        )
        self._keep.append(buffers)
        return step.value

    def set(self, step: int, offset: int, data: np.ndarray) -> None:
        data = np.ascontiguousarray(data)
        N.check(N.lib().phx_pass_set(self.handle, step, offset, data.ctypes.data, data.nbytes))

    def run(self) -> None:
        N.check(N.lib().phx_pass_run(self.handle))

    def run_step(self, step: int) -> None:
        N.check(N.lib().phx_pass_run_step(self.handle, step))

    def clear(self) -> None:
        N.check(N.lib().phx_pass_clear(self.handle))
        self._keep.clear()

    def __len__(self) -> int:
        return N.lib().phx_pass_len(self.handle)

    def compiled(self) -> int:
        return N.lib().phx_pass_compiled(self.handle)

    def close(self) -> None:
        if self.handle:
            N.lib().phx_pass_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
