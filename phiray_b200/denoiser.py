"""The learned denoiser over the C ABI: ``Unet`` (phx_unet_*) and the
per-layer calls its parity tests drive one at a time (phx_nn_*).

phiray has no learned denoiser; ``Unet.denoise(tracer)`` is the drop-in
beside ``Tracer.denoise`` (src/trace/read.rs:78-119): the same px image is
filtered in place, and every tile whose error estimate is above the
threshold keeps the a-trous result of the plain ``Denoise``.

Weights files (``.phxu``): magic ``PHXU``, u32 version 1, u64 count, then
``count`` little-endian float32 in the blob layout (per layer W [cout][9 cin]
with k = (3 ty + tx) cin + ci, then b [cout]).
"""

from __future__ import annotations

import ctypes as C
import struct
from pathlib import Path

import numpy as np

from . import _native as N
from .gpu import Gpu, devptr

HERE = Path(__file__).resolve().parent
WEIGHTS = HERE / "weights" / "kpcn.phxu"
SEED = 0x2545F491

LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 96), (96, 96), (96, 128), (128, 128), (128, 160),
          (160, 160), (288, 128), (128, 128), (224, 96), (96, 96), (160, 64), (64, 64), (96, 32), (32, 32), (32, 32)]
FEATURES = 16
HEAD = 32
TILE = 16
# Mean predicted relative error of a tile above which the a-trous result is kept.
THRESHOLD = 0.1


def padded(n: int) -> int:
    """Image side padded to the network's multiple of 16."""
    return (n + 15) // 16 * 16


def flops_per_pixel() -> int:
    """Multiply-adds x 2 of one forward pass per full-resolution pixel."""
    lv = [0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 3, 3, 2, 2, 1, 1, 0, 0, 0]
    mac = sum(9 * ci * co / 4 ** l for (ci, co), l in zip(LAYERS, lv))
    return int(round(2 * mac))


def read_weights(path) -> np.ndarray:
    raw = Path(path).read_bytes()
    magic, ver, count = struct.unpack_from("<4sIQ", raw, 0)
    if magic != b"PHXU" or ver != 1:
        raise ValueError(f"{path}: not a version-1 phxu weights file")
    data = np.frombuffer(raw, dtype="<f4", count=count, offset=16)
    return data.astype(np.float32)


def write_weights(path, params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, dtype="<f4")
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    Path(path).write_bytes(struct.pack("<4sIQ", b"PHXU", 1, p.size) + p.tobytes())


class Unet:
    """The kernel-predicting U-Net on one Gpu (phx_unet)."""

    def __init__(self, gpu: Gpu, seed: int = SEED, params: np.ndarray | None = None):
        self.gpu = gpu
        h = C.c_void_p()
        N.check(N.lib().phx_unet_create(gpu.handle, seed, C.byref(h)))
        self.handle = h
        c = C.c_uint64()
        N.check(N.lib().phx_unet_param_count(h, C.byref(c)))
        self.count = c.value
        gpu.adopt(self)
        if params is not None:
            self.set_params(params)

    @classmethod
    def pretrained(cls, gpu: Gpu, path=WEIGHTS) -> "Unet":
        return cls(gpu, params=read_weights(path))

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        N.check(N.lib().phx_unet_set_params(self.handle, p.ctypes.data, p.size))

    def _get(self, which: int) -> np.ndarray:
        out = np.empty(self.count, dtype=np.float32)
        N.check(N.lib().phx_unet_get(self.handle, which, out.ctypes.data, out.size))
        return out

    def params(self) -> np.ndarray:
        return self._get(0)

    def grads(self) -> np.ndarray:
        """Gradients of the last ``grads``/``train_step`` (blob layout)."""
        return self._get(1)

    def save(self, path) -> None:
        write_weights(path, self.params())

    def forward(self, feat, irr, alb, B: int, Hp: int, Wp: int, h: int, w: int, out=None, err=None) -> None:
        N.check(N.lib().phx_unet_forward(self.handle, devptr(feat), devptr(irr), devptr(alb), B, Hp, Wp, h, w,
                                         devptr(out), devptr(err)))

    def logits(self) -> int:
        p = C.c_void_p()
        N.check(N.lib().phx_unet_logits(self.handle, C.byref(p)))
        return p.value or 0

    def grad_arena(self) -> tuple[int, int]:
        """(device pointer, fp32 count) of the array holding every layer's
        gradients (phx_unet_grad_arena): what data-parallel ranks reduce."""
        p, c = C.c_void_p(), C.c_uint64()
        N.check(N.lib().phx_unet_grad_arena(self.handle, C.byref(p), C.byref(c)))
        return p.value or 0, c.value

    def grad_tensor(self):
        """The gradient arena as a torch fp32 tensor sharing its memory."""
        import torch

        ptr, count = self.grad_arena()

        class _Arena:
            __cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False), "version": 3}

        return torch.as_tensor(_Arena(), device=f"cuda:{self.gpu.ordinal}")

    def compute_grads(self, feat, irr, alb, ref, B, Hp, Wp, h, w, loss, err_weight: float = 0.1) -> None:
        N.check(N.lib().phx_unet_grads(self.handle, devptr(feat), devptr(irr), devptr(alb), devptr(ref), B, Hp, Wp,
                                       h, w, err_weight, devptr(loss)))

    def adam(self, lr: float) -> None:
        N.check(N.lib().phx_unet_adam(self.handle, lr))

    def train_step(self, feat, irr, alb, ref, B, Hp, Wp, h, w, loss, lr: float, err_weight: float = 0.1) -> None:
        """One Adam step on a batch; the batch loss is ADDED to *loss (device fp32)."""
        N.check(N.lib().phx_unet_train_step(self.handle, devptr(feat), devptr(irr), devptr(alb), devptr(ref), B, Hp,
                                            Wp, h, w, err_weight, lr, devptr(loss)))

    def set_clamp(self, on: bool) -> None:
        """Whether the predicted kernels filter the firefly-clamped irradiance
        or the irradiance as it is (the default; phx_unet_set_clamp)."""
        N.check(N.lib().phx_unet_set_clamp(self.handle, 1 if on else 0))

    def set_flips(self, images: int) -> None:
        """Average the denoised result over 1, 2 (also mirrored in x) or 4
        (also in y and both) network passes (phx_unet_set_flips)."""
        N.check(N.lib().phx_unet_set_flips(self.handle, images))

    def denoise(self, tracer, half=None, tile: int = TILE, threshold: float = THRESHOLD, keep: bool = False,
                count: bool = False) -> int | None:
        """Learned ``Tracer::denoise``; `half`: a snapshot (``Tracer.snapshot``)
        taken part way through the frame's samples, or None. With count=True
        waits and returns the number of tiles that kept the a-trous result."""
        fb = C.c_uint32()
        N.check(N.lib().phx_tracer_denoise_learned(tracer.handle, self.handle, devptr(half), tile, threshold,
                                                   1 if keep else 0, C.byref(fb) if count else None))
        return fb.value if count else None

    def denoise_px(self, px, w: int, h: int, half=None, tile: int = TILE, threshold: float = THRESHOLD,
                   keep: bool = False, view=(0.0, 0.0, 1.0, 0.0), count: bool = False) -> int | None:
        """The same on any device px image (34 w h + 1 words)."""
        fb = C.c_uint32()
        v = (C.c_float * 4)(*view)
        N.check(N.lib().phx_unet_denoise_px(self.handle, devptr(px), devptr(half), w, h, v, tile, threshold,
                                            1 if keep else 0, C.byref(fb) if count else None))
        return fb.value if count else None

    def close(self) -> None:
        if self.handle:
            N.lib().phx_unet_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def features(gpu: Gpu, px, w: int, h: int, Hp: int, Wp: int, feat, irr, alb, half=None) -> None:
    """Network inputs of a traced px image (phx_nn_features); `half`: a
    snapshot taken part way through its samples, or None."""
    N.check(N.lib().phx_nn_features(gpu.handle, devptr(px), devptr(half), w, h, Hp, Wp, devptr(feat), devptr(irr),
                                    devptr(alb)))


def firefly(gpu: Gpu, irr, out, B: int, Hp: int, Wp: int, h: int, w: int) -> None:
    """phx_nn_firefly: the a-trous Denoise's firefly clamp on padded fp32 x 3
    irradiance planes."""
    N.check(N.lib().phx_nn_firefly(gpu.handle, devptr(irr), devptr(out), B, Hp, Wp, h, w))


def snapshot(gpu: Gpu, px, w: int, h: int, snap) -> None:
    """phx_nn_snapshot: the sums and met-sample counts of a px image now."""
    N.check(N.lib().phx_nn_snapshot(gpu.handle, devptr(px), w, h, devptr(snap)))


def snapshot_host(px: np.ndarray, w: int, h: int) -> np.ndarray:
    """The same snapshot from a host px image: (w h, 4) float32."""
    n = w * h
    f = px.view(np.float32)
    out = np.empty((n, 4), np.float32)
    out[:, :3] = f[n:4 * n].reshape(n, 3)
    out[:, 3] = px[31 * n:32 * n].astype(np.float32) - f[33 * n:34 * n]
    return out
