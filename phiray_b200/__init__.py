"""phiray-b200: phiray's Rendered-mode hot path as CUDA kernels for sm_100a.

The native library (``libphiray_b200.so``, built by ``python -m
phiray_b200.build``) exports the C ABI declared in ``include/phiray_cuda.h``;
this package is a thin host-side mirror of phiray's Rust API over it —
``Gpu``, ``GpuArray``, ``Pass``, ``GpuBvh``, ``Skin``/``Denoise`` and
``Tracer`` — used by the tests and the benchmark. There is no CPU fallback:
without the library or a CUDA device the calls raise.
"""

from ._native import PhxError, lib
from .bvh import Bvh, GpuBvh, aabbs, of_tri
from .gpu import Denoise, Gpu, GpuArray, Karras, Kernel, Morton, Pass, Refit, Skin, devptr
from .kernels import denoise, face_boxes, skin
from .tracer import CAMERA, Tracer, camera

__all__ = [
    "Bvh",
    "CAMERA",
    "Tracer",
    "camera",
    "Denoise",
    "Gpu",
    "GpuArray",
    "GpuBvh",
    "Karras",
    "Kernel",
    "Morton",
    "Pass",
    "PhxError",
    "Refit",
    "Skin",
    "aabbs",
    "denoise",
    "devptr",
    "face_boxes",
    "lib",
    "of_tri",
    "skin",
]
