"""ctypes binding of libphiray_b200.so (the C ABI in include/phiray_cuda.h).

The library is loaded from this package's directory. There is no fallback:
if it is missing, importing the API raises, and on a machine without a CUDA
device every call that needs one returns PHX_ERR_DEVICE.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libphiray_b200.so"

PHX_OK = 0
PHX_REBUILD = 1
PHX_ERR_INVALID = -1
PHX_ERR_OOM = -2
PHX_ERR_TIMEOUT = -3
PHX_ERR_CANCELLED = -4
PHX_ERR_DEVICE = -5
PHX_ERR_KERNEL = -6

KERNEL_SKIN = 1
KERNEL_DENOISE = 2
KERNEL_MORTON = 3
KERNEL_KARRAS = 4
KERNEL_REFIT = 5

LEAF = 0x80000000
STACK = 32

_NAMES = {
    PHX_ERR_INVALID: "PHX_ERR_INVALID",
    PHX_ERR_OOM: "PHX_ERR_OOM",
    PHX_ERR_TIMEOUT: "PHX_ERR_TIMEOUT",
    PHX_ERR_CANCELLED: "PHX_ERR_CANCELLED",
    PHX_ERR_DEVICE: "PHX_ERR_DEVICE",
    PHX_ERR_KERNEL: "PHX_ERR_KERNEL",
}


class PhxError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{_NAMES.get(code, code)}: {message}")
        self.code = code


vp = C.c_void_p
u32 = C.c_uint32
i32 = C.c_int32
u64 = C.c_uint64
f32p = C.POINTER(C.c_float)

# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "phx_version": (C.c_char_p, []),
    "phx_last_error": (i32, [C.c_char_p, C.c_size_t]),
    "phx_device_count": (i32, []),
    "phx_ctx_create": (i32, [i32, C.POINTER(vp)]),
    "phx_ctx_destroy": (i32, [vp]),
    "phx_ctx_wait": (i32, [vp, u32]),
    "phx_tracer_create_instanced": (i32, [vp, vp, vp, u32, vp, u32, vp]),
    "phx_tracer_reinstance": (i32, [vp, vp, u32]),
    "phx_tracer_trace_rows": (i32, [vp, vp, u32, u32, u32, u32, u32, u32]),
    "phx_tracer_set_tree": (i32, [vp, u32]),
    "phx_tracer_autotune_tree": (i32, [vp, vp, u32, u32, u32, u32, vp, vp]),
    "phx_tracer_copy_rows": (i32, [vp, u32, u32, vp, i32]),
    "phx_selftest_wait": (i32, [vp, i32, u32, i32]),
    "phx_ctx_stream": (vp, [vp]),
    "phx_ctx_set_stream": (i32, [vp, vp]),
    "phx_buf_alloc": (i32, [vp, u64, C.POINTER(vp)]),
    "phx_buf_wrap": (i32, [vp, vp, u64, C.POINTER(vp)]),
    "phx_buf_free": (i32, [vp]),
    "phx_buf_write": (i32, [vp, u64, vp, u64]),
    "phx_buf_assign": (i32, [vp, vp, u64, C.POINTER(i32)]),
    "phx_buf_read": (i32, [vp, u64, vp, u64, u32]),
    "phx_buf_size": (u64, [vp]),
    "phx_buf_ptr": (vp, [vp]),
    "phx_pass_create": (i32, [vp, C.POINTER(vp)]),
    "phx_pass_destroy": (i32, [vp]),
    "phx_pass_add": (i32, [vp, i32, u32, u32, vp, u32, C.POINTER(vp), u32, C.POINTER(u32)]),
    "phx_pass_set": (i32, [vp, u32, u32, vp, u32]),
    "phx_pass_run": (i32, [vp]),
    "phx_pass_run_step": (i32, [vp, u32]),
    "phx_pass_clear": (i32, [vp]),
    "phx_pass_len": (u32, [vp]),
    "phx_pass_compiled": (u32, [vp]),
    "phx_bvh_build": (i32, [vp, vp, u32, u32, C.POINTER(vp)]),
    "phx_bvh_build_sah": (i32, [vp, vp, u32, u32, vp, vp, C.POINTER(u32), C.POINTER(u32)]),
    "phx_bvh_build_device": (i32, [vp, vp, u32, u32, C.POINTER(vp)]),
    "phx_bvh_rebuild_device": (i32, [vp, vp, u32]),
    "phx_bvh_refit": (i32, [vp]),
    "phx_bvh_update": (i32, [vp, vp, u32]),
    "phx_bvh_update_device": (i32, [vp, vp, u32]),
    "phx_bvh_download": (i32, [vp, vp, vp, C.POINTER(u32), u32]),
    "phx_bvh_info": (i32, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)]),
    "phx_bvh_device": (i32, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    "phx_bvh_destroy": (i32, [vp]),
    "phx_morton": (i32, [vp, vp, u32, vp, vp]),
    "phx_sort_codes": (i32, [vp, vp, u32, vp, vp]),
    "phx_sort_codes_static": (i32, [vp, vp, u32, vp, vp]),
    "phx_karras": (i32, [vp, vp, u32, vp]),
    "phx_gemm_bf16": (i32, [vp, vp, vp, vp, u32, u32, u32]),
    "phx_nn_conv_fwd": (i32, [vp, vp, i32, i32, i32, vp, i32, vp, vp, i32, i32, i32, i32, i32, i32, i32, i32]),
    "phx_nn_conv_kpn": (i32, [vp, vp, i32, i32, i32, vp, i32, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp]),
    "phx_nn_conv_wgrad": (i32, [vp, vp, i32, i32, i32, vp, i32, i32, i32, vp, i32, i32, i32, i32]),
    "phx_nn_bias_grad": (i32, [vp, vp, i32, i32, i32, i32, vp]),
    "phx_nn_relu_bwd": (i32, [vp, vp, i32, i32, vp, i32, i32, i32, i32]),
    "phx_nn_pool_fwd": (i32, [vp, vp, i32, i32, i32, i32, i32, i32, vp]),
    "phx_nn_pool_bwd": (i32, [vp, vp, i32, i32, i32, i32, vp, i32, i32]),
    "phx_nn_up_fwd": (i32, [vp, vp, i32, i32, i32, i32, vp, i32, i32]),
    "phx_nn_up_bwd": (i32, [vp, vp, i32, i32, i32, i32, i32, i32, vp]),
    "phx_nn_flip": (i32, [vp, vp, i32, i32, i32, vp, i32]),
    "phx_nn_kpn": (i32, [vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp, vp, vp, C.c_float]),
    "phx_nn_adam": (i32, [vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, C.c_float, C.c_float, C.c_float, C.c_float, i32]),
    "phx_nn_features": (i32, [vp, vp, vp, i32, i32, i32, i32, vp, vp, vp]),
    "phx_nn_snapshot": (i32, [vp, vp, u32, u32, vp]),
    "phx_nn_firefly": (i32, [vp, vp, vp, i32, i32, i32, i32, i32]),
    "phx_nn_compose": (i32, [vp, vp, i32, i32, i32, vp, vp, i32, C.c_float, i32, C.c_float, C.c_float, vp, vp]),
    "phx_unet_create": (i32, [vp, u64, C.POINTER(vp)]),
    "phx_unet_destroy": (i32, [vp]),
    "phx_unet_param_count": (i32, [vp, C.POINTER(u64)]),
    "phx_unet_set_params": (i32, [vp, vp, u64]),
    "phx_unet_get": (i32, [vp, i32, vp, u64]),
    "phx_unet_forward": (i32, [vp, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp]),
    "phx_unet_grads": (i32, [vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, C.c_float, vp]),
    "phx_unet_adam": (i32, [vp, C.c_float]),
    "phx_unet_train_step": (i32, [vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, C.c_float, C.c_float, vp]),
    "phx_unet_logits": (i32, [vp, C.POINTER(vp)]),
    "phx_unet_grad_arena": (i32, [vp, C.POINTER(vp), C.POINTER(C.c_uint64)]),
    "phx_unet_set_clamp": (i32, [vp, i32]),
    "phx_unet_set_flips": (i32, [vp, i32]),
    "phx_unet_denoise_px": (i32, [vp, vp, vp, u32, u32, f32p, i32, C.c_float, i32, C.POINTER(u32)]),
    "phx_tracer_snapshot": (i32, [vp, vp]),
    "phx_tracer_denoise_learned": (i32, [vp, vp, vp, i32, C.c_float, i32, C.POINTER(u32)]),
    "phx_batch_create": (i32, [vp, C.POINTER(vp)]),
    "phx_batch_destroy": (i32, [vp]),
    "phx_batch_add": (i32, [vp, vp, vp, u32, u32, u32, u32, C.POINTER(u32)]),
    "phx_batch_clear": (i32, [vp]),
    "phx_batch_set_config": (i32, [vp, u32, u32, u32]),
    "phx_batch_trace": (i32, [vp]),
    "phx_batch_autotune": (i32, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_float),
                                 C.POINTER(u32)]),
    "phx_batch_capture": (i32, [vp, vp, C.c_float]),
    "phx_batch_replay": (i32, [vp, vp]),
    "phx_batch_results": (i32, [vp, vp, vp]),
    "phx_skin": (i32, [vp, vp, vp, vp, vp, u32, vp, u32, C.c_float]),
    "phx_face_boxes": (i32, [vp, vp, vp, u32, vp]),
    "phx_denoise": (i32, [vp, vp, u32, u32, f32p, f32p, i32]),
    "phx_tracer_create": (i32, [vp, vp, C.POINTER(vp)]),
    "phx_tracer_destroy": (i32, [vp]),
    "phx_tracer_set_samples": (i32, [vp, u32]),
    "phx_tracer_set_kernel": (i32, [vp, u32]),
    "phx_tracer_set_stack": (i32, [vp, u32]),
    "phx_tracer_set_walk": (i32, [vp, u32]),
    "phx_tracer_autotune": (i32, [vp, vp, u32, u32, u32, C.POINTER(u32), C.POINTER(C.c_float)]),
    "phx_tracer_sample": (i32, [vp, vp, u32, u32, u32, vp, C.POINTER(u32), C.POINTER(i32)]),
    "phx_tracer_trace": (i32, [vp, vp, u32, u32, u32, u32]),
    "phx_tracer_read": (i32, [vp, u64, vp, u64, u32]),
    "phx_tracer_set_adaptive": (i32, [vp, vp]),
    "phx_tracer_show": (i32, [vp, vp, u64]),
    "phx_tracer_unconverged": (i32, [vp, C.POINTER(u32), u32]),
    "phx_tracer_image": (i32, [vp, C.POINTER(vp), C.POINTER(u64)]),
    "phx_tracer_verts": (i32, [vp, C.POINTER(vp), C.POINTER(u32)]),
    "phx_tracer_denoise": (i32, [vp, i32]),
    "phx_tracer_time": (i32, [vp, C.POINTER(C.c_float), C.POINTER(u64)]),
    "phx_tracer_repose_device": (i32, [vp, vp, i32]),
    "phx_tracer_primary": (i32, [vp, vp, u32, u32, u32, vp, vp]),
    "phx_tracer_secondary_rays": (i32, [vp, vp, u32, u32, u32, vp]),
    "phx_trace_rays": (i32, [vp, vp, u32, vp, i32]),
    "phx_trace_rays_stats": (i32, [vp, vp, u32, vp, i32, C.POINTER(u64)]),
    "phx_tracer_trace_stats": (i32, [vp, vp, u32, u32, u32, u32, C.POINTER(u64)]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded native library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python -m phiray_b200.build` (phiray-b200 has no CPU fallback)"
            )
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().phx_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> int:
    """Raises PhxError for a negative status, returns it otherwise."""
    if rc < 0:
        raise PhxError(rc, last_error())
    return rc


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
