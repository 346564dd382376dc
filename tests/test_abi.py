"""The C ABI library loads, exports every entry point include/*.h declares,
and fails loudly (no CPU fallback) where there is no device."""

import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w\s\*]*?\b(phx_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from phiray_b200 import _native

    lib = _native.lib()
    names = declared()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes signatures cover all of them
    assert set(names) <= set(_native.SIGNATURES), set(names) - set(_native.SIGNATURES)


def test_version_string():
    from phiray_b200 import _native

    assert b"sm_100a" in _native.lib().phx_version()


def test_no_device_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from phiray_b200 import _native

    lib = _native.lib()
    assert lib.phx_device_count() == 0
    h = C.c_void_p()
    rc = lib.phx_ctx_create(0, C.byref(h))
    assert rc == _native.PHX_ERR_DEVICE
    assert "device" in _native.last_error().lower()
    with pytest.raises(_native.PhxError):
        import phiray_b200 as px

        px.Gpu(0)


def test_null_arguments_are_invalid():
    from phiray_b200 import _native

    lib = _native.lib()
    assert lib.phx_ctx_wait(None, 1) == _native.PHX_ERR_INVALID
    assert lib.phx_bvh_refit(None) == _native.PHX_ERR_INVALID
    assert lib.phx_pass_run(None) == _native.PHX_ERR_INVALID
