"""phx_sort_codes_static: the radix sort that allocates nothing at call time.

Some callers cannot allocate device memory when they sort — a host that gave
the renderer a fixed budget up front, or a frame loop that must not stall on
cudaMalloc/cudaFree. This entry point takes its working memory from one fixed
array compiled into the library instead.
Its output must be the allocating sort's (phx_sort_codes), bit for bit, on
two calls in a row (the shared array keeps the first call's contents, so the
second call shows that everything that must start at zero does). This file
runs last so a failure here comes after every other test has run.
"""

import ctypes as C

import numpy as np
import pytest

from phiray_b200 import _native as N

pytestmark = pytest.mark.gpu


def _sort(lib, ctx, fn, codes_dev, n, torch):
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    sorted_ = torch.empty(n, dtype=torch.int32, device="cuda")
    N.check(fn(ctx, codes_dev.data_ptr(), n, order.data_ptr(), sorted_.data_ptr()))
    N.check(lib.phx_ctx_wait(ctx, 0))
    return order.cpu().numpy().view(np.uint32), sorted_.cpu().numpy().view(np.uint32)


def test_static_sort_matches_the_allocating_sort_twice():
    import torch

    lib = N.lib()
    ctx = C.c_void_p()
    N.check(lib.phx_ctx_create(0, C.byref(ctx)))
    try:
        rng = np.random.default_rng(2024)
        for n in (1 << 20, 300_001):
            codes = rng.integers(0, 1 << 30, n, dtype=np.uint32)
            codes[::5] = codes[3]  # many equal codes: the order must be stable
            d = torch.tensor(codes.view(np.int32), device="cuda")
            want = _sort(lib, ctx, lib.phx_sort_codes, d, n, torch)
            got = _sort(lib, ctx, lib.phx_sort_codes_static, d, n, torch)
            # errors inside the sort's kernels surface at the next status read
            assert lib.phx_ctx_wait(ctx, 0) == 0
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
            assert np.array_equal(got[0], np.argsort(codes, kind="stable").astype(np.uint32))
        # beyond the stated maximum: a clear error, nothing launched
        big = torch.zeros((1 << 20) + 1, dtype=torch.int32, device="cuda")
        rc = lib.phx_sort_codes_static(ctx, big.data_ptr(), (1 << 20) + 1, big.data_ptr(), big.data_ptr())
        assert rc == N.PHX_ERR_INVALID
        assert "at most" in N.last_error()
    finally:
        lib.phx_ctx_destroy(ctx)
