"""The bounded device waits give up instead of hanging: each wait helper the
kernels use (the tensor-core engine's mbarrier wait, the radix sort's
look-back) is run on a flag nothing sets with a short poll limit; the call
reports PHX_ERR_KERNEL with the spin-limit text, and the same context then
sorts keys correctly. With the flag set the same waits return at once."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import _native as N

pytestmark = pytest.mark.gpu

MBARRIER, LOOKBACK = 0, 1


@pytest.mark.parametrize("which", [MBARRIER, LOOKBACK], ids=["mbarrier", "lookback"])
def test_a_wait_nothing_satisfies_reports_the_spin_limit(gpu, which):
    lib = N.lib()
    rc = lib.phx_selftest_wait(gpu.handle, which, 1 << 12, 0)
    assert rc == N.PHX_ERR_KERNEL
    assert "spin limit" in N.last_error()
    # the status was read and cleared: the context goes on working
    assert lib.phx_selftest_wait(gpu.handle, which, 1 << 12, 1) == N.PHX_OK
    import torch

    rng = np.random.default_rng(4)
    codes = rng.integers(0, 1 << 30, 100_000, dtype=np.uint32)
    d = torch.tensor(codes.view(np.int32), device="cuda")
    order = torch.empty_like(d)
    sorted_ = torch.empty_like(d)
    N.check(lib.phx_sort_codes(gpu.handle, d.data_ptr(), len(codes), order.data_ptr(), sorted_.data_ptr()))
    gpu.wait()
    assert np.array_equal(order.cpu().numpy().view(np.uint32), np.argsort(codes, kind="stable"))


def test_selftest_rejects_bad_arguments(gpu):
    lib = N.lib()
    assert lib.phx_selftest_wait(gpu.handle, 2, 16, 0) == N.PHX_ERR_INVALID
    assert lib.phx_selftest_wait(gpu.handle, 0, 0, 0) == N.PHX_ERR_INVALID
    assert px is not None
