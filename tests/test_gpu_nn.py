"""The tcgen05 BF16 engine and the denoiser network's kernels against plain
fp32/fp64 products on the same bf16 inputs."""

import numpy as np
import pytest

from phiray_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32, 64, 96, 128, 160])
@pytest.mark.parametrize("m,k", [(128, 64), (256, 576), (1024, 1472)])
def test_gemm_bf16_matches_fp32_product(gpu, m, n, k):
    import torch

    g = torch.Generator(device="cpu").manual_seed(m * 1000 + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    want = a.double() @ b.double().T
    da, db = a.cuda(), b.cuda()
    d = torch.empty(m, n, dtype=torch.float32, device="cuda")
    N.check(N.lib().phx_gemm_bf16(gpu.handle, da.data_ptr(), db.data_ptr(), d.data_ptr(), m, n, k))
    gpu.wait()
    got = d.cpu().double()
    err = (got - want).abs().max().item()
    scale = want.abs().max().item()
    assert err <= 1e-5 * scale + 1e-4, (err, scale)  # fp32 accumulation of exact bf16 products
