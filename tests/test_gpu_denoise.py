"""Denoise on the GPU == the oracle's denoise.wgsl restatement, bit for bit:
the fused path on every plane it writes, the Pass path on the whole buffer."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200.kernels import DENOISE_STRENGTH, VIEW_STANDARD
from tests import pxgen

pytestmark = pytest.mark.gpu


def planes(a, n):
    return {"packed": a[:n], "linear": a[n: 4 * n], "shown": a[4 * n: 7 * n]}


@pytest.mark.parametrize("w,h", [(1, 1), (7, 5), (64, 48), (333, 97)])
@pytest.mark.parametrize("keep", [False, True])
def test_fused_denoise_matches_oracle(gpu, orc, w, h, keep):
    img = pxgen.px_image(w, h, seed=w * h)
    n = w * h
    want = orc.denoise(img, w, h, keep=keep)
    d = px.GpuArray.from_(gpu, img)
    px.denoise(gpu, d, w, h, keep=keep)
    got = d.read(np.uint32)
    for name in ("packed", "linear", "shown"):
        assert np.array_equal(planes(got, n)[name], planes(want, n)[name]), name
    if keep:
        assert np.array_equal(got[n: 4 * n], img[n: 4 * n])


def test_pass_denoise_matches_oracle_everywhere(gpu, orc):
    # Tracer::denoise_with (read.rs:96-118): four Denoise steps in a Pass.
    w, h = 96, 64
    n = w * h
    img = pxgen.px_image(w, h, seed=11)
    want = orc.denoise(img, w, h)
    d = px.GpuArray.from_(gpu, img)
    ps = px.Pass(gpu)
    for i, step in enumerate([1, 2, 4, 8]):
        ps.add(px.Denoise, n, px.Denoise.params(w=w, h=h, step=step, round=i, last=int(step == 8), keep=0,
                                                 strength=DENOISE_STRENGTH, view=VIEW_STANDARD), [d])
    ps.run()
    got = d.read(np.uint32)
    assert np.array_equal(got, want)


def test_denoise_reduces_noise_toward_the_mean(gpu, orc):
    # tests/denoise.rs:79-106 in spirit: on a flat-lit image the filtered
    # radiance is closer to the true mean than the noisy one.
    w, h = 128, 128
    img = pxgen.px_image(w, h, seed=3)
    n = w * h
    f = img.view(np.float32)
    count = img[31 * n: 32 * n].astype(np.float32)
    before = f[n: 4 * n].reshape(n, 3) / count[:, None]
    d = px.GpuArray.from_(gpu, img)
    px.denoise(gpu, d, w, h)
    after = d.read(np.float32)[n: 4 * n].reshape(n, 3) / count[:, None]
    truth = 0.4  # gamma(2, 0.2) mean
    hit = f[13 * n: 14 * n] >= 0
    assert np.abs(after[hit] - truth).mean() < 0.75 * np.abs(before[hit] - truth).mean()
