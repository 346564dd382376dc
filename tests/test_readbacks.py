"""The tracer's readbacks (read.rs:182-327) on oracle images, on the CPU:
radiance / albedo / normal / depth divide the px planes by the samples each
pixel took, display is the shown plane, and show's display step (show.wgsl)
over unchanged sums reproduces exactly what emit wrote."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from phiray_b200.tracer import albedo_of, depth_of, display_of, lit_of, normal_of, radiance_of
from tests import oracle_lib


@pytest.fixture(scope="module")
def traced(orc):
    s = scenes.c1_plain(ntris=2048, width=40, height=30, spp=4)
    cam = px.camera(s)
    cam["w"], cam["h"] = s.width, s.height
    img, _ = oracle_lib.TraceOracle(orc, s).trace(cam, 0, 6)
    return s, cam, img


def test_means_over_the_samples_taken(traced):
    s, _, img = traced
    w, h = s.width, s.height
    n = w * h
    f = img.view(np.float32)
    k = img[31 * n:32 * n].astype(np.float32)
    assert np.all(k == 6)
    assert np.array_equal(radiance_of(img, w, h), (f[n:4 * n].reshape(n, 3) / k[:, None]).reshape(h, w, 3))
    assert np.array_equal(albedo_of(img, w, h), (f[7 * n:10 * n].reshape(n, 3) / k[:, None]).reshape(h, w, 3))
    gone = f[33 * n:34 * n]
    hit = (gone == 0).reshape(h, w)
    assert hit.any() and (~hit).any()
    # the metric's mean and Tracer::radiance agree wherever every sample met something
    assert np.array_equal(lit_of(img, w, h)[hit], radiance_of(img, w, h)[hit])


def test_normal_and_depth(traced):
    s, _, img = traced
    w, h = s.width, s.height
    n = w * h
    nrm = normal_of(img, w, h).reshape(n, 3)
    ln = np.linalg.norm(nrm, axis=1)
    assert np.allclose(ln[ln > 0], 1.0, atol=1e-5)
    gone = img.view(np.float32)[33 * n:34 * n]
    d = depth_of(img, w, h).reshape(n)
    assert np.all(d[gone == 6] == np.float32(1e10))  # every sample missed: Cycles' far value
    assert np.all((d[gone == 0] > 0) & (d[gone == 0] < 1e10))


def test_show_over_unchanged_sums_reproduces_emit(orc, traced):
    s, cam, img = traced
    n = s.width * s.height
    again = img.copy()
    again[:n] = 0
    again[4 * n:7 * n] = 0
    orc.lib.orc_show(cam.ctypes.data, again.ctypes.data)
    assert np.array_equal(again, img)
    assert np.array_equal(display_of(img, s.width, s.height).reshape(-1), img.view(np.float32)[4 * n:7 * n])
