"""Adaptive Sampling in the oracle (adapt.wgsl's convergence check and
dilation, gather.wgsl's open-pixel list, util.wgsl's half image, shade.wgsl
skipping settled pixels), checked against its definition on the CPU: the
rules the CUDA tracer is then held to bit for bit."""

import numpy as np
import pytest

import phiray_b200 as px
from phiray_b200 import scenes
from tests import oracle_lib

ADAPT = [0.03, 4.0, 4.0, 1.0]  # threshold, min samples, step, on
SPP = 32


def _scene():
    s = scenes.c1_plain(ntris=2048, width=48, height=32, spp=4)
    cam = px.camera(s)
    cam["w"], cam["h"] = s.width, s.height
    return s, cam


@pytest.fixture(scope="module")
def adaptive(orc):
    s, cam = _scene()
    cam["adapt"] = ADAPT
    img, rays = oracle_lib.TraceOracle(orc, s).trace(cam, 0, SPP)
    return s, cam, img, rays


def test_settled_pixels_stop_at_a_step_boundary(adaptive):
    s, _, img, _ = adaptive
    n = s.width * s.height
    count = img[31 * n:32 * n]
    seen = img[30 * n:31 * n]
    assert 0 < int(seen.sum()) < n  # some settled, some not
    # the first check follows sample 7 (past the minimum 4, the last of a step of 4)
    assert count.min() == 8
    assert np.all(count[seen == 0] == SPP)
    settled = count[seen != 0]
    assert np.all((settled <= SPP) & ((settled - 8) % 4 == 0))  # the last tail may settle some at 32


def test_open_list_and_dilation(adaptive):
    s, _, img, _ = adaptive
    w, h = s.width, s.height
    n = w * h
    flag = img[29 * n:30 * n].reshape(h, w)
    seen = img[30 * n:31 * n].reshape(h, w)
    want = flag.copy()
    want[:, 1:] = np.minimum(want[:, 1:], flag[:, :-1])
    want[:, :-1] = np.minimum(want[:, :-1], flag[:, 1:])
    want[1:, :] = np.minimum(want[1:, :], flag[:-1, :])
    want[:-1, :] = np.minimum(want[:-1, :], flag[1:, :])
    assert np.array_equal(seen, want)  # settled only with all four neighbours settled
    m = int(img[34 * n])
    assert m == int((seen == 0).sum())
    assert np.array_equal(img[32 * n:32 * n + m], np.flatnonzero(seen.reshape(-1) == 0))


def test_convergence_rule_on_open_pixels(adaptive):
    # every pixel still open failed the check at the last boundary (sample 31)
    s, cam, img, _ = adaptive
    n = s.width * s.height
    f = img.view(np.float32)
    full = f[n:4 * n].reshape(n, 3).astype(np.float32)
    half = f[26 * n:29 * n].reshape(n, 3).astype(np.float32)
    scale = np.float32(1.0) / img[31 * n:32 * n].astype(np.float32)
    err_d = (np.abs(full[:, 0] - half[:, 0]) + np.abs(full[:, 1] - half[:, 1]) + np.abs(full[:, 2] - half[:, 2])) * scale
    inten = (full[:, 0] + full[:, 1] + full[:, 2]) * scale
    norm = np.where(inten < 1.0, np.sqrt(inten), inten).astype(np.float32)
    err = err_d / (np.float32(0.0001) + norm)
    flag = img[29 * n:30 * n]
    assert np.all(err[flag == 0] >= np.float32(ADAPT[0]))


def test_two_calls_equal_one_and_off_is_plain(orc, adaptive):
    s, cam, img, rays = adaptive
    o = oracle_lib.TraceOracle(orc, s)
    a, r1 = o.trace(cam, 0, 13)
    b, r2 = o.trace(cam, 13, SPP - 13, px=a)
    assert np.array_equal(b, img) and r1 + r2 == rays
    plain_cam = cam.copy()
    plain_cam["adapt"] = [0.0, 0.0, 0.0, 0.0]
    plain, prays = o.trace(plain_cam, 0, SPP)
    n = s.width * s.height
    assert prays > rays  # settled pixels cost no rays
    assert not plain[26 * n:29 * n].any()  # no half image without it
