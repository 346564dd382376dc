"""The trainer's host logic on the CPU: pair draws weighted by samples, the
px image of the samples between two accumulations, and the snapshot the
network's sample-spread input is read from."""

import types

import numpy as np

from phiray_b200 import train as T
from phiray_b200.denoiser import snapshot_host
from phiray_b200.tracer import PX_LEN


def test_pair_weights_follow_samples():
    ds = types.SimpleNamespace(n=4, spp=np.array([1, 4, 16, 64, 0], np.int32))
    assert T.DataSet.weights(ds, 0.0) is None  # uniform draws
    p = T.DataSet.weights(ds, 0.5)
    assert np.allclose(p, np.array([1, 2, 4, 8]) / 15.0)
    assert np.isclose(p.sum(), 1.0)
    q = T.DataSet.weights(ds, 1.0)
    assert np.all(np.diff(q) > 0) and np.isclose(q[-1], 64 / 85)


def _px(rng, n, count):
    px = np.zeros(PX_LEN * n + 1, np.uint32)
    f = px.view(np.float32)
    f[n:4 * n] = rng.uniform(0, 5, 3 * n)
    f[7 * n:14 * n] = rng.uniform(-1, 1, 7 * n)
    f[33 * n:34 * n] = rng.integers(0, 3, n)
    px[31 * n:32 * n] = count
    return px


def test_difference_of_accumulations_is_the_later_samples():
    rng = np.random.default_rng(3)
    n = 50
    a = _px(rng, n, 8)
    b = a.copy()
    f = b.view(np.float32)
    extra = rng.uniform(0, 2, 3 * n).astype(np.float32)
    f[n:4 * n] += extra
    f[33 * n:34 * n] += 1.0
    b[31 * n:32 * n] += 4
    d = T.px_diff(b, a, n)
    assert np.all(d[31 * n:32 * n] == 4)
    assert np.allclose(d.view(np.float32)[n:4 * n], extra, atol=1e-5)
    assert np.all(d.view(np.float32)[33 * n:34 * n] == 1.0)
    assert np.array_equal(T.px_diff(a, None, n)[n:4 * n], a[n:4 * n])


def test_snapshot_holds_sums_and_met_samples():
    rng = np.random.default_rng(4)
    n = 30
    px = _px(rng, n, 6)
    s = snapshot_host(px, 6, 5)
    f = px.view(np.float32)
    assert s.shape == (n, 4)
    assert np.array_equal(s[:, :3].reshape(-1), f[n:4 * n])
    assert np.array_equal(s[:, 3], 6.0 - f[33 * n:34 * n])
