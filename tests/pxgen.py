"""Synthetic px images (phiray's Tracer image buffer, src/trace/read.rs:37-56:
34 w h + 1 words) with plausible sums in every plane the denoiser reads."""

import numpy as np


def px_image(w: int, h: int, seed: int = 0, samples: int = 12) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = w * h
    px = np.zeros(34 * n + 1, dtype=np.uint32)
    f = px.view(np.float32)
    k = samples
    count = np.full(n, k, np.uint32)
    count[rng.random(n) < 0.05] = rng.integers(1, k, 1)[0]
    px[31 * n: 32 * n] = count
    # radiance sums with fireflies
    rad = rng.gamma(2.0, 0.2, (n, 3)).astype(np.float32) * count[:, None]
    hot = rng.random(n) < 0.01
    rad[hot] *= 80.0
    f[1 * n: 4 * n] = rad.reshape(-1)
    # albedo (two regions with an edge), normals, depth (misses negative)
    x = np.arange(n) % w
    alb = np.where((x < w // 2)[:, None], 0.05, 0.8).astype(np.float32) + rng.random((n, 3)).astype(np.float32) * 0.05
    f[7 * n: 10 * n] = (alb * count[:, None]).reshape(-1)
    nrm = rng.standard_normal((n, 3)).astype(np.float32) * 0.1 + np.array([0, 0, 1], np.float32)
    f[10 * n: 13 * n] = (nrm * count[:, None]).reshape(-1)
    dep = (1.0 + rng.random(n)).astype(np.float32)
    miss = rng.random(n) < 0.1
    dep[miss] = -1.0
    f[13 * n: 14 * n] = dep * count
    missed = np.where(miss, count, 0).astype(np.float32)
    f[33 * n: 34 * n] = missed
    f[24 * n: 25 * n] = count.astype(np.float32)  # film coverage: opaque
    f[20 * n: 23 * n] = (rng.random((n, 3)) * 0.01).astype(np.float32).reshape(-1)
    f[23 * n: 24 * n] = (rng.random(n) * 0.1).astype(np.float32)
    return px
