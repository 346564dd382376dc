"""The reference's own test generators, restated (bit-exact f32 arithmetic).

- ``bvh_prims(n, shift)``: tests/bvh.rs:5-19 (seed 0x2545F491, every 13th
  prim the same box at 5, so Morton codes collide).
- ``test_prims(n)``: src/bvh/test.rs:6-23 (seed 0x9E3779B9, every 10th prim
  a duplicate box).
- ``rig(n)`` and ``translate``: tests/gpu.rs:6-35 (i % 4 influences over
  two translation bones).
"""

from __future__ import annotations

import numpy as np

F = np.float32


def _xorshift(seed: int):
    x = seed & 0xFFFFFFFF

    def step():
        nonlocal x
        x ^= (x << 13) & 0xFFFFFFFF
        x ^= x >> 17
        x ^= (x << 5) & 0xFFFFFFFF
        return x

    return step


def of_tri_rows(a, b, c):
    lo = [min(min(a[k], b[k]), c[k]) for k in range(3)]
    hi = [max(max(a[k], b[k]), c[k]) for k in range(3)]
    return [lo[0], lo[1], lo[2], F(0), hi[0], hi[1], hi[2], F(0)]


def bvh_prims(n: int, shift: float) -> np.ndarray:
    step = _xorshift(0x2545F491)
    k = F(0.001)
    sh = F(shift)

    def r():
        return F(step() % 100_000) * k

    rows = []
    for i in range(n):
        if i % 13 == 0:
            a = [F(5.0), F(5.0), F(5.0)]
        else:
            a = [r(), r() + sh, r()]
        b = [a[0] + F(0.3), a[1], a[2]]
        c = [a[0], a[1] + F(0.3), a[2] + F(0.05)]
        rows.append(of_tri_rows(a, b, c))
    return np.array(rows, dtype=np.float32).reshape(-1, 8)


def test_prims(n: int) -> np.ndarray:
    step = _xorshift(0x9E3779B9)
    k = F(0.01)

    def r():
        return F(step() % 10_000) * k

    rows = []
    for i in range(n):
        if i % 10 == 9:
            rows.append([F(1), F(1), F(1), F(0), F(1.5), F(1.5), F(1.5), F(0)])
            continue
        a = [r(), r(), r()]
        b = [a[0] + F(1.0), a[1], a[2]]
        c = [a[0], a[1] + F(1.0), a[2] + r() * F(0.1)]
        rows.append(of_tri_rows(a, b, c))
    return np.array(rows, dtype=np.float32).reshape(-1, 8)


def translate(x: float, y: float, z: float) -> np.ndarray:
    m = np.zeros(16, dtype=np.float32)
    m[0] = m[5] = m[10] = m[15] = 1.0
    m[12], m[13], m[14] = x, y, z
    return m


PAIR = np.dtype([("bone", "<u4"), ("weight", "<f4"), ("next", "<u4"), ("blend", "<f4")])


def rig(n: int):
    i = np.arange(n)
    rest = np.zeros((n, 4), dtype=np.float32)
    rest[:, 0] = i.astype(np.float32) * F(0.01)
    rest[:, 1] = (i % 7).astype(np.float32)
    rest[:, 2] = -np.sqrt(i.astype(np.float32))
    rest[:, 3] = 1.0
    counts = i % 4
    offsets = np.zeros(n + 1, dtype=np.uint32)
    offsets[1:] = np.cumsum(counts)
    pairs = np.zeros(int(offsets[-1]), dtype=PAIR)
    ks = np.concatenate([np.arange(c) for c in counts]) if n else np.zeros(0, int)
    pairs["bone"] = ks % 2
    pairs["next"] = ks % 2
    pairs["weight"] = F(0.25) + ks.astype(np.float32) * F(0.5)
    pairs["blend"] = 0.0
    return rest, offsets, pairs


def check_tree(nodes: np.ndarray, order: np.ndarray, depth: int, prims: np.ndarray, reachable) -> None:
    """src/bvh/test.rs:25-43 `check`: every prim exactly once under the
    reachable leaves, leaves contain their prims, inner nodes contain their
    children, depth below STACK."""
    words = nodes.view(np.uint32)
    seen = np.zeros(len(prims), dtype=np.int64)
    for i in reachable:
        lo, hi = int(words[i, 3]), int(words[i, 7])
        blo, bhi = nodes[i, 0:3], nodes[i, 4:7]
        if lo & 0x80000000:
            for s in range(lo & 0x7FFFFFFF, hi):
                p = int(order[s])
                seen[p] += 1
                assert np.all(blo <= prims[p, 0:3]) and np.all(bhi >= prims[p, 4:7])
        else:
            for c in (lo, hi):
                assert np.all(blo <= nodes[c, 0:3]) and np.all(bhi >= nodes[c, 4:7])
    assert np.all(seen == 1), "every prim exactly once"
    assert depth < 32
