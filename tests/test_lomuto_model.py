"""A data-parallel form of the binned SAH builder's in-place partition
(src/bvh/sah.rs:180-187, a Lomuto partition), checked against the
sequential swap loop on the CPU. A GPU builder that reproduces the
reference's tree node for node needs the slot order this loop leaves:

- the left elements (bin <= the split bin) end up first, in their order;
- the right block behaves as a queue: a right element joins at the back,
  and every left element met after the first right one moves the front
  element to the back.

So the right block's final order is the last k entries of an append log
E: a right element appends itself; the q-th rotation appends E[q]. Each
entry's position and its link to an earlier entry come from prefix sums
of the flags, and pointer jumping (log2 of the length rounds) resolves
every entry to the right element it carries."""

import numpy as np
import pytest


def lomuto(slots: np.ndarray, left: np.ndarray) -> tuple[np.ndarray, int]:
    """sah.rs:180-187 as written: swap each left element to the front."""
    s = slots.copy()
    m = 0
    for j in range(len(s)):
        if left[s[j]]:
            s[j], s[m] = s[m], s[j]
            m += 1
    return s, m


def lomuto_parallel(slots: np.ndarray, left: np.ndarray) -> tuple[np.ndarray, int]:
    """The same result from scans and pointer jumping only."""
    is_left = left[slots]
    c = len(slots)
    m = int(is_left.sum())
    out = np.empty_like(slots)
    out[:m] = slots[is_left]  # stable on the left
    k = c - m
    if k == 0:
        return out, m
    right_before = np.cumsum(~is_left) - (~is_left)  # rights strictly before j
    seen_right = right_before > 0
    rotate = is_left & seen_right  # a left element after the first right: one rotation
    # every event (a right element, or a rotation) appends one log entry, in
    # the order the loop meets them
    event = (~is_left) | rotate
    pos = np.cumsum(event) - 1  # log position of each event
    rot_index = np.cumsum(rotate) - 1  # q of each rotation
    total = int(event.sum())
    q_total = int(rotate.sum())
    value = np.full(total, -1, dtype=np.int64)  # the right element an entry carries, once known
    link = np.arange(total)  # an entry copies log[link] (itself for a right element)
    value[pos[~is_left]] = slots[~is_left]
    link[pos[rotate]] = rot_index[rotate]
    # pointer jumping: follow links until every entry reaches a right element
    for _ in range(int(np.ceil(np.log2(max(total, 2)))) + 1):
        unresolved = value < 0
        if not unresolved.any():
            break
        nxt = link[unresolved]
        value[unresolved] = value[nxt]
        link[unresolved] = link[nxt]
    assert (value >= 0).all()
    out[m:] = value[q_total:q_total + k]
    return out, m


@pytest.mark.parametrize("seed", range(40))
def test_parallel_partition_equals_the_swap_loop(seed):
    rng = np.random.default_rng(seed)
    c = int(rng.integers(1, 400))
    slots = rng.permutation(10_000)[:c].astype(np.int64)
    p = rng.uniform(0.05, 0.95)
    left = rng.random(10_000) < p
    want, m = lomuto(slots, left)
    got, m2 = lomuto_parallel(slots, left)
    assert m == m2 and np.array_equal(got, want)


def test_edge_cases():
    slots = np.arange(7, dtype=np.int64)
    for left in (np.zeros(7, bool), np.ones(7, bool), np.array([0, 0, 0, 1, 1, 1, 1], bool),
                 np.array([1, 1, 1, 0, 0, 0, 0], bool), np.array([0, 1, 0, 1, 0, 1, 0], bool)):
        assert np.array_equal(lomuto_parallel(slots, left)[0], lomuto(slots, left)[0])
