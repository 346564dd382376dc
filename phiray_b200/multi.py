"""Several GPUs, one process each (torch.distributed over NCCL).

The Rendered path shards with no exchange inside the work: pixels and tile
rows of a frame are independent, and so are the scenes of a batch. Two
splits:

- ``FrameSplit``: one frame cut into bands of tile rows dealt round-robin
  across the ranks (so each rank gets rows from the top, the middle and the
  bottom of the frame, whose costs differ); each rank traces only its rows
  (phx_tracer_trace_rows) into its own tracer, packs their planes
  (phx_tracer_copy_rows, PHX_ROW_WORDS words a pixel) and one all-gather
  (ncclAllGather under torch.distributed) hands every rank the finished
  rows, which are unpacked into its image: the presenting rank then holds
  the whole frame, bit for bit what one GPU would have traced.
- ``balance``: a batch of scenes split by cost (faces x pixels x samples),
  largest first onto the least-loaded rank; each rank traces its own scenes
  and writes its own images, so nothing crosses between GPUs.

The reference renders on one device (src/gpu/mod.rs): this is new, and
tested with gloo ranks on the CPU, where the oracle traces each rank's rows
(tests/test_dist_cpu.py), and on one GPU by emulating the ranks.
"""

from __future__ import annotations

import numpy as np

from . import _native as N

ROW_WORDS = 22
# (first plane, words a pixel) of the planes a traced row carries, in the
# packed order phx_tracer_copy_rows uses (read.rs:37-56).
ROW_PLANES = ((0, 1), (1, 3), (4, 3), (7, 3), (10, 3), (13, 1), (20, 3), (23, 1), (24, 1), (25, 1), (31, 1), (33, 1))
assert sum(k for _, k in ROW_PLANES) == ROW_WORDS


def bands(h: int, world: int, rank: int, tile: int = 16) -> list[tuple[int, int]]:
    """Rank `rank`'s rows of an h-row frame: tiles of `tile` rows, tile k to
    rank k mod world, as (first row, rows) bands."""
    out = []
    for k, r0 in enumerate(range(0, h, tile)):
        if k % world == rank:
            out.append((r0, min(tile, h - r0)))
    return out


def max_rows(h: int, world: int, tile: int = 16) -> int:
    """The most rows any rank holds (every rank's packed buffer is this size,
    so the all-gather moves equal blocks)."""
    return max(sum(n for _, n in bands(h, world, r, tile)) for r in range(world))


def pack_rows(px: np.ndarray, w: int, h: int, bands_: list[tuple[int, int]], out: np.ndarray | None = None) -> np.ndarray:
    """Host form of phx_tracer_copy_rows over several bands: the bands'
    words of every row plane, band after band."""
    n = w * h
    words = sum(ROW_WORDS * rows * w for _, rows in bands_)
    out = np.zeros(words, np.uint32) if out is None else out
    at = 0
    for r0, rows in bands_:
        for plane, k in ROW_PLANES:
            a = plane * n + k * r0 * w
            m = k * rows * w
            out[at:at + m] = px[a:a + m]
            at += m
    return out


def unpack_rows(px: np.ndarray, w: int, h: int, bands_: list[tuple[int, int]], buf: np.ndarray) -> None:
    """The inverse of pack_rows: the bands' planes written into px."""
    n = w * h
    at = 0
    for r0, rows in bands_:
        for plane, k in ROW_PLANES:
            a = plane * n + k * r0 * w
            m = k * rows * w
            px[a:a + m] = buf[at:at + m]
            at += m


def balance(costs, world: int) -> list[list[int]]:
    """Scenes to ranks by cost, largest first onto the least-loaded rank
    (longest-processing-time order); each rank's list keeps cost order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += costs[i]
    return out


def scene_cost(scene, w: int | None = None, h: int | None = None, spp: int | None = None) -> float:
    """Faces x pixels x samples: the split's cost model of a frame."""
    w = scene.width if w is None else w
    h = scene.height if h is None else h
    spp = scene.spp if spp is None else spp
    return float(len(scene.faces)) * w * h * spp


class FrameSplit:
    """One frame of `tracer` across the ranks of `group` (torch.distributed),
    by tile rows; after ``gather`` every rank's tracer image holds the whole
    frame. The tracers must hold the same scene."""

    def __init__(self, tracer, w: int, h: int, rank: int, world: int, tile: int = 16, group=None):
        import torch

        self.tracer, self.w, self.h = tracer, w, h
        self.rank, self.world, self.tile, self.group = rank, world, tile, group
        self.mine = bands(h, world, rank, tile)
        self.block = ROW_WORDS * max_rows(h, world, tile) * w
        self.send = torch.zeros(self.block, dtype=torch.int32, device="cuda")
        self.recv = torch.zeros(self.block * world, dtype=torch.int32, device="cuda")

    def trace(self, cam: np.ndarray, first: int, spp: int) -> None:
        lib = N.lib()
        for r0, rows in self.mine:
            N.check(lib.phx_tracer_trace_rows(self.tracer.handle, cam.ctypes.data, self.w, self.h, first, spp, r0, rows))
        self.tracer.w, self.tracer.h = self.w, self.h

    def gather(self) -> None:
        """Every rank's rows to every rank (one all-gather), then into the
        tracer's image. Collective: every rank calls it."""
        import torch
        import torch.distributed as dist

        lib = N.lib()
        t = self.tracer.handle
        at = 0
        for r0, rows in self.mine:
            N.check(lib.phx_tracer_copy_rows(t, r0, rows, self.send.data_ptr() + 4 * at, 0))
            at += ROW_WORDS * rows * self.w
        self.tracer.gpu.wait()
        dist.all_gather_into_tensor(self.recv, self.send, group=self.group)
        torch.cuda.synchronize()
        for r in range(self.world):
            if r == self.rank:
                continue
            at = r * self.block
            for r0, rows in bands(self.h, self.world, r, self.tile):
                N.check(lib.phx_tracer_copy_rows(t, r0, rows, self.recv.data_ptr() + 4 * at, 1))
                at += ROW_WORDS * rows * self.w
        self.tracer.gpu.wait()
