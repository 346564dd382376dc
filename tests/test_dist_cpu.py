"""The multi-process path of bench.py on CPU ranks (gloo, world size 2):
max-over-ranks timing, the whole-job rate of replicas, and the reference arm
running on rank 0 only."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    t = bench.max_over_ranks(10.0 + rank, "cpu")
    rate = bench.whole_job_rate(1000.0, world, t)
    w, r, loc = bench.dist_env()
    out.put((rank, t, rate, w, r, loc))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rate_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate, w, r, loc in res:
        assert t == 11.0  # the slower rank's time on every rank
        assert rate == pytest.approx(1000.0 * 2 / 11e-3)
        assert (w, r, loc) == (2, rank, rank)


def test_reference_arm_runs_on_rank_zero_only(capsys, monkeypatch):
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    bench.reference_arm(argparse.Namespace(steps=1, warmup=0))
    assert capsys.readouterr().out == ""


def _train_rank(rank: int, world: int, port: int, out) -> None:
    """One data-parallel training rank on CPU: its own gradients, the
    all-reduce average of phiray_b200.train, then the oracle's Adam step."""
    import datetime
    import sys

    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
    from oracle import nn as O
    from phiray_b200 import train as T

    r, size = T.world()
    rng = np.random.default_rng(100 + rank)
    w = np.random.default_rng(5).standard_normal(257).astype(np.float32)  # same start on every rank
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    seen = []
    for step in range(1, 4):
        g_local = rng.standard_normal(257).astype(np.float32)  # this rank's own batch
        t = torch.from_numpy(g_local.copy())
        T.average_grads(t, size)
        everyone = [torch.zeros(257) for _ in range(size)]
        dist.all_gather(everyone, torch.from_numpy(g_local))
        seen.append(float(np.abs(t.numpy() - np.mean([e.numpy() for e in everyone], axis=0)).max()))
        w, m, v = O.adam(w, t.numpy(), m, v, 1e-3, step)
    out.put((rank, r, size, T.shard(range(10), r, size), seen, float(np.sum(w, dtype=np.float64))))
    dist.barrier()
    dist.destroy_process_group()


def test_data_parallel_training_ranks_stay_in_lockstep():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_train_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, r0, s0, sh0, seen0, sum0), (_, r1, s1, sh1, seen1, sum1) = res
    assert (r0, r1, s0, s1) == (0, 1, 2, 2)
    assert sorted(sh0 + sh1) == list(range(10)) and not set(sh0) & set(sh1)  # disjoint scene shards
    assert max(seen0 + seen1) < 1e-6  # the reduced gradient is the mean of the ranks' gradients
    assert sum0 == sum1  # same start, same averaged gradient, same Adam: identical weights


def _split_rank(rank: int, world: int, port: int, out) -> None:
    """One rank of a frame split by tile rows, on CPU: the oracle traces this
    rank's bands, the bands' planes are packed (phiray_b200.multi's layout,
    the one phx_tracer_copy_rows uses on the device), one all-gather (gloo)
    hands every rank every band, and each rank unpacks them into its image."""
    import datetime
    import sys

    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
    import phiray_b200 as px
    from phiray_b200 import multi, scenes
    from tests import oracle_lib

    orc = oracle_lib.load()
    s = scenes.c1_plain(ntris=2048, width=40, height=37, spp=2)
    w, h = s.width, s.height
    cam = px.camera(s)
    cam["w"], cam["h"] = w, h
    T = oracle_lib.TraceOracle(orc, s)
    img = np.zeros(34 * w * h + 1, np.uint32)
    mine = multi.bands(h, world, rank, tile=8)
    for r0, rows in mine:
        T.trace(cam, 0, s.spp, px=img, rows=(r0, rows))
    block = multi.ROW_WORDS * multi.max_rows(h, world, 8) * w
    send = np.zeros(block, np.uint32)
    multi.pack_rows(img, w, h, mine, send)
    recv = torch.zeros(block * world, dtype=torch.int32)
    dist.all_gather_into_tensor(recv, torch.from_numpy(send.view(np.int32)))
    got = recv.numpy().view(np.uint32)
    for r in range(world):
        if r != rank:
            multi.unpack_rows(img, w, h, multi.bands(h, world, r, 8), got[r * block:(r + 1) * block])
    whole, _ = T.trace(cam, 0, s.spp)
    same = all(np.array_equal(img[p * w * h: (p + k) * w * h], whole[p * w * h: (p + k) * w * h])
               for p, k in multi.ROW_PLANES)
    out.put((rank, same, mine))
    dist.barrier()
    dist.destroy_process_group()


def test_frame_split_by_tile_rows_and_gathered_on_two_gloo_ranks():
    """The frame split across ranks and gathered equals one whole trace,
    every row plane bit for bit, on every rank (unmeasured on GPUs: this
    pool runs one GPU a call)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, same0, mine0), (_, same1, mine1) = res
    assert same0 and same1
    rows = sorted(r for b in mine0 + mine1 for r in range(b[0], b[0] + b[1]))
    assert rows == list(range(37))  # every row traced by exactly one rank


def test_bands_and_balance():
    from phiray_b200 import multi

    for h, world in ((1080, 1), (1080, 2), (1080, 8), (37, 3)):
        got = sorted(r for k in range(world) for b in multi.bands(h, world, k) for r in range(b[0], b[0] + b[1]))
        assert got == list(range(h))
        assert multi.max_rows(h, world) >= h / world
    costs = [9.0, 7.0, 6.0, 5.0, 4.0, 3.0, 2.0]
    split = multi.balance(costs, 3)
    assert sorted(i for part in split for i in part) == list(range(7))
    loads = [sum(costs[i] for i in part) for part in split]
    assert max(loads) - min(loads) <= max(costs)  # the greedy bound
    assert split[0][0] == 0  # the costliest scene goes first
