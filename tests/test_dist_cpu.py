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
