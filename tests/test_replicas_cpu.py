"""The multi-GPU path of bench.py on CPU: one process per GPU running an independent replica, with a collective only
for the timing (the slowest rank's time of the timed region) and the whole-job rate over all ranks; checked with two
gloo ranks. The reference arm runs on rank 0 alone and the other ranks leave without work or output."""

import argparse
import os
import socket
from datetime import timedelta

import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, port: int, seconds, queue):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(seconds[rank], 2, dist, device="cpu")
        queue.put((rank, t, bench.whole_job_rate(1000.0, 2, t)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, port, [1.5, 2.5], queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(queue.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in results] == [0, 1]
    assert all(t == 2.5 for _, t, _ in results)
    assert all(v == 800.0 for _, _, v in results)


def test_single_rank_needs_no_collective():
    assert bench.max_over_ranks(3.0, 1, None) == 3.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    bench.run_reference(argparse.Namespace(steps=1, warmup=0, gpus=2))
    assert capsys.readouterr().out == ""
