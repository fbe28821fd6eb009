"""The bench's multi-rank logic on CPU with the gloo backend, world size 2 (the GPU run uses NCCL
and one process per GPU; the path shards by instance, so the only collectives are the barrier and
the max-over-ranks time):

  * ranks_timed returns the same time on every rank, the slowest rank's;
  * whole_job_value counts every rank's pairs;
  * the reference arm does its work on rank 0 only (the others return at once).
"""
import os
import sys
import time

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    calls = []

    def step():
        calls.append(1)
        time.sleep(0.05 * (rank + 1))  # rank 1 is the slow one

    def timer(fn):
        t0 = time.perf_counter()
        fn()
        return (time.perf_counter() - t0) * 1e3

    ms = bench.ranks_timed(step, 3, 2, dist, timer, device="cpu")
    q.put((rank, ms, len(calls), bench.whole_job_value(1000, 3, world, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_share_the_slowest_time():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, n0, v0), (r1, ms1, n1, v1) = res
    assert n0 == n1 == 5                       # 2 warm-up + 3 timed steps on each rank
    assert ms0 == ms1                          # every rank reports the maximum
    assert ms0 >= 3 * 0.05 * 2 * 1e3 * 0.95    # ... which is the slow rank's time
    assert v0 == v1 == pytest.approx(1000 * 3 * 2 / (ms0 * 1e-3))


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, REPO)
    import bench
    monkeypatch.setenv("RANK", "1")
    import argparse
    a = argparse.Namespace(config="twolayer3072", steps=1, warmup=0, gpus=2, cpu_budget=1.0)
    t0 = time.perf_counter()
    assert bench.run_reference(a) is None
    assert time.perf_counter() - t0 < 1.0
    assert capsys.readouterr().out == ""
