"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one independent replica per GPU (the step has no exchange
between ranks); the only cross-rank steps are the barrier around the timed
region and the reductions of its numbers: the max of the per-rank device
times and the sum of the per-rank particle counts.  The reference arm runs
on rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    w, r, _ = bench._dist_init()
    bench._barrier(w)
    ms = bench._allreduce(10.0 + rank, w, "max")      # per-rank device time
    total = bench._allreduce(1000.0 * (rank + 1), w, "sum")  # per-rank particles
    bench._barrier(w)
    q.put((r, w, ms, total))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_bench():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 11.0, 3000.0), (1, 2, 11.0, 3000.0)]


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=3, gpus=2)
    assert bench.run_reference(args, world=2, rank=1) == 0
    assert capsys.readouterr().out == ""
