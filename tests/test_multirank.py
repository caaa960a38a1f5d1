"""The multi-process logic of bench.py as two gloo ranks on CPU: the step time is the
maximum over ranks, each rank works on its own pair, and only rank 0 prints.  The data
path has no collective (each rank runs its own pair), so nothing else is exchanged."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mx = bench.max_over_ranks(10.0 * (rank + 1), world)
        # --impl reference: rank 0 alone runs and prints; the others return without work
        args = type("A", (), {"config": "small", "warmup": 0, "steps": 1, "gpus": world})()
        out = io.StringIO()
        if rank != 0:
            with redirect_stdout(out):
                bench.run_reference(args, bench.WORKLOADS["small"], rank, world)
        q.put((rank, mx, bench.pair_seed(rank), bench.batch_seed(rank), out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

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
    assert [r[1] for r in res] == [20.0, 20.0]
    assert res[0][2] != res[1][2] and res[0][3] != res[1][3]
    assert res[1][4] == ""


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.5, 1) == 12.5
