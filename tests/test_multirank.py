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


# ---- a batch split over ranks (cvt_b200.shard) ---------------------------------------------
# Seven small pairs of uneven sizes; each rank runs its share through the CPU oracle (the
# same arithmetic as the GPU path) and the per-pair results are gathered to rank 0.
SHARD_PAIRS = [(40, 30, 2, 8.0), (24, 18, 1, 6.0), (36, 22, 2, 10.0), (20, 16, 1, 4.0), (44, 26, 2, 8.0),
               (28, 20, 1, 6.0), (32, 24, 2, 8.0)]


def _shard_result(i):
    """sha256 of pair i's disparity map and final planes (1 iteration, both views, LR check)"""
    import hashlib

    from cvt_b200 import scene
    from oracle.pyoracle import Oracle

    W, H, r, dmax = SHARD_PAIRS[i]
    L, R = scene.generate(500 + i, W, H, 4, 1.0, dmax - 1.0)
    res = Oracle("orc").disparity_map(L, R, r, dmax, 1, pp=1, views=2, fused=0)
    h = hashlib.sha256()
    for k in ("dmap", "planesL", "planesR"):
        h.update(res[k].tobytes())
    return h.hexdigest()


def _shard_rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    from cvt_b200 import shard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        w, h, r, d = zip(*SHARD_PAIRS)
        rank_of, load = shard.partition(w, h, r, d, world)
        mine = shard.my_pairs(rank_of, rank)
        got = shard.gather_to_rank0({i: _shard_result(i) for i in mine}, rank, world)
        q.put((rank, list(map(int, rank_of)), list(load), mine, got))
    finally:
        dist.destroy_process_group()


def test_batch_split_over_two_gloo_ranks(orc):
    import torch.multiprocessing as mp

    from cvt_b200 import shard

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, split0, load0, mine0, got0), (_, split1, load1, mine1, got1) = res
    # every rank computes the same split; the shares are a disjoint cover of the batch
    assert split0 == split1
    assert sorted(mine0 + mine1) == list(range(len(SHARD_PAIRS))) and not set(mine0) & set(mine1)
    # balance: longest processing time first leaves the ranks within one pair's work
    work = [shard.pair_work(*p) for p in SHARD_PAIRS]
    assert abs(load0[0] - load0[1]) <= max(work)
    assert load0[0] == sum(work[i] for i in mine0) and load0[1] == sum(work[i] for i in mine1)
    # rank 0 holds every pair's result, equal to one rank running the whole batch
    assert got1 is None
    assert got0 == {i: _shard_result(i) for i in range(len(SHARD_PAIRS))}


def test_partition_balances_the_uneven_batch():
    """the 64-pair uneven workload over 1, 2, 4 and 8 ranks: a disjoint cover, loads within
    one pair's work of each other, and the split is the same when recomputed"""
    sys.path.insert(0, ROOT)
    from cvt_b200 import scene, shard

    specs = scene.batch_specs()
    args = ([s["width"] for s in specs], [s["height"] for s in specs], [10] * len(specs),
            [s["dispmax"] for s in specs])
    work = [shard.pair_work(*a) for a in zip(*args)]
    for ranks in (1, 2, 4, 8):
        rank_of, load = shard.partition(*args, ranks)
        assert sorted(sum((shard.my_pairs(rank_of, k) for k in range(ranks)), [])) == list(range(len(specs)))
        assert abs(load.sum() - sum(work)) <= 1e-9 * sum(work)
        assert load.max() - load.min() <= max(work)
        again, _ = shard.partition(*args, ranks)
        assert (again == rank_of).all()
    with pytest.raises(Exception):
        shard.partition([10], [10], [1], [0.0], 2)   # a pair without work is refused
