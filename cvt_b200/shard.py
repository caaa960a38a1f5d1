"""Split of a stereo batch over GPUs (one process per GPU), the multi-GPU form of the
batched workloads.

Stereo pairs are independent, so a batch shards by pair with no collective on the data
path: every rank computes the same split (pm_batch_partition, longest processing time
first by W*H*(2r+1)^2*dispmax), runs its own pairs, and small per-pair results travel to
rank 0 in one host gather at the end.  The reference runs one pair per call on a single
device (cvt/cl/OpenCL.cpp:30-45) and has no counterpart.
"""
import ctypes as C

import numpy as np

from . import _lib


def partition(widths, heights, patchsizes, dispmaxs, ranks):
    """rank of each pair and the work given to each rank (pm_batch_partition)"""
    n = len(widths)
    w = np.ascontiguousarray(widths, np.int32)
    h = np.ascontiguousarray(heights, np.int32)
    r = np.ascontiguousarray(patchsizes, np.int32)
    d = np.ascontiguousarray(dispmaxs, np.float32)
    if not (len(h) == len(r) == len(d) == n):
        raise ValueError("per-pair arrays differ in length")
    rank_of = np.zeros(n, np.int32)
    load = np.zeros(max(int(ranks), 1), np.float64)
    _lib.check(_lib.lib().pm_batch_partition(n, int(ranks), w.ctypes.data, h.ctypes.data, r.ctypes.data,
                                             d.ctypes.data, rank_of.ctypes.data, load.ctypes.data))
    return rank_of, load


def pair_work(width, height, patchsize, dispmax):
    """the balancing weight of one pair"""
    return float(width) * float(height) * float(2 * patchsize + 1) ** 2 * float(dispmax)


def my_pairs(rank_of, rank):
    """indices of the pairs of `rank`, in batch order"""
    return [int(i) for i in np.flatnonzero(np.asarray(rank_of) == rank)]


def gather_to_rank0(items, rank, world):
    """per-pair results {pair index: value} of every rank, merged on rank 0 (None elsewhere);
    one host-side gather over the process group, after the data path"""
    if world <= 1:
        return dict(items)
    import torch.distributed as dist

    got = [None] * world if rank == 0 else None
    dist.gather_object(dict(items), got, dst=0)
    if rank != 0:
        return None
    out = {}
    for part in got:
        dup = set(out) & set(part)
        if dup:
            raise RuntimeError("pairs %s were processed by two ranks" % sorted(dup))
        out.update(part)
    return out
