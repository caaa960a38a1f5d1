"""Autotuner of the batched schedule (pm_disparity_map_batch_device).

A batch of uneven pairs runs either in lockstep (every iteration's propagate passes and
smoothing stages of all pairs as persistent launches over one tile list, the pairs' prep and
post-processing as concurrent graph branches) or branched (each pair's whole pipeline a
branch of one graph).  The knobs trade overlap, tails and cache locality against each other:
the schedule, the propagate CTAs per SM (the persistent grid; 0 = as many as fit), the tile
shape (32 x 4 or 16 x 8 pixels), the tile order (pair after pair, or the pairs' tile rows
interleaved) and the number of concurrent branches.  tune_batch times the caller's own batch, with a short iteration count, under each
candidate and keeps the fastest on the handle; results are the same bit for bit under every
candidate, only the time differs.
"""
import statistics

# candidates tried by default: {schedule, ctas_per_sm, tile_order, tile_w, branches}
DEFAULT_CANDIDATES = (
    {"schedule": "lockstep", "ctas_per_sm": 0, "tile_order": 0, "tile_w": 32, "branches": 16},
    {"schedule": "lockstep", "ctas_per_sm": 0, "tile_order": 0, "tile_w": 16, "branches": 16},
    {"schedule": "lockstep", "ctas_per_sm": 0, "tile_order": 1, "tile_w": 32, "branches": 16},
    {"schedule": "branched", "ctas_per_sm": 0, "tile_order": 0, "tile_w": 32, "branches": 16},
)


def cuda_event_ms(fn):
    """milliseconds of one call of fn between CUDA events on the current stream"""
    import torch

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def _full(c):
    d = {"schedule": "lockstep", "ctas_per_sm": 0, "tile_order": 0, "tile_w": 32, "branches": 16}
    d.update(c)
    return d


def label(c):
    c = _full(c)
    if c["schedule"] == "branched":
        return "branched/%d" % c["branches"]
    return "lockstep/ctas%d/order%d/tile%dx%d/%d" % (c["ctas_per_sm"], c["tile_order"], c["tile_w"],
                                                      128 // c["tile_w"], c["branches"])


def apply(pm, c):
    """set candidate c on the handle of pm"""
    c = _full(c)
    pm.set_batch_schedule(c["schedule"], c["ctas_per_sm"], c["tile_order"], c["tile_w"])
    pm.set_batch_branches(c["branches"])


def tune_batch(pm, lefts, rights, patchsizes, disparitymaxs, iterations=1, candidates=DEFAULT_CANDIDATES, reps=2,
               pp=1, timer=cuda_event_ms):
    """Returns {"best": candidate, "ms": {label: median ms}} and leaves the best candidate set on
    pm.  Each candidate's first call (graph capture, table upload) is not timed; ties go to the
    earlier candidate."""
    def run():
        pm.disparity_map_batch(lefts, rights, patchsizes, disparitymaxs, iterations, pp=pp)

    timings, best, best_ms = {}, None, None
    for c in candidates:
        apply(pm, c)
        timer(run)   # capture, warm
        ms = statistics.median(timer(run) for _ in range(reps))
        timings[label(c)] = ms
        if best_ms is None or ms < best_ms:
            best, best_ms = c, ms
    apply(pm, best)
    return {"best": best, "ms": timings}
