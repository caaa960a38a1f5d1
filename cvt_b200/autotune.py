"""Autotuner of the batched schedule (pm_disparity_map_batch_device).

A batch of uneven pairs runs as one CUDA graph whose branches execute concurrently;
how many branches share the GPU trades overlap (small pairs and short smoothing
kernels beside long propagate kernels) against contention.  tune_batch times the
caller's own batch, with a short iteration count, at each candidate branch count and
keeps the fastest on the handle (pm_set_batch_branches); results equal those of any
other setting (every pair's arithmetic is the same), only the time differs.
"""
import statistics


def cuda_event_ms(fn):
    """milliseconds of one call of fn between CUDA events on the current stream"""
    import torch

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def tune_batch(pm, lefts, rights, patchsizes, disparitymaxs, iterations=1, candidates=(2, 4, 8, 16), reps=2, pp=1,
               timer=cuda_event_ms):
    """Returns {"branches": best, "ms": {candidate: median ms}} and leaves `best` set on pm.
    Each candidate's first call (graph capture) is not timed; ties go to the earlier candidate."""
    def run():
        pm.disparity_map_batch(lefts, rights, patchsizes, disparitymaxs, iterations, pp=pp)

    timings = {}
    for nb in candidates:
        pm.set_batch_branches(nb)
        timer(run)   # capture, warm
        timings[nb] = statistics.median(timer(run) for _ in range(reps))
    best = min(timings, key=timings.get)
    pm.set_batch_branches(best)
    return {"branches": best, "ms": timings}
