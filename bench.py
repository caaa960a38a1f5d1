"""Benchmark of the PatchMatch-Huber stereo path (cvt::PMHuberStereo::disparityMap).

Workload (default `hd`): one 1280x720 RGBA8 pair from the procedural generator
(40 slanted planes, disparity 2-120 px), disparity range 0-128, 21x21 window
(patch half-width 10), 8 iterations (9 executed, the reference rounds up to
odd), both views with view propagation, left-right check at 1 px / 5 deg.
A step is one full disparityMap call: prep, init, 9 x (propagate L + R,
40-step ROF smoothing per view), LR check, disparity conversion.

Metric: Mpixel*iterations/s = width * height * executed iterations / step time.
  value  device time (CUDA events per step) with inputs resident in HBM; L2 is
         flushed (256 MiB write) between steps, outside the timed events
  e2e    the public host API (numpy in, numpy out) including the host->device
         copy of both images from pinned memory and the device->host copy of the
         disparity map, timed with CUDA events around the call
One process per GPU: each rank processes its own pair (weak scaling, no
collective on the data path); the step time is the maximum over ranks.

`--mode vpm` measures the sibling path cvt::VPMStereoCL::disparitySimple
(VPMStereoCL.cpp:54-85) on the same pair: 21x21 window, disparity range 0-128,
8 iterations, the same metric (one iteration = one vpmstereo_iter_simple pass).

`--mode svpm` measures the optical-flow sibling cvt::SVPMFlowCL::flow
(SVPMFlowCL.cpp:58-89) on the same pair taken as two frames: 7x7 window, flow
range 128, the reference's 200 passes; metric Mpixel*passes/s.

`--mode learned` measures the second half of the metric, "ms to plain-8-iter cost": a
BF16 plane-proposal CNN (cvt_b200/learn.py; tcgen05 convolutions) is trained on the
GPU (outside the timed region) on 128 procedural 512x384 pairs (both views) against plain
8-iteration PatchMatch, then on the hd pair the GPU time of proposals for both views + k
PatchMatch iterations is
timed for growing k until its mean matching cost is within 1% of plain 8-iteration
PatchMatch and its disparity within 1 px of it on >= 98% of the pixels plain
PatchMatch keeps (LR check); value = that time in ms (null if no k up to 9 reaches it).

`--impl reference` times the reference's CPU implementation instead: the
reference kernel sources compiled through the OpenCL-C shim (oracle/_ref) when
built, otherwise the CPU restatement (oracle/), on a bounded crop of the same
workload, using every host thread.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpixel·iterations/s"
WORKLOADS = {
    # name: (W, H, planes, dlo, dhi, patch half-width, dispmax, iterations, views, pp)
    "hd": (1280, 720, 40, 2.0, 120.0, 10, 128.0, 8, 2, 1),
    "small": (320, 240, 12, 2.0, 30.0, 7, 32.0, 4, 1, 0),
    # one pair of the 4K configuration (3840x2160, 120 planes, disparity 0-256, 35x35 window)
    "4k": (3840, 2160, 120, 2.0, 240.0, 17, 256.0, 8, 2, 1),
    # a quarter-size pair with the hd window (the small case of ncu captures of the hd kernels)
    "quarter": (640, 360, 20, 2.0, 60.0, 10, 64.0, 2, 2, 1),
}
# SVPMFlowCL::flow: window half-width, flow range, passes (the reference's MAXITER), and the
# passes of the bounded CPU samples
SVPM = {"r": 3, "flowmax": 128.0, "passes": 200, "cpu_passes": 40, "ref_passes": 20}
# bounded CPU samples (crop of the same scene, same window / range / iterations)
CPU_CROP = {"hd": (256, 144), "small": (320, 240), "4k": (192, 108), "quarter": (160, 90)}
REF_CROP = {"hd": (96, 54), "small": (96, 72), "4k": (64, 36), "quarter": (64, 36)}


def executed(iters):
    return iters | 1


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and "Active" in s[3 + i]
                          and "Not" not in s[3 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def max_over_ranks(ms, world):
    """Maximum over ranks of a per-rank elapsed time in ms (one all-reduce, made outside the
    timed region; the tensor lives where the process group's backend wants it)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def pair_seed(rank):
    """scene seed of a rank's pair: every rank works on its own pair"""
    return rank


def batch_seed(rank):
    return 1234 + 1000 * rank


def window_positions(W, H, r):
    """sum over pixels of in-image window positions (the support weights computed once per pixel)"""
    def axis(n):
        i = np.arange(n)
        return (np.minimum(r, n - 1 - i) + np.minimum(r, i) + 1).sum()
    return int(axis(W)) * int(axis(H))


def window_scale(crop, full, r):
    """in-image window positions per pixel of a crop over those of the full image: a small crop
    clips more of every window at its borders, so its per-pixel work is lower; a crop's rate
    times this factor is its rate normalised to the full image's per-pixel work"""
    (cw, ch), (W, H) = crop, full
    return (window_positions(cw, ch, r) / (cw * ch)) / (window_positions(W, H, r) / (W * H))


def cpu_sample(kind_pref, crop, wl, scene_lr, mode="disparity", fused=0):
    """time the CPU implementation on a crop; returns (Mpx*it/s, seconds, kind, cores)"""
    from oracle import build as obuild
    from oracle.pyoracle import Oracle, available

    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    cw, ch = crop
    L, R = scene_lr
    L = np.ascontiguousarray(L[:ch, :cw])
    R = np.ascontiguousarray(R[:ch, :cw])
    kind = "port"
    if kind_pref == "reference" and available("ref"):
        kind = "reference"
    if kind == "port":
        obuild.build_oracle()
    o = Oracle("ref" if kind == "reference" else "orc")
    t0 = time.perf_counter()
    extra = {} if kind == "reference" else {"fused": int(fused)}
    if mode == "svpm":
        passes = SVPM["ref_passes"] if kind == "reference" else SVPM["cpu_passes"]
        o.svpm_flow(L, R, SVPM["r"], SVPM["flowmax"], passes)
        dt = time.perf_counter() - t0
        return cw * ch * passes / dt / 1e6, dt, kind, os.cpu_count()
    if mode == "vpm":
        o.vpm_disparity_simple(L, R, r, iters, dmax)
    elif mode == "depth":
        o.depth_map(L, R, r, dmax, iters, pp=pp, views=views, **extra)
    else:
        o.disparity_map(L, R, r, dmax, iters, pp=pp, views=views, levels=3 if mode == "pyramid" else 1, **extra)
    dt = time.perf_counter() - t0
    rate = cw * ch * (iters if mode in ("depth", "vpm") else executed(iters)) / dt / 1e6
    return rate, dt, kind, os.cpu_count()


def run_reference(args, wl, rank, world):
    """--impl reference: the reference's CPU implementation, rank 0 only"""
    if rank != 0:
        return
    from cvt_b200 import scene

    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    crop = REF_CROP[args.config]
    L, R = scene.generate(0, crop[0], crop[1], max(2, npl * crop[0] * crop[1] // (W * H) + 2), dlo, dhi)
    mode = args.mode if args.mode in ("disparity", "vpm", "svpm") else "disparity"
    n_it = {"vpm": iters, "svpm": SVPM["ref_passes"]}.get(mode, executed(iters))
    for _ in range(args.warmup):
        cpu_sample("reference", crop, wl, (L, R), mode=mode)
    rates, secs = [], []
    kind, cores = None, None
    for _ in range(args.steps):
        rate, dt, kind, cores = cpu_sample("reference", crop, wl, (L, R), mode=mode)
        rates.append(rate)
        secs.append(dt)
    raw = crop[0] * crop[1] * n_it * len(secs) / sum(secs) / 1e6
    # normalised to the full image's window work per pixel (SVPM's 7x7 windows: the same rule)
    norm = window_scale(crop, (W, H), SVPM["r"] if mode == "svpm" else r)
    value = raw * norm
    if mode == "svpm":
        sample = "%dx%d crop, SVPMFlowCL::flow, window %dx%d, flowmax %g, %d passes" % (
            crop[0], crop[1], 2 * SVPM["r"] + 1, 2 * SVPM["r"] + 1, SVPM["flowmax"], n_it)
    elif mode == "vpm":
        sample = "%dx%d crop, VPMStereoCL::disparitySimple, window %dx%d, dispmax %g, %d iterations" % (
            crop[0], crop[1], 2 * r + 1, 2 * r + 1, dmax, n_it)
    else:
        sample = "%dx%d crop, window %dx%d, dispmax %g, %d iterations executed, %s" % (
            crop[0], crop[1], 2 * r + 1, 2 * r + 1, dmax, n_it, "both views, LR check" if views == 2 else
            "left view")
    metric = "Mpixel·passes/s" if mode == "svpm" else METRIC
    line = {"impl": "reference", "metric": metric, "value": value, "unit": "Mpixel·iterations/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "mode": mode, "sample": sample},
            "crop_value": raw, "window_normalisation": norm,
            "cpu_baseline": {"value": value, "unit": "Mpixel·iterations/s", "cores": cores, "kind": kind,
                             "sample": sample + "; rate normalised to the full image's in-image window positions per "
                                                "pixel (x %.4f)" % norm},
            "e2e": {"value": value, "unit": "Mpixel·iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if mode == "svpm":
        line["unit"] = line["cpu_baseline"]["unit"] = line["e2e"]["unit"] = metric
    print(json.dumps(line))


def run_batch(args, rank, world, local):
    """--config batch: 64 pairs of uneven sizes (batch_specs: W x H uniform in [320,1920] x
    [240,1080], 8-60 planes, disparity range max(32, W/10)), 21x21 window, 8 (9) iterations,
    both views, LR check, as one graph launch (pm_disparity_map_batch_device), against the
    same pairs as eager single-pair calls.  With N ranks the one seeded list of 64 pairs is split
    over them (pm_batch_partition: longest processing time first by W*H*(2r+1)^2*dispmax; no
    collective on the data path), each rank runs its share as one graph, and the per-pair mean
    costs are gathered to rank 0 afterwards (strong scaling: the total work is fixed)."""
    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene, shard

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    specs = scene.batch_specs(seed=batch_seed(0))
    rs_all = [10] * len(specs)
    rank_of, load = shard.partition([s["width"] for s in specs], [s["height"] for s in specs], rs_all,
                                    [s["dispmax"] for s in specs], world)
    mine = shard.my_pairs(rank_of, rank)
    pairs = scene.batch([specs[i] for i in mine])
    dl = [torch.from_numpy(a).cuda() for a, _ in pairs]
    dr = [torch.from_numpy(b).cuda() for _, b in pairs]
    rs = [rs_all[i] for i in mine]
    dm = [specs[i]["dispmax"] for i in mine]
    iters = 8
    px_it_all = sum(s["width"] * s["height"] for s in specs) * executed(iters)
    fused = args.arith == "fused"
    pm = PMHuberStereo(views=2, fused=fused, device=local)
    seq = PMHuberStereo(views=2, fused=fused, device=local, use_graph=False)

    def timed(fn, steps):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(steps):
            ev[k][0].record()
            fn()
            ev[k][1].record()
        torch.cuda.synchronize()
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), world)

    def batched():
        return pm.disparity_map_batch(dl, dr, rs, dm, iters, pp=1)

    def sequential():
        for a, b, r, d in zip(dl, dr, rs, dm):
            seq.disparity_map(a, b, r, d, iters, pp=1)

    # the schedule of the batch (lockstep persistent launches or branches, CTAs per SM, tile
    # order, branch count), picked by timing this batch at 1 iteration (untimed)
    from cvt_b200.autotune import label, tune_batch
    tuned = tune_batch(pm, dl, dr, rs, dm, iterations=1, reps=1)
    for _ in range(args.warmup):
        batched()
    clocks = Clocks(local).start()
    tb = timed(batched, args.steps)
    clk = clocks.stop()
    res = pm.disparity_map_batch(dl, dr, rs, dm, iters, pp=1, planes=True)   # after the timed region
    torch.cuda.synchronize()
    costs = {}
    for i, rr in zip(mine, res):
        c = rr["planes_left"][..., 3]
        costs[i] = float(c[c < 2.0].mean().item())
    gathered = shard.gather_to_rank0(costs, rank, world)   # one host gather after the data path
    sequential()
    ts = timed(sequential, args.steps)
    value = px_it_all * args.steps / (tb * 1e-3) / 1e6
    line = {"metric": METRIC, "value": value, "unit": "Mpixel·iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tb / args.steps, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch", "arith": args.arith, "pairs": len(specs),
                       "megapixels": px_it_all / executed(iters) / 1e6, "window": 21, "iterations": iters,
                       "iterations_executed": executed(iters), "views": 2, "pp": "lrcheck",
                       "parallelism": "pairs split over %d ranks (pm_batch_partition)" % world,
                       "rank_load_share": [float(x) for x in (load / load.sum())],
                       "schedule": "one graph launch per rank: %s (autotuned; ms per 1-iteration batch: %s)" % (
                           label(tuned["best"]), {k: round(v, 1) for k, v in tuned["ms"].items()}),
                       "autotuned": tuned["best"],
                       "l2": "inputs and workspaces (~25 GB) far larger than L2"},
            "sequential": {"value": px_it_all * args.steps / (ts * 1e-3) / 1e6, "ms_per_step": ts / args.steps,
                           "schedule": "eager single-pair calls"},
            "clocks": clk}
    if rank == 0:
        line["pairs_gathered"] = len(gathered)
        line["mean_cost_over_pairs"] = float(np.mean(list(gathered.values())))
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_4kbatch(args, rank, world, local):
    """--config 4kbatch: 8 pairs at 3840x2160 (120 planes, disparity range 0-256, 35x35 window,
    both views, LR check): the learned proposal for both views + 3 PatchMatch iterations, all 8
    pairs as one captured CUDA graph, against plain random-init 8-iteration PatchMatch of the same
    pairs as another captured graph, on the same GPU.  Reported: both graphs' device times, the
    mean-cost gap and the fraction of plain's kept pixels within 1 px.  With N ranks the 8 pairs
    are split over them (pm_batch_partition)."""
    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene, shard
    from cvt_b200.learn import PlaneProposal, default_weights

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=1800))
    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = WORKLOADS["4k"]
    n, k_learned = 8, 3
    rank_of, _ = shard.partition([W] * n, [H] * n, [r] * n, [dmax] * n, world)
    mine = shard.my_pairs(rank_of, rank)
    imgs = [scene.generate(100 + i, W, H, npl, dlo, dhi) for i in mine]
    dL = [torch.from_numpy(a).cuda() for a, _ in imgs]
    dR = [torch.from_numpy(b).cuda() for _, b in imgs]
    pm = PMHuberStereo(views=views, fused=args.arith == "fused", device=local)
    prop = PlaneProposal.load(default_weights(), device=local)
    bufs = [(torch.empty((H, W), device="cuda"), torch.empty((H, W, 4), device="cuda"),
             torch.empty((H, W), device="cuda"), torch.empty((H, W, 4), device="cuda")) for _ in mine]

    def plain_all():
        return [pm.disparity_map(a, b, r, dmax, iters, pp=pp, planes=True) for a, b in zip(dL, dR)]

    def learned_all():
        out = []
        for (a, b), (dl, nl, drr, nr) in zip(zip(dL, dR), bufs):
            prop.propose(a, b, dmax, 0, dl, nl)
            prop.propose(a, b, dmax, 1, drr, nr)
            out.append(pm.disparity_map(a, b, r, dmax, k_learned, pp=pp, planes=True, initdisparity=dl,
                                        initnormalmap=nl, initdisparity_right=drr, initnormalmap_right=nr))
        return out

    # size every workspace with one eager call of each kind on the first pair, then capture
    pm.disparity_map(dL[0], dR[0], r, dmax, 1, pp=pp, planes=True)
    prop.propose(dL[0], dR[0], dmax, 0, *bufs[0][:2])
    torch.cuda.synchronize()
    graphs, outs = {}, {}
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    for name, fn in (("plain", plain_all), ("learned", learned_all)):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            g.capture_begin()
            outs[name] = fn()
            g.capture_end()
        graphs[name] = g
    torch.cuda.current_stream().wait_stream(s)
    clocks = Clocks(local).start()
    ms = {}
    for name in ("plain", "learned"):
        t = []
        for _ in range(max(args.steps, 1)):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            if world > 1:
                dist.barrier()
            a.record()
            graphs[name].replay()
            b.record()
            torch.cuda.synchronize()
            t.append(a.elapsed_time(b))
        ms[name] = max_over_ranks(statistics.median(t), world)
    clk = clocks.stop()
    prop.check_error()
    rows = {}
    for i, po, lo in zip(mine, outs["plain"], outs["learned"]):
        cp = po["planes_left"][..., 3]
        cl = lo["planes_left"][..., 3]
        keep = po["dmap"] > 0
        rows[i] = {"plain_cost": float(cp[cp < 2].mean().item()), "learned_cost": float(cl[cl < 2].mean().item()),
                   "within_1px": float(((lo["dmap"] - po["dmap"]).abs() < 1.0)[keep].float().mean().item())}
    got = shard.gather_to_rank0(rows, rank, world)
    for g in graphs.values():
        del g
    if rank == 0:
        pc = float(np.mean([v["plain_cost"] for v in got.values()]))
        lc = float(np.mean([v["learned_cost"] for v in got.values()]))
        line = {"metric": "learned + 3 iterations vs plain 8 (8 x 3840x2160, one captured graph each)",
                "value": ms["learned"], "unit": "ms", "n_gpus": world, "steps": max(args.steps, 1), "warmup": 0,
                "ms_per_step": ms["learned"], "higher_is_better": False, "scaling": "strong" if world > 1 else "weak",
                "vs_baseline": None, "dtype": "bf16 (CNN) / f32 (PatchMatch, %s)" % args.arith, "data": "synthetic",
                "config": {"workload": "4kbatch", "pairs": n, "width": W, "height": H, "planes": npl,
                           "dispmax": dmax, "window": 2 * r + 1, "plain_iterations": iters,
                           "learned_iterations": k_learned, "iterations_executed": [executed(iters), executed(k_learned)],
                           "views": views, "pp": "lrcheck", "parallelism": "pairs split over %d ranks" % world},
                "plain_ms": ms["plain"], "fraction_of_plain_time": ms["learned"] / ms["plain"],
                "mean_cost_plain": pc, "mean_cost_learned": lc, "cost_gap": lc / pc - 1.0,
                "within_1px_of_plain": float(np.mean([v["within_1px"] for v in got.values()])),
                "per_pair": {str(k): v for k, v in sorted(got.items())}, "clocks": clk}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_vpm(args, wl, rank, world, local):
    """--mode vpm: VPMStereoCL::disparitySimple on the workload's pair (same size, window,
    disparity range and iteration count), one pair per rank (weak scaling)."""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from cvt_b200 import _lib, scene
    from cvt_b200.vpm import VPMStereoCL

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    L, R = scene.generate(pair_seed(rank), W, H, npl, dlo, dhi)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    vpm = VPMStereoCL(r, iters, dmax, device=local)
    vpm0 = VPMStereoCL(r, 0, dmax, device=local)   # gradients, init and |x' - x| only
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # counting pass (untimed): window taps of the iteration kernel
    vpm.set_counting(True)
    vpm.disparity_simple(dL, dR)
    torch.cuda.synchronize()
    taps = vpm.counters()
    vpm.set_counting(False)
    for _ in range(args.warmup):
        vpm.disparity_simple(dL, dR)
        vpm0.disparity_simple(dL, dR)
    torch.cuda.synchronize()

    def timed(v):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            ev[k][0].record()
            v.disparity_simple(dL, dR)
            ev[k][1].record()
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    clocks = Clocks(local).start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = timed(vpm)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms), world)
    base_ms = timed(vpm0)   # outside the timed region: the per-call work other than the iterations
    px_it = W * H * iters
    value = world * px_it * args.steps / (total_ms * 1e-3) / 1e6

    # end to end through the host API: pinned host images in, disparity map out
    pl = torch.from_numpy(L).pin_memory().numpy()
    pr = torch.from_numpy(R).pin_memory().numpy()
    vpm.disparity_simple(pl, pr)
    e2e = []
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        vpm.disparity_simple(pl, pr)
        b.record()
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(b))
    e2e_value = world * px_it * args.steps / (max_over_ranks(sum(e2e), world) * 1e-3) / 1e6

    # roofline of the iteration kernel (FP32-bound): 61 flop per cost-window tap + 178 flop per
    # Gauss-Newton tap (taps counted by the kernel), over its average duration = (step time
    # - step time of a 0-iteration call) / iterations
    flops_launch = (61.0 * taps[0] + 178.0 * taps[1]) / iters
    iter_ms = (statistics.median(step_ms) - statistics.median(base_ms)) / iters
    pk = C.c_float(0.0)
    peak = float(pk.value) if _lib.lib().pm_measure_fp32_peak(local, 200.0, C.byref(pk)) == 0 else None
    achieved = flops_launch / (iter_ms * 1e-3) / 1e12
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "vpm_iter_%s_dram.json" % args.config)
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get("bytes_per_launch")
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None, "traffic": traffic, "kernel": "k_iter (vpmstereo_iter_simple)",
            "avg_launch_ms": iter_ms, "flops_per_launch": flops_launch,
            "peak_source": "FP32 fma probe measured in this run (pm_measure_fp32_peak)"}
    line = {"metric": METRIC, "value": value, "unit": "Mpixel·iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "mode": "vpm", "width": W, "height": H, "planes": npl,
                       "dispmax": dmax, "window": 2 * r + 1, "iterations": iters, "parallelism": "pairs%d" % world,
                       "l2": "flushed between steps (256 MiB write)"},
            "e2e": {"value": e2e_value, "unit": "Mpixel·iterations/s", "h2d_bytes_per_step": 2 * W * H * 4,
                    "d2h_bytes_per_step": W * H * 4},
            "roofline": roof, "clocks": clk, "gpu_launches": (4 + iters) * args.steps,
            "counters": {"cost_taps": taps[0], "gn_taps": taps[1]},
            "phase_ms": {"iterations": iter_ms * iters, "rest": statistics.median(base_ms)}}
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, dt, kind, cores = cpu_sample("port", CPU_CROP[args.config], wl, (L, R), mode="vpm")
        cw, ch = CPU_CROP[args.config]
        line["cpu_baseline"] = {"value": rate, "unit": "Mpixel·iterations/s", "cores": cores, "kind": kind,
                                "sample": "%dx%d crop of the same pair, same window/range/iterations, %.1f s" % (
                                    cw, ch, dt)}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_svpm(args, wl, rank, world, local):
    """--mode svpm: SVPMFlowCL::flow on the workload's pair as two frames (7x7 window, flow
    range 128, 200 passes), one pair per rank (weak scaling)."""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from cvt_b200 import _lib, scene
    from cvt_b200.svpm import SVPMFlowCL

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    W, H, npl, dlo, dhi = wl[:5]
    r, fmax, passes = SVPM["r"], SVPM["flowmax"], SVPM["passes"]
    L, R = scene.generate(pair_seed(rank), W, H, npl, dlo, dhi)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    f = SVPMFlowCL(device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    metric = "Mpixel·passes/s"

    f.set_counting(True)   # counting pass (untimed): cost-window taps of the propagation passes
    f.flow(dL, dR, r, fmax, passes)
    torch.cuda.synchronize()
    taps = f.counters()
    f.set_counting(False)
    for _ in range(args.warmup):
        f.flow(dL, dR, r, fmax, passes)
    torch.cuda.synchronize()

    def timed(n):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            ev[k][0].record()
            f.flow(dL, dR, r, fmax, n)
            ev[k][1].record()
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    clocks = Clocks(local).start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = timed(passes)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms), world)
    base_ms = timed(0)   # outside the timed region: colour planes, init, flow extraction
    px_it = W * H * passes
    value = world * px_it * args.steps / (total_ms * 1e-3) / 1e6

    pl = torch.from_numpy(L).pin_memory().numpy()
    pr = torch.from_numpy(R).pin_memory().numpy()
    f.flow(pl, pr, r, fmax, passes)
    e2e = []
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        f.flow(pl, pr, r, fmax, passes)
        b.record()
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(b))
    e2e_value = world * px_it * args.steps / (max_over_ranks(sum(e2e), world) * 1e-3) / 1e6

    # roofline of the propagation pass (FP32-bound): 52 flop per cost-window tap (taps counted by
    # the kernel), over its average duration = (step time - time of a 0-pass call) / passes
    flops_launch = 52.0 * taps / passes
    pass_ms = (statistics.median(step_ms) - statistics.median(base_ms)) / passes
    pk = C.c_float(0.0)
    peak = float(pk.value) if _lib.lib().pm_measure_fp32_peak(local, 200.0, C.byref(pk)) == 0 else None
    achieved = flops_launch / (pass_ms * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None, "traffic": None,
            "kernel": "k_prop (svpmflow_prop_local_tv_admm)", "avg_launch_ms": pass_ms, "flops_per_launch": flops_launch,
            "peak_source": "FP32 fma probe measured in this run (pm_measure_fp32_peak)"}
    line = {"metric": metric, "value": value, "unit": metric, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "mode": "svpm", "width": W, "height": H, "planes": npl,
                       "flowmax": fmax, "window": 2 * r + 1, "passes": passes, "parallelism": "pairs%d" % world,
                       "l2": "flushed between steps (256 MiB write)"},
            "e2e": {"value": e2e_value, "unit": metric, "h2d_bytes_per_step": 2 * W * H * 4,
                    "d2h_bytes_per_step": W * H * 8},
            "roofline": roof, "clocks": clk, "gpu_launches": (4 + passes) * args.steps,
            "counters": {"cost_taps": taps},
            "phase_ms": {"passes": pass_ms * passes, "rest": statistics.median(base_ms)}}
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, dt, kind, cores = cpu_sample("port", CPU_CROP[args.config], wl, (L, R), mode="svpm")
        cw, ch = CPU_CROP[args.config]
        line["cpu_baseline"] = {"value": rate, "unit": metric, "cores": cores, "kind": kind,
                                "sample": "%dx%d crop of the same frames, same window/range, %d passes, %.1f s" % (
                                    cw, ch, SVPM["cpu_passes"], dt)}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def learned_sweep(pm, prop, dL, dR, wl, timed, plain_ms, plain_res, ks=(1, 2, 4, 6, 8)):
    """ms of learned init (proposals for both views + k iterations, both views and the LR check
    as plain runs) for growing k, against plain random-init PatchMatch's result `plain_res`
    (the configured 8 iterations): mean final matching cost within 1% of plain's and >= 98% of
    plain's kept pixels within 1 px.  Random-init runs of the same k stand beside each row."""
    import torch

    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl

    def stats(res):
        c = res["planes_left"][..., 3]
        c = c[c < 2.0]
        return float(c.mean().item()), res["dmap"]

    c_plain, d_plain = stats(plain_res)
    keep = d_plain > 0
    # fixed proposal buffers: the disparityMap graph is captured once and replayed
    dl = torch.empty((H, W), dtype=torch.float32, device="cuda")
    nl = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    drr = torch.empty((H, W), dtype=torch.float32, device="cuda")
    nr = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")

    def learned(k):
        prop.propose(dL, dR, dmax, 0, dl, nl)
        prop.propose(dL, dR, dmax, 1, drr, nr)
        return pm.disparity_map(dL, dR, r, dmax, k, pp=pp, planes=True, initdisparity=dl, initnormalmap=nl,
                                initdisparity_right=drr, initnormalmap_right=nr)

    rows, found = [], None
    for k in ks:
        res, t_k = timed(lambda: learned(k))
        c_k, d_k = stats(res)
        agree = float(((d_k - d_plain).abs() < 1.0)[keep].float().mean().item())
        rnd, t_r = timed(lambda: pm.disparity_map(dL, dR, r, dmax, k, pp=pp, planes=True))
        c_r, d_r = stats(rnd)
        agree_r = float(((d_r - d_plain).abs() < 1.0)[keep].float().mean().item())
        row = {"iterations": k, "iterations_executed": executed(k), "learned_ms": t_k,
               "learned_cost_ratio": c_k / c_plain, "learned_agree_1px": agree, "random_ms": t_r,
               "random_cost_ratio": c_r / c_plain, "random_agree_1px": agree_r}
        rows.append(row)
        if found is None and c_k <= 1.01 * c_plain and agree >= 0.98:
            found = row
    # plain random-init PatchMatch run on past the configured 8 iterations, against its own
    # 8-iteration result: how far plain itself still moves (the agreement criterion compares with
    # a field that is not converged)
    longer = []
    for k in (12, 16):
        rnd, t_r = timed(lambda: pm.disparity_map(dL, dR, r, dmax, k, pp=pp, planes=True))
        c_r, d_r = stats(rnd)
        longer.append({"iterations": k, "iterations_executed": executed(k), "random_ms": t_r,
                       "random_cost_ratio": c_r / c_plain,
                       "random_agree_1px": float(((d_r - d_plain).abs() < 1.0)[keep].float().mean().item())})
    _, t_prop = timed(lambda: (prop.propose(dL, dR, dmax, 0, dl, nl), prop.propose(dL, dR, dmax, 1, drr, nr)))
    prop.check_error()
    cfg4 = next((x for x in rows if x["iterations"] == 2), None)
    return {"metric": "ms to plain-8-iter cost", "value": found["learned_ms"] if found else None, "unit": "ms",
            "iterations": found["iterations"] if found else None,
            "fraction_of_plain_time": (found["learned_ms"] / plain_ms) if found else None,
            "met_one_third": bool(found and found["learned_ms"] <= plain_ms / 3.0),
            "plain_ms": plain_ms, "plain_mean_cost": c_plain, "proposal_ms_both_views": t_prop,
            "criterion": "mean cost <= 1.01 x plain and >= 98% of plain's kept pixels within 1 px, both views, "
                         "LR check",
            "learned_plus_2": cfg4, "sweep": rows, "plain_longer": longer}


def run_learned(args, wl, rank, world, local):
    """--mode learned: the learned plane proposal (committed weights, cvt_b200/weights/proposal.npz,
    trained by cvt_b200/train_proposal.py) against plain 8-iteration PatchMatch on the workload's
    pair: "ms to plain-8-iter cost" and the sweep over iteration counts"""
    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene
    from cvt_b200.learn import PlaneProposal, default_weights

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900))
    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    L, R = scene.generate(pair_seed(rank), W, H, npl, dlo, dhi)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    pm = PMHuberStereo(views=views, fused=args.arith == "fused", device=local)
    prop = PlaneProposal.load(default_weights(), device=local)
    timed = make_timer(args.warmup, args.steps)
    clocks = Clocks(local).start()
    plain, t_plain = timed(lambda: pm.disparity_map(dL, dR, r, dmax, iters, pp=pp, planes=True))
    out = learned_sweep(pm, prop, dL, dR, wl, timed, t_plain, plain, ks=(1, 2, 4, 6, 8))
    clk = clocks.stop()
    line = {"metric": "ms to plain-8-iter cost (learned vs random init)", "value": out["value"], "unit": "ms",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["value"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 (CNN) / f32 (PatchMatch, %s)" % args.arith, "data": "synthetic",
            "config": {"workload": args.config, "mode": "learned", "width": W, "height": H, "dispmax": dmax,
                       "window": 2 * r + 1, "plain_iterations": iters, "parallelism": "pairs%d" % world,
                       "weights": os.path.relpath(default_weights(), ROOT)},
            "learned": out, "clocks": clk}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def make_timer(warmup, steps):
    """fn -> (last result, median ms over `steps` calls after `warmup`), CUDA events per call"""
    import torch

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        out = None
        for _ in range(steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn()
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return out, statistics.median(ms)

    return timed


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="hd", choices=sorted(WORKLOADS) + ["batch", "4kbatch"])
    ap.add_argument("--mode", default="disparity", choices=["disparity", "depth", "pyramid", "vpm", "svpm", "learned"],
                    help="disparityMap (default), depthMap (Huber variant, iterations not made odd), "
                         "disparityMap over 3 pyramid levels (value counts the full-size pixels) or "
                         "VPMStereoCL::disparitySimple, SVPMFlowCL::flow (200 passes) or the learned plane "
                         "proposal (ms to plain 8-iteration cost)")
    ap.add_argument("--arith", default="strict", choices=["strict", "fused"],
                    help="strict (default): every operation rounds as in the reference kernels, bit-exact with them; "
                         "fused: the window loops contract multiply-adds into fma (faster, not bit-exact)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--no-extra", action="store_true",
                    help="hd: skip the other arithmetic's and the learned proposal's objects of the line")
    ap.add_argument("--profile-run", action="store_true",
                    help="only run warmup + steps of the device pipeline (for ncu captures) and print the step times")
    args = ap.parse_args()
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.config in ("batch", "4kbatch"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched workloads are timed on the GPU only"}))
            return
        (run_batch if args.config == "batch" else run_4kbatch)(args, rank, world, local)
        return
    wl = WORKLOADS[args.config]
    if args.impl == "reference":
        run_reference(args, wl, rank, world)
        return
    if args.mode == "vpm":
        run_vpm(args, wl, rank, world, local)
        return
    if args.mode == "svpm":
        run_svpm(args, wl, rank, world, local)
        return
    if args.mode == "learned":
        run_learned(args, wl, rank, world, local)
        return

    run_disparity(args, wl, rank, world, local)


def measure_disparity(args, wl, pm, call, dL, dR, L, R, local, world, levels, run_iters, steps, flush):
    """time the workload's call on device-resident inputs (value), through the host API with the
    copies (e2e), and one profiled call (per-phase device times, the propagate roofline)"""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from cvt_b200 import _lib

    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    # counting pass (untimed): window samples of the propagate launches
    pm.set_counting(True)
    call(dL, dR)
    torch.cuda.synchronize()
    ctr = pm.counters()
    pm.set_counting(False)
    for _ in range(args.warmup):
        call(dL, dR)
    torch.cuda.synchronize()

    # timed region: the product path (each call one CUDA graph launch, enqueued back to back)
    clocks = Clocks(local).start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(k & 0xff)
        ev[k][0].record()
        call(dL, dR)
        ev[k][1].record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(sum(step_ms), world)
    px_it = W * H * run_iters
    value = world * px_it * steps / (total_ms * 1e-3) / 1e6

    # one more step with per-phase events (eager launches), outside the timed region: the
    # propagate kernels' device time for the roofline and the launch count per step
    flush.fill_(0x5a)
    pm.set_profiling(True)
    call(dL, dR)
    ph = pm.phase_times()
    pm.set_profiling(False)
    prop_ms = ph["propagate"][0]
    launches = ph["total"][1] * steps

    # end to end through the host API: pinned host images in, disparity map out
    pl = torch.from_numpy(L).pin_memory().numpy()
    pr = torch.from_numpy(R).pin_memory().numpy()
    call(pl, pr)
    e2e = []
    for k in range(steps):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        call(pl, pr)
        b.record()
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(b))
    e2e_value = world * px_it * steps / (max_over_ranks(sum(e2e), world) * 1e-3) / 1e6

    # roofline of the propagate kernel (FP32-bound): algorithmic flops per launch
    # = 10 per hoisted support weight + 41 per cost-window sample + 129 per
    #   Gauss-Newton window sample, over the launch's measured average duration
    # one propagate pass = the three kernels of one view and iteration (pm_propagate.cu)
    sizes = [(W, H)]
    for _ in range(1, levels):
        sizes.append((int(np.float32(sizes[-1][0]) * np.float32(0.35)), int(np.float32(sizes[-1][1]) * np.float32(0.35))))
    nlaunch = views * run_iters * levels
    wpos = sum(window_positions(w, h, r) for w, h in sizes) * views * run_iters
    flops_launch = (10.0 * wpos + 41.0 * ctr[0] + 129.0 * ctr[1]) / nlaunch
    avg_launch_s = prop_ms / nlaunch * 1e-3
    peak = None
    pk = C.c_float(0.0)
    if _lib.lib().pm_measure_fp32_peak(local, 200.0, C.byref(pk)) == 0:
        peak = float(pk.value)
    achieved = flops_launch / avg_launch_s / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None, "traffic": None,
            "kernel": "propagate pass (k_prop_chain + k_prop_klt + k_prop_final)", "avg_launch_ms": avg_launch_s * 1e3,
            "flops_per_launch": flops_launch,
            "peak_source": "FP32 fma probe measured in this run (pm_measure_fp32_peak)"}
    return {"value": value, "ms_per_step": total_ms / steps, "e2e_value": e2e_value, "roofline": roof, "clocks": clk,
            "launches": launches, "ctr": ctr, "phases": ph, "step_ms": step_ms}


def run_disparity(args, wl, rank, world, local):
    """the default: disparityMap (or depthMap / the 3-level pyramid) on the workload's pair, one
    pair per rank (weak scaling), in the chosen arithmetic (strict: bit-exact with the reference
    kernels; the default); on the hd workload also the other arithmetic and the learned
    proposal's "ms to plain-8-iter cost" beside it"""
    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    L, R = scene.generate(pair_seed(rank), W, H, npl, dlo, dhi)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    levels = 3 if args.mode == "pyramid" else 1
    fused = args.arith == "fused"
    pm = PMHuberStereo(views=views, fused=fused, device=local, levels=levels)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    depth = args.mode == "depth"
    run_iters = iters if depth else executed(iters)   # depthMap does not make the count odd

    def caller(p):
        def call(a, b):
            if depth:
                return p.depth_map(a, b, r, dmax, iters, pp=pp)
            return p.disparity_map(a, b, r, dmax, iters, pp=pp)
        return call

    call = caller(pm)
    if args.profile_run:
        for _ in range(args.warmup):
            call(dL, dR)
        pm.set_profiling(True)
        for k in range(args.steps):
            call(dL, dR)
            print(json.dumps({"step": k, "phase_ms": pm.phase_times()}))
        return

    m = measure_disparity(args, wl, pm, call, dL, dR, L, R, local, world, levels, run_iters, args.steps, flush)
    tfile = os.path.join(ROOT, "profiles", "propagate_%s_%s_dram.json" % (args.config, args.arith))
    if args.mode == "disparity" and os.path.exists(tfile):
        m["roofline"]["traffic"] = json.load(open(tfile)).get("bytes_per_launch")
    line = {"metric": METRIC, "value": m["value"], "unit": "Mpixel·iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "mode": args.mode, "arith": args.arith, "levels": levels,
                       "width": W, "height": H, "planes": npl, "dispmax": dmax, "window": 2 * r + 1,
                       "iterations": iters, "iterations_executed": run_iters,
                       "views": views, "pp": "lrcheck" if pp == 1 else "none", "parallelism": "pairs%d" % world,
                       "l2": "flushed between steps (256 MiB write)",
                       "parity": "strict: bit-exact with the reference kernels (tests/test_gpu_parity.py, "
                                 "hd fixture tests/golden/hd_strict_hashes.json)" if not fused else
                                 "fused: fma-contracted window loops, not bit-exact with the reference"},
            "e2e": {"value": m["e2e_value"], "unit": "Mpixel·iterations/s", "h2d_bytes_per_step": 2 * W * H * 4,
                    "d2h_bytes_per_step": W * H * 4},
            "roofline": m["roofline"], "clocks": m["clocks"], "gpu_launches": m["launches"],
            "counters": {"cost_samples": m["ctr"][0], "gn_samples": m["ctr"][1], "cost_evals": m["ctr"][2],
                         "early_exits": m["ctr"][3]},
            "phase_ms": {k: v[0] for k, v in m["phases"].items()}}
    extras = args.config == "hd" and args.mode == "disparity" and not args.no_extra
    if extras:
        # the other arithmetic on the same pair, fewer steps (outside the headline's timed region)
        other = "fused" if not fused else "strict"
        pm2 = PMHuberStereo(views=views, fused=not fused, device=local)
        m2 = measure_disparity(args, wl, pm2, caller(pm2), dL, dR, L, R, local, world, levels, run_iters,
                               min(args.steps, 5), flush)
        line[other] = {"value": m2["value"], "ms_per_step": m2["ms_per_step"], "e2e": m2["e2e_value"],
                       "roofline_frac": m2["roofline"]["frac"], "roofline_achieved": m2["roofline"]["achieved"],
                       "propagate_ms": m2["phases"]["propagate"][0], "steps": min(args.steps, 5)}
        pm2.close()
        # the learned proposal against plain 8-iteration PatchMatch (committed weights)
        from cvt_b200.learn import PlaneProposal, default_weights

        if os.path.exists(default_weights()):
            timed = make_timer(1, 3)   # plain and learned calls timed alike (planes requested in both)
            plain, t_plain = timed(lambda: pm.disparity_map(dL, dR, r, dmax, iters, pp=pp, planes=True))
            line["learned"] = learned_sweep(pm, PlaneProposal.load(default_weights(), device=local), dL, dR, wl,
                                            timed, t_plain, plain)
        else:
            line["learned"] = {"unavailable": "no committed weights at %s" % os.path.relpath(default_weights(), ROOT)}
    if rank == 0 and world == 1 and not args.no_cpu:
        crop = CPU_CROP[args.config]
        rate, dt, kind, cores = cpu_sample("port", crop, wl, (L, R), mode=args.mode, fused=int(fused))
        norm = window_scale(crop, (W, H), r)
        line["cpu_baseline"] = {"value": rate * norm, "unit": "Mpixel·iterations/s", "cores": cores, "kind": kind,
                                "sample": "%dx%d crop of the same pair, same window/range/iterations, %s arithmetic, "
                                          "%.1f s; crop rate %.5f normalised to the full image's in-image window "
                                          "positions per pixel (x %.4f)" % (crop[0], crop[1], args.arith, dt, rate, norm)}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
