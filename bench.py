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
}
# SVPMFlowCL::flow: window half-width, flow range, passes (the reference's MAXITER), and the
# passes of the bounded CPU samples
SVPM = {"r": 3, "flowmax": 128.0, "passes": 200, "cpu_passes": 40, "ref_passes": 20}
# bounded CPU samples (crop of the same scene, same window / range / iterations)
CPU_CROP = {"hd": (256, 144), "small": (320, 240), "4k": (192, 108)}
REF_CROP = {"hd": (96, 54), "small": (96, 72), "4k": (64, 36)}


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


def cpu_sample(kind_pref, crop, wl, scene_lr, mode="disparity"):
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
    extra = {} if kind == "reference" else {"fused": 0}
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
    value = crop[0] * crop[1] * n_it * len(secs) / sum(secs) / 1e6
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
            "cpu_baseline": {"value": value, "unit": "Mpixel·iterations/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "Mpixel·iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if mode == "svpm":
        line["unit"] = line["cpu_baseline"]["unit"] = line["e2e"]["unit"] = metric
    print(json.dumps(line))


def run_batch(args, rank, world, local):
    """--config batch: 64 pairs of uneven sizes (batch_specs: W x H uniform in [320,1920] x
    [240,1080], 8-60 planes, disparity range max(32, W/10)), 21x21 window, 8 (9) iterations,
    both views, LR check, as one graph launch (pm_disparity_map_batch_device), against the
    same 64 pairs as 64 eager single-pair calls.  Each rank runs the whole batch of its own
    seed (weak scaling)."""
    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    specs = scene.batch_specs(seed=batch_seed(rank))
    pairs = scene.batch(specs)
    dl = [torch.from_numpy(a).cuda() for a, _ in pairs]
    dr = [torch.from_numpy(b).cuda() for _, b in pairs]
    rs = [10] * len(specs)
    dm = [s["dispmax"] for s in specs]
    iters = 8
    px_it = sum(s["width"] * s["height"] for s in specs) * executed(iters)
    pm = PMHuberStereo(views=2, fused=True, device=local)
    seq = PMHuberStereo(views=2, fused=True, device=local, use_graph=False)

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
        pm.disparity_map_batch(dl, dr, rs, dm, iters, pp=1)

    def sequential():
        for a, b, r, d in zip(dl, dr, rs, dm):
            seq.disparity_map(a, b, r, d, iters, pp=1)

    # the branch count of the batch graph, picked by timing this batch at 1 iteration (untimed)
    from cvt_b200.autotune import tune_batch
    tuned = tune_batch(pm, dl, dr, rs, dm, iterations=1, candidates=(4, 8, 16))
    for _ in range(args.warmup):
        batched()
    clocks = Clocks(local).start()
    tb = timed(batched, args.steps)
    clk = clocks.stop()
    sequential()
    ts = timed(sequential, args.steps)
    value = world * px_it * args.steps / (tb * 1e-3) / 1e6
    line = {"metric": METRIC, "value": value, "unit": "Mpixel·iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tb / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch", "pairs": len(specs), "megapixels": px_it / executed(iters) / 1e6,
                       "window": 21, "iterations": iters, "iterations_executed": executed(iters), "views": 2,
                       "pp": "lrcheck", "parallelism": "pairs%d" % world,
                       "schedule": "one graph launch, %d concurrent branches (autotuned: %s ms per "
                                   "1-iteration batch)" % (tuned["branches"],
                                                           {k: round(v, 1) for k, v in tuned["ms"].items()}),
                       "l2": "inputs and workspaces (~25 GB) far larger than L2"},
            "sequential": {"value": world * px_it * args.steps / (ts * 1e-3) / 1e6, "ms_per_step": ts / args.steps,
                           "schedule": "64 eager single-pair calls"},
            "clocks": clk}
    if rank == 0:
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


def run_learned(args, wl, rank, world, local):
    """--mode learned: time to plain 8-iteration PatchMatch's cost with the learned proposal"""
    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene
    from cvt_b200.learn import PlaneProposal, make_training_set

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900))
    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    # the proposal's 32 hypotheses cover 124 px at step 1 and 248 px at step 2
    step = 1 if dmax <= 128 else 2
    tw, th, tpairs = (512, 384, 128) if step == 1 else (1024, 576, 64)
    t0 = time.perf_counter()
    feats, target = make_training_set(tpairs, tw, th, seed=100 + 1000 * rank, device=local, step=step, dmax=dmax)
    t1 = time.perf_counter()
    prop = PlaneProposal(seed=rank, device=local, step=step)
    losses = prop.train(feats, target, steps=3000, batch=16, lr=1e-3, seed=rank)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    L, R = scene.generate(pair_seed(rank), W, H, npl, dlo, dhi)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    pm = PMHuberStereo(views=views, fused=True, device=local)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn()
            b.record()
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return out, statistics.median(ms)

    def stats(res):
        c = res["planes_left"][..., 3]
        c = c[c < 2.0]
        return float(c.mean().item()), res["dmap"]

    clocks = Clocks(local).start()
    plain, t_plain = timed(lambda: pm.disparity_map(dL, dR, r, dmax, iters, pp=pp, planes=True))
    c_plain, d_plain = stats(plain)
    keep = d_plain > 0
    # fixed proposal buffers: the disparityMap graph is captured once and replayed
    iL = torch.empty((H, W), dtype=torch.float32, device="cuda")
    iR = torch.empty((H, W), dtype=torch.float32, device="cuda")
    rows, found, found_cost = [], None, None
    for k in ((1, 3, 5, 7, 9) if step == 1 else (3, 5, 9)):
        res, t_k = timed(lambda: pm.disparity_map(dL, dR, r, dmax, k, pp=pp, planes=True,
                                                  initdisparity=prop.propose(dL, dR, 0, out=iL),
                                                  initdisparity_right=prop.propose(dL, dR, 1, out=iR)))
        c_k, d_k = stats(res)
        agree = float(((d_k - d_plain).abs() < 1.0)[keep].float().mean().item())
        rnd, t_r = timed(lambda: pm.disparity_map(dL, dR, r, dmax, k, pp=pp, planes=True))
        c_r, d_r = stats(rnd)
        agree_r = float(((d_r - d_plain).abs() < 1.0)[keep].float().mean().item())
        rows.append({"iterations": k, "learned_ms": t_k, "learned_cost": c_k, "learned_agree_1px": agree,
                     "random_ms": t_r, "random_cost": c_r, "random_agree_1px": agree_r})
        if found is None and c_k <= 1.01 * c_plain and agree >= 0.98:
            found = rows[-1]
        if found_cost is None and c_k <= 1.01 * c_plain:
            found_cost = rows[-1]
    # the learned start reproduces plain's left disparity without the right view: PatchMatch on
    # the left view alone (the left-view-only mode of the 320x240 workload, no LR check), against
    # the same plain run and criteria, with random starts in the same mode beside it
    rows_left = []
    if views == 2:
        pm1 = PMHuberStereo(views=1, fused=True, device=local)
        for k in ((3, 5, 7, 9) if step == 1 else (5, 9)):
            res, t_k = timed(lambda: pm1.disparity_map(dL, dR, r, dmax, k, pp=0, planes=True,
                                                       initdisparity=prop.propose(dL, dR, 0, out=iL)))
            c_k, d_k = stats(res)
            agree = float(((d_k - d_plain).abs() < 1.0)[keep].float().mean().item())
            rnd, t_r = timed(lambda: pm1.disparity_map(dL, dR, r, dmax, k, pp=0, planes=True))
            c_r, d_r = stats(rnd)
            agree_r = float(((d_r - d_plain).abs() < 1.0)[keep].float().mean().item())
            rows_left.append({"iterations": k, "learned_ms": t_k, "learned_cost": c_k, "learned_agree_1px": agree,
                              "random_ms": t_r, "random_cost": c_r, "random_agree_1px": agree_r})
        pm1.close()
    best, best_cfg = found, "both views, LR check"
    for row in rows_left:
        if row["learned_cost"] <= 1.01 * c_plain and row["learned_agree_1px"] >= 0.98:
            if best is None or row["learned_ms"] < best["learned_ms"]:
                best, best_cfg = row, "left view only"
            break
    clk = clocks.stop()
    _, t_prop = timed(lambda: (prop.propose(dL, dR, 0, out=iL), prop.propose(dL, dR, 1, out=iR)))
    prop.check_error()
    value = best["learned_ms"] if best else None
    line = {"metric": "ms to plain-8-iter cost (learned vs random init)", "value": value, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (CNN) / f32 (PatchMatch)", "data": "synthetic",
            "config": {"workload": args.config, "mode": "learned", "width": W, "height": H, "dispmax": dmax,
                       "window": 2 * r + 1, "plain_iterations": iters, "parallelism": "pairs%d" % world,
                       "criterion": "mean cost <= 1.01 x plain and >= 98% of plain's kept pixels within 1 px",
                       "training": {"pairs": tpairs, "maps": 2 * tpairs, "size": "%dx%d" % (tw, th),
                                    "hypothesis_step": step, "steps": 3000, "batch": 16,
                                    "data_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2),
                                    "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-20:]))}},
            "plain": {"ms": t_plain, "cost": c_plain, "fraction_of_plain_time": None},
            "proposal_ms": t_prop, "sweep": rows, "sweep_left_view_only": rows_left,
            "value_from": None if best is None else {"config": best_cfg, "iterations": best["iterations"]},
            "clocks": clk,
            "cost_criterion_only": None if found_cost is None else {
                "iterations": found_cost["iterations"], "ms": found_cost["learned_ms"],
                "fraction_of_plain_time": found_cost["learned_ms"] / t_plain},
            "target": "<= 1/3 of plain's time", "met": bool(best and best["learned_ms"] <= t_plain / 3.0)}
    if best:
        line["plain"]["fraction_of_plain_time"] = best["learned_ms"] / t_plain
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="hd", choices=sorted(WORKLOADS) + ["batch"])
    ap.add_argument("--mode", default="disparity", choices=["disparity", "depth", "pyramid", "vpm", "svpm", "learned"],
                    help="disparityMap (default), depthMap (Huber variant, iterations not made odd), "
                         "disparityMap over 3 pyramid levels (value counts the full-size pixels) or "
                         "VPMStereoCL::disparitySimple, SVPMFlowCL::flow (200 passes) or the learned plane "
                         "proposal (ms to plain 8-iteration cost)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--profile-run", action="store_true",
                    help="only run warmup + steps of the device pipeline (for ncu captures) and print the step times")
    args = ap.parse_args()
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.config == "batch":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched workload is timed on the GPU only"}))
            return
        run_batch(args, rank, world, local)
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

    import torch
    import torch.distributed as dist

    from cvt_b200 import PMHuberStereo, scene
    from cvt_b200 import _lib

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    W, H, npl, dlo, dhi, r, dmax, iters, views, pp = wl
    L, R = scene.generate(pair_seed(rank), W, H, npl, dlo, dhi)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    levels = 3 if args.mode == "pyramid" else 1
    pm = PMHuberStereo(views=views, fused=True, device=local, levels=levels)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    depth = args.mode == "depth"
    run_iters = iters if depth else executed(iters)   # depthMap does not make the count odd

    def call(a, b):
        if depth:
            return pm.depth_map(a, b, r, dmax, iters, pp=pp)
        return pm.disparity_map(a, b, r, dmax, iters, pp=pp)

    if args.profile_run:
        for _ in range(args.warmup):
            call(dL, dR)
        pm.set_profiling(True)
        for k in range(args.steps):
            call(dL, dR)
            print(json.dumps({"step": k, "phase_ms": pm.phase_times()}))
        return

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
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
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
    value = world * px_it * args.steps / (total_ms * 1e-3) / 1e6

    # one more step with per-phase events (eager launches), outside the timed region: the
    # propagate kernels' device time for the roofline and the launch count per step
    flush.fill_(0x5a)
    pm.set_profiling(True)
    call(dL, dR)
    ph = pm.phase_times()
    pm.set_profiling(False)
    prop_ms = ph["propagate"][0]
    launches = ph["total"][1] * args.steps

    # end to end through the host API: pinned host images in, disparity map out
    pl = torch.from_numpy(L).pin_memory().numpy()
    pr = torch.from_numpy(R).pin_memory().numpy()
    call(pl, pr)
    e2e = []
    for k in range(args.steps):
        flush.fill_(k & 0xff)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        call(pl, pr)
        b.record()
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(b))
    e2e_value = world * px_it * args.steps / (max_over_ranks(sum(e2e), world) * 1e-3) / 1e6

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
    import ctypes as C
    pk = C.c_float(0.0)
    if _lib.lib().pm_measure_fp32_peak(local, 200.0, C.byref(pk)) == 0:
        peak = float(pk.value)
    achieved = flops_launch / avg_launch_s / 1e12
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "propagate_%s_dram.json" % args.config)
    if args.mode == "disparity" and os.path.exists(tfile):
        traffic = json.load(open(tfile)).get("bytes_per_launch")
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if peak else None, "traffic": traffic,
            "kernel": "propagate pass (k_prop_chain + k_prop_klt + k_prop_final)", "avg_launch_ms": avg_launch_s * 1e3, "flops_per_launch": flops_launch,
            "peak_source": "FP32 fma probe measured in this run (pm_measure_fp32_peak)"}

    line = {"metric": METRIC, "value": value, "unit": "Mpixel·iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "mode": args.mode, "levels": levels, "width": W, "height": H,
                       "planes": npl, "dispmax": dmax, "window": 2 * r + 1, "iterations": iters,
                       "iterations_executed": run_iters,
                       "views": views, "pp": "lrcheck" if pp == 1 else "none", "parallelism": "pairs%d" % world,
                       "l2": "flushed between steps (256 MiB write)"},
            "e2e": {"value": e2e_value, "unit": "Mpixel·iterations/s", "h2d_bytes_per_step": 2 * W * H * 4,
                    "d2h_bytes_per_step": W * H * 4},
            "roofline": roof, "clocks": clk, "gpu_launches": launches,
            "counters": {"cost_samples": ctr[0], "gn_samples": ctr[1], "cost_evals": ctr[2], "early_exits": ctr[3]},
            "phase_ms": {k: v[0] for k, v in ph.items()}}
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, dt, kind, cores = cpu_sample("port", CPU_CROP[args.config], wl, (L, R), mode=args.mode)
        cw, ch = CPU_CROP[args.config]
        line["cpu_baseline"] = {"value": rate, "unit": "Mpixel·iterations/s", "cores": cores, "kind": kind,
                                "sample": "%dx%d crop of the same pair, same window/range/iterations, %.1f s" % (
                                    cw, ch, dt)}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
