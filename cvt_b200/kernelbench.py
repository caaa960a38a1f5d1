"""Per-kernel timing of the PatchMatch-Huber kernels on one workload, through the C ABI.

    python -m cvt_b200.kernelbench --kernel klt --workload hd --reps 5

Kernels: `cost` (one full-window ASW evaluation per pixel, no early exit), `klt`
(one Gauss-Newton step per pixel), `init`, `propagate` (one view, second
iteration of a real run), `rof` (40 smoothing steps).  Prints one JSON line per
kernel with the mean CUDA-event time of a launch and, for the window kernels,
the time per window sample.
"""
import argparse
import ctypes as C
import json

import numpy as np

from . import _lib, scene

WORKLOADS = {"hd": (1280, 720, 40, 2.0, 120.0, 10, 128.0), "small": (320, 240, 12, 2.0, 30.0, 7, 32.0)}


def window_samples(W, H, r, klt):
    def axis(n, lo_edge):
        i = np.arange(n)
        lo = np.maximum(-r, lo_edge - i)
        hi = np.minimum(r, (n - 1 - lo_edge) - i)
        return np.maximum(hi - lo + 1, 0).sum()
    return int(axis(W, 1 if klt else 0)) * int(axis(H, 0))


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="klt", choices=["cost", "klt", "init", "propagate", "rof", "all"])
    ap.add_argument("--workload", default="hd", choices=sorted(WORKLOADS))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--fused", type=int, default=1)
    args = ap.parse_args()
    W, H, npl, dlo, dhi, r, dmax = WORKLOADS[args.workload]
    L = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    left, right = scene.generate(0, W, H, npl, dlo, dhi)
    f4 = lambda: torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")  # noqa: E731
    views = []
    for img in (left, right):
        d = torch.from_numpy(img).cuda()
        bw, g, dt = f4(), f4(), f4()
        _lib.check(L.pm_k_prep(d.data_ptr(), W, H, W * 4, r, args.fused, bw.data_ptr(), g.data_ptr(), dt.data_ptr(), st))
        views.append((bw, g, dt))
    (bwL, gL, dtL), (bwR, gR, dtR) = views
    planes = f4()
    _lib.check(L.pm_k_init(planes.data_ptr(), bwL.data_ptr(), bwR.data_ptr(), gL.data_ptr(), gR.data_ptr(), W, H, r,
                           dmax, 1, None, None, args.fused, st))
    smooth = f4()
    out, cost = f4(), torch.zeros((H, W), dtype=torch.float32, device="cuda")
    scratch = torch.zeros(L.pm_rof_scratch_bytes(W, H), dtype=torch.uint8, device="cuda")
    lam = (C.c_float * 4)(1.0, 1.0, 1.0, 1.0)
    p = lambda t: t.data_ptr()  # noqa: E731
    calls = {
        "cost": lambda: L.pm_k_cost(p(cost), p(planes), p(bwL), p(bwR), p(gL), p(gR), W, H, r, 1e10, args.fused, st),
        "klt": lambda: L.pm_k_klt(p(out), p(planes), p(bwL), p(bwR), p(gL), p(gR), W, H, r, args.fused, st),
        "init": lambda: L.pm_k_init(p(out), p(bwL), p(bwR), p(gL), p(gR), W, H, r, dmax, 1, None, None, args.fused, st),
        "propagate": lambda: L.pm_k_propagate(p(out), p(planes), p(bwL), p(bwR), p(gL), p(gR), p(smooth), 0.005, W, H,
                                              r, dmax, 1, 1, None, None, None, None, None, args.fused, None, st),
        "rof": lambda: L.pm_k_rof(p(out), p(planes), p(dtL), lam, 40, W, H, p(scratch), st),
    }
    names = list(calls) if args.kernel == "all" else [args.kernel]
    for name in names:
        _lib.check(calls[name]())
        torch.cuda.synchronize()
        ts = []
        for _ in range(args.reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            _lib.check(calls[name]())
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        ms = float(np.mean(ts))
        line = {"kernel": name, "workload": args.workload, "fused": args.fused, "ms": ms, "min_ms": float(min(ts))}
        if name in ("cost", "klt"):
            n = window_samples(W, H, r, name == "klt")
            line["window_samples"] = n
            line["ns_per_sample"] = ms * 1e6 / n
        print(json.dumps(line))


if __name__ == "__main__":
    main()
