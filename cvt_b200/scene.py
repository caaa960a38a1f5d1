"""Procedural stereo pairs for tests and benchmarks (pm_scene_generate).

Shapes and value ranges follow the benchmark workloads: slanted planar patches
(disparity in [dlo, dhi], plane normals with |nx|, |ny| <= 0.3) textured with
4-octave value noise in [0, 255]; the right image is the left warped by the
ground-truth disparity plus noise of standard deviation 2.
"""
import ctypes as C

import numpy as np

from . import _lib


def generate(seed, width, height, nplanes, dlo, dhi, nmax=0.3, sigma=2.0, with_gt=False):
    """Return (left, right) RGBA8 arrays of shape (H, W, 4), plus (gt_disp, gt_normal) if with_gt."""
    L = _lib.lib()
    left = np.zeros((height, width, 4), np.uint8)
    right = np.zeros((height, width, 4), np.uint8)
    gd = np.zeros((height, width), np.float32) if with_gt else None
    gn = np.zeros((height, width, 4), np.float32) if with_gt else None
    st = L.pm_scene_generate(C.c_uint64(seed), width, height, nplanes, dlo, dhi, nmax, sigma,
                             left.ctypes.data, right.ctypes.data, width * 4,
                             gd.ctypes.data if with_gt else None, gn.ctypes.data if with_gt else None)
    _lib.check(st)
    if with_gt:
        return left, right, gd, gn
    return left, right


def workload(name, seed=0):
    """Scenes of the benchmark configurations: 'small' (320x240, 12 planes, d 2..30) and
    'hd' (1280x720, 40 planes, d 2..120)."""
    if name == "small":
        return generate(seed, 320, 240, 12, 2.0, 30.0)
    if name == "hd":
        return generate(seed, 1280, 720, 40, 2.0, 120.0)
    raise ValueError(name)


def batch_specs(n=64, seed=1234, wmin=320, wmax=1920, hmin=240, hmax=1080):
    """Pair specifications of the uneven batched workload: width and height uniform in
    [wmin, wmax] x [hmin, hmax], 8-60 planes, disparity range 0..max(32, width / 10)
    (scene disparities 2..0.9 of that range).  Pair i is generated with seed + i.
    Returns a list of dicts {seed, width, height, planes, dispmax, dlo, dhi}."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        w = int(rng.integers(wmin, wmax + 1))
        h = int(rng.integers(hmin, hmax + 1))
        npl = int(rng.integers(8, 61))
        dmax = float(max(32, w // 10))
        out.append({"seed": seed + i, "width": w, "height": h, "planes": npl, "dispmax": dmax, "dlo": 2.0,
                    "dhi": 0.9 * dmax})
    return out


def batch(specs):
    """(left, right) arrays for each spec of batch_specs."""
    return [generate(s["seed"], s["width"], s["height"], s["planes"], s["dlo"], s["dhi"]) for s in specs]
