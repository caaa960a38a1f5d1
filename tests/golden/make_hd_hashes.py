"""Writes tests/golden/hd_strict_hashes.json: digests of the strict CPU restatement's result
for the 1280x720 workload (the generator's pair of seed 0 with 40 planes and disparities
2-120, disparity range 0-128, 21x21 window, 8 iterations (9 executed), both views,
left-right check at 1 px / 5 degrees, normal map requested).

The full-size fields are too large to commit (the planes alone are 29 MB), so the fixture
holds a SHA-256 digest of every row of each output (disparity map, normal map, final planes
of both views) and of each whole field.  NaNs are canonicalised to 0x7fc00000 before
hashing, since the comparison treats every NaN as equal.  The restatement equals the
reference's kernels compiled from their own source bit for bit (tests/test_oracle.py), so
a GPU result with the same digests is the reference's result.

Usage: python tests/golden/make_hd_hashes.py    (about 15 minutes on 8 host threads)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CONFIG = {"seed": 0, "width": 1280, "height": 720, "planes": 40, "dlo": 2.0, "dhi": 120.0, "patch_radius": 10,
          "dispmax": 128.0, "iterations": 8, "pp": 1, "views": 2, "arith": "strict"}
FIELDS = ("dmap", "normal", "planes_left", "planes_right")


def canonical(a):
    """float32 array with every NaN as 0x7fc00000, as little-endian bytes"""
    a = np.ascontiguousarray(a, np.float32).copy()
    a[np.isnan(a)] = np.float32("nan")
    b = a.view(np.uint32)
    b[np.isnan(a)] = 0x7FC00000
    return b.astype("<u4")


def digests(fields):
    """{name: {"rows": [hex per row], "all": hex}} of the fields (numpy arrays, H x W [x 4])"""
    out = {}
    for k in FIELDS:
        c = canonical(fields[k])
        rows = [hashlib.sha256(c[y].tobytes()).hexdigest()[:32] for y in range(c.shape[0])]
        out[k] = {"rows": rows, "all": hashlib.sha256(c.tobytes()).hexdigest()}
    return out


def main():
    from cvt_b200 import scene
    from oracle import build as obuild
    from oracle.pyoracle import Oracle

    obuild.build_oracle()
    c = CONFIG
    L, R = scene.generate(c["seed"], c["width"], c["height"], c["planes"], c["dlo"], c["dhi"])
    t = time.time()
    res = Oracle("orc").disparity_map(L, R, c["patch_radius"], c["dispmax"], c["iterations"], pp=c["pp"],
                                      views=c["views"], fused=0)
    secs = time.time() - t
    fields = {"dmap": res["dmap"], "normal": res["normal"], "planes_left": res["planesL"],
              "planes_right": res["planesR"]}
    kept = res["dmap"] > 0
    cost = res["planesL"][..., 3]
    doc = {"config": c, "generator": "tests/golden/make_hd_hashes.py", "cpu_seconds": round(secs, 1),
           "threads": os.cpu_count(), "kept_fraction": float(kept.mean()),
           "mean_cost_left": float(cost[cost < 2.0].mean()), "digests": digests(fields)}
    with open(os.path.join(HERE, "hd_strict_hashes.json"), "w") as f:
        json.dump(doc, f, indent=0)
    print("wrote hd_strict_hashes.json in %.0f s" % secs)


if __name__ == "__main__":
    main()
