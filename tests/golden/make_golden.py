"""Generate the golden fixtures of tests/golden/ from the reference kernels.

The outputs come from cvt/cl/kernel/pmhstereo.cl, PDDiffTensor.cl,
PDDROFDiffTensor.cl, PDDHuberDiffTensor.cl, pyr/pyrdown.cl, pyr/pyrupmul.cl,
VPMStereo.cl, gradxy.cl and SVPMFlow.cl compiled from their own source through the OpenCL-C shim
(oracle/build.py -> oracle/_ref/libpmref.so), driven by the restated host loops
of PMHuberStereo::disparityMap / depthMap, VPMStereoCL::disparitySimple and SVPMFlowCL::flow.  Inputs are seeded procedural scenes from
cvt_b200.scene.  Run from the repository root where the reference tree is
available:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cvt_b200 import scene  # noqa: E402
from oracle import build as obuild  # noqa: E402
from oracle.pyoracle import Oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name: (seed, W, H, nplanes, dlo, dhi, r, dmax, iterations, pp, views, init_from_gt)
CASES = {
    "lr_40x28": (3, 40, 28, 5, 2.0, 10.0, 3, 12.0, 3, 1, 2, False),
    "odd_33x19": (7, 33, 19, 4, 1.0, 8.0, 2, 10.0, 2, 2, 2, False),
    "left_36x24": (4, 36, 24, 4, 2.0, 8.0, 2, 10.0, 2, 0, 1, False),
    "init_40x28": (5, 40, 28, 5, 2.0, 10.0, 3, 12.0, 1, 2, 2, True),
}

# coarse-to-fine runs (pyramid levels > 1); name: (seed, W, H, nplanes, dlo, dhi, r, dmax,
# iterations, pp, views, levels, init_from_gt)
PYR_CASES = {
    "pyr_96x64": (11, 96, 64, 6, 2.0, 20.0, 2, 24.0, 1, 1, 2, 2, False),
    "pyr3_100x70": (12, 100, 70, 6, 2.0, 30.0, 1, 32.0, 1, 2, 2, 3, True),
}

# VPMStereoCL::disparitySimple; name: (seed, W, H, nplanes, dlo, dhi, r, dmax, iterations, init_from_gt)
VPM_CASES = {
    "vpm_48x32": (21, 48, 32, 5, 2.0, 12.0, 3, 16.0, 3, False),
    "vpm_init_41x27": (22, 41, 27, 4, 1.0, 9.0, 2, 12.0, 2, True),
}

# SVPMFlowCL::flow; name: (seed, W, H, nplanes, dlo, dhi, r, flowmax, passes).  The reference
# runs 200 passes; the fixtures keep 7 and 12 (the TV pull starts at pass 5).
SVPM_CASES = {
    "svpm_40x30": (31, 40, 30, 4, 1.0, 8.0, 2, 8.0, 7),
    "svpm_53x37": (32, 53, 37, 5, 1.0, 10.0, 3, 24.0, 12),
}


def make_case(ref, name, spec):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, pp, views, init = spec
    left, right, gtd, gtn = scene.generate(seed, W, H, npl, dlo, dhi, with_gt=True)
    initd = gtd.copy() if init else None
    if init:
        initd[::5, ::3] = 0.0   # some pixels without a given disparity take the random init
    res = ref.disparity_map(left, right, r, dmax, iters, pp=pp, views=views, initdisp=initd, dump=True)
    arrays = {"left": left, "right": right, "dmap": res["dmap"], "normal": res["normal"],
              "planesL": res["planesL"], "spec": np.array([seed, W, H, npl, dlo, dhi, r, dmax, iters, pp, views,
                                                           int(init)], np.float64)}
    if views == 2:
        arrays["planesR"] = res["planesR"]
    if init:
        arrays["initdisp"] = initd
    for (stage, it), v in res["stages"].items():
        arrays["stage_%s_%d" % (stage, it)] = v
    # per-kernel fixtures on the first view
    bwL, gL, dtL = ref.prep(left, r)
    bwR, gR, dtR = ref.prep(right, r)
    arrays.update(bwL=bwL, gL=gL, dtL=dtL, bwR=bwR, gR=gR, dtR=dtR)
    rng = np.random.default_rng(seed)
    planes = res["stages"][("init_left", -1)].copy()
    # a few awkward planes: non-finite, steep, far outside the image
    planes[0, 0] = [np.nan, 0, 0, 0]
    planes[1, 1] = [np.inf, 1, 1, 0]
    planes[2, 2] = [40.0, 3.0, -900.0, 0]
    planes[3, 3] = [1.0, 0.0, -1e6, 0]
    arrays["k_planes"] = planes
    arrays["k_cost_inf"] = ref.cost(planes, bwL, bwR, gL, gR, r, 1e10)
    arrays["k_cost_02"] = ref.cost(planes, bwL, bwR, gL, gR, r, 0.2)
    arrays["k_klt"] = ref.klt(planes, bwL, bwR, gL, gR, r)
    smooth = (rng.random((H, W, 4), np.float32) * np.array([0.2, 0.2, 1.0, 1.0], np.float32)).astype(np.float32)
    arrays["k_smooth"] = smooth
    pout, vn, vv, _ = ref.propagate(planes, bwL, bwR, gL, gR, smooth, 0.37, r, dmax, 1, 1)
    arrays.update(k_prop=pout, k_prop_vn=vn, k_prop_vv=vv)
    nd = ref.normal_depth(planes, 1.0 / dmax, 1)
    arrays["k_nd"] = nd
    arrays["k_rof"] = ref.rof(nd, dtL, [1.3, 1.3, 1.3, 1.0], 40)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)


def make_pyr_case(ref, name, spec):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, pp, views, levels, init = spec
    left, right, gtd, gtn = scene.generate(seed, W, H, npl, dlo, dhi, with_gt=True)
    initd = gtd.copy() if init else None
    if init:
        initd[::4, ::3] = 0.0
    res = ref.disparity_map(left, right, r, dmax, iters, pp=pp, views=views, initdisp=initd, levels=levels,
                            dump=True)
    arrays = {"left": left, "right": right, "dmap": res["dmap"], "normal": res["normal"],
              "planesL": res["planesL"], "planesR": res["planesR"],
              "spec": np.array([seed, W, H, npl, dlo, dhi, r, dmax, iters, pp, views, levels, int(init)], np.float64)}
    if init:
        arrays["initdisp"] = initd
    for (stage, it), v in res["stages"].items():
        if "init" in stage:   # each level's initial planes (the rest is pinned by the outputs)
            arrays["stage_%s_%d" % (stage, it)] = v
    # per-kernel fixtures: one pyramid step down of the left image and one step up of a
    # disparity and a normal field (the sizes of the first level step)
    W1, H1 = int(np.float32(W) * np.float32(0.35)), int(np.float32(H) * np.float32(0.35))
    arrays["k_pyrdown"] = ref.pyrdown(left, W1, H1)
    rng = np.random.default_rng(seed)
    d1 = (rng.random((H1, W1), np.float32) * 10).astype(np.float32)
    n1 = rng.standard_normal((H1, W1, 4)).astype(np.float32)
    up = np.float32(W) / np.float32(W1)
    arrays.update(k_pyr_d1=d1, k_pyr_n1=n1, k_pyrup_d=ref.pyrup_mul(d1, W, H, [up] * 4),
                  k_pyrup_n=ref.pyrup_mul(n1, W, H, [1.0] * 4))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)


# depthMap runs; name: (seed, W, H, nplanes, dlo, dhi, r, dmax, iterations, dscale, pp, init_from_gt)
DEPTH_CASES = {
    "depth_48x32": (21, 48, 32, 5, 2.0, 14.0, 2, 16.0, 6, -1.0, 1, False),
    "depth_init_44x30": (22, 44, 30, 5, 2.0, 12.0, 2, 14.0, 3, 0.5, 2, True),
}


def make_depth_case(ref, name, spec):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, dscale, pp, init = spec
    left, right, gtd, gtn = scene.generate(seed, W, H, npl, dlo, dhi, with_gt=True)
    initd = gtd.copy() if init else None
    if init:
        initd[::4, ::3] = 0.0
    res = ref.depth_map(left, right, r, dmax, iters, dscale=dscale, pp=pp, initdisp=initd, dump=True)
    arrays = {"left": left, "right": right, "dmap": res["dmap"], "normal": res["normal"],
              "planesL": res["planesL"], "planesR": res["planesR"],
              "spec": np.array([seed, W, H, npl, dlo, dhi, r, dmax, iters, dscale, pp, int(init)], np.float64)}
    if init:
        arrays["initdisp"] = initd
    for (stage, it), v in res["stages"].items():
        if stage.startswith("init") or it == 0:
            arrays["stage_%s_%d" % (stage, it)] = v
    # per-kernel fixtures: the raw prep, fill_state of a plane field with gaps, the Huber smoother
    colour, grad, dt = ref.prep_raw(left, 12.0)
    arrays.update(k_colour=colour, k_grad=grad, k_dt12=dt)
    planes = res["stages"][("prop_left", 0)].copy()
    planes[3, :, 3] = -1.0
    planes[5, 7:20, 3] = -2.0
    arrays["k_fs_planes"] = planes
    arrays["k_fill_state_l"] = ref.fill_state(planes, 1.0 / dmax, 1)
    arrays["k_fill_state_r"] = ref.fill_state(planes, 1.0 / dmax, 0)
    arrays["k_huber"] = ref.huber(arrays["k_fill_state_l"], dt, [2.3] * 4, 1e-4, 40)
    arrays["k_huber_odd"] = ref.huber(arrays["k_fill_state_l"], dt, [2.3] * 4, 1e-4, 7)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)


def make_vpm_case(ref, name, spec):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, init = spec
    left, right, gtd, gtn = scene.generate(seed, W, H, npl, dlo, dhi, with_gt=True)
    initd = None
    if init:
        initd = gtd.copy()
        initd[::4, ::3] = -1.0          # below the range: the van der Corput init
        initd[2::5, 1::4] = dmax + 1.0  # above the range: the van der Corput init
    disp, states = ref.vpm_disparity_simple(left, right, r, iters, dmax, initd)
    arrays = {"left": left, "right": right, "disparity": disp, "states": states,
              "spec": np.array([seed, W, H, npl, dlo, dhi, r, dmax, iters, int(init)], np.float64)}
    if init:
        arrays["initdisp"] = initd
    # per-kernel fixtures: both gradients, init, two iterations (the neighbour offsets rotate
    # with the iteration index), the scaled disparity
    g0, g1 = ref.vpm_grad(left), ref.vpm_grad(right)
    s0 = ref.vpm_init(left, g0, right, g1, r, dmax, initd)
    s1 = ref.vpm_iter(s0, left, g0, right, g1, r, dmax, 0)
    s5 = ref.vpm_iter(s1, left, g0, right, g1, r, dmax, 5)
    arrays.update(k_grad0=g0, k_grad1=g1, k_init=s0, k_iter0=s1, k_iter5=s5,
                  k_disp_scaled=ref.vpm_disparity(s5, 1.0 / dmax))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)


def make_svpm_case(ref, name, spec):
    seed, W, H, npl, dlo, dhi, r, flowmax, passes = spec
    first, second = scene.generate(seed, W, H, npl, dlo, dhi)
    flow, states, duals = ref.svpm_flow(first, second, r, flowmax, passes)
    arrays = {"first": first, "second": second, "flow": flow, "states": states, "duals": duals,
              "spec": np.array([seed, W, H, npl, dlo, dhi, r, flowmax, passes], np.float64)}
    # per-kernel fixtures: init, the first pass (no pull) and pass 6 (pull on) from fixed inputs
    s0 = ref.svpm_init(first, second, r, flowmax)
    s1, p1 = ref.svpm_prop(s0, np.zeros_like(s0), first, second, r, flowmax, 1)
    s6, p6 = ref.svpm_prop(s1, p1 + 0.25, first, second, r, flowmax, 6)
    arrays.update(k_init=s0, k_prop1=s1, k_dual1=p1, k_prop6=s6, k_dual6=p6, k_flow=ref.svpm_to_flow(s6))
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)


def main():
    so = obuild.build_ref()
    if so is None:
        sys.exit("the reference kernels are not available (no reference tree and no prebuilt oracle/_ref)")
    obuild.build_oracle()
    ref = Oracle("ref")
    for name, spec in CASES.items():
        make_case(ref, name, spec)
        print("wrote", name)
    for name, spec in PYR_CASES.items():
        make_pyr_case(ref, name, spec)
        print("wrote", name)
    for name, spec in DEPTH_CASES.items():
        make_depth_case(ref, name, spec)
        print("wrote", name)
    for name, spec in VPM_CASES.items():
        make_vpm_case(ref, name, spec)
        print("wrote", name)
    for name, spec in SVPM_CASES.items():
        make_svpm_case(ref, name, spec)
        print("wrote", name)


if __name__ == "__main__":
    main()
