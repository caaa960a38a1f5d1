"""The CPU oracle: pinned against the reference kernels (golden fixtures and, where
the reference tree is present, a live build of its own source), plus known-answer
tests for the arithmetic it fixes."""
import numpy as np
import pytest

from conftest import depth_cases, golden_cases, load_golden, pyramid_cases, svpm_cases, vpm_cases
from oracle.pyoracle import bits_equal


def spec_of(g):
    s = g["spec"]
    seed, W, H, npl, dlo, dhi, r, dmax, iters, pp, views, init = s
    return dict(W=int(W), H=int(H), r=int(r), dmax=float(dmax), iters=int(iters), pp=int(pp), views=int(views),
                init=bool(init))


@pytest.mark.parametrize("case", golden_cases())
def test_restatement_matches_reference_golden(orc, case):
    """Every stage of PMHuberStereo::disparityMap, bit for bit (strict arithmetic)."""
    g = load_golden(case)
    s = spec_of(g)
    res = orc.disparity_map(g["left"], g["right"], s["r"], s["dmax"], s["iters"], pp=s["pp"], views=s["views"],
                            initdisp=g.get("initdisp"), dump=True, fused=0)
    for (stage, it), v in res["stages"].items():
        ok = bits_equal(v, g["stage_%s_%d" % (stage, it)])
        assert ok.all(), (case, stage, it, ok.mean())
    for k in ("dmap", "normal", "planesL") + (("planesR",) if s["views"] == 2 else ()):
        assert bits_equal(res[k], g[k]).all(), (case, k)


@pytest.mark.parametrize("case", golden_cases())
def test_restatement_kernels_match_reference_golden(orc, case):
    g = load_golden(case)
    s = spec_of(g)
    r, dmax = s["r"], s["dmax"]
    bwL, gL, dtL = orc.prep(g["left"], r)
    bwR, gR, dtR = orc.prep(g["right"], r)
    for a, k in ((bwL, "bwL"), (gL, "gL"), (dtL, "dtL"), (bwR, "bwR"), (gR, "gR"), (dtR, "dtR")):
        assert bits_equal(a, g[k]).all(), k
    P = g["k_planes"]
    assert bits_equal(orc.cost(P, bwL, bwR, gL, gR, r, 1e10), g["k_cost_inf"]).all()
    assert bits_equal(orc.cost(P, bwL, bwR, gL, gR, r, 0.2), g["k_cost_02"]).all()
    assert bits_equal(orc.klt(P, bwL, bwR, gL, gR, r), g["k_klt"]).all()
    out, vn, vv, vs = orc.propagate(P, bwL, bwR, gL, gR, g["k_smooth"], 0.37, r, dmax, 1, 1)
    assert bits_equal(out, g["k_prop"]).all()
    assert (vn == g["k_prop_vn"]).all()
    keep = np.minimum(vn, 2)
    for k in range(2):
        m = keep > k
        assert bits_equal(vv[..., 4 * k:4 * k + 4][m], g["k_prop_vv"][..., 4 * k:4 * k + 4][m]).all()
    nd = orc.normal_depth(P, 1.0 / dmax, 1)
    assert bits_equal(nd, g["k_nd"]).all()
    assert bits_equal(orc.rof(nd, dtL, [1.3, 1.3, 1.3, 1.0], 40), g["k_rof"]).all()


def test_restatement_matches_reference_live(orc, ref):
    """A fresh seed through both CPU builds (needs the reference tree or a prebuilt oracle/_ref)."""
    from cvt_b200 import scene

    L, R = scene.generate(11, 37, 23, 5, 1.0, 9.0)
    a = orc.disparity_map(L, R, 2, 11.0, 2, pp=1, dump=True)
    b = ref.disparity_map(L, R, 2, 11.0, 2, pp=1, dump=True)
    for k in a["stages"]:
        assert bits_equal(a["stages"][k], b["stages"][k]).all(), k
    assert bits_equal(a["dmap"], b["dmap"]).all()


@pytest.mark.parametrize("W,H,r", [(1, 1, 2), (3, 2, 1), (5, 7, 4), (17, 3, 3)])
def test_tiny_images_match_reference(orc, ref, W, H, r):
    """Images smaller than the window and than a 16x16 work-group."""
    from cvt_b200 import scene

    L, R = scene.generate(W * 100 + H, W, H, 2, 1.0, 3.0)
    a = orc.disparity_map(L, R, r, 4.0, 1, pp=2, dump=True)
    b = ref.disparity_map(L, R, r, 4.0, 1, pp=2, dump=True)
    for k in a["stages"]:
        assert bits_equal(a["stages"][k], b["stages"][k]).all(), k
    assert bits_equal(a["dmap"], b["dmap"]).all()
    assert bits_equal(a["normal"], b["normal"]).all()


def _sweep_cases(n=8, seed=2024):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        W, H, r, it = int(rng.integers(9, 33)), int(rng.integers(5, 21)), int(rng.integers(0, 5)), int(rng.integers(1, 4))
        views = int(rng.choice([1, 2]))
        pp = 0 if views == 1 else int(rng.choice([0, 1, 2]))
        out.append((W, H, r, it, views, pp, float(rng.uniform(3, 12)), bool(rng.integers(0, 2))))
    return out


@pytest.mark.parametrize("W,H,r,it,views,pp,dmax,init", _sweep_cases())
def test_restatement_matches_reference_parameter_sweep(orc, ref, W, H, r, it, views, pp, dmax, init):
    """Seeded draws of size, window radius (0 included), iterations, views, post-processing and
    disparity range; half start from a given disparity whose negative entries take the random
    start per pixel (pmhstereo_init_disparity_normal).  Every stage equal bit for bit."""
    from cvt_b200 import scene

    L, R = scene.generate(W * 31 + H, W, H, 3, 0.5, dmax - 1.0)
    idisp = np.random.default_rng(W + H).uniform(-1.0, dmax, (H, W)).astype(np.float32) if init else None
    a = orc.disparity_map(L, R, r, dmax, it, pp=pp, views=views, initdisp=idisp, dump=True)
    b = ref.disparity_map(L, R, r, dmax, it, pp=pp, views=views, initdisp=idisp, dump=True)
    assert a["stages"].keys() == b["stages"].keys()
    for k in a["stages"]:
        assert bits_equal(a["stages"][k], b["stages"][k]).all(), k
    for k in ("dmap", "normal", "planesL"):
        assert bits_equal(a[k], b[k]).all(), k


def _sibling_cases(seed=77):
    rng = np.random.default_rng(seed)
    vpm = [(int(rng.integers(9, 41)), int(rng.integers(5, 25)), int(rng.integers(0, 6)), int(rng.integers(0, 4)),
            float(rng.uniform(3, 16)), bool(rng.integers(0, 2))) for _ in range(6)]
    svpm = [(int(rng.integers(5, 40)), int(rng.integers(5, 40)), int(rng.integers(0, 5)), int(rng.integers(1, 9)),
             float(rng.uniform(2, 12))) for _ in range(6)]
    depth = []
    for i in range(4):
        views = 1 + i % 2
        depth.append((int(rng.integers(9, 33)), int(rng.integers(5, 21)), int(rng.integers(0, 4)), int(rng.integers(1, 4)),
                      float(rng.uniform(3, 12)), views, 0 if views == 1 else int(rng.choice([0, 1, 2])),
                      float(rng.choice([-1.0, 0.5]))))
    return vpm, svpm, depth


_VPM_SWEEP, _SVPM_SWEEP, _DEPTH_SWEEP = _sibling_cases()


@pytest.mark.parametrize("W,H,r,it,dmax,init", _VPM_SWEEP)
def test_vpm_restatement_matches_reference_parameter_sweep(orc, ref, W, H, r, it, dmax, init):
    """VPMStereoCL::disparitySimple over seeded sizes, radius 0-5, 0-3 iterations and disparity
    ranges; half start from a given disparity with entries outside [0, dmax)"""
    from cvt_b200 import scene

    L, R = scene.generate(W * 13 + H, W, H, 3, 0.5, min(dmax - 1.0, 8.0))
    idisp = np.random.default_rng(W * H).uniform(-1.0, dmax + 1.0, (H, W)).astype(np.float32) if init else None
    a = orc.vpm_disparity_simple(L, R, r, it, dmax, idisp)
    b = ref.vpm_disparity_simple(L, R, r, it, dmax, idisp)
    assert bits_equal(a[0], b[0]).all() and bits_equal(a[1], b[1]).all()


@pytest.mark.parametrize("W,H,r,passes,flowmax", _SVPM_SWEEP)
def test_svpm_restatement_matches_reference_parameter_sweep(orc, ref, W, H, r, passes, flowmax):
    """SVPMFlowCL::flow over seeded sizes (below, at and past one 16x16 group), radius 0-4,
    1-8 passes and flow ranges"""
    from cvt_b200 import scene

    a1, a2 = scene.generate(W * 17 + H, W, H, 3, 0.5, 4.0)
    for x, y in zip(orc.svpm_flow(a1, a2, r, flowmax, passes), ref.svpm_flow(a1, a2, r, flowmax, passes)):
        assert bits_equal(x, y).all()


@pytest.mark.parametrize("W,H,r,it,dmax,views,pp,dscale", _DEPTH_SWEEP)
def test_depth_restatement_matches_reference_parameter_sweep(orc, ref, W, H, r, it, dmax, views, pp, dscale):
    """PMHuberStereo::depthMap over seeded sizes, radius 0-3, iterations, views, post-processing
    and the output scale (1 / dmax by default, or given); every stage equal bit for bit"""
    from cvt_b200 import scene

    L, R = scene.generate(W * 7 + H, W, H, 3, 0.5, dmax - 1.0)
    a = orc.depth_map(L, R, r, dmax, it, dscale=dscale, pp=pp, views=views, dump=True)
    b = ref.depth_map(L, R, r, dmax, it, dscale=dscale, pp=pp, views=views, dump=True)
    assert a["stages"].keys() == b["stages"].keys()
    for k in a["stages"]:
        assert bits_equal(a["stages"][k], b["stages"][k]).all(), k
    assert bits_equal(a["dmap"], b["dmap"]).all()


@pytest.mark.parametrize("W,H,r,it,levels", [(24, 20, 1, 1, 3), (30, 18, 2, 1, 2)])
def test_pyramid_restatement_matches_reference_parameter_sweep(orc, ref, W, H, r, it, levels):
    """the coarse-to-fine loop at sizes whose levels round down unevenly"""
    from cvt_b200 import scene

    L, R = scene.generate(W * 5 + H, W, H, 3, 0.5, 8.0)
    a = orc.disparity_map(L, R, r, 10.0, it, pp=1, levels=levels, dump=True)
    b = ref.disparity_map(L, R, r, 10.0, it, pp=1, levels=levels, dump=True)
    for k in a["stages"]:
        assert bits_equal(a["stages"][k], b["stages"][k]).all(), k
    assert bits_equal(a["dmap"], b["dmap"]).all()


def _mwc_step(x, c):
    A = 4294883355
    xn = (A * x + c) & 0xffffffff
    carry = 1 if xn < c else 0
    cn = ((A * x) >> 32) + carry
    return xn, cn & 0xffffffff


def test_mwc64x_skip_equals_stepping(orc):
    """MWC64X skip-ahead (MWC64X.cl:104-141) against plain stepping from the common seed."""
    A, BASE = 4294883355, 4077358422479273989
    x, c = BASE // A, BASE % A
    states = []
    for _ in range(64):
        states.append((x, c))
        x, c = _mwc_step(x, c)
    for d in (0, 1, 2, 3, 17, 63):
        sx, sc = states[d]
        expect = np.float32(np.float32(sx ^ sc) * np.float32(2.3283064365386962890625e-10))
        got = orc.rng_floats(d, 1, 1)[0]
        assert got == expect, d


def test_libm_within_opencl_bounds(orc):
    """exp <= 3 ulp, sin/cos <= 4 ulp, acospi <= 5 ulp (OpenCL 1.2 s7.4), in fact ~1-2.5."""
    L = orc.L
    xs = np.linspace(-40, 0, 20001, dtype=np.float32)
    got = np.array([L.orc_exp(float(x)) for x in xs], np.float32)
    want = np.exp(xs.astype(np.float64))
    ulp = np.spacing(want.astype(np.float32)).astype(np.float64)
    assert (np.abs(got - want) / ulp).max() <= 1.0
    assert L.orc_exp(0.0) == 1.0
    xs = np.linspace(0, 6.3, 20001, dtype=np.float32)
    for fn, ref_fn in ((L.orc_sin, np.sin), (L.orc_cos, np.cos)):
        got = np.array([fn(float(x)) for x in xs], np.float32)
        want = ref_fn(xs.astype(np.float64))
        ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
        m = np.abs(want) > 1e-6
        assert (np.abs(got - want)[m] / ulp[m]).max() <= 2.0
    xs = np.linspace(-1, 1, 20001, dtype=np.float32)
    got = np.array([L.orc_acospi(float(x)) for x in xs], np.float32)
    want = np.arccos(xs.astype(np.float64)) / np.pi
    ulp = np.spacing(want.astype(np.float32)).astype(np.float64)
    m = want > 1e-6
    assert (np.abs(got - want)[m] / ulp[m]).max() <= 3.0


def test_fused_mode_differs_only_by_rounding(orc):
    """Fused arithmetic changes last bits, not the method: final disparities stay close."""
    from cvt_b200 import scene

    L, R, gt, _ = scene.generate(2, 48, 32, 4, 2.0, 10.0, with_gt=True)
    a = orc.disparity_map(L, R, 3, 12.0, 3, pp=0, fused=0)
    b = orc.disparity_map(L, R, 3, 12.0, 3, pp=0, fused=1)
    assert np.mean(np.abs(a["dmap"] - b["dmap"]) < 1.0) > 0.9


def pyr_spec(g):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, pp, views, levels, init = g["spec"]
    return dict(W=int(W), H=int(H), r=int(r), dmax=float(dmax), iters=int(iters), pp=int(pp), views=int(views),
                levels=int(levels), init=bool(init))


@pytest.mark.parametrize("case", pyramid_cases())
def test_pyramid_restatement_matches_reference_golden(orc, case):
    """The coarse-to-fine loop of PMHuberStereo::disparityMap (levels > 1), bit for bit."""
    g = load_golden(case)
    s = pyr_spec(g)
    res = orc.disparity_map(g["left"], g["right"], s["r"], s["dmax"], s["iters"], pp=s["pp"], views=s["views"],
                            initdisp=g.get("initdisp"), levels=s["levels"], dump=True, fused=0)
    n = 0
    for (stage, it), v in res["stages"].items():
        k = "stage_%s_%d" % (stage, it)
        if k in g:
            assert bits_equal(v, g[k]).all(), (case, stage)
            n += 1
    assert n == 2 * s["levels"]
    for k in ("dmap", "normal", "planesL", "planesR"):
        assert bits_equal(res[k], g[k]).all(), (case, k)
    W1, H1 = g["k_pyrdown"].shape[1], g["k_pyrdown"].shape[0]
    assert (orc.pyrdown(g["left"], W1, H1) == g["k_pyrdown"]).all()
    up = np.float32(s["W"]) / np.float32(W1)
    assert bits_equal(orc.pyrup_mul(g["k_pyr_d1"], s["W"], s["H"], [up] * 4), g["k_pyrup_d"]).all()
    assert bits_equal(orc.pyrup_mul(g["k_pyr_n1"], s["W"], s["H"], [1.0] * 4), g["k_pyrup_n"]).all()


@pytest.mark.parametrize("Wi,Hi,Wo,Ho", [(37, 23, 12, 8), (5, 3, 1, 1), (8, 6, 19, 13), (64, 1, 22, 1)])
def test_pyramid_kernels_match_reference_live(orc, ref, Wi, Hi, Wo, Ho):
    """pyrdown and pyrup_mul4f for down- and upsampling and degenerate sizes"""
    rng = np.random.default_rng(Wi * 100 + Ho)
    img = rng.integers(0, 256, (Hi, Wi, 4), dtype=np.uint8)
    assert (orc.pyrdown(img, Wo, Ho) == ref.pyrdown(img, Wo, Ho)).all()
    f1 = rng.standard_normal((Hi, Wi)).astype(np.float32)
    f4 = rng.standard_normal((Hi, Wi, 4)).astype(np.float32)
    mul = [1.7, -0.5, 3.0, 1.0]
    assert bits_equal(orc.pyrup_mul(f1, Wo, Ho, mul), ref.pyrup_mul(f1, Wo, Ho, mul)).all()
    assert bits_equal(orc.pyrup_mul(f4, Wo, Ho, mul), ref.pyrup_mul(f4, Wo, Ho, mul)).all()


def depth_spec(g):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, dscale, pp, init = g["spec"]
    return dict(W=int(W), H=int(H), r=int(r), dmax=float(dmax), iters=int(iters), dscale=float(dscale), pp=int(pp),
                init=bool(init))


@pytest.mark.parametrize("case", depth_cases())
def test_depth_restatement_matches_reference_golden(orc, case):
    """PMHuberStereo::depthMap, bit for bit (strict arithmetic), and its kernels"""
    g = load_golden(case)
    s = depth_spec(g)
    res = orc.depth_map(g["left"], g["right"], s["r"], s["dmax"], s["iters"], dscale=s["dscale"], pp=s["pp"],
                        initdisp=g.get("initdisp"), dump=True, fused=0)
    n = 0
    for (stage, it), v in res["stages"].items():
        k = "stage_%s_%d" % (stage, it)
        if k in g:
            assert bits_equal(v, g[k]).all(), (case, stage, it)
            n += 1
    assert n >= 6
    for k in ("dmap", "normal", "planesL", "planesR"):
        assert bits_equal(res[k], g[k]).all(), (case, k)
    c, gr, dt = orc.prep_raw(g["left"], 12.0)
    assert bits_equal(c, g["k_colour"]).all() and bits_equal(gr, g["k_grad"]).all() and bits_equal(dt, g["k_dt12"]).all()
    P = g["k_fs_planes"]
    assert bits_equal(orc.fill_state(P, 1.0 / s["dmax"], 1), g["k_fill_state_l"]).all()
    assert bits_equal(orc.fill_state(P, 1.0 / s["dmax"], 0), g["k_fill_state_r"]).all()
    assert bits_equal(orc.huber(g["k_fill_state_l"], dt, [2.3] * 4, 1e-4, 40), g["k_huber"]).all()
    assert bits_equal(orc.huber(g["k_fill_state_l"], dt, [2.3] * 4, 1e-4, 7), g["k_huber_odd"]).all()


def test_depth_restatement_matches_reference_live(orc, ref):
    """a fresh seed and a single-view-free edge: 4 iterations (theta's schedule divides by 0 after the last)"""
    from cvt_b200 import scene

    L, R = scene.generate(31, 41, 27, 5, 1.0, 9.0)
    for iters in (1, 4):
        a = orc.depth_map(L, R, 2, 11.0, iters, pp=2, dump=True)
        b = ref.depth_map(L, R, 2, 11.0, iters, pp=2, dump=True)
        for k in a["stages"]:
            assert bits_equal(a["stages"][k], b["stages"][k]).all(), (iters, k)
        assert bits_equal(a["dmap"], b["dmap"]).all()


def vpm_spec(g):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, init = g["spec"]
    return dict(W=int(W), H=int(H), r=int(r), dmax=float(dmax), iters=int(iters), init=bool(init))


@pytest.mark.parametrize("case", vpm_cases())
def test_vpm_restatement_matches_reference_golden(orc, case):
    """VPMStereoCL::disparitySimple and each of its kernels, bit for bit"""
    g = load_golden(case)
    s = vpm_spec(g)
    r, dmax = s["r"], s["dmax"]
    initd = g.get("initdisp")
    disp, states = orc.vpm_disparity_simple(g["left"], g["right"], r, s["iters"], dmax, initd)
    assert bits_equal(disp, g["disparity"]).all() and bits_equal(states, g["states"]).all()
    g0, g1 = orc.vpm_grad(g["left"]), orc.vpm_grad(g["right"])
    assert bits_equal(g0, g["k_grad0"]).all() and bits_equal(g1, g["k_grad1"]).all()
    s0 = orc.vpm_init(g["left"], g0, g["right"], g1, r, dmax, initd)
    assert bits_equal(s0, g["k_init"]).all()
    assert bits_equal(orc.vpm_iter(g["k_init"], g["left"], g0, g["right"], g1, r, dmax, 0), g["k_iter0"]).all()
    assert bits_equal(orc.vpm_iter(g["k_iter0"], g["left"], g0, g["right"], g1, r, dmax, 5), g["k_iter5"]).all()
    assert bits_equal(orc.vpm_disparity(g["k_iter5"], 1.0 / dmax), g["k_disp_scaled"]).all()


@pytest.mark.parametrize("W,H,r,iters", [(1, 1, 2, 2), (2, 3, 0, 1), (3, 2, 1, 2), (37, 5, 4, 1), (33, 34, 2, 0)])
def test_vpm_restatement_matches_reference_live(orc, ref, W, H, r, iters):
    """edge sizes: a single pixel, images narrower than the Gauss-Newton taps' column range
    (singular steps), r = 0, zero iterations, sizes off the 32x32 work-group grid"""
    from cvt_b200 import scene

    L, R = scene.generate(40 + W, W, H, 3, 0.5, 4.0)
    a = orc.vpm_disparity_simple(L, R, r, iters, 6.0)
    b = ref.vpm_disparity_simple(L, R, r, iters, 6.0)
    assert bits_equal(a[0], b[0]).all() and bits_equal(a[1], b[1]).all()


@pytest.mark.parametrize("case", svpm_cases())
def test_svpm_restatement_matches_reference_golden(orc, case):
    """SVPMFlowCL::flow and each of its kernels, bit for bit"""
    g = load_golden(case)
    seed, W, H, npl, dlo, dhi, r, flowmax, passes = g["spec"]
    r, flowmax, passes = int(r), float(flowmax), int(passes)
    flow, states, duals = orc.svpm_flow(g["first"], g["second"], r, flowmax, passes)
    for a, k in ((flow, "flow"), (states, "states"), (duals, "duals")):
        assert bits_equal(a, g[k]).all(), k
    assert bits_equal(orc.svpm_init(g["first"], g["second"], r, flowmax), g["k_init"]).all()
    s1, p1 = orc.svpm_prop(g["k_init"], np.zeros_like(g["k_init"]), g["first"], g["second"], r, flowmax, 1)
    assert bits_equal(s1, g["k_prop1"]).all() and bits_equal(p1, g["k_dual1"]).all()
    s6, p6 = orc.svpm_prop(g["k_prop1"], g["k_dual1"] + np.float32(0.25), g["first"], g["second"], r, flowmax, 6)
    assert bits_equal(s6, g["k_prop6"]).all() and bits_equal(p6, g["k_dual6"]).all()
    assert bits_equal(orc.svpm_to_flow(g["k_prop6"]), g["k_flow"]).all()


@pytest.mark.parametrize("W,H,r,passes", [(1, 1, 1, 6), (5, 3, 0, 6), (17, 33, 2, 7), (16, 16, 3, 5)])
def test_svpm_restatement_matches_reference_live(orc, ref, W, H, r, passes):
    """edge sizes: a single pixel, r = 0, sizes one past the 16x16 work-group, exactly one group"""
    from cvt_b200 import scene

    a, b = scene.generate(60 + W, W, H, 3, 0.5, 4.0)
    x = orc.svpm_flow(a, b, r, 6.0, passes)
    y = ref.svpm_flow(a, b, r, 6.0, passes)
    for u, v in zip(x, y):
        assert bits_equal(u, v).all()


def test_log_within_a_ulp(orc):
    """the oracle's log (Box-Muller of SVPMFlow.cl:42) against double precision: <= 1 ulp,
    and its special values"""
    rng = np.random.default_rng(3)
    bits = np.concatenate([rng.integers(1, 0x7f800000, 200000, dtype=np.uint32),
                           np.arange(0x3f000000, 0x3f000000 + 20000, dtype=np.uint32),
                           np.arange(0x3f800000 - 10000, 0x3f800000 + 10000, dtype=np.uint32)])
    xs = bits.view(np.float32)
    got = np.array([orc.L.orc_log(float(x)) for x in xs], np.float32)
    want = np.log(xs.astype(np.float64))
    ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
    err = np.abs(got.astype(np.float64) - want) / ulp
    assert err.max() <= 1.0, (err.max(), xs[err.argmax()])
    assert orc.L.orc_log(1.0) == 0.0 and np.isneginf(orc.L.orc_log(0.0)) and np.isnan(orc.L.orc_log(-1.0))
    assert np.isposinf(orc.L.orc_log(float("inf")))


def test_known_candidates_leave_the_state_unchanged(orc):
    """Candidates whose plane equals the current plane, with the current cost below the
    early-exit value, are skipped by the CUDA kernels.  The restatement still evaluates them and
    records any that changed the state: none may, on scenes that make many (converged planes
    copied between neighbours), in both arithmetic modes and with the depth variant."""
    from cvt_b200 import scene

    L, R = scene.generate(21, 160, 96, 5, 2.0, 30.0)
    known0, changed0 = orc.known_counts()
    for fused in (0, 1):
        o = orc.disparity_map(L, R, 5, 32.0, 5, pp=1, fused=fused)
        assert np.isfinite(o["dmap"]).all()
    orc.depth_map(L, R, 5, 32.0, 4, fused=1)
    known, changed = orc.known_counts()
    assert known - known0 > 1000, known - known0
    assert changed == changed0 == 0

