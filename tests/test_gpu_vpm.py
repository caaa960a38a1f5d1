"""Parity of the VPMStereoCL kernels (cvt/vision/VPMStereoCL.cpp, cvt/cl/kernel/VPMStereo.cl)
with the reference through the C ABI: the golden fixtures bit for bit, the oracle bit for bit
on fresh seeds and edge sizes, and size-independent properties at the benchmark size."""
import numpy as np
import pytest

from conftest import load_golden, vpm_cases
from oracle.pyoracle import bits_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(native):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def vpm_spec(g):
    seed, W, H, npl, dlo, dhi, r, dmax, iters, init = g["spec"]
    return int(W), int(H), int(r), float(dmax), int(iters), bool(init)


class K:
    """One reference kernel per call (pm_k_vpm_*) on device buffers."""

    def __init__(self, torch, L):
        self.t, self.L = torch, L

    def s(self):
        return self.t.cuda.current_stream().cuda_stream

    def f4(self, H, W):
        return self.t.zeros((H, W, 4), dtype=self.t.float32, device="cuda")

    def grad(self, img):
        H, W = img.shape[:2]
        out = self.f4(H, W)
        d = dev(self.t, img)
        assert self.L.pm_k_vpm_grad(out.data_ptr(), d.data_ptr(), W, H, W * 4, self.s()) == 0
        return host(out)

    def init(self, c1, g1, c2, g2, r, dmax, initd=None):
        H, W = c1.shape[:2]
        out = self.f4(H, W)
        a, b, ga, gb = dev(self.t, c1), dev(self.t, c2), dev(self.t, g1), dev(self.t, g2)
        di = None if initd is None else dev(self.t, initd.astype(np.float32))
        assert self.L.pm_k_vpm_init(out.data_ptr(), a.data_ptr(), ga.data_ptr(), b.data_ptr(), gb.data_ptr(), W, H,
                                    W * 4, r, dmax, None if di is None else di.data_ptr(), self.s()) == 0
        return host(out)

    def iter(self, st, c1, g1, c2, g2, r, dmax, it):
        H, W = c1.shape[:2]
        out = self.f4(H, W)
        i = dev(self.t, st)
        a, b, ga, gb = dev(self.t, c1), dev(self.t, c2), dev(self.t, g1), dev(self.t, g2)
        assert self.L.pm_k_vpm_iter(out.data_ptr(), i.data_ptr(), a.data_ptr(), ga.data_ptr(), b.data_ptr(),
                                    gb.data_ptr(), W, H, W * 4, r, dmax, it, self.s()) == 0
        return host(out)

    def disparity(self, st, scale):
        H, W = st.shape[:2]
        out = self.t.zeros((H, W), dtype=self.t.float32, device="cuda")
        i = dev(self.t, st)
        assert self.L.pm_k_vpm_disparity(out.data_ptr(), i.data_ptr(), W, H, scale, self.s()) == 0
        return host(out)


@pytest.mark.parametrize("case", vpm_cases())
def test_vpm_kernels_match_reference_golden(torch_cuda, native, case):
    g = load_golden(case)
    W, H, r, dmax, iters, init = vpm_spec(g)
    k = K(torch_cuda, native)
    g0, g1 = k.grad(g["left"]), k.grad(g["right"])
    assert bits_equal(g0, g["k_grad0"]).all() and bits_equal(g1, g["k_grad1"]).all()
    assert bits_equal(k.init(g["left"], g0, g["right"], g1, r, dmax, g.get("initdisp")), g["k_init"]).all()
    for it, src, dst in ((0, "k_init", "k_iter0"), (5, "k_iter0", "k_iter5")):
        out = k.iter(g[src], g["left"], g0, g["right"], g1, r, dmax, it)
        ok = bits_equal(out, g[dst])
        assert ok.all(), (case, it, ok.mean())
    assert bits_equal(k.disparity(g["k_iter5"], 1.0 / dmax), g["k_disp_scaled"]).all()


@pytest.mark.parametrize("case", vpm_cases())
def test_vpm_disparity_simple_matches_reference_golden(torch_cuda, native, case):
    """host and device entries of disparitySimple"""
    from cvt_b200.vpm import VPMStereoCL

    g = load_golden(case)
    W, H, r, dmax, iters, init = vpm_spec(g)
    v = VPMStereoCL(r, iters, dmax)
    d, st = v.disparity_simple(g["left"], g["right"], g.get("initdisp"), states=True)
    assert bits_equal(d, g["disparity"]).all() and bits_equal(st, g["states"]).all()
    ini = None if g.get("initdisp") is None else dev(torch_cuda, g["initdisp"])
    dd, sd = v.disparity_simple(dev(torch_cuda, g["left"]), dev(torch_cuda, g["right"]), ini, states=True)
    assert bits_equal(host(dd), g["disparity"]).all() and bits_equal(host(sd), g["states"]).all()


@pytest.mark.parametrize("W,H,r,iters", [(1, 1, 2, 2), (2, 3, 0, 1), (3, 2, 1, 2), (37, 5, 4, 1), (33, 34, 2, 0),
                                         (160, 96, 5, 3), (4096, 3, 3, 1), (4, 4096, 2, 1), (40, 24, 32, 1)])
def test_vpm_matches_oracle_edge_sizes(torch_cuda, native, orc, W, H, r, iters):
    """a single pixel, images narrower than the Gauss-Newton taps' column range (singular
    steps: NaN states whose costs are finite), r = 0, zero iterations, sizes off every tile,
    the largest accepted width, height and window radius"""
    from cvt_b200 import scene
    from cvt_b200.vpm import VPMStereoCL

    L, R = scene.generate(40 + W, W, H, 3, 0.5, 4.0 if W < 64 else 24.0)
    dmax = 6.0 if W < 64 else 32.0
    a = orc.vpm_disparity_simple(L, R, r, iters, dmax)
    b = VPMStereoCL(r, iters, dmax).disparity_simple(L, R, states=True)
    assert bits_equal(b[0], a[0]).all() and bits_equal(b[1], a[1]).all()


def test_vpm_padded_rows_and_stream(torch_cuda, native, orc):
    """a row stride beyond 4 W (device entry) and a side stream"""
    import ctypes as C

    from cvt_b200 import scene

    torch = torch_cuda
    W, H, r, dmax, iters = 70, 45, 3, 20.0, 2
    L, R = scene.generate(5, W, H, 4, 1.0, 16.0)
    pad = np.zeros((H, W + 6, 4), np.uint8)
    padR = pad.copy()
    pad[:, :W], padR[:, :W] = L, R
    want = orc.vpm_disparity_simple(L, R, r, iters, dmax)
    h = C.c_void_p()
    assert native.pm_vpm_create(C.byref(h), r, iters, dmax, 0) == 0
    try:
        a, b = dev(torch, pad), dev(torch, padR)
        d = torch.zeros((H, W), dtype=torch.float32, device="cuda")
        st = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
        s = torch.cuda.Stream()
        with torch.cuda.stream(s):
            assert native.pm_vpm_disparity_simple_device(h, a.data_ptr(), b.data_ptr(), W, H, (W + 6) * 4,
                                                         d.data_ptr(), None, st.data_ptr(), s.cuda_stream) == 0
        s.synchronize()
        assert bits_equal(d.cpu().numpy(), want[0]).all() and bits_equal(st.cpu().numpy(), want[1]).all()
    finally:
        native.pm_vpm_destroy(h)


def test_vpm_hd_properties(torch_cuda, native):
    """1280x720 (the benchmark size): deterministic across calls, the returned disparities
    equal |x' - x| of the returned states, costs in [0, 1] or the out-of-range 1, and most
    pixels near the scene's true disparity"""
    from cvt_b200 import scene
    from cvt_b200.vpm import VPMStereoCL

    W, H = 1280, 720
    L, R, gd, gn = scene.generate(0, W, H, 40, 2.0, 120.0, with_gt=True)
    v = VPMStereoCL(7, 4, 128.0)
    d1, s1 = v.disparity_simple(L, R, states=True)
    d2, s2 = v.disparity_simple(L, R, states=True)
    assert bits_equal(d1, d2).all() and bits_equal(s1, s2).all()
    xs = np.arange(W, dtype=np.float32)[None, :]
    ys = np.arange(H, dtype=np.float32)[:, None]
    with np.errstate(all="ignore"):
        xp = (s1[..., 0] * xs + s1[..., 1] * ys + s1[..., 2]).astype(np.float32)
        assert bits_equal(np.abs(xp - xs).astype(np.float32), d1).all()
    c = s1[..., 3]
    assert np.nanmin(c) >= 0.0 and np.nanmax(c) <= 1.0 + 1e-6
    good = np.abs(d1 - gd) < 1.0
    assert np.mean(good[:, 160:]) > 0.5, np.mean(good[:, 160:])


def test_vpm_cpp_drop_in_matches_oracle(native, torch_cuda, orc, tmp_path):
    """cvt::VPMStereoCL::disparitySimple through the C++ header (tests/cpp/drop_in.cpp)"""
    import subprocess

    from cvt_b200 import scene
    from test_abi import build_drop_in

    exe = build_drop_in(tmp_path)
    outv = tmp_path / "vpm.raw"
    subprocess.run([exe, str(tmp_path / "d.raw"), str(tmp_path / "depth.raw"), str(tmp_path / "d.pfm"), str(outv)],
                   check=True)
    d = np.fromfile(str(outv), np.float32).reshape(64, 96)
    L, R = scene.generate(7, 96, 64, 6, 2.0, 20.0)
    assert bits_equal(d, orc.vpm_disparity_simple(L, R, 3, 4, 24.0)[0]).all()
