"""Parity of the SVPMFlowCL kernels (cvt/vision/SVPMFlowCL.cpp, cvt/cl/kernel/SVPMFlow.cl) with
the reference through the C ABI: the golden fixtures bit for bit, the oracle bit for bit on
fresh seeds and edge sizes, and properties at the benchmark size."""
import numpy as np
import pytest

from conftest import load_golden, svpm_cases
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


def spec(g):
    seed, W, H, npl, dlo, dhi, r, flowmax, passes = g["spec"]
    return int(W), int(H), int(r), float(flowmax), int(passes)


@pytest.mark.parametrize("case", svpm_cases())
def test_svpm_kernels_match_reference_golden(torch_cuda, native, case):
    torch = torch_cuda
    g = load_golden(case)
    W, H, r, flowmax, passes = spec(g)
    s = torch.cuda.current_stream().cuda_stream
    a, b = dev(torch, g["first"]), dev(torch, g["second"])
    out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    assert native.pm_k_svpm_init(out.data_ptr(), a.data_ptr(), b.data_ptr(), W, H, W * 4, r, flowmax, s) == 0
    assert bits_equal(host(out), g["k_init"]).all()
    for it, src, pin, dst, pdst in ((1, "k_init", None, "k_prop1", "k_dual1"), (6, "k_prop1", "k_dual1", "k_prop6",
                                                                              "k_dual6")):
        i = dev(torch, g[src])
        p = dev(torch, np.zeros_like(g[src]) if pin is None else g[pin] + np.float32(0.25))
        o, po = torch.zeros_like(i), torch.zeros_like(i)
        assert native.pm_k_svpm_prop(o.data_ptr(), po.data_ptr(), i.data_ptr(), p.data_ptr(), a.data_ptr(),
                                     b.data_ptr(), W, H, W * 4, r, flowmax, it, s) == 0
        ok = bits_equal(host(o), g[dst])
        assert ok.all(), (case, it, ok.mean())
        assert bits_equal(host(po), g[pdst]).all()
    st = dev(torch, g["k_prop6"])
    fl = torch.zeros((H, W, 2), dtype=torch.float32, device="cuda")
    assert native.pm_k_svpm_to_flow(fl.data_ptr(), st.data_ptr(), W, H, s) == 0
    assert bits_equal(host(fl), g["k_flow"]).all()


@pytest.mark.parametrize("case", svpm_cases())
def test_svpm_flow_matches_reference_golden(torch_cuda, native, case):
    """host and device entries of SVPMFlowCL::flow"""
    from cvt_b200.svpm import SVPMFlowCL

    g = load_golden(case)
    W, H, r, flowmax, passes = spec(g)
    f = SVPMFlowCL()
    res = f.flow(g["first"], g["second"], r, flowmax, passes, states=True)
    for a, k in zip(res, ("flow", "states", "duals")):
        assert bits_equal(a, g[k]).all(), k
    res = f.flow(dev(torch_cuda, g["first"]), dev(torch_cuda, g["second"]), r, flowmax, passes, states=True)
    for a, k in zip(res, ("flow", "states", "duals")):
        assert bits_equal(host(a), g[k]).all(), k


@pytest.mark.parametrize("W,H,r,passes,flowmax", [(1, 1, 1, 6, 6.0), (5, 3, 0, 6, 6.0), (17, 33, 2, 7, 6.0),
                                                  (16, 16, 3, 5, 6.0), (130, 75, 3, 9, 24.0), (4096, 2, 2, 3, 16.0),
                                                  (3, 4096, 1, 3, 6.0), (20, 18, 32, 3, 6.0)])
def test_svpm_matches_oracle_edge_sizes(torch_cuda, native, orc, W, H, r, passes, flowmax):
    """a single pixel, r = 0, one past a 16x16 group, exactly one group, several groups, the
    largest accepted width, height and window radius"""
    from cvt_b200 import scene
    from cvt_b200.svpm import SVPMFlowCL

    a, b = scene.generate(60 + W, W, H, 3, 0.5, 4.0 if W < 64 else 16.0)
    want = orc.svpm_flow(a, b, r, flowmax, passes)
    got = SVPMFlowCL().flow(a, b, r, flowmax, passes, states=True)
    for u, v in zip(got, want):
        assert bits_equal(u, v).all()


def test_svpm_hd_properties(torch_cuda, native):
    """1280x720 (the benchmark size), the reference's 200 passes: deterministic across calls,
    the flow equals the states' (u, v), costs finite, and most pixels within 3 px of the
    scene's true motion (-d, 0)"""
    from cvt_b200 import scene
    from cvt_b200.svpm import SVPMFlowCL

    W, H = 1280, 720
    a, b, gd, gn = scene.generate(0, W, H, 40, 2.0, 120.0, with_gt=True)
    f = SVPMFlowCL()
    f1, s1, p1 = f.flow(a, b, 3, 128.0, 200, states=True)
    f2, s2, p2 = f.flow(a, b, 3, 128.0, 200, states=True)
    assert bits_equal(f1, f2).all() and bits_equal(s1, s2).all() and bits_equal(p1, p2).all()
    assert bits_equal(f1, s1[..., :2]).all()
    assert np.isfinite(s1[..., 2]).all()
    epe = np.hypot(f1[..., 0] + gd, f1[..., 1])[:, 160:]
    print("EPE median %.3f, within 1 px %.3f, within 3 px %.3f" % (np.median(epe), np.mean(epe < 1), np.mean(epe < 3)))
    assert np.mean(epe < 3.0) > 0.5, np.mean(epe < 3.0)


def test_svpm_cpp_drop_in_matches_oracle(native, torch_cuda, orc, tmp_path):
    """cvt::SVPMFlowCL::flow through the C++ header (tests/cpp/drop_in.cpp); flowInit throws"""
    import subprocess

    from cvt_b200 import scene
    from test_abi import build_drop_in

    exe = build_drop_in(tmp_path)
    outf = tmp_path / "flow.raw"
    subprocess.run([exe, str(tmp_path / "d.raw"), str(tmp_path / "depth.raw"), str(tmp_path / "d.pfm"),
                    str(tmp_path / "vpm.raw"), str(outf)], check=True)
    fl = np.fromfile(str(outf), np.float32).reshape(64, 96, 2)
    L, R = scene.generate(7, 96, 64, 6, 2.0, 20.0)
    assert bits_equal(fl, orc.svpm_flow(L, R, 2, 16.0, 8)[0]).all()
