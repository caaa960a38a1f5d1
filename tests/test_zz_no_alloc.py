"""pm_k_rof_static (library-owned static scratch) against pm_k_rof (caller scratch).

Some callers of this library cannot allocate device memory on the smoothing path: a
binding that hands over only image pointers and has no device allocator to make a scratch
buffer with, or a loop that runs under a fixed device-memory budget and must not stall
other streams behind cudaMalloc/cudaFree.  pm_k_rof_static serves them from a static
device array instead.  Both entry points launch the same ROF steps, so the tolerance is
zero: results must be bit-identical.  Calls made after a larger call has filled the shared
scratch show that what one call leaves there does not reach the next call's result; a
device reset between two calls shows that the array's address is looked up again in the
new context.  The file is named to be collected last, after every other test has used
the library in the same process.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, load_golden
from oracle.pyoracle import bits_equal

pytestmark = pytest.mark.gpu

PM_EINVAL_SHAPE, PM_EINVAL_ARG = 1, 2
LAM = (1.3, 1.3, 1.3, 1.0)
# tolerance: 0 ulp (bits_equal), since both entry points run the same kernels in the same order


@pytest.fixture(scope="module")
def torch_cuda(native):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _rof_both(torch, L, nd, dt, lam, iters):
    H, W = nd.shape[:2]
    st = torch.cuda.current_stream().cuda_stream
    a = torch.from_numpy(np.ascontiguousarray(nd)).cuda()
    d = torch.from_numpy(np.ascontiguousarray(dt)).cuda()
    ref = torch.empty_like(a)
    out = torch.full_like(a, float("nan"))
    scratch = torch.zeros(L.pm_rof_scratch_bytes(W, H), dtype=torch.uint8, device="cuda")
    lm = (C.c_float * 4)(*lam)
    assert L.pm_k_rof(ref.data_ptr(), a.data_ptr(), d.data_ptr(), lm, iters, W, H, scratch.data_ptr(), st) == 0
    rc = L.pm_k_rof_static(out.data_ptr(), a.data_ptr(), d.data_ptr(), lm, iters, W, H, st)
    assert rc == 0, L.pm_last_error(None)
    torch.cuda.synchronize()
    return ref.cpu().numpy(), out.cpu().numpy()


def _big_case(g):
    # a 320x224 image (64 times the golden case, mirrored tiles)
    big_nd = np.tile(np.concatenate([g["k_nd"], g["k_nd"][:, ::-1]], 1), (8, 4, 1))
    big_dt = np.tile(np.concatenate([g["dtL"], g["dtL"][:, ::-1]], 1), (8, 4, 1))
    assert big_nd.shape == (224, 320, 4)
    return big_nd, big_dt


def test_rof_static_matches_caller_scratch_twice(native, torch_cuda):
    g = load_golden("lr_40x28")
    big_nd, big_dt = _big_case(g)
    # call 1: the large image, odd step count
    ref1, out1 = _rof_both(torch_cuda, native, big_nd, big_dt, LAM, 7)
    assert np.isfinite(ref1).all()
    assert bits_equal(out1, ref1).all()
    # call 2: the golden case on the scratch call 1 left behind
    ref2, out2 = _rof_both(torch_cuda, native, g["k_nd"], g["dtL"], LAM, 40)
    assert bits_equal(out2, ref2).all()
    assert bits_equal(out2, g["k_rof"]).all()


@pytest.mark.parametrize("iters", [0, 1, 2])
def test_rof_static_short_step_counts_on_used_scratch(native, torch_cuda, iters):
    """0, 1 and 2 steps after a larger call has filled the scratch (0 and 1 run the single-step
    kernel once: the step count is rounded up to odd, PDOptCL.cpp:1152-1166; 2 is one two-step
    launch)"""
    g = load_golden("lr_40x28")
    big_nd, big_dt = _big_case(g)
    ref1, out1 = _rof_both(torch_cuda, native, big_nd, big_dt, LAM, 9)
    assert bits_equal(out1, ref1).all()
    ref2, out2 = _rof_both(torch_cuda, native, g["k_nd"], g["dtL"], LAM, iters)
    assert bits_equal(out2, ref2).all()
    assert np.isfinite(ref2).all() and not bits_equal(ref2, g["k_nd"]).all()


def test_rof_static_rejects_oversized_image_and_negative_steps(native, torch_cuda):
    W, H = 1024, 512   # 524288 pixels > PM_ROF_STATIC_MAX_PIXELS = 262144
    lm = (C.c_float * 4)(1.0, 1.0, 1.0, 1.0)
    x = torch_cuda.zeros(16, dtype=torch_cuda.uint8, device="cuda")
    rc = native.pm_k_rof_static(x.data_ptr(), x.data_ptr() + 8, x.data_ptr(), lm, 2, W, H, None)
    assert rc == PM_EINVAL_SHAPE
    msg = native.pm_last_error(None)
    msg = msg.decode() if isinstance(msg, bytes) else msg
    assert "PM_ROF_STATIC_MAX_PIXELS" in msg
    a = torch_cuda.zeros((4, 4, 4), dtype=torch_cuda.float32, device="cuda")
    b = torch_cuda.zeros_like(a)
    assert native.pm_k_rof_static(b.data_ptr(), a.data_ptr(), a.data_ptr(), lm, -1, 4, 4, None) == PM_EINVAL_ARG
    s = torch_cuda.zeros(native.pm_rof_scratch_bytes(4, 4), dtype=torch_cuda.uint8, device="cuda")
    assert native.pm_k_rof(b.data_ptr(), a.data_ptr(), a.data_ptr(), lm, -1, 4, 4, s.data_ptr(), None) == PM_EINVAL_ARG


# Child process for the reset and capture cases: both need a CUDA context that no other
# test has used.  It talks to the CUDA runtime directly (the same libcudart the library
# links), so no allocator holds addresses across the reset.
_CHILD = r'''
import ctypes as C, sys
import numpy as np
sys.path.insert(0, ROOT)
sys.path.insert(0, ROOT + "/tests")
from conftest import load_golden
from cvt_b200 import _lib
from oracle.pyoracle import bits_equal
L = _lib.lib()
rt = C.CDLL("libcudart.so.12")
g = load_golden("lr_40x28")
nd, dt, want = (np.ascontiguousarray(g[k], np.float32) for k in ("k_nd", "dtL", "k_rof"))
H, W = nd.shape[:2]
n = nd.nbytes
lm = (C.c_float * 4)(1.3, 1.3, 1.3, 1.0)

def dev(a=None):
    p = C.c_void_p()
    assert rt.cudaMalloc(C.byref(p), C.c_size_t(n)) == 0
    if a is not None:
        assert rt.cudaMemcpy(p, a.ctypes.data, C.c_size_t(n), 1) == 0
    return p

def run():
    i, d, o = dev(nd), dev(dt), dev()
    rc = L.pm_k_rof_static(o, i, d, lm, 40, W, H, None)
    assert rc == 0, L.pm_last_error(None)
    out = np.empty_like(nd)
    assert rt.cudaMemcpy(out.ctypes.data, o, C.c_size_t(n), 2) == 0
    for p in (i, d, o):
        rt.cudaFree(p)
    return out

mode = sys.argv[1]
if mode == "reset":
    a = run()
    assert rt.cudaDeviceReset() == 0
    b = run()
    assert bits_equal(a, want).all() and bits_equal(b, want).all()
    print("reset ok")
else:
    import torch
    i = torch.from_numpy(nd).cuda()
    o = torch.empty_like(i)
    s = torch.cuda.Stream()
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        gr.capture_begin()
        rc = L.pm_k_rof_static(o.data_ptr(), i.data_ptr(), i.data_ptr(), lm, 2, W, H, C.c_void_p(s.cuda_stream))
        gr.capture_end()
    msg = L.pm_last_error(None)
    msg = msg.decode() if isinstance(msg, bytes) else msg
    assert rc == 2 and "before stream capture" in msg, (rc, msg)
    print("capture ok")
'''


def _child(mode):
    code = "ROOT = %r\n" % ROOT + _CHILD
    r = subprocess.run([sys.executable, "-c", code, mode], capture_output=True, text=True, timeout=300,
                       cwd=ROOT, env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_rof_static_after_device_reset(native):
    """a call, cudaDeviceReset (which ends only this process's context), another call: both
    equal the reference fixture"""
    assert "reset ok" in _child("reset")


def test_rof_static_first_call_under_capture_is_refused(native):
    """the first call in a fresh context, made while the stream is being captured, returns
    PM_EINVAL_ARG with a message instead of looking the array up inside the capture"""
    assert "capture ok" in _child("capture")
