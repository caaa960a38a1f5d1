"""pm_k_rof_static (library-owned static scratch) against pm_k_rof (caller scratch).

Both entry points launch the same ROF steps, so the tolerance is zero: results must be
bit-identical.  Two calls in a row, the first on a larger image, show that what one call
leaves in the shared scratch does not reach the next call's result.  The file is named to
be collected last, after every other test has used the library in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden
from oracle.pyoracle import bits_equal

pytestmark = pytest.mark.gpu

PM_EINVAL_SHAPE = 1
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


def test_rof_static_matches_caller_scratch_twice(native, torch_cuda):
    g = load_golden("lr_40x28")
    lam = (1.3, 1.3, 1.3, 1.0)
    # call 1: a 320x224 image (64 times the golden case, mirrored tiles), odd step count
    big_nd = np.tile(np.concatenate([g["k_nd"], g["k_nd"][:, ::-1]], 1), (8, 4, 1))
    big_dt = np.tile(np.concatenate([g["dtL"], g["dtL"][:, ::-1]], 1), (8, 4, 1))
    assert big_nd.shape == (224, 320, 4)
    ref1, out1 = _rof_both(torch_cuda, native, big_nd, big_dt, lam, 7)
    assert np.isfinite(ref1).all()
    assert bits_equal(out1, ref1).all()
    # call 2: the golden case on the scratch call 1 left behind
    ref2, out2 = _rof_both(torch_cuda, native, g["k_nd"], g["dtL"], lam, 40)
    assert bits_equal(out2, ref2).all()
    assert bits_equal(out2, g["k_rof"]).all()


def test_rof_static_rejects_oversized_image(native, torch_cuda):
    W, H = 1024, 512   # 524288 pixels > PM_ROF_STATIC_MAX_PIXELS = 262144
    lm = (C.c_float * 4)(1.0, 1.0, 1.0, 1.0)
    x = torch_cuda.zeros(16, dtype=torch_cuda.uint8, device="cuda")
    rc = native.pm_k_rof_static(x.data_ptr(), x.data_ptr() + 8, x.data_ptr(), lm, 2, W, H, None)
    assert rc == PM_EINVAL_SHAPE
    msg = native.pm_last_error(None)
    msg = msg.decode() if isinstance(msg, bytes) else msg
    assert "PM_ROF_STATIC_MAX_PIXELS" in msg
