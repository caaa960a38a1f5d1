"""The learned plane proposal on the GPU (cvt_b200/csrc/pm_learn.cu, cvt_b200/learn.py): the
tcgen05 convolutions (forward and data gradient) and weight gradients of every layer against
the CUDA cores and the numpy oracle, the whole backward pass against the oracle, the input,
target and upsampling kernels, checkpoint / resume with the Adam state, the committed weights,
and what a short training run gains over random initialisation.

Tolerances: a convolution's FP32 sums on the tensor cores and on the CUDA cores differ in
order, so their BF16 outputs may differ by one BF16 rounding (|a - b| <= 2^-7 |b| + 1e-6);
weight gradients within 1e-4 relative of their largest entry; the whole backward pass (BF16
data gradients rounded at every layer) within 2e-2 relative with cosine similarity > 0.999 at
the last layer, the bound widening by 1e-2 and 5e-4 per layer below it."""
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import lpp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(native):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def bf(torch, a):
    return torch.from_numpy(np.ascontiguousarray(O.bf16(a))).cuda().to(torch.bfloat16)


def to_np(t):
    import torch

    torch.cuda.synchronize()
    return t.float().cpu().numpy()


def one_rounding(a, b):
    return np.abs(a - b) <= 2.0 ** -7 * np.abs(b) + 1e-6


def run_conv(torch, native, layer, mode, tc, x, w, b, mask, B, H, W):
    ci, co, _ = O.SHAPES[layer]
    cout = ci if mode else co
    last = layer == 7 and mode == 0
    out = torch.zeros((B, H, W, cout), dtype=torch.float32 if last else torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = native.pm_lpp_conv(layer, mode, tc, x.data_ptr(), w.data_ptr(), None if b is None else b.data_ptr(),
                            None if mask is None else mask.data_ptr(), out.data_ptr(), B, H, W, err.data_ptr(), s)
    assert rc == 0, native.pm_lpp_last_error()
    assert int(err.item()) == 0
    return to_np(out)


@pytest.mark.parametrize("dims", [(2, 11, 37), (1, 5, 9), (3, 24, 40)])
@pytest.mark.parametrize("layer", range(8))
def test_conv_layers_tensor_cores_match_cuda_cores_and_oracle(torch_cuda, native, layer, dims):
    """forward and data gradient of each layer (its channel counts and dilation) on B maps of
    H x W feature pixels: 11 x 37 (partial 16 x 8 tiles at the right and bottom; dilation 16
    reaches past the map), 5 x 9 (a map smaller than one tile), 3 maps of 24 x 40 (several
    tiles per map and per CTA)"""
    torch = torch_cuda
    ci, co, dil = O.SHAPES[layer]
    B, H, W = dims
    rng = np.random.default_rng(layer + 100 * H)
    xn = O.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    wn = O.bf16((rng.standard_normal((co, 9 * ci)) * 0.1).astype(np.float32))
    bn = (rng.standard_normal(co) * 0.1).astype(np.float32)
    z = O.conv(xn, wn, dil) + bn
    got_tc = run_conv(torch, native, layer, 0, 1, bf(torch, xn), bf(torch, wn), torch.from_numpy(bn).cuda(), None, B,
                      H, W)
    got_cc = run_conv(torch, native, layer, 0, 0, bf(torch, xn), bf(torch, wn), torch.from_numpy(bn).cuda(), None, B,
                      H, W)
    want = z if layer == 7 else O.bf16(np.maximum(z, 0).astype(np.float32))
    assert one_rounding(got_tc, got_cc).all()
    assert one_rounding(got_tc, want).all()
    if layer == 0:
        return
    # data gradient: the transposed, tap-mirrored weights (pm_lpp_weights_bf16 builds them)
    p = np.concatenate([wn.ravel(), bn]).astype(np.float32)
    wm = torch.zeros(co * 9 * ci, dtype=torch.bfloat16, device="cuda")
    wt = torch.zeros(co * 9 * ci, dtype=torch.bfloat16, device="cuda")
    assert native.pm_lpp_weights_bf16(layer, torch.from_numpy(p).cuda().data_ptr(), wm.data_ptr(), wt.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream) == 0
    assert (to_np(wm) == wn.ravel()).all()
    dyn = O.bf16(rng.standard_normal((B, H, W, co)).astype(np.float32))
    mn = O.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    w3 = wn.astype(np.float64).reshape(co, 9, ci)
    dx = np.zeros((B, H, W, ci))
    for t, (ty, tx) in enumerate(O.TAPS):
        dx += O.shift(dyn.astype(np.float64) @ w3[:, t, :], -ty * dil, -tx * dil)
    want = O.bf16(np.where(mn > 0, dx, 0.0).astype(np.float32))
    got_tc = run_conv(torch, native, layer, 1, 1, bf(torch, dyn), wt, None, bf(torch, mn), B, H, W)
    got_cc = run_conv(torch, native, layer, 1, 0, bf(torch, dyn), wt, None, bf(torch, mn), B, H, W)
    assert one_rounding(got_tc, got_cc).all()
    assert one_rounding(got_tc, want).all()


@pytest.mark.parametrize("dims", [(3, 19, 41), (4, 40, 64)])
@pytest.mark.parametrize("layer", range(8))
def test_weight_gradients_tensor_cores_match_cuda_cores_and_oracle(torch_cuda, native, layer, dims):
    """weight and bias gradients of each layer over 3 maps of 19 x 41 (45 units of 16 x 4
    pixels, partial at the right and bottom) and 4 maps of 40 x 64 (160 units: CTAs that sum
    two units, partial sums reduced in groups)"""
    torch = torch_cuda
    ci, co, dil = O.SHAPES[layer]
    B, H, W = dims
    rng = np.random.default_rng(10 + layer + H)
    xn = O.bf16(rng.standard_normal((B, H, W, ci)).astype(np.float32))
    dyn = O.bf16(rng.standard_normal((B, H, W, co)).astype(np.float32))
    x, dy = bf(torch, xn), bf(torch, dyn)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    scratch = torch.zeros(native.pm_lpp_wgrad_scratch_floats(layer, B, H, W), dtype=torch.float32, device="cuda")
    out = {}
    for tc in (1, 0):
        g = torch.zeros(co * 9 * ci + co, dtype=torch.float32, device="cuda")
        assert native.pm_lpp_wgrad(layer, tc, x.data_ptr(), dy.data_ptr(), scratch.data_ptr() if tc else None,
                                   g.data_ptr(), B, H, W, err.data_ptr(), s) == 0, native.pm_lpp_last_error()
        out[tc] = to_np(g)
    assert int(err.item()) == 0
    dw = np.zeros((co, 9, ci))
    flat = dyn.astype(np.float64).reshape(-1, co)
    for t, (ty, tx) in enumerate(O.TAPS):
        dw[:, t, :] = flat.T @ O.shift(xn.astype(np.float64), ty * dil, tx * dil).reshape(-1, ci)
    want = np.concatenate([dw.ravel(), flat.sum(0)])
    scale = np.abs(want).max()
    assert np.abs(out[1] - want).max() <= 1e-4 * scale
    assert np.abs(out[0] - want).max() <= 1e-4 * scale


def _net(torch):
    from cvt_b200.learn import PlaneProposal

    return PlaneProposal(seed=3)


def test_backward_pass_matches_oracle(torch_cuda):
    """loss and all eight layers' gradients of one batch, against the oracle's backward pass on
    the same BF16 weights"""
    torch = torch_cuda
    pp = _net(torch)
    rng = np.random.default_rng(5)
    B, H, W = 2, 12, 20
    xn = np.zeros((B, H, W, 16), np.float32)
    xn[..., :6] = rng.random((B, H, W, 6)) - 0.5
    xn = O.bf16(xn)
    tn = np.zeros((B, H, W, 4), np.float32)
    tn[..., 0] = rng.random((B, H, W)) * 12
    tn[..., 1:3] = rng.standard_normal((B, H, W, 2)) * 0.2
    tn[..., 3] = (rng.random((B, H, W)) > 0.1).astype(np.float32)
    loss, grads = pp.gradients(bf(torch, xn), torch.from_numpy(tn).cuda())
    pp.check_error()
    layers = [(p[:pp.nweights(l)].reshape(pp.shapes[l][1], -1), p[pp.nweights(l):]) for l, p in enumerate(pp.params())]
    acts, out = O.forward(xn, layers)
    want_loss, dl = O.loss_grad(out, tn, 4.0)
    want = O.backward(acts, layers, dl)
    assert abs(float(loss) - want_loss) <= 1e-3 * abs(want_loss)
    # the data gradients are rounded to BF16 at every layer, in both; where the two FP32 sums round
    # to neighbouring BF16 values the difference travels down, so the bound widens with depth
    for l in range(8):
        got = to_np(grads[l])
        w = np.concatenate([want[l][0].ravel(), want[l][1]])
        cos = float(got @ w / (np.linalg.norm(got) * np.linalg.norm(w) + 1e-30))
        rel = float(np.linalg.norm(got - w) / (np.linalg.norm(w) + 1e-30))
        depth = 7 - l
        assert cos > 0.999 - 0.0005 * depth and rel < 0.02 + 0.01 * depth, (l, cos, rel)


def test_input_target_upsample_match_oracle(torch_cuda, native):
    import torch

    from cvt_b200 import PMHuberStereo, scene
    from cvt_b200.learn import PlaneProposal

    L, R = scene.generate(4, 96, 64, 5, 2.0, 20.0)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    pp = PlaneProposal(seed=0)
    for view in (0, 1):
        got = to_np(pp.net_input(dL, dR, 4, view))[0]
        assert np.abs(got - O.net_input(L, R, 4, view)).max() <= 2.0 ** -8
    # targets from the planes of both views, against the oracle's restatement of k_target; the
    # left view's target disparity agrees with the pipeline's disparity map where both keep pixels
    res = PMHuberStereo().disparity_map(dL, dR, 3, 24.0, 3, pp=1, planes=True)
    st = torch.cuda.current_stream().cuda_stream
    pl, pr = to_np(res["planes_left"]), to_np(res["planes_right"])
    for view, (a, b) in enumerate(((res["planes_left"], res["planes_right"]), (res["planes_right"], res["planes_left"]))):
        t = torch.zeros((16, 24, 4), dtype=torch.float32, device="cuda")
        assert native.pm_lpp_target(a.data_ptr(), b.data_ptr(), 96, 64, 4, view, 24.0, t.data_ptr(), st) == 0
        tn = to_np(t)
        want = O.target(pl if view == 0 else pr, pr if view == 0 else pl, 4, view, 24.0)
        assert (tn[..., 3] == want[..., 3]).mean() > 0.99   # validity (a rounding at the 1 px test may flip)
        both = (tn[..., 3] > 0) & (want[..., 3] > 0)
        assert both.mean() > 0.3
        assert np.abs(tn[..., :3] - want[..., :3])[both].max() < 1e-4
    # upsampling of a random output map, both views
    o4 = torch.from_numpy(np.random.default_rng(1).standard_normal((16, 24, 16)).astype(np.float32) * 0.3).cuda()
    o4[..., 0] = o4[..., 0].abs() * 10
    for view in (0, 1):
        disp = torch.zeros((64, 96), dtype=torch.float32, device="cuda")
        nm = torch.zeros((64, 96, 4), dtype=torch.float32, device="cuda")
        assert native.pm_lpp_upsample(o4.data_ptr(), 24, 16, 96, 64, 4, view, 24.0, disp.data_ptr(), nm.data_ptr(),
                                      st) == 0
        wd, wnm = O.upsample(to_np(o4), 96, 64, 4, view, 24.0)
        assert np.abs(to_np(disp) - wd).max() <= 1e-4 * 24 and np.abs(to_np(nm) - wnm).max() <= 1e-5


def test_propose_matches_oracle_forward(torch_cuda):
    """the single native call (input, 8 convolutions, upsampling) against the oracle's forward
    pass on the same BF16 weights; one BF16 rounding of slack per layer on the disparity"""
    import torch

    from cvt_b200 import scene
    from cvt_b200.learn import PlaneProposal

    pp = PlaneProposal(seed=7)
    L, R = scene.generate(8, 160, 96, 6, 2.0, 50.0)
    dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    layers = [(p[:pp.nweights(l)].reshape(pp.shapes[l][1], -1), p[pp.nweights(l):]) for l, p in enumerate(pp.params())]
    for view in (0, 1):
        d, n = pp.propose(dL, dR, 64.0, view)
        pp.check_error()
        _, out = O.forward(O.net_input(L, R, 4, view)[None], layers)
        wd, wn = O.upsample(out[0], 160, 96, 4, view, 64.0)
        assert np.abs(to_np(d) - wd).max() <= 0.05 * max(np.abs(wd).max(), 1.0)
        assert np.abs(to_np(n) - wn).max() <= 0.05


def _small_set(torch, pairs, seed):
    from cvt_b200.learn import make_training_set

    return make_training_set(pairs, 192, 128, seed=seed, dmax=32.0, patch=3, iterations=4)


def test_checkpoint_resume_equals_uninterrupted_training(torch_cuda, tmp_path):
    """train 6 steps, save (weights, Adam moments, step, seed), train 6 more; a network loaded
    from the checkpoint and trained the same 6 steps ends with the same parameters, bit for bit"""
    import torch

    from cvt_b200.learn import PlaneProposal

    x, t = _small_set(torch, 8, 300)
    a = PlaneProposal(seed=11)
    a.train(x, t, epochs=3, batch=8, lr=1e-3, seed=1)
    ck = str(tmp_path / "ck.npz")
    a.save(ck)
    a.train(x, t, epochs=3, batch=8, lr=1e-3, seed=2)
    b = PlaneProposal.load(ck)
    assert b.step == 6
    b.train(x, t, epochs=3, batch=8, lr=1e-3, seed=2)
    for pa, pb in zip(a.params(), b.params()):
        assert (pa == pb).all()


def test_training_beats_random_initialisation(torch_cuda):
    """a short training run on 48 small procedural pairs lowers the loss, and on held-out pairs
    the learned start + 1 iteration has a lower mean matching cost than a random start + 1"""
    import torch

    from cvt_b200 import PMHuberStereo, scene
    from cvt_b200.learn import PlaneProposal

    x, t = _small_set(torch, 48, 400)
    pp = PlaneProposal(seed=1)
    losses = pp.train(x, t, epochs=40, batch=16, lr=2e-3, seed=0)
    ls = losses.cpu().numpy()
    assert ls[-10:].mean() < 0.7 * ls[:10].mean(), (ls[:10].mean(), ls[-10:].mean())
    pm = PMHuberStereo()
    wins = 0
    for s in range(3):
        L, R = scene.generate(900 + s, 192, 128, 10, 2.0, 28.0)
        dL, dR = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
        d, n = pp.propose(dL, dR, 32.0, 0)
        dr, nr = pp.propose(dL, dR, 32.0, 1)
        lrn = pm.disparity_map(dL, dR, 3, 32.0, 1, pp=1, planes=True, initdisparity=d, initnormalmap=n,
                               initdisparity_right=dr, initnormalmap_right=nr)
        rnd = pm.disparity_map(dL, dR, 3, 32.0, 1, pp=1, planes=True)
        cl = to_np(lrn["planes_left"])[..., 3]
        cr = to_np(rnd["planes_left"])[..., 3]
        wins += float(cl[cl < 2].mean()) < float(cr[cr < 2].mean())
    assert wins == 3


def test_committed_weights_load_and_propose(torch_cuda):
    """the weights trained at the full recipe (cvt_b200/weights/, written by
    cvt_b200/train_proposal.py) load and give finite proposals in range"""
    import torch

    from cvt_b200 import scene
    from cvt_b200.learn import PlaneProposal, default_weights

    path = default_weights()
    assert os.path.exists(path), path
    pp = PlaneProposal.load(path)
    L, R = scene.generate(2, 256, 192, 8, 2.0, 100.0)
    d, n = pp.propose(torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(), 128.0, 0)
    d, n = to_np(d), to_np(n)
    assert np.isfinite(d).all() and (d >= 0).all() and (d <= 128).all() and np.isfinite(n).all()
