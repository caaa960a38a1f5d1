"""The learned plane proposal on the GPU (cvt_b200/csrc/pm_learn.cu, cvt_b200/learn.py):
the tcgen05 convolution against the CUDA-core kernel and the numpy oracle, the weight
gradients and the whole backward pass against the oracle, the features, and what a short
training run gains over random initialisation."""
import numpy as np
import pytest

from oracle import lpp_oracle as O

pytestmark = pytest.mark.gpu

CH, KTOT = 32, 288


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


def conv(torch, native, epi, tc, x, w, b, mask, B, H, W):
    out = torch.zeros((B, H, W, CH), dtype=torch.float32 if epi == 1 else torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert native.pm_lpp_conv(epi, tc, x.data_ptr(), w.data_ptr(), None if b is None else b.data_ptr(),
                              None if mask is None else mask.data_ptr(), out.data_ptr(), B, H, W, err.data_ptr(), s) == 0
    assert int(err.item()) == 0
    return to_np(out)


@pytest.mark.parametrize("B,H,W", [(1, 4, 32), (2, 9, 13), (1, 23, 37)])
def test_tensor_core_conv_matches_cuda_cores_and_oracle(torch_cuda, native, B, H, W):
    """all three epilogues; sizes with a partial last tile of 128 pixels"""
    torch = torch_cuda
    rng = np.random.default_rng(B * 100 + H)
    xn = O.bf16(rng.standard_normal((B, H, W, CH)).astype(np.float32))
    wn = O.bf16((rng.standard_normal((CH, KTOT)) * 0.1).astype(np.float32))
    bn = (rng.standard_normal(CH) * 0.1).astype(np.float32)
    mn = O.bf16(rng.standard_normal((B, H, W, CH)).astype(np.float32))
    x, w, b, mk = bf(torch, xn), bf(torch, wn), torch.from_numpy(bn).cuda(), bf(torch, mn)
    z = O.conv(xn, wn)
    for epi in (0, 1, 2):
        tc = conv(torch, native, epi, 1, x, w, b, mk, B, H, W)
        ref = conv(torch, native, epi, 0, x, w, b, mk, B, H, W)
        if epi == 0:
            want = O.bf16(np.maximum(z + bn, 0).astype(np.float32))
        elif epi == 1:
            want = (z + bn).astype(np.float32)
        else:
            want = O.bf16(np.where(mn > 0, z, 0).astype(np.float32))
        tol = 1e-4 if epi == 1 else 2 ** -7
        for got in (tc, ref):
            err = np.abs(got - want) / (np.abs(want) + 1e-2)
            assert err.max() < tol, (epi, err.max())


def test_weight_gradient_matches_oracle(torch_cuda, native):
    torch = torch_cuda
    rng = np.random.default_rng(5)
    B, H, W = 2, 11, 17
    xn = O.bf16(rng.standard_normal((B, H, W, CH)).astype(np.float32))
    dyn = O.bf16((rng.standard_normal((B, H, W, CH)) * 0.01).astype(np.float32))
    x, dy = bf(torch, xn), bf(torch, dyn)
    scratch = torch.empty(native.pm_lpp_wgrad_scratch_floats(B, H, W, 64), dtype=torch.float32, device="cuda")
    g = torch.empty(CH * KTOT + CH, dtype=torch.float32, device="cuda")
    assert native.pm_lpp_wgrad(x.data_ptr(), dy.data_ptr(), scratch.data_ptr(), g.data_ptr(), B, H, W, 64,
                               torch.cuda.current_stream().cuda_stream) == 0
    g = to_np(g)
    gw = np.zeros((CH, 9, CH))
    for t, (ddy, ddx) in enumerate(O.TAPS):
        gw[:, t, :] = np.einsum("bhwn,bhwc->nc", dyn.astype(np.float64), O.shift(xn.astype(np.float64), ddy, ddx))
    assert np.abs(g[:CH * KTOT] - gw.ravel()).max() < 1e-4 * np.abs(gw).max() + 1e-7
    assert np.abs(g[CH * KTOT:] - dyn.astype(np.float64).sum((0, 1, 2))).max() < 1e-5


@pytest.mark.parametrize("tc,step", [(1, 1), (0, 1), (1, 2)])
def test_backward_matches_oracle(torch_cuda, native, tc, step):
    """loss and the gradients of all six layers against the oracle's backward pass on the same
    BF16 weights and inputs: relative error of each layer's gradient < 1e-2, cosine > 0.999"""
    torch = torch_cuda
    from cvt_b200.learn import PlaneProposal

    pp = PlaneProposal(seed=3, tensor_cores=bool(tc), step=step)
    rng = np.random.default_rng(7)
    B, H, W = 2, 12, 20
    feats = O.bf16((rng.random((B, H, W, CH)) * 2).astype(np.float32))
    target = (rng.random((B, H, W)) * 20).astype(np.float32)
    target[0, :2, :] = -1.0
    loss, grads = pp.gradients(bf(torch, feats), torch.from_numpy(target).cuda())
    layers = [(a[:CH * KTOT].reshape(CH, KTOT), a[CH * KTOT:]) for a in pp.params()]
    acts, logits = O.forward(feats, layers)
    oloss, dl = O.loss_grad(logits, target, feats, step)
    og = O.backward(acts, layers, dl)
    assert abs(loss - oloss) < 1e-3 * max(1.0, abs(oloss)), (loss, oloss)
    for l in range(6):
        g = to_np(grads[l])
        want = np.concatenate([og[l][0].ravel(), og[l][1]])
        rel = np.linalg.norm(g - want) / np.linalg.norm(want)
        cos = float(g @ want / (np.linalg.norm(g) * np.linalg.norm(want)))
        assert rel < 1e-2 and cos > 0.999, (l, rel, cos)


def test_features_match_oracle(torch_cuda, native):
    torch = torch_cuda
    from cvt_b200 import scene
    from cvt_b200.learn import PlaneProposal

    L, R = scene.generate(3, 203, 121, 6, 2.0, 60.0)
    for view in (0, 1):
        for step, scale in ((1, 4), (2, 4), (2, 2)):
            f = to_np(PlaneProposal(step=step, scale=scale).features(torch.from_numpy(L).cuda(),
                                                                     torch.from_numpy(R).cuda(), view))
            want = O.features(L, R, view, step, scale)
            assert f.shape == want.shape
            assert (np.abs(f - want) <= 2 ** -7 * np.abs(want) + 1e-6).all(), (view, step, scale)


def test_training_gains_over_random_init(torch_cuda, native):
    """a short training run on 24 scenes; on 3 held-out scenes the learned initialisation plus
    one PatchMatch iteration ends at a lower mean matching cost, and closer to plain 8-iteration
    PatchMatch, than the random initialisation plus one iteration"""
    torch = torch_cuda
    from cvt_b200 import scene
    from cvt_b200.learn import PlaneProposal, make_training_set
    from cvt_b200.stereo import PMHuberStereo

    feats, target = make_training_set(24, 256, 192, seed=500)
    pp = PlaneProposal(seed=1)
    losses = pp.train(feats, target, steps=300, batch=8, lr=2e-3)
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:20]), (losses[:3], losses[-3:])
    pm = PMHuberStereo()
    gains = []
    for i in range(3):
        l, r = scene.generate(900 + i, 256, 192, 10, 2.0, 60.0)
        dl, dr = torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()
        ref = pm.disparity_map(dl, dr, 7, 128.0, 8, pp=0, planes=True)
        rnd = pm.disparity_map(dl, dr, 7, 128.0, 1, pp=0, planes=True)
        lrn = pm.disparity_map(dl, dr, 7, 128.0, 1, pp=0, planes=True, initdisparity=pp.propose(dl, dr, 0),
                               initdisparity_right=pp.propose(dl, dr, 1))
        d8 = to_np(ref["dmap"])
        res = []
        for run in (rnd, lrn):
            cost = to_np(run["planes_left"])[..., 3]
            agree = np.mean(np.abs(to_np(run["dmap"]) - d8) < 1.0)
            res.append((float(np.mean(cost[cost < 2])), float(agree)))
        print("scene %d: random+1 cost %.4f agree %.3f | learned+1 cost %.4f agree %.3f" % (i, *res[0], *res[1]))
        gains.append((res[0][0] - res[1][0], res[1][1] - res[0][1]))
    assert all(c > 0 for c, _ in gains) and all(a > 0 for _, a in gains), gains


def test_init2_without_right_equals_disparity_map(torch_cuda, native):
    """pm_disparity_map_init2_device with no right initial disparity is disparityMap itself, bit
    for bit; with one it is deterministic and its right view starts from it (cost after one
    iteration below the random start's)"""
    torch = torch_cuda
    from cvt_b200 import scene
    from cvt_b200.stereo import PMHuberStereo
    from oracle.pyoracle import bits_equal

    l, r, gd, gn = scene.generate(41, 160, 96, 6, 2.0, 24.0, with_gt=True)
    dl, dr = torch.from_numpy(l).cuda(), torch.from_numpy(r).cuda()
    pm = PMHuberStereo()
    initl = torch.from_numpy(gd).cuda()
    a = pm.disparity_map(dl, dr, 4, 32.0, 1, pp=1, planes=True, initdisparity=initl)
    b = {k: torch.empty_like(v) for k, v in a.items()}
    assert native.pm_disparity_map_init2_device(pm._h, dl.data_ptr(), dr.data_ptr(), 160, 96, 640, 4, 32.0, 1, 1,
                                                b["dmap"].data_ptr(), None, initl.data_ptr(), None,
                                                b["planes_left"].data_ptr(), b["planes_right"].data_ptr(),
                                                torch.cuda.current_stream().cuda_stream) == 0
    for k in ("dmap", "planes_left", "planes_right"):
        assert bits_equal(to_np(a[k]), to_np(b[k])).all(), k
    # right view from the left ground truth warped to the right image (x_R = x_L - d)
    dgr = np.zeros_like(gd)
    ys, xs = np.nonzero(gd > 0)
    xr = np.round(xs - gd[ys, xs]).astype(int)
    ok = (xr >= 0) & (xr < 160)
    dgr[ys[ok], xr[ok]] = gd[ys[ok], xs[ok]]
    initr = torch.from_numpy(dgr).cuda()
    c1 = pm.disparity_map(dl, dr, 4, 32.0, 1, pp=0, planes=True, initdisparity=initl, initdisparity_right=initr)
    c2 = pm.disparity_map(dl, dr, 4, 32.0, 1, pp=0, planes=True, initdisparity=initl, initdisparity_right=initr)
    assert bits_equal(to_np(c1["planes_right"]), to_np(c2["planes_right"])).all()
    rc = to_np(c1["planes_right"])[..., 3]
    rr = to_np(a["planes_right"])[..., 3]
    assert np.mean(rc[rc < 2]) < np.mean(rr[rr < 2])


def test_one_call_proposal_equals_the_step_by_step_path(torch_cuda, native):
    """pm_lpp_propose_device (one native call) equals features -> six convolutions ->
    soft-argmin -> upsampling run call by call, bit for bit, for both views"""
    torch = torch_cuda
    from cvt_b200 import scene
    from cvt_b200.learn import SKIP, PlaneProposal
    from oracle.pyoracle import bits_equal

    pp = PlaneProposal(seed=4)
    L, R = scene.generate(8, 150, 93, 6, 2.0, 60.0)
    dl, dr = torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda()
    s = torch.cuda.current_stream().cuda_stream
    for view in (0, 1):
        one = to_np(pp.propose(dl, dr, view))
        f = pp.features(dl, dr, view)
        _, logits = pp.forward(f)
        H4, W4 = f.shape[1:3]
        d4 = torch.empty((H4, W4), dtype=torch.float32, device="cuda")
        assert native.pm_lpp_softargmin(logits.data_ptr(), f.data_ptr(), SKIP, float(pp.hstep), None, d4.data_ptr(),
                                        None, None, H4 * W4, 0.0, s) == 0
        up = torch.empty((93, 150), dtype=torch.float32, device="cuda")
        assert native.pm_lpp_upsample(d4.data_ptr(), W4, H4, 150, 93, pp.scale, up.data_ptr(), s) == 0
        assert bits_equal(one, to_np(up)).all(), view
