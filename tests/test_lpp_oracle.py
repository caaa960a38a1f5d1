"""The learned proposal's numpy oracle (oracle/lpp_oracle.py): its backward pass against
finite differences, in exact (float64, no BF16 rounding) arithmetic, and its pieces against
their definitions."""
import numpy as np

from oracle import lpp_oracle as L


def _layers(rng):
    return [(rng.standard_normal((co, 9 * ci)) * np.sqrt(2.0 / (9 * ci)), rng.standard_normal(co) * 0.05)
            for ci, co, _ in L.SHAPES]


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(L, "bf16", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(1)
    x = np.zeros((1, 6, 9, 16))
    x[..., :6] = rng.random((1, 6, 9, 6)) - 0.5
    layers = _layers(rng)
    t = np.zeros((1, 6, 9, 4))
    t[..., 0] = rng.random((1, 6, 9)) * 10
    t[..., 1:3] = rng.standard_normal((1, 6, 9, 2)) * 0.2
    t[..., 3] = 1.0
    t[0, 1, 2, 3] = 0.0   # an invalid target pixel
    wn = 4.0

    def loss(ls):
        return L.loss_grad(L.forward(x, ls)[1], t, wn)[0]

    acts, out = L.forward(x, layers)
    _, dl = L.loss_grad(out, t, wn)
    g = L.backward(acts, layers, dl)
    worst = 0.0
    for li, (ci, co, _) in enumerate(L.SHAPES):
        for (i, j) in ((0, 0), (co - 1, 9 * ci - 1), (co // 2, 4 * ci + 1), (1, 7 * ci + 2)):
            e = 1e-6
            lp = [(w.copy(), b.copy()) for w, b in layers]
            lm = [(w.copy(), b.copy()) for w, b in layers]
            lp[li][0][i, j] += e
            lm[li][0][i, j] -= e
            fd = (loss(lp) - loss(lm)) / (2 * e)
            worst = max(worst, abs(fd - g[li][0][i, j]) / max(abs(fd), 1e-3))
        lp = [(w.copy(), b.copy()) for w, b in layers]
        lm = [(w.copy(), b.copy()) for w, b in layers]
        lp[li][1][1] += 1e-6
        lm[li][1][1] -= 1e-6
        fd = (loss(lp) - loss(lm)) / 2e-6
        worst = max(worst, abs(fd - g[li][1][1]) / max(abs(fd), 1e-3))
    assert worst < 1e-5, worst


def test_dilated_conv_taps():
    """a single tap of weight 1 moves the image by the tap offset times the dilation"""
    x = np.zeros((1, 20, 24, 16))
    x[0, 10, 12, 3] = 1.0
    w = np.zeros((16, 9 * 16))
    w[5, 2 * 16 + 3] = 1.0   # tap (dy, dx) = (-1, +1), input channel 3 -> output channel 5
    y = L.conv(x, w, 4)
    assert y[0, 14, 8, 5] == 1.0 and np.count_nonzero(y) == 1


def test_input_and_upsample_mirror():
    rng = np.random.default_rng(2)
    left = rng.integers(0, 256, (16, 24, 4), dtype=np.uint8)
    right = rng.integers(0, 256, (16, 24, 4), dtype=np.uint8)
    a = L.net_input(left, right, 4, 0)
    b = L.net_input(left, right, 4, 1)
    assert a.shape == (4, 6, 16) and (a[..., 6:] == 0).all()
    # the mirrored pair holds the right image's blocks first, in mirrored order
    assert np.allclose(b[..., :3], a[:, ::-1, 3:6], atol=1e-2) and np.allclose(b[..., 3:6], a[:, ::-1, :3], atol=1e-2)
    o4 = np.zeros((4, 6, 16), np.float32)
    o4[..., 0] = np.arange(6)[None, :]
    o4[..., 2] = 0.25
    d, n = L.upsample(o4, 24, 16, 4, 0, 100.0)
    dr, nr = L.upsample(o4, 24, 16, 4, 1, 100.0)
    assert np.allclose(dr, d[:, ::-1]) and np.allclose(nr[..., 1], -n[:, ::-1, 1])
    assert (d >= 0).all() and np.allclose(np.linalg.norm(n[..., :3], axis=-1), 1.0, atol=1e-6)


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.00390625, 1.01171875, 1.0078125 + 2 ** -9, -3.3, 0.0], np.float32)
    b = L.bf16(a)
    assert b[0] == 1.0 and b[1] == 1.0 and b[2] == 1.015625 and b[3] == 1.0078125
    assert (b.view(np.uint32) & 0xFFFF == 0).all()
