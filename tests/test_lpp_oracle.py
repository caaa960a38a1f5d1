"""The learned proposal's numpy oracle (oracle/lpp_oracle.py): its backward pass against
finite differences, in exact (float64, no BF16 rounding) arithmetic."""
import numpy as np

from oracle import lpp_oracle as L


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(L, "bf16", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(1)
    x = rng.random((1, 4, 6, 32))
    layers = [(rng.standard_normal((32, 288)) * 0.08, rng.standard_normal(32) * 0.05) for _ in range(6)]
    t = rng.random((1, 4, 6)) * 10
    t[0, 1, 2] = -1.0   # masked target

    def fwd(ls):
        acts, h = [x], x
        for i, (w, b) in enumerate(ls):
            z = L.conv(h, w) + b
            if i < 5:
                h = np.maximum(z, 0)
                acts.append(h)
        return acts, z

    acts, lg = fwd(layers)
    _, dl = L.loss_grad(lg, t)
    g = L.backward(acts, layers, dl)
    worst = 0.0
    for li in range(6):
        for (i, j) in ((5, 100), (31, 287), (7, 33), (20, 200)):
            e = 1e-6
            lp = [(w.copy(), b.copy()) for w, b in layers]
            lm = [(w.copy(), b.copy()) for w, b in layers]
            lp[li][0][i, j] += e
            lm[li][0][i, j] -= e
            fd = (L.loss_grad(fwd(lp)[1], t)[0] - L.loss_grad(fwd(lm)[1], t)[0]) / (2 * e)
            worst = max(worst, abs(fd - g[li][0][i, j]) / max(abs(fd), 1e-3))
        lp = [(w.copy(), b.copy()) for w, b in layers]
        lm = [(w.copy(), b.copy()) for w, b in layers]
        lp[li][1][3] += 1e-6
        lm[li][1][3] -= 1e-6
        fd = (L.loss_grad(fwd(lp)[1], t)[0] - L.loss_grad(fwd(lm)[1], t)[0]) / 2e-6
        worst = max(worst, abs(fd - g[li][1][3]) / max(abs(fd), 1e-3))
    assert worst < 1e-5, worst


def test_bf16_rounding_is_nearest_even():
    a = np.array([1.0, 1.00390625, 1.01171875, 1.0078125 + 2 ** -9, -3.3, 0.0], np.float32)
    b = L.bf16(a)
    assert b[0] == 1.0 and b[1] == 1.0 and b[2] == 1.015625 and b[3] == 1.0078125
    assert (b.view(np.uint32) & 0xFFFF == 0).all()
