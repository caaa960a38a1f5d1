"""ORACLE — test infrastructure only (tests/).

numpy restatement of the learned plane proposal's network (cvt_b200/csrc/pm_learn.cu): the
cost-volume features, the 3x3 convolutions with BF16 inputs and FP32 accumulation, ReLU,
soft-argmin, the smooth-L1 loss and the backward pass (data gradients through the ReLU
masks, weight and bias gradients), with the BF16 roundings the kernels make at the same
points.  Activations are NHWC (batch, rows, columns, 32 channels); a layer's weights are
wmat[n][t][c] (output channel, tap t = (dy + 1) * 3 + (dx + 1), input channel) and bias[n].
"""
import numpy as np

CH = 32
TAPS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]


def bf16(a):
    """round float32 to the nearest BF16 (ties to even), returned as float32"""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def shift(x, dy, dx):
    """x[b, y + dy, x + dx, :] with zeros outside"""
    B, H, W, C = x.shape
    out = np.zeros_like(x)
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[:, yd, xd, :] = x[:, ys, xs, :]
    return out


def conv(x, wmat):
    """sum over taps and channels in float64 of the (BF16-valued) inputs"""
    x = x.astype(np.float64)
    w = wmat.astype(np.float64).reshape(CH, 9, CH)
    out = np.zeros(x.shape[:3] + (CH,), np.float64)
    for t, (dy, dx) in enumerate(TAPS):
        out += shift(x, dy, dx) @ w[:, t, :].T
    return out


def forward(feat, layers):
    """feat: (B, H4, W4, 32) BF16 values; layers: [(wmat (32, 288), bias (32,))] * 6.
    Returns (acts, logits): acts[0] = feat, acts[l] = BF16 ReLU output of layer l - 1."""
    acts = [feat]
    x = feat
    for i, (w, b) in enumerate(layers):
        z = conv(x, bf16(w)) + b
        if i < len(layers) - 1:
            x = bf16(np.maximum(z, 0.0).astype(np.float32))
            acts.append(x)
        else:
            logits = z.astype(np.float32)
    return acts, logits


SKIP = 4.0


def softargmin(logits, feat=None, step=1.0):
    """soft-argmin over the logits plus SKIP times the cost volume (the features); hypotheses
    `step` quarter pixels apart"""
    l = logits.astype(np.float64)
    if feat is not None:
        l = l + SKIP * feat.astype(np.float64)
    p = np.exp(-(l - l.min(-1, keepdims=True)))
    p /= p.sum(-1, keepdims=True)
    d = step * (p * np.arange(CH)).sum(-1)
    return p, d


def loss_grad(logits, target, feat=None, step=1.0):
    """smooth-L1 mean over targets >= 0; returns (loss, dlogits as BF16)"""
    p, d = softargmin(logits, feat, step)
    valid = target >= 0
    n = max(int(valid.sum()), 1)
    r = d - target
    l = np.where(np.abs(r) < 1, 0.5 * r * r, np.abs(r) - 0.5)
    g = np.where(np.abs(r) < 1, r, np.sign(r)) / n
    g = np.where(valid, g, 0.0)
    dl = -p * (step * np.arange(CH) - d[..., None]) * g[..., None]
    return float(np.where(valid, l, 0).sum() / n), bf16(dl.astype(np.float32))


def backward(acts, layers, dlogits):
    """weight and bias gradients of every layer (float64), with the data gradients rounded to
    BF16 after the ReLU mask, as the kernels store them"""
    grads = [None] * len(layers)
    dy = dlogits.astype(np.float64)
    for i in range(len(layers) - 1, -1, -1):
        x = acts[i].astype(np.float64)
        gw = np.zeros((CH, 9, CH))
        for t, (ddy, ddx) in enumerate(TAPS):
            gw[:, t, :] = np.einsum("bhwn,bhwc->nc", dy, shift(x, ddy, ddx))
        grads[i] = (gw.reshape(CH, 9 * CH), dy.sum((0, 1, 2)))
        if i > 0:
            w = bf16(layers[i][0]).astype(np.float64).reshape(CH, 9, CH)
            dx = np.zeros_like(x)
            for t, (ddy, ddx) in enumerate(TAPS):
                dx += shift(dy, -ddy, -ddx) @ w[:, t, :]
            dx = np.where(acts[i] > 0, dx, 0.0)
            dy = bf16(dx.astype(np.float32)).astype(np.float64)
    return grads


def features(left, right, view=0, step=1, scale=4):
    """grey of scale x scale blocks and the 32-hypothesis cost volume (BF16 values) of the left
    (view 0) or right view (1), hypotheses `step` feature pixels apart, as k_grey / k_costvol"""
    def grey4(img):
        H4, W4 = img.shape[0] // scale, img.shape[1] // scale
        f = img[:scale * H4, :scale * W4, :3].astype(np.float32)
        g = (f[..., 0] * np.float32(0.2126) + f[..., 1] * np.float32(0.7152) + f[..., 2] * np.float32(0.0722))
        return g.reshape(H4, scale, W4, scale).sum((1, 3)) / np.float32(scale * scale * 255)
    gl, gr = grey4(left).astype(np.float64), grey4(right).astype(np.float64)
    if view:
        gl, gr = gr, gl
    sgn = 1 if view else -1
    H4, W4 = gl.shape
    cv = np.zeros((H4, W4, CH))
    xs = np.arange(W4)
    for d in range(CH):
        xm = xs + sgn * step * d
        inside = (xm >= 0) & (xm < W4)
        other = gr[:, np.clip(xm, 0, W4 - 1)]
        diff = np.where(inside[None, :], np.abs(gl - other), 1.0)
        s = np.zeros_like(diff)
        n = np.zeros_like(diff)
        for j in (-1, 0, 1):
            for i in (-1, 0, 1):
                ok = np.zeros_like(diff, bool)
                ok[max(0, -j):H4 - max(0, j), max(0, -i):W4 - max(0, i)] = True
                sh = np.zeros_like(diff)
                sh[max(0, -j):H4 - max(0, j), max(0, -i):W4 - max(0, i)] = diff[max(0, j):H4 + min(0, j), max(0, i):W4 + min(0, i)]
                s += sh
                n += ok
        cv[:, :, d] = 8.0 * s / n
    return bf16(cv.astype(np.float32))[None]
