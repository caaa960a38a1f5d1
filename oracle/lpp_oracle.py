"""ORACLE — test infrastructure only (tests/).

numpy restatement of the learned plane proposal's network (cvt_b200/csrc/pm_learn.cu): the
input (block means of both views' RGB), the dilated 3x3 convolutions with BF16 inputs and FP32
accumulation, ReLU, the L1 loss on (d, nx, ny) and the backward pass (data gradients through
the ReLU masks, weight and bias gradients), with the BF16 roundings the kernels make at the
same points, and the upsampling to full resolution.  Activations are NHWC (batch, rows,
columns, channels); layer l's weights are w[co][t][ci] (tap t = (dy + 1) * 3 + (dx + 1) in
units of the layer's dilation) and bias[co].
"""
import numpy as np

# (input channels, output channels, dilation) of the eight layers (pm_lpp_layer_shape)
SHAPES = [(16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 4), (64, 64, 8), (64, 64, 16), (64, 32, 1), (32, 16, 1)]
NL = len(SHAPES)
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
    if abs(dy) >= H or abs(dx) >= W:
        return out
    ys, yd = (slice(dy, H), slice(0, H - dy)) if dy >= 0 else (slice(0, H + dy), slice(-dy, H))
    xs, xd = (slice(dx, W), slice(0, W - dx)) if dx >= 0 else (slice(0, W + dx), slice(-dx, W))
    out[:, yd, xd, :] = x[:, ys, xs, :]
    return out


def conv(x, w, dil):
    """sum over taps and channels in float64 of the (BF16-valued) inputs; w (COUT, 9 * CIN)"""
    x = x.astype(np.float64)
    cout = w.shape[0]
    cin = x.shape[3]
    wr = np.asarray(w, np.float64).reshape(cout, 9, cin)
    out = np.zeros(x.shape[:3] + (cout,), np.float64)
    for t, (dy, dx) in enumerate(TAPS):
        out += shift(x, dy * dil, dx * dil) @ wr[:, t, :].T
    return out


def net_input(left, right, scale, right_view=0):
    """(H4, W4, 16) float32 BF16 values: first then second view's RGB block means of k / 255
    minus 0.5 (k_input); right_view: the mirrored pair, right image first"""
    H, W = left.shape[:2]
    H4, W4 = H // scale, W // scale
    a, b = (right[:, ::-1], left[:, ::-1]) if right_view else (left, right)
    out = np.zeros((H4, W4, 16), np.float32)
    for k, img in enumerate((a, b)):
        blk = img[:H4 * scale, :W4 * scale, :3].astype(np.float32) / np.float32(255.0)
        blk = blk.reshape(H4, scale, W4, scale, 3)
        s = np.zeros((H4, W4, 3), np.float32)
        for dy in range(scale):   # the kernel's summation order: rows of the block, then columns
            for dx in range(scale):
                s = s + blk[:, dy, :, dx, :]
        out[..., 3 * k:3 * k + 3] = s * np.float32(1.0 / (scale * scale)) - np.float32(0.5)
    return bf16(out)


def forward(x, layers):
    """x: (B, H4, W4, 16) BF16 values; layers: [(w (COUT, 9 CIN), bias (COUT,))] * 8.
    Returns (acts, out): acts[0] = x, acts[l] = BF16 ReLU output of layer l - 1; out = the last
    layer's FP32 output (B, H4, W4, 16)."""
    acts = [x]
    h = x
    for i, ((w, b), (_, _, dil)) in enumerate(zip(layers, SHAPES)):
        z = conv(h, bf16(w), dil) + b
        if i < NL - 1:
            h = bf16(np.maximum(z, 0.0))
            acts.append(h)
    return acts, z


def loss_grad(out, target, wn):
    """L1 loss of out[..., :3] against target (d, nx, ny, valid) and its gradient (BF16-rounded
    after scaling by 1 / the number of valid pixels, as k_loss)"""
    valid = target[..., 3] > 0
    e = out[..., :3] - target[..., :3]
    w = np.array([1.0, wn, wn])
    loss = float((np.abs(e) * w)[valid].sum())
    count = max(int(valid.sum()), 1)
    g = np.zeros(out.shape, np.float64)
    g[..., :3] = np.sign(e) * w / count
    g[~valid] = 0.0
    return loss / count, bf16(g)


def backward(acts, layers, dout):
    """weight and bias gradients of every layer (list of (dW (COUT, 9 CIN), db (COUT,))) for the
    output gradient dout; data gradients are BF16-rounded and masked by the ReLU as in the
    kernels"""
    grads = [None] * NL
    dy = np.asarray(dout, np.float64)
    for l in range(NL - 1, -1, -1):
        cin, cout, dil = SHAPES[l]
        x = acts[l].astype(np.float64)
        dw = np.zeros((cout, 9, cin), np.float64)
        flat = dy.reshape(-1, cout)
        for t, (ty, tx) in enumerate(TAPS):
            dw[:, t, :] = flat.T @ shift(x, ty * dil, tx * dil).reshape(-1, cin)
        grads[l] = (dw.reshape(cout, 9 * cin), flat.sum(0))
        if l > 0:
            w = bf16(layers[l][0]).astype(np.float64).reshape(cout, 9, cin)
            dx = np.zeros(x.shape, np.float64)
            for t, (ty, tx) in enumerate(TAPS):
                dx += shift(dy @ w[:, t, :], -ty * dil, -tx * dil)
            dy = bf16(np.where(acts[l] > 0, dx, 0.0)).astype(np.float64)
    return grads


def upsample(out4, W, H, scale, right_view, dmax):
    """full-resolution disparity and normal map (k_upsample)"""
    H4, W4 = out4.shape[:2]
    xs = np.arange(W)
    if right_view:
        xs = W - 1 - xs
    u = np.clip((xs.astype(np.float32) + np.float32(0.5)) / np.float32(scale) - np.float32(0.5), 0, W4 - 1)
    v = np.clip((np.arange(H).astype(np.float32) + np.float32(0.5)) / np.float32(scale) - np.float32(0.5), 0, H4 - 1)
    u0, v0 = u.astype(int), v.astype(int)
    u1, v1 = np.minimum(u0 + 1, W4 - 1), np.minimum(v0 + 1, H4 - 1)
    a, b = (u - u0)[None, :, None], (v - v0)[:, None, None]
    o = out4[..., :3].astype(np.float64)
    r = (1 - b) * ((1 - a) * o[v0][:, u0] + a * o[v0][:, u1]) + b * ((1 - a) * o[v1][:, u0] + a * o[v1][:, u1])
    d = np.clip(r[..., 0] * scale, 0.0, dmax)
    nx, ny = r[..., 1], (-r[..., 2] if right_view else r[..., 2])
    n = np.stack([nx, ny, np.sqrt(np.maximum(1 - nx * nx - ny * ny, 0.01)), np.zeros_like(nx)], -1)
    return d, n


def target(planes, other, scale, right_view, dmax):
    """training target (k_target): per feature block the means over valid pixels of d / scale,
    nx, ny and 1 when at least half of the block is valid; planes of this view and the other
    (H, W, 4) float32; float32 arithmetic per pixel as in the kernel (sums in float64 here)"""
    H, W = planes.shape[:2]
    H4, W4 = H // scale, W // scale
    out = np.zeros((H4, W4, 4), np.float32)
    f = np.float32
    for y4 in range(H4):
        for x4 in range(W4):
            acc, n = np.zeros(3), 0
            for dy in range(scale):
                for dx in range(scale):
                    y, xf = y4 * scale + dy, x4 * scale + dx
                    x = W - 1 - xf if right_view else xf
                    a, b, c = (f(v) for v in planes[y, x, :3])
                    if not (np.isfinite(a) and np.isfinite(b) and np.isfinite(c)):
                        continue
                    tx = f(f(a * f(x)) + f(b * f(y))) + c
                    dv = f(tx - f(x)) if right_view else f(f(x) - tx)
                    if not (dv > 0 and dv <= dmax):
                        continue
                    xo = int(np.rint(tx))
                    if xo < 0 or xo >= W:
                        continue
                    ao, bo, co = (f(v) for v in other[y, xo, :3])
                    txo = f(f(ao * f(xo)) + f(bo * f(y))) + co
                    dov = f(f(xo) - txo) if right_view else f(txo - f(xo))
                    if not (abs(dov - dv) <= 1.0):
                        continue
                    vx, vy = float(a) - 1.0, (-float(b) if right_view else float(b))
                    inv = 1.0 / np.sqrt(vx * vx + vy * vy + 1.0)
                    acc += (float(dv), vx * inv, vy * inv)
                    n += 1
            if n > 0 and 2 * n >= scale * scale:
                out[y4, x4] = (acc[0] / n / scale, acc[1] / n, acc[2] / n, 1.0)
    return out
