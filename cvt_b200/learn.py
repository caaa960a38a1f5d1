"""Learned plane proposal for PMHuberStereo.disparity_map: a BF16 CNN whose per-pixel
(disparity, nx, ny) replaces the random initialisation, through the reference's
initdisparity / initnormalmap arguments (PMHuberStereo.cpp:92-93 ->
pmhstereo_init_disparity_normal, pmhstereo.cl:802-828), so that fewer PatchMatch iterations
reach plain PatchMatch's result.

The kernels are the library's (cvt_b200/csrc/pm_learn.cu, pm_lpp_* in cvtpm.h): the network
input, tcgen05 convolutions (forward and data gradient), tcgen05 weight gradients, the L1 loss,
Adam, the upsampling to full resolution.  This module only orders them: torch tensors serve as
device buffers; torch operators only pick training batches and sum per-block losses for logging.

    pp = PlaneProposal(seed=0)
    x, t = make_training_set(pairs=20000, width=512, height=384, seed=100, dmax=64.0)
    pp.train(x, t, epochs=30, batch=32)
    pp.save("weights.npz")
    d, n = pp.propose(left, right, dmax=128.0)            # (H, W), (H, W, 4) CUDA tensors
    res = PMHuberStereo().disparity_map(left, right, r, 128.0, 2, initdisparity=d, initnormalmap=n)

Scale.  The network always sees disparities of 0-16 feature pixels: it runs at 1 / scale of
the image with scale = 4 * max(1, round(dmax / 64)) (a quarter of the resolution for disparity
ranges up to 64, an eighth up to 128, a sixteenth up to 256).
"""
import concurrent.futures as cf

import numpy as np

from . import _lib

NL = 8
IN_CH, OUT_CH = 16, 16
WN = 4.0   # weight of the normal terms in the L1 loss


def _check(status):
    if status != _lib.PM_OK:
        L = _lib.lib()
        raise _lib.StereoError(status, (L.pm_lpp_last_error() or b"pm_lpp error").decode())


def _p(t):
    return None if t is None else t.data_ptr()


def layer_shapes():
    """[(cin, cout, dilation)] of the eight layers, from the library"""
    import ctypes as C

    L = _lib.lib()
    out = []
    for l in range(L.pm_lpp_layers()):
        ci, co, di = C.c_int(), C.c_int(), C.c_int()
        _check(L.pm_lpp_layer_shape(l, C.byref(ci), C.byref(co), C.byref(di)))
        out.append((ci.value, co.value, di.value))
    return out


def scale_for(dmax):
    """the network's resolution divisor for a disparity range"""
    return 4 * max(1, int(round(float(dmax) / 64.0)))


class PlaneProposal:
    """The network's FP32 master weights, their BF16 copies and Adam state, on one device."""

    def __init__(self, seed=0, device=0, tensor_cores=True):
        import torch

        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.tc = int(bool(tensor_cores))
        self.shapes = layer_shapes()
        self.seed = int(seed)
        rng = np.random.default_rng(seed)
        params = []
        for l, (ci, co, _) in enumerate(self.shapes):
            std = np.sqrt(2.0 / (9 * ci)) if l < NL - 1 else 0.01
            w = (rng.standard_normal((co, 9 * ci)) * std).astype(np.float32)
            if l == 0:
                w.reshape(co, 9, ci)[:, :, 6:] = 0.0   # input channels 6-15 are always zero
            b = np.zeros(co, np.float32)
            if l == NL - 1:
                b[0] = 4.0   # start at a mid-range disparity (feature pixels)
            params.append(np.concatenate([w.ravel(), b]))
        self.set_params(params)
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)

    # ---- parameters ------------------------------------------------------------
    def nweights(self, l):
        ci, co, _ = self.shapes[l]
        return co * 9 * ci

    def set_params(self, params, m1=None, m2=None):
        torch = self.torch
        self.p = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.dev) for a in params]
        self.m1 = [torch.zeros_like(a) for a in self.p] if m1 is None else \
            [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.dev) for a in m1]
        self.m2 = [torch.zeros_like(a) for a in self.p] if m2 is None else \
            [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.dev) for a in m2]
        # BF16 weights of all layers back to back (pm_lpp_propose_device), 256-byte aligned
        tot = sum(self.nweights(l) for l in range(NL))
        self.wall = torch.empty(tot + 128, dtype=torch.bfloat16, device=self.dev)
        base = (-self.wall.data_ptr() // 2) % 128
        self.wmat, off = [], base
        for l in range(NL):
            self.wmat.append(self.wall[off:off + self.nweights(l)])
            off += self.nweights(l)
        self.wt = [torch.empty(self.nweights(l), dtype=torch.bfloat16, device=self.dev) for l in range(NL)]
        self.ball = torch.empty(sum(co for _, co, _ in self.shapes), dtype=torch.float32, device=self.dev)
        self._refresh()

    def _refresh(self):
        L, s = _lib.lib(), self._stream()
        off = 0
        for l in range(NL):
            _check(L.pm_lpp_weights_bf16(l, _p(self.p[l]), _p(self.wmat[l]), _p(self.wt[l]), s))
            co = self.shapes[l][1]
            self.ball[off:off + co].copy_(self.p[l][self.nweights(l):])
            off += co

    def bias(self, l):
        return self.p[l][self.nweights(l):]

    def params(self):
        return [a.cpu().numpy() for a in self.p]

    def save(self, path, weights_only=False, **extra):
        """the FP32 master parameters, and unless weights_only the Adam moments, the step count and
        the seed (a checkpoint that training resumes from exactly)"""
        arrs = {"p%d" % l: a for l, a in enumerate(self.params())}
        if not weights_only:
            arrs.update({"m1_%d" % l: a.cpu().numpy() for l, a in enumerate(self.m1)})
            arrs.update({"m2_%d" % l: a.cpu().numpy() for l, a in enumerate(self.m2)})
        np.savez_compressed(path, step=self.step, seed=self.seed, **arrs, **extra)

    @classmethod
    def load(cls, path, device=0, tensor_cores=True):
        z = np.load(path)
        pp = cls(seed=int(z["seed"]), device=device, tensor_cores=tensor_cores)
        m1 = [z["m1_%d" % l] for l in range(NL)] if "m1_0" in z else None
        m2 = [z["m2_%d" % l] for l in range(NL)] if "m2_0" in z else None
        pp.set_params([z["p%d" % l] for l in range(NL)], m1, m2)
        pp.step = int(z["step"])
        return pp

    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def check_error(self):
        if int(self.err.item()):
            raise _lib.StereoError(_lib.PM_ETIMEOUT, "a tensor-core kernel's bounded wait ran out")

    # ---- network ---------------------------------------------------------------
    def net_input(self, left, right, scale, view=0):
        """(H, W, 4) uint8 CUDA tensors -> (1, H/scale, W/scale, 16) BF16 input of the left view
        (0) or of the mirrored pair (1, the right view's proposal)"""
        torch = self.torch
        H, W = left.shape[:2]
        out = torch.empty((1, H // scale, W // scale, IN_CH), dtype=torch.bfloat16, device=self.dev)
        _check(_lib.lib().pm_lpp_input(_p(left.contiguous()), _p(right.contiguous()), W, H, W * 4, int(scale),
                                       int(view), _p(out), self._stream()))
        return out

    def forward(self, x):
        """x (B, H4, W4, 16) BF16 -> (activations, output (B, H4, W4, 16) FP32)"""
        torch, L = self.torch, _lib.lib()
        B, H4, W4 = x.shape[:3]
        acts = [x]
        h = x
        for l in range(NL):
            last = l == NL - 1
            co = self.shapes[l][1]
            out = torch.empty((B, H4, W4, co), dtype=torch.float32 if last else torch.bfloat16, device=self.dev)
            _check(L.pm_lpp_conv(l, 0, self.tc, _p(h), _p(self.wmat[l]), _p(self.bias(l)), None, _p(out), B, H4, W4,
                                 _p(self.err), self._stream()))
            if not last:
                acts.append(out)
            h = out
        return acts, h

    def gradients(self, x, target, count=None):
        """loss (a device scalar) and the FP32 gradients of every layer's parameters for one batch;
        count = the batch's valid target pixels (counted here, with a device sync, when None)"""
        torch, L = self.torch, _lib.lib()
        B, H4, W4 = x.shape[:3]
        M = B * H4 * W4
        acts, out = self.forward(x)
        dy = torch.empty((B, H4, W4, OUT_CH), dtype=torch.bfloat16, device=self.dev)
        parts = torch.empty((M + 255) // 256, dtype=torch.float32, device=self.dev)
        if count is None:
            count = int((target[..., 3] > 0).sum().item())
        count = max(int(count), 1)
        _check(L.pm_lpp_loss(_p(out), _p(target.contiguous()), WN, 1.0 / count, M, _p(dy), _p(parts), self._stream()))
        grads = [None] * NL
        for l in range(NL - 1, -1, -1):
            ci, co, _ = self.shapes[l]
            g = torch.empty(self.nweights(l) + co, dtype=torch.float32, device=self.dev)
            n = L.pm_lpp_wgrad_scratch_floats(l, B, H4, W4)
            if getattr(self, "_scr", None) is None or self._scr.numel() < n:
                self._scr = torch.empty(n, dtype=torch.float32, device=self.dev)
            _check(L.pm_lpp_wgrad(l, self.tc, _p(acts[l]), _p(dy), _p(self._scr), _p(g), B, H4, W4, _p(self.err),
                                  self._stream()))
            grads[l] = g
            if l > 0:
                dx = torch.empty((B, H4, W4, ci), dtype=torch.bfloat16, device=self.dev)
                _check(L.pm_lpp_conv(l, 1, self.tc, _p(dy), _p(self.wt[l]), None, _p(acts[l]), _p(dx), B, H4, W4,
                                     _p(self.err), self._stream()))
                dy = dx
        return parts.sum() / count, grads

    def train_step(self, x, target, lr=1e-3, count=None):
        L = _lib.lib()
        loss, grads = self.gradients(x, target, count)
        self.step += 1
        for l in range(NL):
            _check(L.pm_lpp_adam(_p(self.p[l]), _p(grads[l]), _p(self.m1[l]), _p(self.m2[l]), self.p[l].numel(), lr,
                                 self.step, self._stream()))
        self._refresh()
        return loss

    def train(self, x, target, epochs=30, batch=32, lr=1e-3, seed=0, log_every=0, on_epoch=None):
        """Adam over `epochs` passes of the training maps in seeded random order, batches of
        `batch` (the last partial batch of an epoch is dropped); the learning rate falls by 10x
        for the last fifth of the epochs.  Returns the per-step losses (a float tensor)."""
        torch = self.torch
        g = np.random.default_rng(seed)
        n = x.shape[0]
        valid = (target[..., 3] > 0).sum((1, 2)).cpu().numpy()   # valid pixels per map, counted once
        losses = []
        for e in range(epochs):
            perm = g.permutation(n)
            order = torch.from_numpy(perm).to(self.dev)
            lr_e = lr * (0.1 if e >= int(0.8 * epochs) else 1.0)
            for i in range(0, n - batch + 1, batch):
                idx = order[i:i + batch]
                losses.append(self.train_step(x.index_select(0, idx), target.index_select(0, idx), lr_e,
                                              int(valid[perm[i:i + batch]].sum())))
                if log_every and len(losses) % log_every == 0:
                    print("epoch %d step %d loss %.4f" % (e, len(losses), float(losses[-1])), flush=True)
            if on_epoch:
                on_epoch(e, self)
        self.check_error()
        return torch.stack(losses) if losses else torch.zeros(0)

    def propose(self, left, right, dmax, view=0, disp=None, normal=None):
        """full-resolution initial disparity (pixels) and normal map of the left (view 0) or the
        right view (1) for a pair of (H, W, 4) uint8 CUDA tensors, through the single native call
        pm_lpp_propose_device; disp ((H, W) float32) and normal ((H, W, 4) float32) are filled in
        place when given, so that a following disparity_map call sees the same buffers and
        replays its graph"""
        torch, L = self.torch, _lib.lib()
        H, W = left.shape[:2]
        sc = scale_for(dmax)
        nbytes = L.pm_lpp_propose_workspace_bytes(W, H, sc) + 256
        if getattr(self, "_ws", None) is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.dev)
        ws = self._ws
        off = (-ws.data_ptr()) % 256
        if disp is None:
            disp = torch.empty((H, W), dtype=torch.float32, device=self.dev)
        if normal is None:
            normal = torch.empty((H, W, 4), dtype=torch.float32, device=self.dev)
        _check(L.pm_lpp_propose_device(_p(self.wmat[0]), _p(self.ball), sc, _p(left.contiguous()),
                                       _p(right.contiguous()), W, H, W * 4, int(view), float(dmax), _p(disp),
                                       _p(normal), ws.data_ptr() + off, ws.numel() - off, _p(self.err),
                                       self._stream()))
        return disp, normal


def make_training_set(pairs, width, height, seed, dmax=64.0, patch=5, iterations=8, device=0, fused=True,
                      workers=8, log_every=0):
    """Training maps from seeded procedural scenes, two per pair: the left view's input with the
    1 / scale resolution (d, nx, ny, valid) of plain (random-init) two-view PatchMatch's final left
    planes after `iterations` iterations, and the mirrored pair's input with the right view's.
    Scenes: 8-60 planes, disparities 2 to 0.9 dmax; they are generated on `workers` host threads
    ahead of the GPU.  Returns (inputs (2 pairs, H4, W4, 16) BF16, targets (2 pairs, H4, W4, 4) FP32)."""
    import torch

    from . import scene
    from .stereo import PMHuberStereo

    dev = torch.device("cuda", device)
    pm = PMHuberStereo(device=device, fused=fused)
    sc = scale_for(dmax)
    pp_in = PlaneProposal.__new__(PlaneProposal)   # only for net_input
    pp_in.torch, pp_in.dev = torch, dev
    H4, W4 = height // sc, width // sc
    inputs = torch.empty((2 * pairs, H4, W4, IN_CH), dtype=torch.bfloat16, device=dev)
    target = torch.empty((2 * pairs, H4, W4, 4), dtype=torch.float32, device=dev)
    L = _lib.lib()

    def gen(i):
        s = seed + i
        return scene.generate(s, width, height, 8 + s % 53, 2.0, 0.9 * dmax)

    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        futs = [ex.submit(gen, i) for i in range(min(pairs, 4 * workers))]
        for i in range(pairs):
            l, r = futs[i].result()
            futs[i] = None
            if i + 4 * workers < pairs:
                futs.append(ex.submit(gen, i + 4 * workers))
            dl, dr = torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)
            st = torch.cuda.current_stream(dev).cuda_stream
            inputs[2 * i] = PlaneProposal.net_input(pp_in, dl, dr, sc, 0)[0]
            inputs[2 * i + 1] = PlaneProposal.net_input(pp_in, dl, dr, sc, 1)[0]
            res = pm.disparity_map(dl, dr, patch, dmax, iterations, pp=1, planes=True)
            pl, pr = res["planes_left"], res["planes_right"]
            _check(L.pm_lpp_target(_p(pl), _p(pr), width, height, sc, 0, float(dmax), _p(target[2 * i]), st))
            _check(L.pm_lpp_target(_p(pr), _p(pl), width, height, sc, 1, float(dmax), _p(target[2 * i + 1]), st))
            if log_every and (i + 1) % log_every == 0:
                torch.cuda.synchronize(dev)
                print("training set: %d / %d pairs" % (i + 1, pairs), flush=True)
    pm.close()
    return inputs, target


def default_weights():
    """path of the committed weights, trained at the cfg4 recipe by cvt_b200/train_proposal.py"""
    import os

    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "proposal.npz")
