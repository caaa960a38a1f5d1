"""Learned plane proposal for PMHuberStereo.disparity_map: a small BF16 CNN that replaces
the random initialisation (through the reference's initdisparity argument,
PMHuberStereo.cpp:92-93) so that fewer PatchMatch iterations reach the same cost.

The kernels are the library's (cvt_b200/csrc/pm_learn.cu, pm_lpp_* in cvtpm.h):
cost-volume features, tcgen05 convolutions, soft-argmin, smooth-L1 loss, data and
weight gradients, Adam.  This module only orders them: torch tensors serve as device
buffers; torch operators only pick training batches, count valid targets and sum the
per-block loss for logging.

    pp = PlaneProposal(seed=0)
    feats, target = make_training_set(pairs=48, width=512, height=384, seed=100)
    pp.train(feats, target, steps=400)
    init = pp.propose(left, right)                      # (H, W) float32 CUDA tensor
    dmap = PMHuberStereo().disparity_map(left, right, r, dmax, 1, initdisparity=init)

At 1280x720 (21x21, disparity 0-128) the left view alone, started from the proposal,
reproduces plain 8-iteration two-view PatchMatch's left disparity (cost within 1%, 98% of
its kept pixels within 1 px) after 7 iterations, in 0.34 of plain's time:

    dmap = PMHuberStereo(views=1).disparity_map(left, right, r, dmax, 7, pp=DISPARITY_PP_NONE,
                                                 initdisparity=init)
"""
import ctypes as C

import numpy as np

from . import _lib

CH = 32
KTOT = 9 * CH
NLAYERS = 6
SKIP = 4.0   # the cost volume's weight in the soft-argmin: the network learns a correction to it
EPI_RELU, EPI_LOGITS, EPI_DGRAD = 0, 1, 2


def _check(status):
    if status != _lib.PM_OK:
        L = _lib.lib()
        raise _lib.StereoError(status, (L.pm_lpp_last_error() or b"pm_lpp error").decode())


def _p(t):
    return None if t is None else t.data_ptr()


class PlaneProposal:
    """The network's FP32 master weights, their BF16 copies and Adam state, on one device."""

    def __init__(self, seed=0, device=0, tensor_cores=True, step=1, scale=4):
        """scale: the network's resolution is 1 / scale of the image's (4 or 2); step: feature
        pixels between the 32 disparity hypotheses (scale 4: step 1 reaches 124 px, 2 reaches
        248 px; scale 2: step 2 reaches 124 px)"""
        import torch

        self.torch = torch
        self.hstep = int(step)
        self.scale = int(scale)
        self.dev = torch.device("cuda", device)
        self.tc = int(bool(tensor_cores))
        rng = np.random.default_rng(seed)
        params = []
        for l in range(NLAYERS):
            std = np.sqrt(2.0 / KTOT) if l < NLAYERS - 1 else 0.02
            w = (rng.standard_normal((CH, KTOT)) * std).astype(np.float32)
            params.append(np.concatenate([w.ravel(), np.zeros(CH, np.float32)]))
        self.set_params(params)
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)

    # ---- parameters ------------------------------------------------------------
    def set_params(self, params):
        torch = self.torch
        self.p = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(self.dev) for a in params]
        self.m1 = [torch.zeros_like(a) for a in self.p]
        self.m2 = [torch.zeros_like(a) for a in self.p]
        # BF16 weights of all layers in one 256-byte aligned buffer (pm_lpp_propose_device)
        self.wall = torch.empty(NLAYERS * CH * KTOT + 128, dtype=torch.bfloat16, device=self.dev)
        base = (-self.wall.data_ptr() // 2) % 128
        self.wmat = [self.wall[base + l * CH * KTOT: base + (l + 1) * CH * KTOT] for l in range(NLAYERS)]
        self.wt = [torch.empty(CH * KTOT, dtype=torch.bfloat16, device=self.dev) for _ in range(NLAYERS)]
        self.ball = torch.empty(NLAYERS * CH, dtype=torch.float32, device=self.dev)
        self._refresh()

    def _refresh(self):
        L, s = _lib.lib(), self._stream()
        for l in range(NLAYERS):
            _check(L.pm_lpp_weights_bf16(_p(self.p[l]), _p(self.wmat[l]), _p(self.wt[l]), s))
            self.ball[l * CH:(l + 1) * CH].copy_(self.p[l][CH * KTOT:])

    def bias(self, l):
        return self.p[l][CH * KTOT:]

    def params(self):
        return [a.cpu().numpy() for a in self.p]

    def save(self, path):
        np.savez_compressed(path, *self.params(), step=self.step, hstep=self.hstep, scale=self.scale)

    @classmethod
    def load(cls, path, device=0, tensor_cores=True):
        z = np.load(path)
        pp = cls(device=device, tensor_cores=tensor_cores, step=int(z["hstep"]) if "hstep" in z else 1,
                 scale=int(z["scale"]) if "scale" in z else 4)
        pp.set_params([z["arr_%d" % l] for l in range(NLAYERS)])
        pp.step = int(z["step"])
        return pp

    def _stream(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def check_error(self):
        if int(self.err.item()):
            raise _lib.StereoError(_lib.PM_ETIMEOUT, "a tensor-core convolution's bounded wait ran out")

    # ---- network ---------------------------------------------------------------
    def features(self, left, right, view=0):
        """(H, W, 4) uint8 CUDA tensors -> (1, H/4, W/4, 32) BF16 cost volume of the left (view 0)
        or the right view (1)"""
        torch = self.torch
        H, W = left.shape[:2]
        H4, W4 = H // self.scale, W // self.scale
        grey = torch.empty(2 * H4 * W4, dtype=torch.float32, device=self.dev)
        out = torch.empty((1, H4, W4, CH), dtype=torch.bfloat16, device=self.dev)
        _check(_lib.lib().pm_lpp_features(_p(left.contiguous()), _p(right.contiguous()), W, H, W * 4, int(view),
                                          self.hstep, self.scale, _p(grey), _p(out), self._stream()))
        return out

    def forward(self, feats):
        """feats (B, H4, W4, 32) BF16 -> (activations, logits (B, H4, W4, 32) FP32)"""
        torch, L = self.torch, _lib.lib()
        B, H4, W4 = feats.shape[:3]
        acts = [feats]
        x = feats
        for l in range(NLAYERS):
            last = l == NLAYERS - 1
            out = torch.empty((B, H4, W4, CH), dtype=torch.float32 if last else torch.bfloat16, device=self.dev)
            _check(L.pm_lpp_conv(EPI_LOGITS if last else EPI_RELU, self.tc, _p(x), _p(self.wmat[l]), _p(self.bias(l)),
                                 None, _p(out), B, H4, W4, _p(self.err), self._stream()))
            if not last:
                acts.append(out)
            x = out
        return acts, x

    def disparity4(self, feats):
        """quarter-resolution disparity (quarter pixels) of each map in the batch"""
        torch = self.torch
        _, logits = self.forward(feats)
        B, H4, W4 = feats.shape[:3]
        d = torch.empty((B, H4, W4), dtype=torch.float32, device=self.dev)
        _check(_lib.lib().pm_lpp_softargmin(_p(logits), _p(feats), SKIP, float(self.hstep), None, _p(d), None, None,
                                            B * H4 * W4, 0.0, self._stream()))
        return d

    def gradients(self, feats, target4):
        """loss and the FP32 weight / bias gradients of every layer for one batch"""
        torch, L = self.torch, _lib.lib()
        B, H4, W4 = feats.shape[:3]
        M = B * H4 * W4
        acts, logits = self.forward(feats)
        disp = torch.empty(M, dtype=torch.float32, device=self.dev)
        dy = torch.empty((B, H4, W4, CH), dtype=torch.bfloat16, device=self.dev)
        parts = torch.empty((M + 255) // 256, dtype=torch.float32, device=self.dev)
        count = max(int((target4 >= 0).sum().item()), 1)
        _check(L.pm_lpp_softargmin(_p(logits), _p(feats), SKIP, float(self.hstep), _p(target4.contiguous()), _p(disp),
                                   _p(dy), _p(parts), M, 1.0 / count, self._stream()))
        per_block = 256
        scratch = torch.empty(L.pm_lpp_wgrad_scratch_floats(B, H4, W4, per_block), dtype=torch.float32, device=self.dev)
        grads = [None] * NLAYERS
        for l in range(NLAYERS - 1, -1, -1):
            g = torch.empty(CH * KTOT + CH, dtype=torch.float32, device=self.dev)
            _check(L.pm_lpp_wgrad(_p(acts[l]), _p(dy), _p(scratch), _p(g), B, H4, W4, per_block, self._stream()))
            grads[l] = g
            if l > 0:
                dx = torch.empty((B, H4, W4, CH), dtype=torch.bfloat16, device=self.dev)
                _check(L.pm_lpp_conv(EPI_DGRAD, self.tc, _p(dy), _p(self.wt[l]), None, _p(acts[l]), _p(dx), B, H4, W4,
                                     _p(self.err), self._stream()))
                dy = dx
        return float(parts.sum().item()) / count, grads

    def train_step(self, feats, target4, lr=1e-3):
        L = _lib.lib()
        loss, grads = self.gradients(feats, target4)
        self.step += 1
        for l in range(NLAYERS):
            _check(L.pm_lpp_adam(_p(self.p[l]), _p(grads[l]), _p(self.m1[l]), _p(self.m2[l]), self.p[l].numel(), lr,
                                 self.step, self._stream()))
        self._refresh()
        return loss

    def train(self, feats, target4, steps=400, batch=8, lr=1e-3, seed=0, log_every=0):
        """Adam over random batches of the training maps; returns the losses"""
        torch = self.torch
        g = np.random.default_rng(seed)
        n = feats.shape[0]
        losses = []
        for s in range(steps):
            idx = torch.from_numpy(g.choice(n, size=min(batch, n), replace=False)).to(self.dev)
            lr_s = lr * (0.1 if s >= int(0.8 * steps) else 1.0)
            losses.append(self.train_step(feats.index_select(0, idx).contiguous(),
                                          target4.index_select(0, idx).contiguous(), lr_s))
            if log_every and s % log_every == 0:
                print("step %d loss %.4f" % (s, losses[-1]))
        self.check_error()
        return losses

    def propose(self, left, right, view=0, out=None):
        """full-resolution initial disparity (pixels) of the left (view 0) or right view (1) for a
        pair of (H, W, 4) uint8 CUDA tensors, through the single native call pm_lpp_propose_device;
        `out` (an (H, W) float32 CUDA tensor) is filled in place when given, so that a following
        disparity_map call sees the same buffer and replays its graph"""
        torch, L = self.torch, _lib.lib()
        H, W = left.shape[:2]
        nbytes = L.pm_lpp_propose_workspace_bytes(W, H, self.scale) + 256
        if getattr(self, "_ws", None) is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.dev)
        ws = self._ws
        off = (-ws.data_ptr()) % 256
        if out is None:
            out = torch.empty((H, W), dtype=torch.float32, device=self.dev)
        _check(L.pm_lpp_propose_device(_p(self.wmat[0]), _p(self.ball), NLAYERS, SKIP, self.hstep, self.scale,
                                       _p(left.contiguous()),
                                       _p(right.contiguous()), W, H, W * 4, int(view), _p(out), ws.data_ptr() + off,
                                       ws.numel() - off, _p(self.err), self._stream()))
        return out


def make_training_set(pairs, width, height, seed, iterations=8, patch=7, dmax=None, device=0, step=1, scale=4):
    """Training maps from procedural scenes, two per pair: the left view's features with the
    quarter-resolution mean of plain (random-init) PatchMatch's LR-checked left disparity after
    `iterations` iterations, and the right view's features with its right disparity."""
    import torch

    from . import scene
    from .stereo import PMHuberStereo

    dev = torch.device("cuda", device)
    pm = PMHuberStereo(device=device)
    pp = PlaneProposal(device=device, step=step, scale=scale)
    H4, W4 = height // scale, width // scale
    feats = torch.empty((2 * pairs, H4, W4, CH), dtype=torch.bfloat16, device=dev)
    target = torch.empty((2 * pairs, H4, W4), dtype=torch.float32, device=dev)
    dright = torch.empty((height, width), dtype=torch.float32, device=dev)
    L = _lib.lib()
    dmax = float(dmax if dmax is not None else scale * CH * step)
    for i in range(pairs):
        l, r = scene.generate(seed + i, width, height, 8 + (seed + i) % 24, 2.0,
                              min(0.9 * dmax, (30.0 + (i % 4) * 30.0) * step))
        dl, dr = torch.from_numpy(l).to(dev), torch.from_numpy(r).to(dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        feats[2 * i] = pp.features(dl, dr, 0)[0]
        feats[2 * i + 1] = pp.features(dl, dr, 1)[0]
        res = pm.disparity_map(dl, dr, patch, dmax, iterations, pp=1, planes=True)
        _check(L.pm_lpp_target(_p(res["dmap"]), width, height, scale, _p(target[2 * i]), st))
        _lib.check(L.pm_k_to_disparity(_p(dright), _p(res["planes_right"]), width, height, 1.0, 0, st))
        _check(L.pm_lpp_target(_p(dright), width, height, scale, _p(target[2 * i + 1]), st))
    return feats, target
