"""Python mirror of cvt::PMHuberStereo (cvt/vision/PMHuberStereo.h:42-110).

`PMHuberStereo.disparity_map` has the arguments of the reference's
`disparityMap(dmap, left, right, patchsize, disparitymax, iterations, pp,
normalmap, initdisparity, initnormalmap)` (PMHuberStereo.cpp:75): images go in,
the disparity map (and, on request, the normal map and the final plane fields)
come out.  Host numpy arrays run through pm_disparity_map (host copies
included); CUDA torch tensors run through pm_disparity_map_device on the
current stream.  Errors raise StereoError, as the reference raises
cvt::Exception.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import PP_LRCHECK, PP_LRCHECK_FILL, PP_NONE, StereoError  # noqa: F401

DISPARITY_PP_NONE = PP_NONE
DISPARITY_PP_LRCHECK = PP_LRCHECK
DISPARITY_PP_LRCHECK_FILL = PP_LRCHECK_FILL


def _is_torch(x):
    return type(x).__module__.startswith("torch")


class PMHuberStereo:
    """Slanted-plane PatchMatch stereo with ROF-coupled smoothing on one B200."""

    def __init__(self, views=2, fused=False, device=0, thetamin=1e-4, maxdispdiff=1.0, maxanglediff=5.0,
                 rof_iters=40, use_graph=True, levels=1):
        L = _lib.lib()
        opt = _lib.Options()
        _lib.check(L.pm_options_default(C.byref(opt)))
        opt.views, opt.fused, opt.device = int(views), int(bool(fused)), int(device)
        opt.thetamin, opt.maxdispdiff, opt.maxanglediff = thetamin, maxdispdiff, maxanglediff
        opt.rof_iters, opt.use_graph = int(rof_iters), int(bool(use_graph))
        opt.levels = int(levels)
        h = C.c_void_p()
        _lib.check(L.pm_create(C.byref(h), C.byref(opt)))
        self._h = h
        self.views = views
        self.fused = fused

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().pm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_batch_branches(self, n):
        """concurrent branches of later batched calls (0: the library's default, 16)"""
        _lib.check(_lib.lib().pm_set_batch_branches(self._h, int(n)), self._h)

    def set_batch_schedule(self, schedule="branched", ctas_per_sm=0, tile_order=0, tile_w=32):
        """how later batched calls run: "branched" (the default: each pair's pipeline a graph
        branch) or "lockstep" (every iteration's propagate passes and smoothing stages of all
        pairs as persistent launches over one tile list; ctas_per_sm caps the propagate CTAs per
        SM, 0 = as many as fit; tile_order 0 = pair after pair, 1 = the pairs' tile rows
        interleaved; tile_w 32 = tiles of 32 x 4 pixels, 16 = 16 x 8)"""
        mode = {"lockstep": _lib.PM_BATCH_LOCKSTEP, "branched": _lib.PM_BATCH_BRANCHED}[schedule]
        _lib.check(_lib.lib().pm_set_batch_schedule(self._h, mode, int(ctas_per_sm), int(tile_order), int(tile_w)),
                   self._h)

    def set_counting(self, on):
        _lib.check(_lib.lib().pm_set_counting(self._h, int(bool(on))), self._h)

    def counters(self):
        c = (C.c_uint64 * 4)()
        _lib.check(_lib.lib().pm_get_counters(self._h, c), self._h)
        return [int(v) for v in c]

    PHASES = ("prep", "init", "propagate", "smooth", "post", "total")

    def set_profiling(self, on):
        _lib.check(_lib.lib().pm_set_profiling(self._h, int(bool(on))), self._h)

    def phase_times(self):
        """{phase: (ms, kernel launches)} of the last call made with profiling on."""
        ms = (C.c_float * 6)()
        n = (C.c_int * 6)()
        _lib.check(_lib.lib().pm_get_phase_times(self._h, ms, n), self._h)
        return {p: (float(ms[i]), int(n[i])) for i, p in enumerate(self.PHASES)}

    def disparity_map(self, left, right, patchsize, disparitymax, iterations, pp=PP_LRCHECK, normalmap=False,
                      initdisparity=None, initnormalmap=None, planes=False, stream=None, initdisparity_right=None,
                      initnormalmap_right=None):
        """Returns dmap, or a dict {dmap, normal?, planes_left?, planes_right?} when
        normalmap or planes is requested.  left/right: (H, W, 4) uint8.  initdisparity_right
        (CUDA tensors only) also starts the right view from a disparity and, with
        initnormalmap_right, a normal map, as disparityMapAll allows
        (pm_disparity_map_init2_device)."""
        if initdisparity_right is not None:
            return self._device(left, right, patchsize, disparitymax, iterations, pp, normalmap, initdisparity,
                                initnormalmap, planes, stream, None, initdisparity_right, initnormalmap_right)
        return self._run(None, left, right, patchsize, disparitymax, iterations, pp, normalmap, initdisparity,
                         initnormalmap, planes, stream)

    def depth_map(self, left, right, patchsize, depthmax, iterations, dscale=-1.0, pp=PP_LRCHECK, normalmap=False,
                  initdisparity=None, initnormalmap=None, planes=False, stream=None):
        """PMHuberStereo::depthMap (PMHuberStereo.cpp:145-347): the Huber-smoothed variant; dmap is
        the disparity times dscale (dscale <= 0: 1 / depthmax).  Returns as disparity_map."""
        return self._run(float(dscale), left, right, patchsize, depthmax, iterations, pp, normalmap, initdisparity,
                         initnormalmap, planes, stream)

    def _run(self, dscale, left, right, patchsize, disparitymax, iterations, pp, normalmap, initdisparity,
             initnormalmap, planes, stream):
        if _is_torch(left):
            return self._device(left, right, patchsize, disparitymax, iterations, pp, normalmap, initdisparity,
                                initnormalmap, planes, stream, dscale)
        L = _lib.lib()
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        if left.shape != right.shape or left.ndim != 3 or left.shape[2] != 4:
            raise StereoError(_lib.PM_EINVAL_SHAPE, "Left/Right stereo images inconsistent")
        H, W = left.shape[:2]
        dmap = np.zeros((H, W), np.float32)
        nmap = np.zeros((H, W, 4), np.float32) if normalmap else None
        pl = np.zeros((H, W, 4), np.float32) if planes else None
        pr = np.zeros((H, W, 4), np.float32) if planes else None
        idisp = None if initdisparity is None else np.ascontiguousarray(initdisparity, np.float32)
        inorm = None if initnormalmap is None else np.ascontiguousarray(initnormalmap, np.float32)

        def p(a):
            return None if a is None else a.ctypes.data

        if dscale is None:
            _lib.check(L.pm_disparity_map(self._h, left.ctypes.data, right.ctypes.data, W, H, W * 4, int(patchsize),
                                          float(disparitymax), int(iterations), int(pp), dmap.ctypes.data, p(nmap),
                                          p(idisp), p(inorm), p(pl), p(pr)), self._h)
        else:
            _lib.check(L.pm_depth_map(self._h, left.ctypes.data, right.ctypes.data, W, H, W * 4, int(patchsize),
                                      float(disparitymax), int(iterations), dscale, int(pp), dmap.ctypes.data, p(nmap),
                                      p(idisp), p(inorm), p(pl), p(pr)), self._h)
        if not normalmap and not planes:
            return dmap
        out = {"dmap": dmap}
        if normalmap:
            out["normal"] = nmap
        if planes:
            out["planes_left"], out["planes_right"] = pl, pr
        return out

    def disparity_map_batch(self, lefts, rights, patchsizes, disparitymaxs, iterations, pp=PP_LRCHECK, planes=False,
                            stream=None):
        """n pairs of CUDA uint8 tensors (H_i, W_i, 4), each with its own patch size and disparity
        range, run as one graph launch (pm_disparity_map_batch_device).  Returns a list of
        dmaps, or of dicts {dmap, planes_left, planes_right} when planes is requested."""
        import torch

        L = _lib.lib()
        n = len(lefts)
        if len(rights) != n or len(patchsizes) != n or len(disparitymaxs) != n:
            raise StereoError(_lib.PM_EINVAL_ARG, "per-pair lists differ in length")
        ls, rs, outs = [], [], []
        for a, b in zip(lefts, rights):
            if a.shape != b.shape or a.dim() != 3 or a.shape[2] != 4 or a.dtype != torch.uint8 or not a.is_cuda:
                raise StereoError(_lib.PM_EINVAL_SHAPE, "Left/Right stereo images inconsistent")
            ls.append(a.contiguous())
            rs.append(b.contiguous())
        dm = [torch.empty(a.shape[:2], dtype=torch.float32, device=a.device) for a in ls]
        pl = [torch.empty(a.shape, dtype=torch.float32, device=a.device) for a in ls] if planes else None
        pr = [torch.empty(a.shape, dtype=torch.float32, device=a.device) for a in ls] if planes else None

        def arr(ctype, vals):
            return (ctype * max(n, 1))(*vals)

        st = stream if stream is not None else torch.cuda.current_stream(ls[0].device if n else None).cuda_stream
        ptr = C.c_void_p
        _lib.check(L.pm_disparity_map_batch_device(
            self._h, n, arr(ptr, [t.data_ptr() for t in ls]), arr(ptr, [t.data_ptr() for t in rs]),
            arr(C.c_int, [t.shape[1] for t in ls]), arr(C.c_int, [t.shape[0] for t in ls]),
            arr(C.c_size_t, [t.shape[1] * 4 for t in ls]), arr(C.c_int, [int(r) for r in patchsizes]),
            arr(C.c_float, [float(d) for d in disparitymaxs]), int(iterations), int(pp),
            arr(ptr, [t.data_ptr() for t in dm]), arr(ptr, [t.data_ptr() for t in pl]) if planes else None,
            arr(ptr, [t.data_ptr() for t in pr]) if planes else None, st), self._h)
        if not planes:
            return dm
        return [{"dmap": d, "planes_left": a, "planes_right": b} for d, a, b in zip(dm, pl, pr)]

    def _device(self, left, right, patchsize, dmax, iterations, pp, normalmap, initd, initn, planes, stream,
                dscale=None, initd_right=None, initn_right=None):
        import torch

        L = _lib.lib()
        if left.shape != right.shape or left.dim() != 3 or left.shape[2] != 4 or left.dtype != torch.uint8:
            raise StereoError(_lib.PM_EINVAL_SHAPE, "Left/Right stereo images inconsistent")
        left = left.contiguous()
        right = right.contiguous()
        H, W = left.shape[:2]
        dev = left.device
        dmap = torch.empty((H, W), dtype=torch.float32, device=dev)
        nmap = torch.empty((H, W, 4), dtype=torch.float32, device=dev) if normalmap else None
        pl = torch.empty((H, W, 4), dtype=torch.float32, device=dev) if planes else None
        pr = torch.empty((H, W, 4), dtype=torch.float32, device=dev) if planes else None
        initd = None if initd is None else initd.contiguous().float()
        initn = None if initn is None else initn.contiguous().float()
        st = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream

        def p(t):
            return None if t is None else t.data_ptr()

        if initd_right is not None:
            if not _is_torch(left):
                raise StereoError(_lib.PM_EINVAL_ARG, "initdisparity_right: CUDA tensors only")
            ir = initd_right.contiguous().float()
            inr = None if initn_right is None else initn_right.contiguous().float()
            _lib.check(L.pm_disparity_map_init2_device(self._h, p(left), p(right), W, H, W * 4, int(patchsize), float(dmax),
                                                       int(iterations), int(pp), p(dmap), p(nmap), p(initd), p(ir),
                                                       p(initn), p(inr), p(pl), p(pr), st), self._h)
        elif dscale is None:
            _lib.check(L.pm_disparity_map_device(self._h, p(left), p(right), W, H, W * 4, int(patchsize), float(dmax),
                                                 int(iterations), int(pp), p(dmap), p(nmap), p(initd), p(initn), p(pl),
                                                 p(pr), st), self._h)
        else:
            _lib.check(L.pm_depth_map_device(self._h, p(left), p(right), W, H, W * 4, int(patchsize), float(dmax),
                                             int(iterations), dscale, int(pp), p(dmap), p(nmap), p(initd), p(initn),
                                             p(pl), p(pr), st), self._h)
        if not normalmap and not planes:
            return dmap
        out = {"dmap": dmap}
        if normalmap:
            out["normal"] = nmap
        if planes:
            out["planes_left"], out["planes_right"] = pl, pr
        return out
