"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
cpu_baseline leg).

numpy front end of the two CPU checkers:
  Oracle('orc')  the restatement, oracle/liboracle.so
  Oracle('ref')  the reference's own kernel sources compiled through the
                 OpenCL-C shim, oracle/_ref/libpmref.so (present where it was
                 built from the reference tree)
Both expose the same functions with the same arguments.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpmref.so")

vp = C.c_void_p
i32 = C.c_int
f32 = C.c_float
DUMP_FN = C.CFUNCTYPE(None, C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_void_p)


def available(kind):
    return os.path.exists(ORACLE_SO if kind == "orc" else REF_SO)


def _p(a):
    return None if a is None else a.ctypes.data


def _f4(shape):
    return np.zeros(shape + (4,), np.float32)


class Oracle:
    def __init__(self, kind="orc"):
        self.kind = kind
        path = ORACLE_SO if kind == "orc" else REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = C.CDLL(path)
        p = kind + "_"
        sig = {
            "prep": [vp, i32, i32, i32, i32, i32, vp, vp, vp],
            "init": [vp, vp, vp, vp, vp, i32, i32, i32, f32, i32, vp, vp, i32],
            "propagate": [vp, vp, vp, vp, vp, vp, vp, f32, i32, i32, i32, f32, i32, i32, vp, vp, vp, vp, vp, i32, vp],
            "cost": [vp, vp, vp, vp, vp, vp, i32, i32, i32, f32, i32],
            "klt": [vp, vp, vp, vp, vp, vp, i32, i32, i32, i32],
            "normal_depth": [vp, vp, i32, i32, f32, i32],
            "rof": [vp, vp, vp, C.POINTER(C.c_float), i32, i32, i32],
            "consistency": [vp, vp, vp, i32, i32, f32, f32],
            "to_disparity": [vp, vp, i32, i32, f32, i32],
            "fill_depthmap": [vp, vp, i32, i32, f32],
            "fill_normalmap": [vp, vp, i32, i32, i32],
            "disparity_to_normal": [vp, vp, i32, i32],
            "pyrdown": [vp, i32, i32, vp, i32, i32],
            "pyrup_mul": [vp, i32, i32, vp, i32, i32, i32, C.POINTER(C.c_float)],
            "prep_raw": [vp, i32, i32, i32, f32, vp, vp, vp],
            "fill_state": [vp, vp, i32, i32, f32, i32],
            "huber": [vp, vp, vp, C.POINTER(C.c_float), f32, i32, i32, i32],
        }
        for name, args in sig.items():
            fn = getattr(self.L, p + name)
            fn.restype = i32
            fn.argtypes = args
            setattr(self, "_" + name, fn)
        # VPMStereoCL: the restatement takes a row stride for its colour images, the
        # reference glue packed rows
        st = [i32] if kind == "orc" else []
        vsig = {
            "vpm_grad": [vp, vp, i32, i32] + st,
            "vpm_init": [vp, vp, vp, vp, vp, i32, i32] + st + [i32, f32, vp],
            "vpm_iter": [vp, vp, vp, vp, vp, vp, i32, i32] + st + [i32, f32, i32],
            "vpm_disparity": [vp, vp, i32, i32, f32],
            "vpm_disparity_simple": [vp, vp, vp, vp, i32, i32] + st + [i32, i32, f32, vp],
        }
        for name, args in vsig.items():
            fn = getattr(self.L, p + name)
            fn.restype = i32
            fn.argtypes = args
            setattr(self, "_" + name, fn)
        self._st = (lambda W: [W * 4]) if kind == "orc" else (lambda W: [])
        # SVPMFlowCL, same convention
        fsig = {
            "svpm_init": [vp, vp, vp, i32, i32] + st + [i32, f32],
            "svpm_prop": [vp, vp, vp, vp, vp, vp, i32, i32] + st + [i32, f32, i32],
            "svpm_to_flow": [vp, vp, i32, i32],
            "svpm_flow": [vp, vp, vp, vp, vp, i32, i32] + st + [i32, f32, i32],
        }
        for name, args in fsig.items():
            fn = getattr(self.L, p + name)
            fn.restype = i32
            fn.argtypes = args
            setattr(self, "_" + name, fn)
        if kind == "orc":
            self.L.orc_disparity_map_dump.restype = i32
            self.L.orc_disparity_map_dump.argtypes = [vp, vp, i32, i32, i32, i32, f32, i32, i32, i32, i32, vp, vp, vp,
                                                      vp, vp, vp, i32, vp, DUMP_FN, vp]
            self.L.orc_depth_map_dump.restype = i32
            self.L.orc_depth_map_dump.argtypes = [vp, vp, i32, i32, i32, i32, f32, i32, f32, i32, i32, vp, vp, vp,
                                                  vp, vp, vp, i32, vp, DUMP_FN, vp]
            for fn in ("orc_exp", "orc_sin", "orc_cos", "orc_acospi", "orc_log"):
                getattr(self.L, fn).restype = f32
                getattr(self.L, fn).argtypes = [f32]
            self.L.orc_rng_floats.restype = i32
            self.L.orc_rng_floats.argtypes = [C.c_int64, i32, i32, vp]
        else:
            self.L.ref_disparity_map_dump.restype = i32
            self.L.ref_disparity_map_dump.argtypes = [vp, vp, i32, i32, i32, i32, f32, i32, i32, i32, i32, vp, vp, vp,
                                                      vp, vp, vp, DUMP_FN, vp]
            self.L.ref_depth_map_dump.restype = i32
            self.L.ref_depth_map_dump.argtypes = [vp, vp, i32, i32, i32, i32, f32, i32, f32, i32, i32, vp, vp, vp,
                                                  vp, vp, vp, DUMP_FN, vp]

    # ---- kernels -----------------------------------------------------------------
    def prep(self, img, r, fused=0):
        H, W = img.shape[:2]
        img = np.ascontiguousarray(img)
        bw, g, dt = _f4((H, W)), _f4((H, W)), _f4((H, W))
        assert self._prep(img.ctypes.data, W, H, W * 4, r, fused, bw.ctypes.data, g.ctypes.data, dt.ctypes.data) == 0
        return bw, g, dt

    def init(self, bw1, bw2, g1, g2, r, dmax, lr, initdisp=None, initnormal=None, fused=0):
        H, W = bw1.shape[:2]
        out = _f4((H, W))
        assert self._init(out.ctypes.data, _p(bw1), _p(bw2), _p(g1), _p(g2), W, H, r, dmax, lr, _p(initdisp),
                          _p(initnormal), fused) == 0
        return out

    def propagate(self, old, bw1, bw2, g1, g2, smooth, theta, r, dmax, lr, it, vin_n=None, vin_val=None,
                  scatter=True, fused=0, counters=None):
        """Returns (planes, vout_n, vout_val, vout_src); vout_src is None for the reference build."""
        H, W = old.shape[:2]
        out = _f4((H, W))
        vn = np.zeros((H, W), np.int32) if scatter else None
        vv = np.zeros((H, W, 8), np.float32) if scatter else None
        vs = np.full((H, W, 2), -1, np.int32) if (scatter and self.kind == "orc") else None
        assert self._propagate(out.ctypes.data, _p(old), _p(bw1), _p(bw2), _p(g1), _p(g2), _p(smooth), theta, W, H, r,
                               dmax, lr, it, _p(vin_n), _p(vin_val), _p(vn), _p(vv), _p(vs), fused,
                               _p(counters)) == 0
        return out, vn, vv, vs

    def cost(self, planes, bw1, bw2, g1, g2, r, mincost, fused=0):
        H, W = planes.shape[:2]
        out = np.zeros((H, W), np.float32)
        assert self._cost(out.ctypes.data, _p(planes), _p(bw1), _p(bw2), _p(g1), _p(g2), W, H, r, mincost, fused) == 0
        return out

    def klt(self, planes, bw1, bw2, g1, g2, r, fused=0):
        H, W = planes.shape[:2]
        out = _f4((H, W))
        assert self._klt(out.ctypes.data, _p(planes), _p(bw1), _p(bw2), _p(g1), _p(g2), W, H, r, fused) == 0
        return out

    def normal_depth(self, planes, dispscale, lr):
        H, W = planes.shape[:2]
        out = _f4((H, W))
        assert self._normal_depth(out.ctypes.data, _p(planes), W, H, dispscale, lr) == 0
        return out

    def rof(self, inp, dt, lam, iters):
        H, W = inp.shape[:2]
        out = _f4((H, W))
        lam_c = (C.c_float * 4)(*lam)
        assert self._rof(out.ctypes.data, _p(inp), _p(dt), lam_c, iters, W, H) == 0
        return out

    def consistency(self, left, right, maxdd=1.0, maxad=5.0):
        H, W = left.shape[:2]
        out = _f4((H, W))
        assert self._consistency(out.ctypes.data, _p(left), _p(right), W, H, maxdd, maxad) == 0
        return out

    def to_disparity(self, planes, scale=1.0, lr=1):
        H, W = planes.shape[:2]
        out = np.zeros((H, W), np.float32)
        assert self._to_disparity(out.ctypes.data, _p(planes), W, H, scale, lr) == 0
        return out

    def fill_depthmap(self, planes, scale=1.0):
        H, W = planes.shape[:2]
        out = np.zeros((H, W), np.float32)
        assert self._fill_depthmap(out.ctypes.data, _p(planes), W, H, scale) == 0
        return out

    def fill_normalmap(self, planes, lr=1):
        H, W = planes.shape[:2]
        out = _f4((H, W))
        assert self._fill_normalmap(out.ctypes.data, _p(planes), W, H, lr) == 0
        return out

    def disparity_to_normal(self, disp):
        H, W = disp.shape[:2]
        out = _f4((H, W))
        assert self._disparity_to_normal(out.ctypes.data, _p(disp), W, H) == 0
        return out

    def pyrdown(self, img, Wo, Ho):
        """one pyramid step of an RGBA8 image (H, W, 4) to (Ho, Wo, 4)"""
        img = np.ascontiguousarray(img, np.uint8)
        out = np.zeros((Ho, Wo, 4), np.uint8)
        assert self._pyrdown(out.ctypes.data, Wo, Ho, img.ctypes.data, img.shape[1], img.shape[0]) == 0
        return out

    def pyrup_mul(self, img, Wo, Ho, mul):
        """pyrup_mul4f of a float image (H, W) or (H, W, 4) to (Ho, Wo[, 4]), times mul (4 floats)"""
        img = np.ascontiguousarray(img, np.float32)
        ch = 1 if img.ndim == 2 else 4
        out = np.zeros((Ho, Wo) if ch == 1 else (Ho, Wo, 4), np.float32)
        m = (C.c_float * 4)(*[float(v) for v in mul])
        assert self._pyrup_mul(out.ctypes.data, Wo, Ho, img.ctypes.data, img.shape[1], img.shape[0], ch, m) == 0
        return out

    # ---- whole pipeline ------------------------------------------------------------
    def disparity_map(self, left, right, r, dmax, iterations, pp=1, views=2, initdisp=None, initnormal=None,
                      fused=0, dump=False, counters=None, levels=1):
        """PMHuberStereo::disparityMap.  Returns dict with dmap, normal, planesL, planesR
        and, with dump=True, every intermediate stage keyed (stage, iter); stages of pyramid
        level l > 0 are named "l<l>_<stage>"."""
        H, W = left.shape[:2]
        left = np.ascontiguousarray(left)
        right = np.ascontiguousarray(right)
        res = {"dmap": np.zeros((H, W), np.float32), "normal": _f4((H, W)), "planesL": _f4((H, W)),
               "planesR": _f4((H, W)), "stages": {}}
        stages = res["stages"]

        def cb(name, it, w, h, ptr, user):
            stages[(name.decode(), it)] = np.ctypeslib.as_array(ptr, shape=(h, w, 4)).copy()

        fn = DUMP_FN(cb) if dump else DUMP_FN()
        common = [left.ctypes.data, right.ctypes.data, W, H, W * 4, r, dmax, iterations, pp, views, levels,
                  res["dmap"].ctypes.data, res["normal"].ctypes.data, _p(initdisp), _p(initnormal),
                  res["planesL"].ctypes.data, res["planesR"].ctypes.data]
        if self.kind == "orc":
            st = self.L.orc_disparity_map_dump(*common, fused, _p(counters), fn, None)
        else:
            st = self.L.ref_disparity_map_dump(*common, fn, None)
        assert st == 0, st
        return res

    def depth_map(self, left, right, r, dmax, iterations, dscale=-1.0, pp=1, views=2, initdisp=None,
                  initnormal=None, fused=0, dump=False, counters=None):
        """PMHuberStereo::depthMap.  Returns dict with dmap, normal, planesL, planesR (and stages)."""
        H, W = left.shape[:2]
        left = np.ascontiguousarray(left)
        right = np.ascontiguousarray(right)
        res = {"dmap": np.zeros((H, W), np.float32), "normal": _f4((H, W)), "planesL": _f4((H, W)),
               "planesR": _f4((H, W)), "stages": {}}
        stages = res["stages"]

        def cb(name, it, w, h, ptr, user):
            stages[(name.decode(), it)] = np.ctypeslib.as_array(ptr, shape=(h, w, 4)).copy()

        fn = DUMP_FN(cb) if dump else DUMP_FN()
        common = [left.ctypes.data, right.ctypes.data, W, H, W * 4, r, dmax, iterations, dscale, pp, views,
                  res["dmap"].ctypes.data, res["normal"].ctypes.data, _p(initdisp), _p(initnormal),
                  res["planesL"].ctypes.data, res["planesR"].ctypes.data]
        if self.kind == "orc":
            st = self.L.orc_depth_map_dump(*common, fused, _p(counters), fn, None)
        else:
            st = self.L.ref_depth_map_dump(*common, fn, None)
        assert st == 0, st
        return res

    def prep_raw(self, img, alpha):
        H, W = img.shape[:2]
        img = np.ascontiguousarray(img, np.uint8)
        c, g, d = _f4((H, W)), _f4((H, W)), _f4((H, W))
        assert self._prep_raw(img.ctypes.data, W, H, W * 4, alpha, c.ctypes.data, g.ctypes.data, d.ctypes.data) == 0
        return c, g, d

    def fill_state(self, planes, dispscale, lr):
        H, W = planes.shape[:2]
        out = _f4((H, W))
        assert self._fill_state(out.ctypes.data, _p(np.ascontiguousarray(planes, np.float32)), W, H, dispscale,
                                lr) == 0
        return out

    def huber(self, inp, dt, lam, eps, iters):
        H, W = inp.shape[:2]
        out = _f4((H, W))
        lm = (C.c_float * 4)(*[float(v) for v in lam])
        assert self._huber(out.ctypes.data, _p(np.ascontiguousarray(inp, np.float32)),
                           _p(np.ascontiguousarray(dt, np.float32)), lm, eps, iters, W, H) == 0
        return out

    # ---- VPMStereoCL (cvt/vision/VPMStereoCL.cpp) -----------------------------------
    def vpm_grad(self, img):
        """grad_gray_xydiag (gradxy.cl:60-97) of an RGBA8 image: (dx, dy, dx, dy)."""
        H, W = img.shape[:2]
        img = np.ascontiguousarray(img, np.uint8)
        out = _f4((H, W))
        assert self._vpm_grad(out.ctypes.data, img.ctypes.data, W, H, *self._st(W)) == 0
        return out

    def vpm_init(self, c1, g1, c2, g2, r, dmax, initdisp=None):
        """vpmstereo_init, or vpmstereo_init_disparity with initdisp (VPMStereo.cl:260-309)."""
        H, W = c1.shape[:2]
        c1, c2 = np.ascontiguousarray(c1, np.uint8), np.ascontiguousarray(c2, np.uint8)
        g1, g2 = np.ascontiguousarray(g1, np.float32), np.ascontiguousarray(g2, np.float32)
        if initdisp is not None:
            initdisp = np.ascontiguousarray(initdisp, np.float32)
        out = _f4((H, W))
        assert self._vpm_init(out.ctypes.data, c1.ctypes.data, g1.ctypes.data, c2.ctypes.data, g2.ctypes.data, W, H,
                              *self._st(W), r, dmax, _p(initdisp)) == 0
        return out

    def vpm_iter(self, states, c1, g1, c2, g2, r, dmax, it):
        """vpmstereo_iter_simple (VPMStereo.cl:311-361)."""
        H, W = c1.shape[:2]
        c1, c2 = np.ascontiguousarray(c1, np.uint8), np.ascontiguousarray(c2, np.uint8)
        g1, g2 = np.ascontiguousarray(g1, np.float32), np.ascontiguousarray(g2, np.float32)
        states = np.ascontiguousarray(states, np.float32)
        out = _f4((H, W))
        assert self._vpm_iter(out.ctypes.data, states.ctypes.data, c1.ctypes.data, g1.ctypes.data, c2.ctypes.data,
                              g2.ctypes.data, W, H, *self._st(W), r, dmax, it) == 0
        return out

    def vpm_disparity(self, states, scale=1.0):
        """vpmstereo_disparity (VPMStereo.cl:363-377)."""
        H, W = states.shape[:2]
        states = np.ascontiguousarray(states, np.float32)
        out = np.zeros((H, W), np.float32)
        assert self._vpm_disparity(out.ctypes.data, states.ctypes.data, W, H, scale) == 0
        return out

    def vpm_disparity_simple(self, c1, c2, r, iterations, dmax, initdisp=None):
        """VPMStereoCL::disparitySimple (VPMStereoCL.cpp:54-85). Returns (disparity, states)."""
        H, W = c1.shape[:2]
        c1, c2 = np.ascontiguousarray(c1, np.uint8), np.ascontiguousarray(c2, np.uint8)
        if initdisp is not None:
            initdisp = np.ascontiguousarray(initdisp, np.float32)
        disp, states = np.zeros((H, W), np.float32), _f4((H, W))
        assert self._vpm_disparity_simple(disp.ctypes.data, states.ctypes.data, c1.ctypes.data, c2.ctypes.data, W, H,
                                          *self._st(W), r, iterations, dmax, _p(initdisp)) == 0
        return disp, states

    # ---- SVPMFlowCL (cvt/vision/SVPMFlowCL.cpp) --------------------------------------
    def svpm_init(self, img1, img2, r, flowmax):
        """svpmflow_init (SVPMFlow.cl:213-233): states (u, v, cost, 0)."""
        H, W = img1.shape[:2]
        a, b = np.ascontiguousarray(img1, np.uint8), np.ascontiguousarray(img2, np.uint8)
        out = _f4((H, W))
        assert self._svpm_init(out.ctypes.data, a.ctypes.data, b.ctypes.data, W, H, *self._st(W), r, flowmax) == 0
        return out

    def svpm_prop(self, states, duals, img1, img2, r, flowmax, it):
        """svpmflow_prop_local_tv_admm (SVPMFlow.cl:574-731). Returns (states, duals)."""
        H, W = img1.shape[:2]
        a, b = np.ascontiguousarray(img1, np.uint8), np.ascontiguousarray(img2, np.uint8)
        s_in, p_in = np.ascontiguousarray(states, np.float32), np.ascontiguousarray(duals, np.float32)
        out, pout = _f4((H, W)), _f4((H, W))
        assert self._svpm_prop(out.ctypes.data, pout.ctypes.data, s_in.ctypes.data, p_in.ctypes.data, a.ctypes.data,
                               b.ctypes.data, W, H, *self._st(W), r, flowmax, it) == 0
        return out, pout

    def svpm_to_flow(self, states):
        H, W = states.shape[:2]
        s_in = np.ascontiguousarray(states, np.float32)
        out = np.zeros((H, W, 2), np.float32)
        assert self._svpm_to_flow(out.ctypes.data, s_in.ctypes.data, W, H) == 0
        return out

    def svpm_flow(self, img1, img2, r, flowmax, iterations):
        """SVPMFlowCL::flow (SVPMFlowCL.cpp:58-89) with `iterations` passes (reference: 200).
        Returns (flow, states, duals)."""
        H, W = img1.shape[:2]
        a, b = np.ascontiguousarray(img1, np.uint8), np.ascontiguousarray(img2, np.uint8)
        flow, states, duals = np.zeros((H, W, 2), np.float32), _f4((H, W)), _f4((H, W))
        assert self._svpm_flow(flow.ctypes.data, states.ctypes.data, duals.ctypes.data, a.ctypes.data, b.ctypes.data,
                               W, H, *self._st(W), r, flowmax, iterations) == 0
        return flow, states, duals

    # ---- helpers (restatement only) ------------------------------------------------
    def known_counts(self):
        """(candidates with a known outcome, skipped by the CUDA kernels; those of them that
        changed the state when evaluated), since the library was loaded"""
        out = np.zeros(2, np.int64)
        self.L.orc_known_counts(out.ctypes.data_as(C.c_void_p))
        return int(out[0]), int(out[1])

    def rng_floats(self, linpos, nd, n):
        out = np.zeros(n, np.float32)
        assert self.L.orc_rng_floats(linpos, nd, n, out.ctypes.data) == 0
        return out


def bits_equal(a, b):
    """Bitwise equality of float arrays with every NaN treated as equal."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    nan = np.isnan(a) & np.isnan(b)
    return (a.view(np.uint32) == b.view(np.uint32)) | nan
