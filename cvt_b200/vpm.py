"""Python mirror of cvt::VPMStereoCL (cvt/vision/VPMStereoCL.h:33-65).

`VPMStereoCL(patchsize, iterations, disparitymax)` and
`disparity_simple(image0, image1, initdisparity=None)` follow the reference's
constructor and `disparitySimple(output, image0, image1, initdisparity)`
(VPMStereoCL.cpp:36-85): RGBA8 images go in, the disparity map comes out.
Host numpy arrays run through pm_vpm_disparity_simple (host copies included);
CUDA torch tensors run through pm_vpm_disparity_simple_device on the current
stream.  Errors raise StereoError, as the reference raises cvt::Exception.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import StereoError  # noqa: F401


def _check(status, handle=None):
    if status != _lib.PM_OK:
        L = _lib.lib()
        msg = L.pm_vpm_last_error(handle)
        raise StereoError(status, (msg or L.pm_status_string(status)).decode())
    return status


def _is_torch(x):
    return type(x).__module__.startswith("torch")


class VPMStereoCL:
    """One-view slanted-plane PatchMatch stereo (van der Corput candidates, neighbour
    states, Gauss-Newton refinement) on one B200."""

    def __init__(self, patchsize, iterations, disparitymax, device=0):
        h = C.c_void_p()
        _check(_lib.lib().pm_vpm_create(C.byref(h), int(patchsize), int(iterations), float(disparitymax),
                                        int(device)))
        self._h = h
        self.patchsize, self.iterations, self.disparitymax = int(patchsize), int(iterations), float(disparitymax)

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().pm_vpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_counting(self, on):
        _check(_lib.lib().pm_vpm_set_counting(self._h, int(bool(on))), self._h)

    def counters(self):
        """(cost-window taps, Gauss-Newton taps) of the calls made while counting."""
        c = (C.c_uint64 * 2)()
        _check(_lib.lib().pm_vpm_get_counters(self._h, c), self._h)
        return int(c[0]), int(c[1])

    def disparity_simple(self, image0, image1, initdisparity=None, states=False, stream=None):
        """Returns the (H, W) float32 disparity map, or (disparity, states) with states=True.
        image0/image1: (H, W, 4) uint8, numpy (host) or CUDA torch tensors (device)."""
        if _is_torch(image0):
            return self._device(image0, image1, initdisparity, states, stream)
        a = np.ascontiguousarray(image0, np.uint8)
        b = np.ascontiguousarray(image1, np.uint8)
        if a.ndim != 3 or a.shape[2] != 4 or b.shape != a.shape:
            raise ValueError("images must be (H, W, 4) uint8 of equal size")
        H, W = a.shape[:2]
        disp = np.zeros((H, W), np.float32)
        st = np.zeros((H, W, 4), np.float32) if states else None
        ini = None if initdisparity is None else np.ascontiguousarray(initdisparity, np.float32)
        if ini is not None and ini.shape != (H, W):
            raise ValueError("initdisparity must be (H, W)")
        _check(_lib.lib().pm_vpm_disparity_simple(self._h, a.ctypes.data, b.ctypes.data, W, H, W * 4,
                                                  disp.ctypes.data, None if ini is None else ini.ctypes.data,
                                                  None if st is None else st.ctypes.data), self._h)
        return (disp, st) if states else disp

    def _device(self, image0, image1, initdisparity, states, stream):
        import torch

        if image0.dtype != torch.uint8 or image0.dim() != 3 or image0.shape[2] != 4 or image1.shape != image0.shape:
            raise ValueError("images must be (H, W, 4) uint8 CUDA tensors of equal size")
        a, b = image0.contiguous(), image1.contiguous()
        H, W = a.shape[:2]
        disp = torch.empty((H, W), dtype=torch.float32, device=a.device)
        st = torch.empty((H, W, 4), dtype=torch.float32, device=a.device) if states else None
        ini = None if initdisparity is None else initdisparity.to(torch.float32).contiguous()
        s = stream if stream is not None else torch.cuda.current_stream(a.device).cuda_stream
        _check(_lib.lib().pm_vpm_disparity_simple_device(self._h, a.data_ptr(), b.data_ptr(), W, H, W * 4,
                                                         disp.data_ptr(), None if ini is None else ini.data_ptr(),
                                                         None if st is None else st.data_ptr(), s), self._h)
        return (disp, st) if states else disp
