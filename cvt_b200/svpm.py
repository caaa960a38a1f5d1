"""Python mirror of cvt::SVPMFlowCL (cvt/vision/SVPMFlowCL.h).

`SVPMFlowCL().flow(first, second, patchsize, flowmax)` follows the reference's
`flow(flow, first, second, patchsize, flowmax, gtflow)` (SVPMFlowCL.cpp:58-89):
RGBA8 frames go in, the (H, W, 2) float32 flow (u, v) comes out.  The reference
runs MAXITER = 200 passes; `iterations` makes that count a parameter (default
200).  Host numpy arrays run through pm_svpm_flow (host copies included); CUDA
torch tensors run through pm_svpm_flow_device on the current stream.  Errors
raise StereoError, as the reference raises cvt::Exception.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import StereoError  # noqa: F401

MAXITER = 200


def _check(status, handle=None):
    if status != _lib.PM_OK:
        L = _lib.lib()
        msg = L.pm_svpm_last_error(handle)
        raise StereoError(status, (msg or L.pm_status_string(status)).decode())
    return status


def _is_torch(x):
    return type(x).__module__.startswith("torch")


class SVPMFlowCL:
    """PatchMatch optical flow with a TV pull on one B200."""

    def __init__(self, device=0):
        h = C.c_void_p()
        _check(_lib.lib().pm_svpm_create(C.byref(h), int(device)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().pm_svpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_counting(self, on):
        _check(_lib.lib().pm_svpm_set_counting(self._h, int(bool(on))), self._h)

    def counters(self):
        """cost-window taps of the propagation passes of the calls made while counting"""
        c = (C.c_uint64 * 1)()
        _check(_lib.lib().pm_svpm_get_counters(self._h, c), self._h)
        return int(c[0])

    def flow(self, first, second, patchsize, flowmax, iterations=MAXITER, states=False, stream=None):
        """Returns the (H, W, 2) flow, or (flow, states, duals) with states=True."""
        if _is_torch(first):
            return self._device(first, second, patchsize, flowmax, iterations, states, stream)
        a = np.ascontiguousarray(first, np.uint8)
        b = np.ascontiguousarray(second, np.uint8)
        if a.ndim != 3 or a.shape[2] != 4 or b.shape != a.shape:
            raise ValueError("frames must be (H, W, 4) uint8 of equal size")
        H, W = a.shape[:2]
        fl = np.zeros((H, W, 2), np.float32)
        st = np.zeros((H, W, 4), np.float32) if states else None
        du = np.zeros((H, W, 4), np.float32) if states else None
        _check(_lib.lib().pm_svpm_flow(self._h, a.ctypes.data, b.ctypes.data, W, H, W * 4, int(patchsize),
                                       float(flowmax), int(iterations), fl.ctypes.data,
                                       None if st is None else st.ctypes.data, None if du is None else du.ctypes.data),
               self._h)
        return (fl, st, du) if states else fl

    def _device(self, first, second, patchsize, flowmax, iterations, states, stream):
        import torch

        if first.dtype != torch.uint8 or first.dim() != 3 or first.shape[2] != 4 or second.shape != first.shape:
            raise ValueError("frames must be (H, W, 4) uint8 CUDA tensors of equal size")
        a, b = first.contiguous(), second.contiguous()
        H, W = a.shape[:2]
        fl = torch.empty((H, W, 2), dtype=torch.float32, device=a.device)
        st = torch.empty((H, W, 4), dtype=torch.float32, device=a.device) if states else None
        du = torch.empty((H, W, 4), dtype=torch.float32, device=a.device) if states else None
        s = stream if stream is not None else torch.cuda.current_stream(a.device).cuda_stream
        _check(_lib.lib().pm_svpm_flow_device(self._h, a.data_ptr(), b.data_ptr(), W, H, W * 4, int(patchsize),
                                              float(flowmax), int(iterations), fl.data_ptr(),
                                              None if st is None else st.data_ptr(),
                                              None if du is None else du.data_ptr(), s), self._h)
        return (fl, st, du) if states else fl
