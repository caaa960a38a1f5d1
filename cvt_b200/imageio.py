"""Disparity, normal and plane images on disk in cvt's formats (PFM, CVTRaw), through
libcvtpm's host I/O (pm_pfm_* / pm_cvtraw_*).

    save_pfm(path, a)      a: (H, W) or (H, W, 4) float32; RGBA is saved without alpha
    load_pfm(path)         -> (H, W) or (H, W, 4) float32 (alpha 1)
    save_cvtraw(path, a)   a: (H, W) float32, (H, W, 2) float32 (flow), (H, W, 4) float32 or
                           (H, W, 4) uint8
    load_cvtraw(path)      -> array of the saved format
"""
import ctypes as C

import numpy as np

from . import _lib

# IFormat ids of cvt/gfx/IFormat.h:36-65 (PM_IFORMAT_* of cvtpm.h)
_FORMATS = {(1, np.dtype(np.float32)): 4, (2, np.dtype(np.float32)): 8, (4, np.dtype(np.uint8)): 9,
            (4, np.dtype(np.float32)): 12}
_DTYPES = {4: (np.float32, 1), 8: (np.float32, 2), 9: (np.uint8, 4), 12: (np.float32, 4)}


def _check(st):
    if st != 0:
        raise _lib.StereoError(st, (_lib.lib().pm_io_last_error() or b"I/O error").decode())


def save_pfm(path, a):
    a = np.ascontiguousarray(a, np.float32)
    ch = 1 if a.ndim == 2 else a.shape[2]
    if ch not in (1, 4):
        raise ValueError("PFM: grey (H, W) or RGBA (H, W, 4) float images")
    H, W = a.shape[:2]
    _check(_lib.lib().pm_pfm_save(str(path).encode(), a.ctypes.data, W, H, ch, W * ch * 4))


def load_pfm(path):
    L = _lib.lib()
    w, h, ch = C.c_int(), C.c_int(), C.c_int()
    p = str(path).encode()
    _check(L.pm_pfm_load(p, None, 0, C.byref(w), C.byref(h), C.byref(ch)))
    out = np.zeros((h.value, w.value) if ch.value == 1 else (h.value, w.value, 4), np.float32)
    _check(L.pm_pfm_load(p, out.ctypes.data, out.size, C.byref(w), C.byref(h), C.byref(ch)))
    return out


def save_cvtraw(path, a):
    a = np.ascontiguousarray(a)
    ch = 1 if a.ndim == 2 else a.shape[2]
    fid = _FORMATS.get((ch, a.dtype))
    if fid is None:
        raise ValueError("CVTRaw: GRAY_FLOAT, GRAYALPHA_FLOAT, RGBA_FLOAT or RGBA_UINT8 images")
    H, W = a.shape[:2]
    _check(_lib.lib().pm_cvtraw_save(str(path).encode(), a.ctypes.data, W, H, a.strides[0], fid))


def load_cvtraw(path):
    L = _lib.lib()
    w, h, fid = C.c_int(), C.c_int(), C.c_int()
    st = C.c_size_t()
    p = str(path).encode()
    _check(L.pm_cvtraw_load(p, None, 0, 0, C.byref(w), C.byref(h), C.byref(st), C.byref(fid)))
    if fid.value not in _DTYPES:
        raise ValueError("CVTRaw: unsupported format id %d" % fid.value)
    dt, ch = _DTYPES[fid.value]
    shape = (h.value, w.value) if ch == 1 else (h.value, w.value, ch)
    out = np.zeros(shape, dt)
    row = out.strides[0]
    _check(L.pm_cvtraw_load(p, out.ctypes.data, out.nbytes, row, C.byref(w), C.byref(h), C.byref(st), C.byref(fid)))
    return out
