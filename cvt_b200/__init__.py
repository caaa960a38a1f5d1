"""cvt_b200 — B200-native PatchMatch-Huber stereo (the cvt::PMHuberStereo path of phheise/cvt).

The computation runs in libcvtpm.so (hand-written sm_100a CUDA kernels behind the
C ABI of include/cvtpm.h); this package is its Python front end.
"""
from ._lib import StereoError, lib  # noqa: F401
from .stereo import (DISPARITY_PP_LRCHECK, DISPARITY_PP_LRCHECK_FILL, DISPARITY_PP_NONE,  # noqa: F401
                     PMHuberStereo)

__all__ = ["PMHuberStereo", "StereoError", "DISPARITY_PP_NONE", "DISPARITY_PP_LRCHECK",
           "DISPARITY_PP_LRCHECK_FILL", "lib"]
