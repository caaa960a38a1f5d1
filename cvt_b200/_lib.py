"""ctypes binding of libcvtpm.so (include/cvtpm.h).

The library is loaded from this package directory.  It is required: there is
no fallback implementation, and every call below fails loudly if the library
is missing.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcvtpm.so")

PM_OK, PM_EINVAL_SHAPE, PM_EINVAL_ARG, PM_ENOMEM, PM_ECUDA, PM_ETIMEOUT, PM_ENOTIMPL, PM_ENODEV = range(8)
PM_MAX_WIDTH, PM_MAX_HEIGHT, PM_MAX_RADIUS = 4096, 4096, 32   # the image and window limits of cvtpm.h
PM_MAX_BATCH, PM_BATCH_BRANCHES, PM_MAX_RANKS = 4096, 16, 1024   # the batch limits of cvtpm.h
PM_BATCH_LOCKSTEP, PM_BATCH_BRANCHED = 0, 1   # batch schedules (pm_set_batch_schedule)
PP_NONE, PP_LRCHECK, PP_LRCHECK_FILL = 0, 1, 2

# every exported symbol of include/cvtpm.h
SYMBOLS = [
    "pm_options_default", "pm_create", "pm_destroy", "pm_last_error", "pm_status_string",
    "pm_disparity_map", "pm_disparity_map_device", "pm_depth_map", "pm_depth_map_device", "pm_set_counting", "pm_get_counters",
    "pm_set_profiling", "pm_get_phase_times", "pm_measure_fp32_peak",
    "pm_disparity_map_batch_device", "pm_disparity_map_init2_device", "pm_set_batch_branches", "pm_batch_schedule",
    "pm_batch_partition", "pm_set_batch_schedule", "pm_batch_jobs",
    "pm_k_prep", "pm_k_init", "pm_k_cost", "pm_k_klt", "pm_k_propagate", "pm_k_normal_depth",
    "pm_rof_scratch_bytes", "pm_k_rof", "pm_k_rof_static", "pm_k_consistency", "pm_k_to_disparity", "pm_k_fill_depthmap",
    "pm_k_fill_normalmap", "pm_k_disparity_to_normal", "pm_k_pyrdown", "pm_k_pyrup_mul", "pm_pyramid_size",
    "pm_k_fill_state", "pm_k_huber", "pm_k_prep_raw",
    "pm_pfm_save", "pm_pfm_load", "pm_cvtraw_save", "pm_cvtraw_load", "pm_io_last_error",
    "pm_rng_floats", "pm_expf_host", "pm_sinf_host", "pm_cosf_host", "pm_acospif_host",
    "pm_exit_threshold_host", "pm_scene_generate", "pm_logf_host",
    "pm_vpm_create", "pm_vpm_destroy", "pm_vpm_last_error", "pm_vpm_disparity_simple",
    "pm_vpm_disparity_simple_device", "pm_vpm_set_counting", "pm_vpm_get_counters",
    "pm_k_vpm_grad", "pm_k_vpm_init", "pm_k_vpm_iter", "pm_k_vpm_disparity",
    "pm_svpm_create", "pm_svpm_destroy", "pm_svpm_last_error", "pm_svpm_flow", "pm_svpm_flow_device",
    "pm_svpm_set_counting", "pm_svpm_get_counters", "pm_k_svpm_init", "pm_k_svpm_prop", "pm_k_svpm_to_flow",
    "pm_lpp_last_error", "pm_lpp_layers", "pm_lpp_layer_shape", "pm_lpp_param_count", "pm_lpp_input", "pm_lpp_conv",
    "pm_lpp_wgrad_scratch_floats", "pm_lpp_wgrad", "pm_lpp_target", "pm_lpp_loss", "pm_lpp_upsample", "pm_lpp_adam",
    "pm_lpp_weights_bf16", "pm_lpp_propose_workspace_bytes", "pm_lpp_propose_device",
]


class Options(C.Structure):
    _fields_ = [("views", C.c_int), ("fused", C.c_int), ("thetamin", C.c_float), ("maxdispdiff", C.c_float),
                ("maxanglediff", C.c_float), ("rof_iters", C.c_int), ("device", C.c_int), ("use_graph", C.c_int),
                ("levels", C.c_int)]


class StereoError(RuntimeError):
    """Raised for a non-zero status of the native library (the reference throws cvt::Exception)."""

    def __init__(self, status, message):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


_lib = None

vp = C.c_void_p
i32 = C.c_int
f32 = C.c_float
sz = C.c_size_t


def lib():
    """Load libcvtpm.so (built by cvt_b200/build.py) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libcvtpm.so is not built: run `python cvt_b200/build.py` (needs nvcc)")
    L = C.CDLL(LIB_PATH)
    sig = {
        "pm_options_default": (i32, [C.POINTER(Options)]),
        "pm_create": (i32, [C.POINTER(vp), C.POINTER(Options)]),
        "pm_destroy": (i32, [vp]),
        "pm_last_error": (C.c_char_p, [vp]),
        "pm_status_string": (C.c_char_p, [i32]),
        "pm_disparity_map": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, i32, vp, vp, vp, vp, vp, vp]),
        "pm_disparity_map_device": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, i32, vp, vp, vp, vp, vp, vp, vp]),
        "pm_depth_map": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, f32, i32, vp, vp, vp, vp, vp, vp]),
        "pm_depth_map_device": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, f32, i32, vp, vp, vp, vp, vp, vp,
                                      vp]),
        "pm_set_counting": (i32, [vp, i32]),
        "pm_set_batch_branches": (i32, [vp, i32]),
        "pm_batch_schedule": (i32, [i32, i32, vp, vp, vp, vp, vp]),
        "pm_batch_partition": (i32, [i32, i32, vp, vp, vp, vp, vp, vp]),
        "pm_set_batch_schedule": (i32, [vp, i32, i32, i32, i32]),
        "pm_batch_jobs": (i32, [i32, vp, vp, vp, i32, i32, i32, vp, i32, C.POINTER(C.c_int)]),
        "pm_get_counters": (i32, [vp, C.POINTER(C.c_uint64)]),
        "pm_set_profiling": (i32, [vp, i32]),
        "pm_get_phase_times": (i32, [vp, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
        "pm_measure_fp32_peak": (i32, [i32, f32, C.POINTER(C.c_float)]),
        "pm_disparity_map_batch_device": (i32, [vp, i32, vp, vp, vp, vp, vp, vp, vp, i32, i32, vp, vp, vp, vp]),
        "pm_k_prep": (i32, [vp, i32, i32, sz, i32, i32, vp, vp, vp, vp]),
        "pm_k_init": (i32, [vp, vp, vp, vp, vp, i32, i32, i32, f32, i32, vp, vp, i32, vp]),
        "pm_k_cost": (i32, [vp, vp, vp, vp, vp, vp, i32, i32, i32, f32, i32, vp]),
        "pm_k_klt": (i32, [vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, vp]),
        "pm_k_propagate": (i32, [vp, vp, vp, vp, vp, vp, vp, f32, i32, i32, i32, f32, i32, i32,
                                 vp, vp, vp, vp, vp, i32, vp, vp]),
        "pm_k_normal_depth": (i32, [vp, vp, i32, i32, f32, i32, vp]),
        "pm_rof_scratch_bytes": (sz, [i32, i32]),
        "pm_k_rof": (i32, [vp, vp, vp, C.POINTER(C.c_float), i32, i32, i32, vp, vp]),
        "pm_k_rof_static": (i32, [vp, vp, vp, C.POINTER(C.c_float), i32, i32, i32, vp]),
        "pm_k_consistency": (i32, [vp, vp, vp, i32, i32, f32, f32, vp]),
        "pm_k_to_disparity": (i32, [vp, vp, i32, i32, f32, i32, vp]),
        "pm_k_fill_depthmap": (i32, [vp, vp, i32, i32, f32, vp]),
        "pm_k_fill_normalmap": (i32, [vp, vp, i32, i32, i32, vp]),
        "pm_k_disparity_to_normal": (i32, [vp, vp, i32, i32, vp]),
        "pm_pfm_save": (i32, [C.c_char_p, vp, i32, i32, i32, sz]),
        "pm_pfm_load": (i32, [C.c_char_p, vp, sz, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]),
        "pm_cvtraw_save": (i32, [C.c_char_p, vp, i32, i32, sz, i32]),
        "pm_cvtraw_load": (i32, [C.c_char_p, vp, sz, sz, C.POINTER(i32), C.POINTER(i32), C.POINTER(sz),
                                 C.POINTER(i32)]),
        "pm_io_last_error": (C.c_char_p, []),
        "pm_k_fill_state": (i32, [vp, vp, i32, i32, f32, i32, vp]),
        "pm_k_huber": (i32, [vp, vp, vp, C.POINTER(C.c_float), f32, i32, i32, i32, vp, vp]),
        "pm_k_prep_raw": (i32, [vp, i32, i32, sz, f32, vp, vp, vp, vp]),
        "pm_k_pyrdown": (i32, [vp, i32, i32, vp, sz, i32, i32, vp]),
        "pm_k_pyrup_mul": (i32, [vp, i32, i32, vp, i32, i32, i32, C.POINTER(C.c_float), vp]),
        "pm_pyramid_size": (i32, [i32, i32]),
        "pm_rng_floats": (i32, [C.c_int64, i32, i32, vp]),
        "pm_expf_host": (f32, [f32]),
        "pm_sinf_host": (f32, [f32]),
        "pm_cosf_host": (f32, [f32]),
        "pm_acospif_host": (f32, [f32]),
        "pm_logf_host": (f32, [f32]),
        "pm_exit_threshold_host": (f32, [f32, f32]),
        "pm_scene_generate": (i32, [C.c_uint64, i32, i32, i32, f32, f32, f32, f32, vp, vp, i32, vp, vp]),
        "pm_vpm_create": (i32, [C.POINTER(vp), i32, i32, f32, i32]),
        "pm_vpm_destroy": (i32, [vp]),
        "pm_vpm_last_error": (C.c_char_p, [vp]),
        "pm_vpm_disparity_simple": (i32, [vp, vp, vp, i32, i32, sz, vp, vp, vp]),
        "pm_vpm_disparity_simple_device": (i32, [vp, vp, vp, i32, i32, sz, vp, vp, vp, vp]),
        "pm_vpm_set_counting": (i32, [vp, i32]),
        "pm_vpm_get_counters": (i32, [vp, C.POINTER(C.c_uint64)]),
        "pm_k_vpm_grad": (i32, [vp, vp, i32, i32, sz, vp]),
        "pm_k_vpm_init": (i32, [vp, vp, vp, vp, vp, i32, i32, sz, i32, f32, vp, vp]),
        "pm_k_vpm_iter": (i32, [vp, vp, vp, vp, vp, vp, i32, i32, sz, i32, f32, i32, vp]),
        "pm_k_vpm_disparity": (i32, [vp, vp, i32, i32, f32, vp]),
        "pm_svpm_create": (i32, [C.POINTER(vp), i32]),
        "pm_svpm_destroy": (i32, [vp]),
        "pm_svpm_last_error": (C.c_char_p, [vp]),
        "pm_svpm_flow": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, vp, vp, vp]),
        "pm_svpm_flow_device": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, vp, vp, vp, vp]),
        "pm_svpm_set_counting": (i32, [vp, i32]),
        "pm_svpm_get_counters": (i32, [vp, C.POINTER(C.c_uint64)]),
        "pm_k_svpm_init": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, vp]),
        "pm_k_svpm_prop": (i32, [vp, vp, vp, vp, vp, vp, i32, i32, sz, i32, f32, i32, vp]),
        "pm_k_svpm_to_flow": (i32, [vp, vp, i32, i32, vp]),
        "pm_lpp_last_error": (C.c_char_p, []),
        "pm_lpp_layers": (i32, []),
        "pm_lpp_layer_shape": (i32, [i32, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "pm_lpp_param_count": (sz, []),
        "pm_lpp_input": (i32, [vp, vp, i32, i32, sz, i32, i32, vp, vp]),
        "pm_lpp_conv": (i32, [i32, i32, i32, vp, vp, vp, vp, vp, i32, i32, i32, vp, vp]),
        "pm_lpp_wgrad_scratch_floats": (sz, [i32, i32, i32, i32]),
        "pm_lpp_wgrad": (i32, [i32, i32, vp, vp, vp, vp, i32, i32, i32, vp, vp]),
        "pm_lpp_target": (i32, [vp, vp, i32, i32, i32, i32, f32, vp, vp]),
        "pm_lpp_loss": (i32, [vp, vp, f32, f32, i32, vp, vp, vp]),
        "pm_lpp_upsample": (i32, [vp, i32, i32, i32, i32, i32, i32, f32, vp, vp, vp]),
        "pm_lpp_adam": (i32, [vp, vp, vp, vp, i32, f32, i32, vp]),
        "pm_lpp_weights_bf16": (i32, [i32, vp, vp, vp, vp]),
        "pm_lpp_propose_workspace_bytes": (sz, [i32, i32, i32]),
        "pm_lpp_propose_device": (i32, [vp, vp, i32, vp, vp, i32, i32, sz, i32, f32, vp, vp, vp, sz, vp, vp]),
        "pm_disparity_map_init2_device": (i32, [vp, vp, vp, i32, i32, sz, i32, f32, i32, i32, vp, vp, vp, vp, vp, vp,
                                                vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status, handle=None):
    """Raise StereoError for a non-zero status, with the library's message."""
    if status != PM_OK:
        L = lib()
        msg = L.pm_last_error(handle) if handle is not None else L.pm_last_error(None)
        raise StereoError(status, (msg or L.pm_status_string(status)).decode())
    return status
