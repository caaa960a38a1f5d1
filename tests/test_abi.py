"""The C-ABI library without a GPU: it loads, exports every declared entry point,
rejects bad arguments, and its host-evaluated arithmetic (the same code the
kernels run) equals the oracle's."""
import ctypes as C
import hashlib
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "cvtpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pm_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(native):
    from cvt_b200 import _lib

    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(native, n), n
    assert sorted(_lib.SYMBOLS) == names


def test_rejects_bad_shapes_without_touching_the_device(native):
    from cvt_b200 import _lib

    assert native.pm_k_prep(None, 0, 10, 40, 2, 1, None, None, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_prep(None, 10, 10, 40, 99, 1, None, None, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_prep(None, 5000, 10, 20000, 2, 1, None, None, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_prep(None, 10, 10, 40, 2, 1, None, None, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_init(None, None, None, None, None, 8, 8, 2, 4.0, 1, None, None, 1, None) == _lib.PM_EINVAL_ARG
    assert b"null" in native.pm_last_error(None)


def test_size_limits_follow_the_header(native):
    from cvt_b200 import _lib

    hdr = open(os.path.join(ROOT, "include", "cvtpm.h")).read()
    for name in ("PM_MAX_WIDTH", "PM_MAX_HEIGHT", "PM_MAX_RADIUS", "PM_MAX_BATCH", "PM_BATCH_BRANCHES"):
        assert int(re.search(name + r"\s*=\s*(\d+)", hdr).group(1)) == getattr(_lib, name), name
    W, r = _lib.PM_MAX_WIDTH, _lib.PM_MAX_RADIUS
    # one past each limit is refused before any device work
    assert native.pm_k_prep(None, W + 1, 4, 4 * (W + 1), 2, 1, None, None, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_prep(None, 4, _lib.PM_MAX_HEIGHT + 1, 16, 2, 1, None, None, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_prep(None, 4, 4, 16, r + 1, 1, None, None, None, None) == _lib.PM_EINVAL_SHAPE


def test_option_defaults_are_the_reference_constants(native):
    """pm_options_default: both views (disparityMapAll), thetamin 1e-4 (PMHuberStereo.cpp:92),
    LR check at 1 px and 5 degrees (:79-80), 40 ROF steps (PDOPTITER), one pyramid level (:78),
    strict arithmetic (bit-exact with the reference kernels); the structure's layout matches the
    header's; every status has a name"""
    from cvt_b200 import _lib

    o = _lib.Options()
    assert native.pm_options_default(C.byref(o)) == _lib.PM_OK
    assert (o.views, o.fused, o.rof_iters, o.device, o.use_graph, o.levels) == (2, 0, 40, 0, 1, 1)
    assert np.float32(o.thetamin) == np.float32(1e-4)
    assert (o.maxdispdiff, o.maxanglediff) == (1.0, 5.0)
    assert native.pm_options_default(None) == _lib.PM_EINVAL_ARG
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "cvtpm.h")).read(), flags=re.S)
    body = re.search(r"typedef struct\s*(?:pm_options)?\s*\{([^}]*)\}\s*pm_options;", hdr).group(1)
    fields = re.findall(r"(int|float)\s+(\w+);", body)
    assert [(n, {"int": C.c_int, "float": C.c_float}[t]) for t, n in fields] == list(_lib.Options._fields_)
    native.pm_status_string.restype = C.c_char_p
    names = [native.pm_status_string(s) for s in range(8)]
    assert len(set(names)) == 8 and all(n and n != b"unknown status" for n in names)
    assert native.pm_status_string(99) == b"unknown status"


def test_create_fails_loudly_without_device(native):
    import torch

    from cvt_b200 import _lib

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert native.pm_create(C.byref(h), None) == _lib.PM_ENODEV
    from cvt_b200 import PMHuberStereo, StereoError

    with pytest.raises(StereoError):
        PMHuberStereo()


def test_rng_matches_oracle(native, orc):
    for lin, nd in ((0, 3), (1, 3), (1234, 3), (77, 6), (921599 * 6 + 8, 1), (4000000, 6)):
        a = np.zeros(16, np.float32)
        assert native.pm_rng_floats(lin, nd, 16, a.ctypes.data) == 0
        b = orc.rng_floats(lin, nd, 16)
        assert (a.view(np.uint32) == b.view(np.uint32)).all(), (lin, nd)


def test_elementary_functions_match_oracle(native, orc):
    rng = np.random.default_rng(0)
    xs = np.concatenate([np.linspace(-40, 0, 4001), rng.uniform(-104, 89, 4000), [0.0, -0.0, 88.7, -103.9]])
    for x in xs.astype(np.float32):
        assert np.float32(native.pm_expf_host(float(x))).view(np.uint32) == \
            np.float32(orc.L.orc_exp(float(x))).view(np.uint32), x
    for x in np.concatenate([np.linspace(0, 6.3, 4001), rng.uniform(-100, 100, 2000)]).astype(np.float32):
        assert np.float32(native.pm_sinf_host(float(x))).view(np.uint32) == np.float32(orc.L.orc_sin(float(x))).view(np.uint32)
        assert np.float32(native.pm_cosf_host(float(x))).view(np.uint32) == np.float32(orc.L.orc_cos(float(x))).view(np.uint32)
    for x in np.linspace(-1, 1, 4001).astype(np.float32):
        assert np.float32(native.pm_acospif_host(float(x))).view(np.uint32) == \
            np.float32(orc.L.orc_acospi(float(x))).view(np.uint32)
    lx = np.concatenate([rng.integers(0, 0x7f800001, 6000, dtype=np.uint32).view(np.float32),
                         np.float32([0.0, 1.0, 2.3283064e-10, 1e-45, 0.5, 0.70710677, 1.4142135])])
    for x in lx:
        a, b = np.float32(native.pm_logf_host(float(x))), np.float32(orc.L.orc_log(float(x)))
        assert a.view(np.uint32) == b.view(np.uint32) or (np.isnan(a) and np.isnan(b)), x


def test_exit_threshold_is_exact(native):
    """census >= threshold(m, b)  <=>  RN(census / b) >= m, around the threshold."""
    rng = np.random.default_rng(1)
    for _ in range(3000):
        b = np.float32(rng.uniform(1.0, 450.0))
        m = np.float32(rng.choice([rng.uniform(0, 1.2), rng.uniform(1e-8, 1e-3), rng.uniform(0.9, 1.1)]))
        t = np.float32(native.pm_exit_threshold_host(float(m), float(b)))
        assert np.isfinite(t) and t >= 0
        below = np.nextafter(t, np.float32(-1))
        assert np.float32(t / b) >= m
        if t > 0:
            assert not (np.float32(below / b) >= m)
    assert native.pm_exit_threshold_host(0.0, 3.0) == -np.inf
    assert native.pm_exit_threshold_host(-1.0, 3.0) == -np.inf
    assert np.isnan(native.pm_exit_threshold_host(float("nan"), 3.0))
    assert native.pm_exit_threshold_host(float("inf"), 3.0) == np.inf


def test_scene_generator_is_deterministic(native):
    from cvt_b200 import scene

    L1, R1, d1, n1 = scene.generate(1234, 96, 64, 8, 2.0, 30.0, with_gt=True)
    L2, R2 = scene.generate(1234, 96, 64, 8, 2.0, 30.0)
    assert (L1 == L2).all() and (R1 == R2).all()
    assert d1.min() >= 2.0 - 1e-4 and d1.max() <= 30.0 + 1e-4
    assert np.abs(n1[..., :2]).max() <= 0.3 + 1e-6
    # the same bytes on every host: pinned digests
    h = hashlib.sha256(L1.tobytes() + R1.tobytes()).hexdigest()
    assert h == SCENE_DIGEST, h


SCENE_DIGEST = "54e0dc1c90811ccd82790abf7eceef416b3e1e22cc42747722fc6a5d7d1094ca"


def build_drop_in(tmp_path):
    import subprocess

    exe = str(tmp_path / "drop_in")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "drop_in.cpp"), "-L", os.path.join(ROOT, "cvt_b200"), "-lcvtpm",
                    "-Wl,-rpath," + os.path.join(ROOT, "cvt_b200"), "-o", exe], check=True)
    return exe


def test_cpp_drop_in_header_compiles_and_fails_loudly(native, tmp_path):
    """The C++ class with the reference's signatures builds against the library; without a
    device it throws (no CPU fallback)."""
    import subprocess

    import torch

    exe = build_drop_in(tmp_path)
    if not torch.cuda.is_available():
        p = subprocess.run([exe, str(tmp_path / "d.raw")], capture_output=True, text=True)
        assert p.returncode == 1 and "no CUDA device" in p.stderr


def _lpt_schedule(sizes, branches):
    """longest processing time first, as the batched entry documents it"""
    work = [w * h * (2 * r + 1) ** 2 for w, h, r in sizes]
    order = sorted(range(len(sizes)), key=lambda i: -work[i])   # sorted() is stable
    nb = min(len(sizes), branches)
    load, owner = [0] * nb, [0] * len(sizes)
    for i in order:
        b = min(range(nb), key=lambda k: (load[k], k))
        owner[i] = b
        load[b] += work[i]
    return order, owner, load


def test_batch_schedule_is_longest_first_onto_least_loaded(native):
    """the schedule of pm_disparity_map_batch_device, computed on the host: the 64-pair
    workload, ties in work (equal sizes keep their order), fewer pairs than branches"""
    from cvt_b200 import _lib, scene

    specs = scene.batch_specs()
    cases = [([(s["width"], s["height"], 10) for s in specs], b) for b in (1, 4, 16)]
    cases.append(([(64, 48, 2), (320, 240, 7), (64, 48, 2), (320, 240, 7), (96, 16, 32)], 3))
    cases.append(([(5, 5, 1), (7, 3, 0)], 16))
    for sizes, branches in cases:
        n = len(sizes)
        W = np.array([s[0] for s in sizes], np.int32)
        H = np.array([s[1] for s in sizes], np.int32)
        R = np.array([s[2] for s in sizes], np.int32)
        order, owner = np.zeros(n, np.int32), np.zeros(n, np.int32)
        assert native.pm_batch_schedule(n, branches, W.ctypes.data, H.ctypes.data, R.ctypes.data, order.ctypes.data,
                                        owner.ctypes.data) == _lib.PM_OK
        want_order, want_owner, load = _lpt_schedule(sizes, branches)
        assert order.tolist() == want_order and owner.tolist() == want_owner
        assert len(load) == min(n, branches) and sorted(set(owner.tolist())) == list(range(len(load)))
    x = np.zeros(4, np.int32)
    assert native.pm_batch_schedule(2, 0, x.ctypes.data, x.ctypes.data, x.ctypes.data, x.ctypes.data,
                                    x.ctypes.data) == _lib.PM_EINVAL_ARG
    assert native.pm_batch_schedule(2, _lib.PM_BATCH_BRANCHES + 1, x.ctypes.data, x.ctypes.data, x.ctypes.data,
                                    x.ctypes.data, x.ctypes.data) == _lib.PM_EINVAL_ARG
    assert native.pm_batch_schedule(2, 4, None, x.ctypes.data, x.ctypes.data, x.ctypes.data,
                                    x.ctypes.data) == _lib.PM_EINVAL_ARG
    assert native.pm_batch_schedule(0, 4, None, None, None, None, None) == _lib.PM_OK


def _jobs_restatement(sizes, tw, th, tile_order):
    """the job list of a lockstep batch: pairs in decreasing W*H*(2r+1)^2 (stable), tiles
    row-major per pair (order 0) or the pairs' tile rows interleaved (order 1)"""
    order = sorted(range(len(sizes)), key=lambda i: -sizes[i][0] * sizes[i][1] * (2 * sizes[i][2] + 1) ** 2)
    rows = {i: -(-sizes[i][1] // th) for i in order}
    cols = {i: -(-sizes[i][0] // tw) for i in order}
    out = []
    if tile_order == 0:
        for i in order:
            out += [(i, by, bx) for by in range(rows[i]) for bx in range(cols[i])]
    else:
        for by in range(max(rows.values())):
            for i in order:
                if by < rows[i]:
                    out += [(i, by, bx) for bx in range(cols[i])]
    return out


def test_batch_jobs_cover_every_tile_once(native):
    """pm_batch_jobs, the tile list the lockstep batch walks: every tile of every pair exactly
    once, in the documented order, for the 64-pair workload and ragged small cases"""
    from cvt_b200 import _lib, scene

    specs = scene.batch_specs()
    cases = [[(s["width"], s["height"], 10) for s in specs],
             [(64, 48, 2), (320, 240, 7), (64, 48, 2), (33, 17, 1), (1, 1, 0)], [(4096, 4096, 32)]]
    for sizes in cases:
        n = len(sizes)
        W = np.array([s[0] for s in sizes], np.int32)
        H = np.array([s[1] for s in sizes], np.int32)
        R = np.array([s[2] for s in sizes], np.int32)
        for tw, th in ((32, 4), (16, 8), (32, 8), (32, 16)):
            for order in (0, 1):
                cnt = C.c_int()
                assert native.pm_batch_jobs(n, W.ctypes.data, H.ctypes.data, R.ctypes.data, tw, th, order, None, 0,
                                            C.byref(cnt)) == _lib.PM_OK
                jobs = np.zeros(2 * cnt.value, np.uint32)
                assert native.pm_batch_jobs(n, W.ctypes.data, H.ctypes.data, R.ctypes.data, tw, th, order,
                                            jobs.ctypes.data, cnt.value, C.byref(cnt)) == _lib.PM_OK
                got = [(int(p), int(t) >> 16, int(t) & 0xFFFF) for p, t in zip(jobs[0::2], jobs[1::2])]
                want = _jobs_restatement(sizes, tw, th, order)
                assert got == want
                assert len(set(got)) == len(got) == sum(-(-w // tw) * -(-h // th) for w, h, _ in sizes)
        small = C.c_int()
        assert native.pm_batch_jobs(n, W.ctypes.data, H.ctypes.data, R.ctypes.data, 32, 4, 0, jobs.ctypes.data, 0,
                                    C.byref(small)) == _lib.PM_EINVAL_ARG
    x = np.zeros(4, np.int32)
    cnt = C.c_int()
    assert native.pm_batch_jobs(2, x.ctypes.data, x.ctypes.data, x.ctypes.data, 32, 4, 0, None, 0,
                                C.byref(cnt)) == _lib.PM_EINVAL_SHAPE
    w = np.array([8, 8], np.int32)
    assert native.pm_batch_jobs(2, w.ctypes.data, w.ctypes.data, x.ctypes.data, 32, 4, 2, None, 0,
                                C.byref(cnt)) == _lib.PM_EINVAL_ARG
    assert native.pm_batch_jobs(2, w.ctypes.data, w.ctypes.data, x.ctypes.data, 0, 4, 0, None, 0,
                                C.byref(cnt)) == _lib.PM_EINVAL_ARG
    assert native.pm_batch_jobs(0, None, None, None, 32, 4, 0, None, 0, C.byref(cnt)) == _lib.PM_OK
    assert cnt.value == 0
    assert native.pm_set_batch_schedule(None, 0, 0, 0, 32) == _lib.PM_EINVAL_ARG


def test_batch_specs_seeded_and_in_range():
    from cvt_b200 import scene

    a, b = scene.batch_specs(), scene.batch_specs()
    assert a == b and len(a) == 64
    for i, s in enumerate(a):
        assert s["seed"] == 1234 + i
        assert 320 <= s["width"] <= 1920 and 240 <= s["height"] <= 1080
        assert 8 <= s["planes"] <= 60
        assert s["dispmax"] == max(32, s["width"] // 10)
    assert len({(s["width"], s["height"]) for s in a}) > 60


def test_batch_null_handle(native):
    from cvt_b200 import _lib

    # argument checks come before any device work
    assert native.pm_disparity_map_batch_device(None, 1, None, None, None, None, None, None, None, 3, 1,
                                                None, None, None, None) == _lib.PM_EINVAL_ARG


def test_pyramid_sizes_follow_float_scaling(native):
    # CLPyramid::update: (size_t)(size_t(n) * 0.35f) per level, in float arithmetic
    for n in (1, 2, 3, 97, 320, 1280, 1920, 4096):
        m = n
        for levels in range(1, 5):
            assert native.pm_pyramid_size(n, levels) == m, (n, levels)
            m = int(np.float32(m) * np.float32(0.35))


def test_vpm_rejects_bad_arguments_without_touching_the_device(native):
    from cvt_b200 import _lib

    h = C.c_void_p()
    assert native.pm_vpm_create(C.byref(h), 99, 3, 16.0, 0) == _lib.PM_EINVAL_SHAPE
    assert native.pm_vpm_create(C.byref(h), 3, -1, 16.0, 0) == _lib.PM_EINVAL_ARG
    assert native.pm_vpm_create(C.byref(h), 3, 3, 0.0, 0) == _lib.PM_EINVAL_ARG
    assert native.pm_vpm_create(C.byref(h), 3, 3, float("nan"), 0) == _lib.PM_EINVAL_ARG
    assert native.pm_vpm_create(None, 3, 3, 16.0, 0) == _lib.PM_EINVAL_ARG
    assert b"null" in native.pm_vpm_last_error(None)
    assert native.pm_vpm_disparity_simple(None, None, None, 8, 8, 32, None, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_vpm_grad(None, None, 0, 8, 32, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_vpm_grad(None, None, 8, 8, 16, None) == _lib.PM_EINVAL_SHAPE   # stride < 4 W
    assert native.pm_k_vpm_grad(None, None, 8, 8, 32, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_vpm_init(None, None, None, None, None, 8, 8, 32, 40, 4.0, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_vpm_iter(None, None, None, None, None, None, 8, 8, 32, 2, 4.0, -1, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_vpm_disparity(None, None, 8, 0, 1.0, None) == _lib.PM_EINVAL_SHAPE


def test_vpm_create_fails_loudly_without_device(native):
    import torch

    from cvt_b200 import _lib

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert native.pm_vpm_create(C.byref(h), 3, 3, 16.0, 0) == _lib.PM_ENODEV
    from cvt_b200.vpm import StereoError, VPMStereoCL

    with pytest.raises(StereoError):
        VPMStereoCL(3, 3, 16.0)


def test_svpm_rejects_bad_arguments_without_touching_the_device(native):
    from cvt_b200 import _lib

    assert native.pm_svpm_create(None, 0) == _lib.PM_EINVAL_ARG
    assert native.pm_svpm_flow(None, None, None, 8, 8, 32, 2, 4.0, 5, None, None, None) == _lib.PM_EINVAL_ARG
    assert b"null" in native.pm_svpm_last_error(None)
    assert native.pm_k_svpm_init(None, None, None, 0, 8, 32, 2, 4.0, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_svpm_init(None, None, None, 8, 8, 32, 40, 4.0, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_k_svpm_init(None, None, None, 8, 8, 32, 2, -1.0, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_svpm_init(None, None, None, 8, 8, 32, 2, 4.0, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_svpm_prop(None, None, None, None, None, None, 8, 8, 32, 2, 4.0, -1, None) == _lib.PM_EINVAL_ARG
    assert native.pm_k_svpm_to_flow(None, None, 8, 8, None) == _lib.PM_EINVAL_ARG


def test_svpm_create_fails_loudly_without_device(native):
    import torch

    from cvt_b200 import _lib

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert native.pm_svpm_create(C.byref(h), 0) == _lib.PM_ENODEV
    from cvt_b200.svpm import StereoError, SVPMFlowCL

    with pytest.raises(StereoError):
        SVPMFlowCL()


def test_lpp_rejects_bad_arguments_without_touching_the_device(native):
    import ctypes as C

    from cvt_b200 import _lib

    # the network of cfg4: 8 layers of 3x3 convolutions, 32-64 channels, dilations growing to 16
    assert native.pm_lpp_layers() == 8
    shapes = []
    for l in range(8):
        ci, co, di = C.c_int(), C.c_int(), C.c_int()
        assert native.pm_lpp_layer_shape(l, C.byref(ci), C.byref(co), C.byref(di)) == 0
        shapes.append((ci.value, co.value, di.value))
    assert shapes == [(16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 4), (64, 64, 8), (64, 64, 16), (64, 32, 1),
                      (32, 16, 1)]
    assert native.pm_lpp_layer_shape(8, None, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_param_count() == sum(co * 9 * ci + co for ci, co, _ in shapes)
    assert native.pm_lpp_conv(0, 0, 1, None, None, None, None, None, 0, 4, 4, None, None) == _lib.PM_EINVAL_SHAPE
    assert native.pm_lpp_conv(9, 0, 1, None, None, None, None, None, 1, 4, 4, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_conv(0, 1, 1, None, None, None, None, None, 1, 4, 4, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_conv(2, 0, 1, None, None, None, None, None, 1, 4, 4, None, None) == _lib.PM_EINVAL_ARG
    assert b"null" in native.pm_lpp_last_error()
    assert native.pm_lpp_input(None, None, 3, 8, 16, 4, 0, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_loss(None, None, 1.0, 1.0, 0, None, None, None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_adam(None, None, None, None, 10, 1e-3, 0, None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_propose_workspace_bytes(2, 2, 4) == 0
    assert native.pm_lpp_propose_workspace_bytes(64, 48, 4) >= 16 * 12 * (16 * 2 + 2 * 64 * 2 + 16 * 4)
    assert native.pm_lpp_propose_device(None, None, 4, None, None, 64, 48, 256, 0, 64.0, None, None, None, 0, None,
                                        None) == _lib.PM_EINVAL_ARG
    assert native.pm_lpp_wgrad_scratch_floats(8, 1, 4, 4) == 0
    # partial sums per CTA, at most one CTA per 16 x 4-pixel unit and at most 160 CTAs:
    # 9 * CIN + 1 rows (the last one the bias) x COUT
    assert native.pm_lpp_wgrad_scratch_floats(3, 1, 32, 40) == 8 * 3 * (9 * 64 + 1) * 64
    assert native.pm_lpp_wgrad_scratch_floats(3, 32, 96, 128) == 160 * (9 * 64 + 1) * 64


def test_autotuner_keeps_the_fastest_candidate():
    """tune_batch with a stand-in handle and timer: every candidate (schedule, CTAs per SM, tile
    order, branches) is set, warmed once and timed `reps` times; the fastest stays set; ties go to
    the earlier candidate"""
    from cvt_b200.autotune import DEFAULT_CANDIDATES, label, tune_batch

    class FakeHandle:
        def __init__(self):
            self.state, self.calls, self.set_log = None, [], []
            self.sched = self.branches = None

        def set_batch_schedule(self, schedule, ctas, order, tile_w):
            self.sched = (schedule, ctas, order, tile_w)

        def set_batch_branches(self, n):
            self.branches = n
            self.state = self.sched + (n,)
            self.set_log.append(self.state)

        def disparity_map_batch(self, lefts, rights, patchsizes, dmaxs, iterations, pp=1):
            self.calls.append((self.state, iterations, pp))

    cands = [{"schedule": "branched", "branches": 4}, {"schedule": "lockstep", "ctas_per_sm": 3},
             {"schedule": "lockstep", "tile_order": 1, "tile_w": 16, "branches": 8}]
    keys = [("branched", 0, 0, 32, 4), ("lockstep", 3, 0, 32, 16), ("lockstep", 0, 1, 16, 8)]
    for cost, want in (([50.0, 20.0, 30.0], 1), ([9.0, 12.0, 9.0], 0)):
        pm = FakeHandle()
        table = dict(zip(keys, cost))

        def timer(fn):
            fn()
            return table[pm.state]

        res = tune_batch(pm, [], [], [], [], iterations=1, candidates=cands, reps=3, timer=timer)
        assert res["best"] == cands[want] and pm.state == keys[want]
        assert res["ms"] == {label(c): t for c, t in zip(cands, cost)}
        assert pm.set_log == keys + [keys[want]]
        assert [c[0] for c in pm.calls] == [k for k in keys for _ in range(4)]
        assert all(c[1:] == (1, 1) for c in pm.calls)
    assert len({label(c) for c in DEFAULT_CANDIDATES}) == len(DEFAULT_CANDIDATES)

