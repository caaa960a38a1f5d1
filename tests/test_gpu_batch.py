"""Batched pairs of uneven sizes in one graph launch (pm_disparity_map_batch_device) and the
graph replay of single-pair calls, against eager single-pair calls through the C ABI.

All three run the same kernels on the same inputs, so the results must be bit-identical
(tolerance 0); the single-pair device path itself is pinned to the oracle in
test_gpu_parity.py.
"""
import numpy as np
import pytest

from oracle.pyoracle import bits_equal

pytestmark = pytest.mark.gpu

# (width, height, patch half-width, disparity range, planes)
PAIRS = [(72, 40, 3, 16.0, 5), (40, 56, 2, 12.0, 4), (96, 33, 4, 24.0, 6), (33, 17, 1, 8.0, 3)]


@pytest.fixture(scope="module")
def torch_cuda(native):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def _pairs(torch):
    from cvt_b200 import scene

    out = []
    for i, (w, h, r, d, npl) in enumerate(PAIRS):
        L, R = scene.generate(100 + i, w, h, npl, 1.0, 0.9 * d)
        out.append((torch.from_numpy(L).cuda(), torch.from_numpy(R).cuda(), r, d))
    return out


def _host(t):
    return t.cpu().numpy()


def test_batch_equals_single_pair_calls(torch_cuda):
    from cvt_b200 import PMHuberStereo

    pairs = _pairs(torch_cuda)
    eager = PMHuberStereo(views=2, fused=True, use_graph=False)
    ref = [eager.disparity_map(a, b, r, d, 3, planes=True) for a, b, r, d in pairs]
    pm = PMHuberStereo(views=2, fused=True)
    for rep in range(2):   # capture, then replay
        out = pm.disparity_map_batch([p[0] for p in pairs], [p[1] for p in pairs], [p[2] for p in pairs],
                                     [p[3] for p in pairs], 3, planes=True)
        torch_cuda.cuda.synchronize()
        for o, e in zip(out, ref):
            for k in ("dmap", "planes_left", "planes_right"):
                assert bits_equal(_host(o[k]), _host(e[k])).all(), (rep, k)


@pytest.mark.parametrize("schedule,ctas,order,tile_w,fused", [
    ("lockstep", 0, 0, 32, False), ("lockstep", 2, 1, 32, False), ("lockstep", 0, 1, 32, True),
    ("lockstep", 0, 0, 16, False), ("lockstep", 3, 1, 16, True), ("branched", 0, 0, 32, False)])
def test_schedules_equal_single_pair_calls(torch_cuda, schedule, ctas, order, tile_w, fused):
    """the lockstep schedule (persistent launches over the tiles of every pair, tiles of 32 x 4 or
    16 x 8 pixels) and the branched one give the single-pair results bit for bit, on capture and
    on replay, in both arithmetics"""
    from cvt_b200 import PMHuberStereo

    pairs = _pairs(torch_cuda)
    eager = PMHuberStereo(views=2, fused=fused, use_graph=False)
    ref = [eager.disparity_map(a, b, r, d, 3, planes=True) for a, b, r, d in pairs]
    pm = PMHuberStereo(views=2, fused=fused)
    pm.set_batch_schedule(schedule, ctas, order, tile_w)
    for rep in range(2):
        out = pm.disparity_map_batch([p[0] for p in pairs], [p[1] for p in pairs], [p[2] for p in pairs],
                                     [p[3] for p in pairs], 3, planes=True)
        torch_cuda.cuda.synchronize()
        for o, e in zip(out, ref):
            for k in ("dmap", "planes_left", "planes_right"):
                assert bits_equal(_host(o[k]), _host(e[k])).all(), (rep, k)


def test_lockstep_edge_cases(torch_cuda):
    """lockstep batches with one view (no view buffers), an odd smoothing step count (one single
    step, then double steps), no smoothing steps, eager launches (no graph) and counted runs (the
    counting kernel variants) equal single-pair calls"""
    from cvt_b200 import PMHuberStereo

    pairs = _pairs(torch_cuda)
    ls, rs = [p[0] for p in pairs], [p[1] for p in pairs]
    r, d = [p[2] for p in pairs], [p[3] for p in pairs]
    for kw, pp in (({"views": 1}, 0), ({"rof_iters": 7}, 1), ({"use_graph": False}, 1), ({"rof_iters": 0}, 1)):
        eager = PMHuberStereo(fused=False, **dict(kw, use_graph=False))
        ref = [eager.disparity_map(a, b, rr, dd, 4, pp=pp, planes=True) for a, b, rr, dd in pairs]
        pm = PMHuberStereo(fused=False, **kw)
        pm.set_batch_schedule("lockstep")
        out = pm.disparity_map_batch(ls, rs, r, d, 4, pp=pp, planes=True)
        torch_cuda.cuda.synchronize()
        for o, e in zip(out, ref):
            for k in ("dmap", "planes_left") + (("planes_right",) if kw.get("views", 2) == 2 else ()):
                assert bits_equal(_host(o[k]), _host(e[k])).all(), (kw, k)
    pm = PMHuberStereo(fused=False, use_graph=False)
    pm.set_batch_schedule("lockstep")
    pm.set_counting(True)
    out = pm.disparity_map_batch(ls, rs, r, d, 3, planes=True)
    ref = [PMHuberStereo(fused=False, use_graph=False).disparity_map(a, b, rr, dd, 3, planes=True)
           for a, b, rr, dd in pairs]
    torch_cuda.cuda.synchronize()
    for o, e in zip(out, ref):
        assert bits_equal(_host(o["planes_left"]), _host(e["planes_left"])).all()


def test_graph_replay_equals_eager(torch_cuda):
    from cvt_b200 import PMHuberStereo

    a, b, r, d = _pairs(torch_cuda)[0]
    eager = PMHuberStereo(views=2, fused=True, use_graph=False)
    e = eager.disparity_map(a, b, r, d, 3, planes=True)
    pm = PMHuberStereo(views=2, fused=True)
    for rep in range(3):
        o = pm.disparity_map(a, b, r, d, 3, planes=True)
        torch_cuda.cuda.synchronize()
        for k in ("dmap", "planes_left", "planes_right"):
            assert bits_equal(_host(o[k]), _host(e[k])).all(), (rep, k)
    # host entry (legacy default stream) through the graph as well
    h = pm.disparity_map(_host(a), _host(b), r, d, 3)
    assert bits_equal(h, _host(e["dmap"])).all()


def test_batch_rejects_bad_pair(torch_cuda):
    from cvt_b200 import PMHuberStereo, StereoError

    pairs = _pairs(torch_cuda)
    pm = PMHuberStereo(views=2)
    with pytest.raises(StereoError):
        pm.disparity_map_batch([pairs[0][0], pairs[1][0]], [pairs[0][1], pairs[1][1]], [3, 99], [16.0, 12.0], 3)
    assert pm.disparity_map_batch([], [], [], [], 3) == []


def test_branch_counts_and_autotuner_keep_results(torch_cuda, native):
    """every concurrent-branch count gives the same results bit for bit, in both schedules; the
    autotuner picks one of its candidates and leaves it set"""
    from cvt_b200 import PMHuberStereo
    from cvt_b200.autotune import tune_batch

    torch = torch_cuda
    pairs = _pairs(torch)
    ls, rs = [p[0] for p in pairs], [p[1] for p in pairs]
    r, d = [p[2] for p in pairs], [p[3] for p in pairs]
    pm = PMHuberStereo()
    ref = [_host(t) for t in pm.disparity_map_batch(ls, rs, r, d, 3)]
    for schedule in ("lockstep", "branched"):
        pm.set_batch_schedule(schedule)
        for nb in (1, 2, 3):
            pm.set_batch_branches(nb)
            got = [_host(t) for t in pm.disparity_map_batch(ls, rs, r, d, 3)]
            assert all(bits_equal(a, b).all() for a, b in zip(got, ref)), (schedule, nb)
    cands = [{"schedule": "branched", "branches": 2}, {"schedule": "lockstep", "ctas_per_sm": 1},
             {"schedule": "lockstep", "tile_order": 1, "branches": 1}]
    tuned = tune_batch(pm, ls, rs, r, d, iterations=1, candidates=cands, reps=1)
    assert tuned["best"] in cands and len(tuned["ms"]) == 3
    got = [_host(t) for t in pm.disparity_map_batch(ls, rs, r, d, 3)]
    assert all(bits_equal(a, b).all() for a, b in zip(got, ref))
    from cvt_b200 import _lib

    with pytest.raises(_lib.StereoError):
        pm.set_batch_branches(99)
    with pytest.raises(_lib.StereoError):
        pm.set_batch_schedule("lockstep", 0, 0, 24)
