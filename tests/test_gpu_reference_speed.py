"""Speed and agreement against the reference's OWN CUDA path on the same B200 (oracle/_ref:
the reference sources compiled unmodified, texture references mapped onto texture objects),
through the same host-buffer entry point (GPU_CB_K_backproject's arguments,
fastcone.backproject, numpy buffers), on three problems:

* the small circular FDK: 128^3 voxels, 180 views, 192x128 detector, D = 500, pw = 0.5;
* the large circular FDK: 1024^3 voxels, 1440 views, 1536x1024 detector, D = 2000, pw = 0.8
  (the reference's host-side caching makes its call take about 15 s);
* the helix: 512x512x384, 4 turns x 1160 views, 736x64, Katsevich weight (the reference has
  no PI window, so both run dense).

Both calls include their host<->device copies and set-up (best of `reps` after a warm-up;
printed with -s).  Each test asserts the results agree within the 1e-3 rel-L2 of the
reference's 8-bit texture weights, and that ours is faster: by 5x on the two large problems
(the measured margins are larger)."""
import time

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _need_ref():
    if O.reflib() is None:
        pytest.skip("oracle/_ref/libfastcone_ref.so not built")


def _best(fn, reps):
    """(best time of `reps` calls after a warm-up call, the last call's result)"""
    out = fn()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        out = fn()
        best = min(best, time.perf_counter() - t0)
    return best, out


def _compare(vol_xyz, det_wh, nviews, D, pw, reps, mode=2, hmid=None, arc=2 * np.pi):
    from fastcone_b200 import fastcone as fc

    norm = np.full(nviews, 1.0 / nviews, np.float32)
    pb = O.make_problem(vol_xyz, det_wh, nviews, D=D, pw=pw, norm=norm, hmid=hmid, arc=arc)
    proj = np.random.default_rng(0).random(pb.proj_shape, dtype=np.float32)
    upd = float(np.prod(vol_xyz)) * nviews

    def ours():
        vol = np.zeros(pb.vol_shape_zyx, np.float32)
        fc.backproject(vol, proj, pb.angles, pb.D, pb.hMid, norm=norm, kernelMode=mode, pixelWidth=pb.pw)
        return vol

    def ref():
        return O.reflib_backproject(pb, proj, kernel_mode=mode)

    t_ours, v_ours = _best(ours, reps)
    t_ref, v_ref = _best(ref, reps)
    err = O.rel_l2(v_ours, v_ref)
    print(f"\n{vol_xyz} x {nviews} views, mode {mode}: ours {t_ours * 1e3:.1f} ms ({upd / t_ours / 1e9:.1f} GUPS), "
          f"reference CUDA path {t_ref * 1e3:.1f} ms ({upd / t_ref / 1e9:.1f} GUPS), "
          f"ratio {t_ref / t_ours:.1f}, rel-L2 {err:.2e}")
    return t_ours, t_ref, err


def test_faster_than_reference_cuda_path_small_fdk():
    _need_ref()
    t_ours, t_ref, err = _compare((128, 128, 128), (192, 128), 180, 500.0, 0.5, reps=3)
    assert err < 1e-3
    assert t_ours < t_ref


def test_faster_than_reference_cuda_path_large_fdk():
    _need_ref()
    t_ours, t_ref, err = _compare((1024, 1024, 1024), (1536, 1024), 1440, 2000.0, 0.8, reps=1)
    assert err < 1e-3
    assert t_ref > 5.0 * t_ours, (t_ours, t_ref)


def test_faster_than_reference_cuda_path_helical_katsevich():
    """The helical geometry (512x512x384, 4 turns x 1160 views, 736x64 detector) through the
    reference's Katsevich backprojection (kernelMode 1: weight U, every view, no PI window --
    the reference has none) and ours on the same arguments."""
    _need_ref()
    n = 4 * 1160
    hmid = (384 / 2.0 - 0.5 * (n - 1) * (80.0 / 1160) + np.arange(n) * (80.0 / 1160)).astype(np.float32)
    t_ours, t_ref, err = _compare((512, 512, 384), (736, 64), n, 1140.0, 1.096, reps=1, mode=1, hmid=hmid,
                                  arc=4 * 2 * np.pi)
    assert err < 1e-3
    assert t_ref > 5.0 * t_ours, (t_ours, t_ref)
