"""Device-side status paths without a GPU fault, the exact PI-window pair count, and the
measured shared-memory ceiling.

* Timeout: a plan's test hook (fcb_bp_plan_set_test_stall) makes the producer warp stage
  only the first views of each launch, drain its copies and leave; the consumers' next wait
  for a staged view runs out after 1 ms.  The kernel must report FCB_ERR_TIMEOUT through
  fcb_sync_status, leave no copy in flight, and the next normal call on the same context
  must match the FP64 oracle (FP32 storage <= 2e-5 rel-L2, BF16 <= 1e-2).  Covers the plain,
  the PI-window and the 16-bit (tap-pair) consumers.
* fcb_katsevich_pi_pairs equals the FP64 oracle's count of in-window voxel-view pairs on a
  whole small helix.
* fcb_smem_bandwidth returns a plausible rate (between 10 and 80 TB/s on a B200)."""
import ctypes
import dataclasses
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case, smooth_projections

pytestmark = pytest.mark.gpu


def _helix():
    from fastcone_b200.geometry import ConeGeometry

    return ConeGeometry.helical((48, 48, 40), 1.0, (128, 32), 1.0, 150.0, 300.0, 3, 120, 24.0,
                                pi_window=True)


def _stall_then_recover(g, mode, dtype, proj_np, ref, tol):
    import torch

    from fastcone_b200 import _lib, ops

    proj = torch.from_numpy(proj_np).cuda().to(dtype)
    plan = ops.BackprojectPlan(g, mode=mode, dtype=dtype)
    assert plan.info()["box_w"] > 0, "the case must use the staged kernel"
    _lib.check(_lib.lib().fcb_bp_plan_set_test_stall(plan._h, 3, 1000000))
    vol = torch.zeros(g.vol_shape, device="cuda")
    plan(proj, vol)
    with pytest.raises(_lib.FastconeError) as ex:
        ops.sync_status()
    assert ex.value.status == _lib.FCB_ERR_TIMEOUT
    # the context is usable and the status word clear: a normal call is correct
    ops.sync_status()
    _lib.check(_lib.lib().fcb_bp_plan_set_test_stall(plan._h, -1, 2000000000))
    vol.zero_()
    plan(proj, vol)
    ops.sync_status()
    got = vol.cpu().numpy()
    assert O.rel_l2(got, ref) < tol, O.rel_l2(got, ref)


@pytest.mark.parametrize("dtype_name,tol", [("float32", 2e-5), ("bfloat16", 1e-2)])
def test_timeout_reported_and_next_call_correct(dtype_name, tol):
    import torch

    g, pb = make_case(vol_xyz=(48, 40, 36), det_wh=(64, 48), nviews=45)
    proj, _ = smooth_projections(pb)
    ref = O.backproject_f64(pb, proj, kernel_mode=2)
    _stall_then_recover(g, 2, getattr(torch, dtype_name), proj, ref, tol)


def test_timeout_reported_pi_window():
    import torch

    g = _helix()
    dlam = float(g.angles[-1] - g.angles[0]) / (g.nviews - 1)
    g = dataclasses.replace(g, norm=np.full(g.nviews, dlam / (2 * math.pi * g.D), np.float32))
    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid,
                        norm=g.norm)
    proj = np.random.default_rng(4).random(g.proj_shape, dtype=np.float32)
    ref, _ = O.katsevich_piwin_f64(pb, proj, g.helical_pitch)
    _stall_then_recover(g, 1, torch.float32, proj, ref, 2e-5)


def test_set_test_stall_rejects_bad_arguments():
    import torch

    from fastcone_b200 import _lib, ops

    g, _ = make_case()
    plan = ops.BackprojectPlan(g, mode=2, dtype=torch.float32)
    assert _lib.lib().fcb_bp_plan_set_test_stall(plan._h, 1, 0) == _lib.FCB_ERR_INVALID
    assert _lib.lib().fcb_bp_plan_set_test_stall(plan._h, 1, 3000000000) == _lib.FCB_ERR_INVALID
    assert _lib.lib().fcb_bp_plan_set_test_stall(None, 1, 1000) == _lib.FCB_ERR_INVALID


def test_pi_pairs_equal_oracle_count():
    import bench

    g = _helix()
    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid)
    _, want = O.katsevich_piwin_f64(pb, np.zeros(g.proj_shape, np.float32), g.helical_pitch)
    got = bench.pi_pairs(g)
    assert got == want, (got, want)
    # a sub-volume and a single column
    sub = dataclasses.replace(g, vol_start=(5, 9, 3), vol_end=(40, 31, 37))
    pbs = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid,
                         volStart=sub.vol_start, volEnd=sub.vol_end)
    _, want = O.katsevich_piwin_f64(pbs, np.zeros(g.proj_shape, np.float32), g.helical_pitch)
    assert bench.pi_pairs(sub) == want
    pts = O.column_points(g.vol_xyz, (20, 30, 0), (21, 31, 40), 1)
    _, want = O.katsevich_piwin_points_f64(pb, np.zeros(g.proj_shape, np.float32), pts, g.helical_pitch)
    assert bench.pi_pairs(dataclasses.replace(g, vol_start=(20, 30, 0), vol_end=(21, 31, 40))) == want


def test_smem_probe_plausible():
    import torch

    from fastcone_b200 import _lib

    ms, nb = ctypes.c_float(), ctypes.c_double()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.lib().fcb_smem_bandwidth(4, 20000, ctypes.byref(ms), ctypes.byref(nb), st))
    gbs = nb.value / (ms.value / 1e3) / 1e9
    assert 10e3 < gbs < 80e3, gbs
    assert _lib.lib().fcb_smem_bandwidth(3, 10, ctypes.byref(ms), ctypes.byref(nb), st) == _lib.FCB_ERR_INVALID
