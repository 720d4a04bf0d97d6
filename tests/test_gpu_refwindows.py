"""Reference-compatible windows on the GPU (referenceWindows = 1, what the GPU_CB_* entry
points use): where the reference's sub-problem windows cut a footprint, the CUDA kernels
reproduce the reference's result -- the oracle's reference path with exact weights
(texq = 0) is the comparison, and the ideal operator must differ visibly (so the windowed
kernels are the ones that ran)."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case, smooth_projections

pytestmark = pytest.mark.gpu

QUIRK = {
    "48c72": dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5),
    "flat90": dict(vol_xyz=(40, 40, 24), det_wh=(90, 40), nviews=20, D=120.0, pw=0.5),
    "rows56": dict(vol_xyz=(40, 40, 40), det_wh=(64, 56), nviews=30, D=150.0, pw=0.8),
}


def _case(name):
    g, pb = make_case(**QUIRK[name])
    return dataclasses.replace(g, reference_windows=True), pb


@pytest.mark.parametrize("name", sorted(QUIRK))
@pytest.mark.parametrize("mode", [2, 1, 0])
def test_backprojection_reproduces_reference_windows(name, mode):
    import torch

    from fastcone_b200 import ops

    g, pb = _case(name)
    assert ops.reference_windows(g)["bp_matters"]
    proj, _ = smooth_projections(pb)
    got = ops.backproject(torch.from_numpy(proj).cuda(), g, mode=mode).cpu().numpy()
    emu = O.ref_backproject(pb, proj, kernel_mode=mode, texq=0)
    ideal = O.backproject_f64(pb, proj, kernel_mode=mode)
    # the windows matter here (by several times the tolerance below)
    assert O.rel_l2(emu, ideal) > 2e-4
    assert O.rel_l2(got, emu) < 5e-5, O.rel_l2(got, emu)


@pytest.mark.parametrize("name", sorted(QUIRK))
def test_projection_reproduces_reference_windows(name):
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.phantom import random_ellipsoids

    g, pb = _case(name)
    assert ops.reference_windows(g)["proj_matters"]
    vol = O.phantom_voxelize(pb.volDim, random_ellipsoids(6, pb.volDim, 4))
    emu = O.ref_project(pb, vol, texq=0)
    assert O.rel_l2(emu, O.project_f64(pb, vol)) > 1e-3
    for method in (0, 1):
        got = ops.project(torch.from_numpy(vol).cuda(), g, method=method).cpu().numpy()
        assert O.rel_l2(got, emu) < 5e-5, (method, O.rel_l2(got, emu))


def test_sub_volume_with_window_offsets():
    """volStart/volEnd and per-view window offsets through the windowed kernels."""
    import torch

    from fastcone_b200 import ops

    n = 24
    g, pb = make_case(vol_xyz=(48, 44, 40), det_wh=(72, 56), nviews=n, D=160.0, pw=0.6,
                      vol_start=(4, 2, 3), vol_end=(44, 40, 37), window_wh=(64, 48),
                      woff=np.arange(n) % 5 + 2, hoff=np.arange(n) % 3 + 4)
    g = dataclasses.replace(g, reference_windows=True)
    proj, _ = smooth_projections(pb)
    w = ops.reference_windows(g)
    for mode in (2, 0):
        got = ops.backproject(torch.from_numpy(proj).cuda(), g, mode=mode).cpu().numpy()
        emu = O.ref_backproject(pb, proj, kernel_mode=mode, texq=0)
        assert O.rel_l2(got, emu) < 5e-5, (mode, w["bp_matters"], O.rel_l2(got, emu))
    e, s = pb.volEnd, pb.volStart
    vol = np.random.default_rng(2).random((e[2] - s[2], e[1] - s[1], e[0] - s[0]), dtype=np.float32)
    got = ops.project(torch.from_numpy(vol).cuda(), g, method=1).cpu().numpy()
    emu = O.ref_project(pb, vol, texq=0)
    assert O.rel_l2(got, emu) < 5e-5, (w["proj_matters"], O.rel_l2(got, emu))


def test_plans_and_noalloc_refuse_windows_they_cannot_reproduce():
    import torch

    from fastcone_b200 import _lib, ops

    g, pb = _case("48c72")
    with pytest.raises(_lib.FastconeError):
        ops.ProjectPlan(g, method=1)
    proj = torch.zeros(pb.proj_shape, device="cuda")
    vol = torch.zeros(g.vol_shape, device="cuda")
    gs = g.struct()
    import ctypes

    rc = _lib.lib().fcb_backproject_device_noalloc(ctypes.byref(gs), 2, ctypes.c_void_p(proj.data_ptr()),
                                                   _lib.FCB_F32, ctypes.c_void_p(vol.data_ptr()), None)
    assert rc == _lib.FCB_ERR_INVALID
