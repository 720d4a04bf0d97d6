"""GPU parity of the backprojectors against the CPU oracle (FP64 and reference path).

Tolerances: explicit-FP32 kernels vs the FP64 oracle at rel-L2 <= 2e-5 (FP32 arithmetic);
vs the reference path (texture-emulated 8-bit interpolation weights) at rel-L2 <= 1e-3, the
bound set by those weights; 16-bit projection storage vs FP64 at the rounding of the
storage type (fp16 2e-3, bf16 1e-2 rel-L2 on smooth data).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case, smooth_projections

pytestmark = pytest.mark.gpu


def _bp(g, proj, mode, dtype=None):
    import torch

    from fastcone_b200 import ops

    dtype = dtype or torch.float32
    p = torch.from_numpy(proj).cuda().to(dtype)
    vol = ops.backproject(p, g, mode=mode)
    ops.sync_status()
    return vol.cpu().numpy()


@pytest.mark.parametrize("mode", [2, 1, 0])
def test_bp_modes_vs_f64(mode):
    g, pb = make_case()
    proj, _ = smooth_projections(pb)
    got = _bp(g, proj, mode)
    ref64 = O.backproject_f64(pb, proj, kernel_mode=mode)
    assert O.rel_l2(got, ref64) < 2e-5, O.rel_l2(got, ref64)


def test_fdk_vs_reference_path():
    g, pb = make_case(vol_xyz=(64, 64, 64), det_wh=(96, 64), nviews=60, D=250.0, pw=0.5)
    proj, _ = smooth_projections(pb)
    proj = O.rampfilter(O.fbp_cosine_weight(proj, pb.D, pb.hMid)).astype(np.float32)
    got = _bp(g, proj, 2)
    refpath = O.ref_backproject(pb, proj, kernel_mode=2, texq=1)
    assert O.rel_l2(got, refpath) < 1e-3
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(got, ref64) < 2e-5


@pytest.mark.parametrize("case", [
    dict(vol_xyz=(50, 37, 29), det_wh=(60, 41), nviews=7),                        # ragged sizes
    dict(vol_xyz=(40, 40, 40), vol_start=(5, 3, 7), vol_end=(33, 38, 30)),       # sub-volume
    dict(vol_xyz=(40, 40, 40), det_wh=(64, 48), nviews=13, window_wh=(40, 30),
         woff=np.arange(13) % 5 + 8, hoff=np.arange(13) % 3 + 6),              # data windows
    dict(vol_xyz=(24, 24, 24), det_wh=(32, 32), nviews=1),                       # one view
    dict(vol_xyz=(24, 24, 24), det_wh=(32, 32), nviews=1901, D=80.0),           # several launches
])
def test_fdk_edge_cases(case):
    g, pb = make_case(**case)
    rng = np.random.default_rng(3)
    proj = rng.random(pb.proj_shape, dtype=np.float32)
    got = _bp(g, proj, 2)
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(got, ref64) < 3e-5


@pytest.mark.parametrize("vol_xyz", [(80, 48, 40), (40, 96, 36)])
@pytest.mark.parametrize("arc0, arc1, nviews", [
    (-0.17, 0.17, 24),        # views near 0 degrees: tiles run x fastest
    (1.40, 1.74, 24),         # near 90 degrees: y fastest
    (0.0, 2 * np.pi, 400),    # three launches of up to 180 views, each choosing its raster
])
def test_fdk_tile_raster(vol_xyz, arc0, arc1, nviews):
    """Each launch runs its tiles with x or y fastest (the axis that moves the detector column
    less over its views); on tile grids that are not square both orders must cover every tile
    exactly once."""
    angles = np.linspace(arc0, arc1, nviews, endpoint=False).astype(np.float32)
    g, pb = make_case(vol_xyz=vol_xyz, det_wh=(128, 64), nviews=nviews, D=200.0, pw=1.0, angles=angles)
    proj, _ = smooth_projections(pb)
    got = _bp(g, proj, 2)
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(got, ref64) < 2e-5, O.rel_l2(got, ref64)


def test_bp_accumulates():
    import torch

    from fastcone_b200 import ops

    g, pb = make_case()
    proj, _ = smooth_projections(pb)
    init = np.random.default_rng(5).random(g.vol_shape, dtype=np.float32)
    vol = torch.from_numpy(init.copy()).cuda()
    ops.backproject(torch.from_numpy(proj).cuda(), g, mode=2, vol=vol)
    got = vol.cpu().numpy()
    want = init + O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(got, want) < 2e-5


@pytest.mark.parametrize("dtype_name,tol", [("float16", 2e-3), ("bfloat16", 1e-2)])
def test_fdk_half_storage(dtype_name, tol):
    import torch

    g, pb = make_case(vol_xyz=(64, 64, 48), det_wh=(96, 64), nviews=90, D=250.0, pw=0.6)
    proj, _ = smooth_projections(pb)
    dt = getattr(torch, dtype_name)
    got = _bp(g, proj, 2, dtype=dt)
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(got, ref64) < tol


def test_plan_reuse_and_info():
    import torch

    from fastcone_b200 import ops

    g, pb = make_case()
    proj, _ = smooth_projections(pb)
    plan = ops.BackprojectPlan(g, mode=2)
    info = plan.info()
    assert info["box_w"] > 0 and info["box_h"] > 0 and info["box_w"] % 4 == 0
    p = torch.from_numpy(proj).cuda()
    v = torch.zeros(g.vol_shape, device="cuda")
    plan(p, v)
    plan(p, v)
    ops.sync_status()
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(v.cpu().numpy(), 2 * ref64) < 2e-5


def test_fdk_footprint_beyond_shared_memory_runs_generic():
    """Detector pixels much finer than voxels (pw = 0.14 voxel): a 16x16x32-voxel tile's
    footprint is about 155 x 225 pixels at 45 degrees, and two staged FP32 boxes of it
    (2 x 136 KB) exceed a CTA's 227 KB of shared memory, so the plan takes the general-matrix
    kernel (no staging box) instead of failing at launch; the result equals the FP64 oracle."""
    import torch

    from fastcone_b200 import ops

    g, pb = make_case(vol_xyz=(48, 48, 48), det_wh=(512, 352), nviews=16, D=1000.0, pw=0.14)
    proj = np.random.default_rng(9).random(pb.proj_shape, dtype=np.float32)
    plan = ops.BackprojectPlan(g, mode=2)
    info = plan.info()
    assert info["box_w"] == 0 and info["box_h"] == 0, info
    v = torch.zeros(g.vol_shape, device="cuda")
    plan(torch.from_numpy(proj).cuda(), v)
    ops.sync_status()
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(v.cpu().numpy(), ref64) < 3e-5


def test_reference_abi_host_buffers():
    """GPU_CB_K_backproject with host buffers (the reference's entry point) == device API."""
    from fastcone_b200 import fastcone as fc

    g, pb = make_case(vol_xyz=(40, 36, 32), det_wh=(50, 42), nviews=33)
    proj, _ = smooth_projections(pb)
    for mode in (2, 1, 0):
        vol = np.zeros(g.vol_shape, np.float32)
        fc.backproject(vol, proj.copy(), pb.angles, pb.D, pb.hMid, norm=pb.norm, kernelMode=mode,
                       pixelWidth=pb.pw)
        ref64 = O.backproject_f64(pb, proj, kernel_mode=mode)
        assert O.rel_l2(vol, ref64) < 2e-5, mode


@pytest.mark.parametrize("pinned", [False, True])
def test_host_driver_z_slab_pipeline(pinned):
    """A volume deep enough for several z-slabs (volume in/out overlapped with the kernels)
    through the host-buffer entry point, pageable and pinned buffers: equals the device API
    and the FP64 oracle; an accumulating second call doubles it."""
    import torch

    from fastcone_b200 import _lib, ops

    g, pb = make_case(vol_xyz=(40, 36, 200), det_wh=(64, 256), nviews=27, D=400.0, pw=1.0,
                      vol_start=(0, 0, 3), vol_end=(40, 36, 197))
    proj, _ = smooth_projections(pb)
    dev = ops.backproject(torch.from_numpy(proj).cuda(), g, mode=2).cpu().numpy()
    if pinned:
        vol_t = torch.zeros(g.vol_shape, dtype=torch.float32, pin_memory=True)
        proj_t = torch.from_numpy(proj).pin_memory()
        vol, hp = vol_t.numpy(), proj_t.numpy()
    else:
        vol, hp = np.zeros(g.vol_shape, np.float32), proj
    gs = g.struct()
    import ctypes

    for _ in range(2):
        _lib.check(_lib.lib().fcb_backproject_host(0, ctypes.byref(gs), 2, hp.ctypes.data_as(_lib.c_float_p),
                                                   vol.ctypes.data_as(_lib.c_float_p)))
    assert O.rel_l2(vol, 2 * dev) < 1e-6
    ref64 = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(vol, 2 * ref64) < 2e-5


def test_misaligned_unweighted():
    from fastcone_b200 import fastcone as fc

    g, pb = make_case(vol_xyz=(40, 40, 40), det_wh=(64, 56), nviews=30, D=150.0, pw=0.8)
    proj, _ = smooth_projections(pb)
    mis = np.array([1.5, -0.7, 3.0, 0.02, -0.015, 0.03], np.float32)
    vol = np.zeros(g.vol_shape, np.float32)
    fc.backproject(vol, proj.copy(), pb.angles, pb.D, pb.hMid, norm=pb.norm, kernelMode=0,
                   misAlignments=mis, pixelWidth=pb.pw)
    # the detector is smaller than the volume's shadow: the reference's windows cut rows
    # 52-55 off, and the reference-compatible entry point reproduces that
    emu = O.ref_backproject(pb, proj, kernel_mode=0, texq=0, mis=mis)
    assert O.rel_l2(vol, emu) < 5e-5
    # the native API (ideal operator) against the FP64 oracle
    import dataclasses

    import torch

    from fastcone_b200 import ops

    gm = dataclasses.replace(g, misalignments=mis)
    got = ops.backproject(torch.from_numpy(proj).cuda(), gm, mode=0).cpu().numpy()
    ref64 = O.backproject_f64(pb, proj, kernel_mode=0, mis=mis)
    assert O.rel_l2(got, ref64) < 2e-5


def test_katsevich_view_skipping_tall_volume():
    """A volume several z-tiles tall on a 4-turn helix: most views reach only some tiles and
    are not staged for the others; the result still equals the FP64 windowed oracle."""
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.geometry import ConeGeometry

    n, vpt = 480, 120
    P = 32.0
    g = ConeGeometry.helical((64, 64, 96), 1.0, (128, 24), 1.0, 200.0, 400.0, n // vpt, vpt, P,
                             pi_window=True)
    g = g.with_norm(np.full(n, 1.0 / vpt, np.float32))
    pb = O.make_problem(g.vol_xyz, g.det_wh, n, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid, norm=g.norm)
    proj = np.random.default_rng(4).random(pb.proj_shape, dtype=np.float32) + 0.5
    got = ops.backproject(torch.from_numpy(proj).cuda(), g, mode=1).cpu().numpy()
    ops.sync_status()
    ref, pairs = O.katsevich_piwin_f64(pb, proj, g.helical_pitch)
    assert 0 < pairs < 0.6 * np.prod(g.vol_shape) * n
    assert O.rel_l2(got, ref) < 2e-3, O.rel_l2(got, ref)


def test_katsevich_pi_window_vs_f64():
    """Katsevich backprojection restricted to the PI window (Tam-Danielsson bounds, oriented
    by the helix handedness) vs the FP64 oracle.  Voxel-view pairs within rounding of the
    window boundary may flip, hence the looser bound."""
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.geometry import ConeGeometry

    n, vpt = 240, 80
    P = 24.0
    g = ConeGeometry.helical((48, 48, 40), 1.0, (96, 24), 1.0, 150.0, 300.0, n // vpt, vpt, P,
                             pi_window=True)
    g = g.with_norm(np.full(n, 1.0 / vpt, np.float32))
    pb = O.make_problem(g.vol_xyz, g.det_wh, n, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid, norm=g.norm)
    proj = np.random.default_rng(9).random(pb.proj_shape, dtype=np.float32) + 0.5
    got = ops.backproject(torch.from_numpy(proj).cuda(), g, mode=1).cpu().numpy()
    ref, pairs = O.katsevich_piwin_f64(pb, proj, g.helical_pitch)
    assert pairs > 0
    assert O.rel_l2(got, ref) < 2e-3, O.rel_l2(got, ref)


def test_host_driver_staging_of_large_pageable_buffers():
    """Pageable caller buffers larger than one staging piece (64 MB), with a detector width
    that is not a multiple of 4 (rows padded on the device): the staged copies through
    pinned buffers give exactly the result of pinned caller buffers, for the backprojector
    (volume in and out, projections in) and the projector (projections in and out)."""
    import ctypes

    import torch

    from fastcone_b200 import _lib

    g, pb = make_case(vol_xyz=(256, 256, 300), det_wh=(250, 300), nviews=240, D=900.0, pw=1.0, seed=4)
    rng = np.random.default_rng(5)
    proj = rng.random(g.proj_shape, dtype=np.float32)           # 72 MB
    vol0 = rng.random(g.vol_shape, dtype=np.float32)            # 79 MB
    gs = g.struct()
    L = _lib.lib()
    outs = []
    for pinned in (False, True):
        if pinned:
            vol = torch.from_numpy(vol0.copy()).pin_memory().numpy()
            hp = torch.from_numpy(proj.copy()).pin_memory().numpy()
        else:
            vol, hp = vol0.copy(), proj.copy()
        _lib.check(L.fcb_backproject_host(0, ctypes.byref(gs), 2, hp.ctypes.data_as(_lib.c_float_p),
                                          vol.ctypes.data_as(_lib.c_float_p)))
        _lib.check(L.fcb_project_host(0, ctypes.byref(gs), _lib.PROJ_EXPLICIT, vol.ctypes.data_as(_lib.c_float_p),
                                      hp.ctypes.data_as(_lib.c_float_p)))
        outs.append((vol.copy(), hp.copy()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert not np.array_equal(outs[0][0], vol0)


def test_host_driver_device_block_cache(monkeypatch):
    """The host entry points keep a finished call's device blocks for later calls: calls that
    reuse them (blocks holding the previous call's data), calls after the cache was released
    and calls with the cache switched off give the same result, equal to the FP64 oracle."""
    import ctypes

    from fastcone_b200 import _lib

    g, pb = make_case(vol_xyz=(64, 56, 40), det_wh=(96, 64), nviews=90, D=200.0, pw=1.0, seed=6)
    proj, _ = smooth_projections(pb)
    gs = g.struct()
    L = _lib.lib()

    def host_bp(p):
        vol = np.zeros(g.vol_shape, np.float32)
        _lib.check(L.fcb_backproject_host(0, ctypes.byref(gs), 2, p.ctypes.data_as(_lib.c_float_p),
                                          vol.ctypes.data_as(_lib.c_float_p)))
        return vol

    first = host_bp(proj)
    other = host_bp(np.ascontiguousarray(proj[::-1]))     # different data through the same blocks
    again = host_bp(proj)
    _lib.check(L.fcb_release_device_cache())
    released = host_bp(proj)
    monkeypatch.setenv("FCB_HOST_CACHE", "0")
    uncached = host_bp(proj)
    _lib.check(L.fcb_release_device_cache())
    for v in (again, released, uncached):
        assert np.array_equal(v, first)
    assert not np.array_equal(other, first)
    assert O.rel_l2(first, O.backproject_f64(pb, proj, kernel_mode=2)) < 2e-5
