"""Katsevich helical reconstruction: GPU filtering vs the FP64 oracle's filtering
(rel-L2 <= 1e-5), and the full reconstruction (GPU filtering + PI-window backprojection) of a
seeded ellipsoid phantom vs the FP64 oracle pipeline (rel-L2 <= 2e-3) and vs the phantom
itself in the central region (discretisation-limited: rel-L2 <= 0.2, mean within 2 %)."""
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _helix():
    from fastcone_b200.geometry import ConeGeometry

    return ConeGeometry.helical((48, 48, 40), 1.0, (128, 32), 1.0, 150.0, 300.0, 3, 120, 24.0,
                                pi_window=True)


def _data(g):
    from fastcone_b200.phantom import random_ellipsoids

    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid)
    params = random_ellipsoids(4, g.vol_xyz, 5, axes=(0.25, 0.45), centre_radius=0.4)
    vol = O.phantom_voxelize(g.vol_xyz, params)
    return pb, vol, O.project_f64(pb, vol).astype(np.float32)


def test_katsevich_filter_vs_fp64():
    import torch

    from fastcone_b200 import ops

    g = _helix()
    pb, vol, proj = _data(g)
    got = ops.katsevich_filter(torch.from_numpy(proj).cuda(), g).cpu().numpy()
    want = O.katsevich_filter(proj, g.angles, g.D, g.pw, g.helical_pitch)
    assert O.rel_l2(got, want) < 1e-5, O.rel_l2(got, want)


def test_katsevich_reconstruction():
    import torch

    from fastcone_b200 import ops

    g = _helix()
    pb, vol, proj = _data(g)
    rec = ops.katsevich_reconstruct(torch.from_numpy(proj).cuda(), g).cpu().numpy()
    gF = O.katsevich_filter(proj, g.angles, g.D, g.pw, g.helical_pitch)
    dlam = float(g.angles[-1] - g.angles[0]) / (g.nviews - 1)
    pb.norm[:] = dlam / (2 * math.pi * g.D)
    ref, pairs = O.katsevich_piwin_f64(pb, gF.astype(np.float32), g.helical_pitch)
    assert O.rel_l2(rec, ref) < 2e-3, O.rel_l2(rec, ref)
    c = (slice(12, 28), slice(10, 38), slice(10, 38))
    assert O.rel_l2(rec[c], vol[c]) < 0.2
    assert abs(rec[c].mean() / vol[c].mean() - 1.0) < 0.02


def test_fft_hilbert_matches_direct_sum(monkeypatch):
    """The Katsevich filter's Hilbert transform by cuFFT (default) equals the direct
    O(W^2) sum to FP32 rounding."""
    import numpy as np
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.helical((48, 48, 40), 1.0, (96, 24), 1.0, 150.0, 300.0, 3, 80, 24.0, pi_window=True)
    p = torch.from_numpy(np.random.default_rng(3).random(g.proj_shape, dtype=np.float32)).cuda()
    monkeypatch.setenv("FCB_KATS_DIRECT_HILBERT", "1")
    a = ops.katsevich_filter(p, g)
    monkeypatch.setenv("FCB_KATS_DIRECT_HILBERT", "0")
    b = ops.katsevich_filter(p, g)
    torch.cuda.synchronize()
    rel = float((a - b).norm() / a.norm())
    assert rel < 2e-5, rel


def test_katsevich_plan_equals_one_shot():
    """The reusable Katsevich filter plan gives the one-shot filter's result, call after call."""
    import numpy as np
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.helical((48, 48, 40), 1.0, (96, 24), 1.0, 150.0, 300.0, 3, 80, 24.0, pi_window=True)
    p = torch.from_numpy(np.random.default_rng(8).random(g.proj_shape, dtype=np.float32)).cuda()
    ref = ops.katsevich_filter(p, g)
    plan = ops.KatsevichPlan(g)
    for _ in range(2):
        got = plan(p)
        torch.cuda.synchronize()
        assert torch.equal(got, ref)


@pytest.mark.parametrize("dtype_name,tol", [("float16", 2e-3), ("bfloat16", 1e-2)])
def test_pi_window_16bit_storage(dtype_name, tol):
    """The PI-window backprojection with FP16 / BF16-stored projections (fdk_pair_kernel with
    the window) vs the FP64 oracle on the same data, within the storage type's rounding, and
    vs the FP32 kernel on the same 16-bit values (the same window decisions: <= 1e-5)."""
    import dataclasses

    import torch

    from fastcone_b200 import _lib, ops

    g = _helix()
    dlam = float(g.angles[-1] - g.angles[0]) / (g.nviews - 1)
    g = dataclasses.replace(g, norm=np.full(g.nviews, dlam / (2 * math.pi * g.D), np.float32))
    pb, vol, proj = _data(g)
    pb.norm[:] = g.norm
    p16 = torch.from_numpy(proj).cuda().to(getattr(torch, dtype_name))
    plan = ops.BackprojectPlan(g, mode=_lib.MODE_KATSEVICH, dtype=p16.dtype)
    assert plan.info()["box_w"] > 0
    got = plan(p16, torch.zeros(g.vol_shape, device="cuda"))
    ops.sync_status()
    ref, _ = O.katsevich_piwin_f64(pb, proj, g.helical_pitch)
    assert O.rel_l2(got.cpu().numpy(), ref) < tol, O.rel_l2(got.cpu().numpy(), ref)
    same = ops.backproject(p16.float(), g, mode=_lib.MODE_KATSEVICH)
    assert O.rel_l2(got.cpu().numpy(), same.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("dtype_name,tol", [("float32", 2e-5), ("bfloat16", 1e-2)])
def test_pi_window_on_general_kernel(dtype_name, tol):
    """A projection buffer the TMA descriptor cannot take (4 bytes off alignment) runs the
    general-matrix kernel: it applies the same PI window (vs the FP64 oracle, and vs the
    staged kernel on the same values), also when the views of a staged launch (600 here)
    exceed what one launch of the general kernel holds."""
    import ctypes
    import dataclasses

    import torch

    from fastcone_b200 import _lib, ops
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.helical((40, 40, 36), 1.0, (112, 28), 1.0, 150.0, 300.0, 5, 120, 24.0, pi_window=True)
    dlam = float(g.angles[-1] - g.angles[0]) / (g.nviews - 1)
    g = dataclasses.replace(g, norm=np.full(g.nviews, dlam / (2 * math.pi * g.D), np.float32))
    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid,
                        norm=g.norm)
    proj = np.random.default_rng(9).random(g.proj_shape, dtype=np.float32)
    dt = getattr(torch, dtype_name)
    p = torch.from_numpy(proj).cuda().to(dt)
    n = p.numel()
    k = 4 // p.element_size()
    buf = torch.zeros(n + 16, dtype=dt, device="cuda")
    buf[k:k + n] = p.reshape(-1)
    L = _lib.lib()
    s = g.struct()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    got = torch.zeros(g.vol_shape, device="cuda")
    _lib.check(L.fcb_backproject_device(ctypes.byref(s), _lib.MODE_KATSEVICH, ctypes.c_void_p(buf[k:].data_ptr()),
                                        {"float32": 0, "bfloat16": 2}[dtype_name], ctypes.c_void_p(got.data_ptr()), st))
    ops.sync_status()
    got = got.cpu().numpy()
    ref, _ = O.katsevich_piwin_f64(pb, p.float().cpu().numpy(), g.helical_pitch)
    assert O.rel_l2(got, ref) < tol, O.rel_l2(got, ref)
    staged = ops.backproject(p, g, mode=_lib.MODE_KATSEVICH).cpu().numpy()
    assert O.rel_l2(got, staged) < 2e-5, O.rel_l2(got, staged)
