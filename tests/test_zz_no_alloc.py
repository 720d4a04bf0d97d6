"""fcb_backproject_device_noalloc: the backprojection entry point for callers that cannot
allocate device memory while they run (GPU memory owned by another allocator or a fixed
budget, or a timing-critical loop that must not stop for an allocation).  Its scratch is a
static device array shared by all calls, so each case here calls it twice in a row through
the C ABI and checks both results against the allocating entry point (and the FP64 oracle):
the second call clears and reuses what the first left in the array.  Cases: FP32 / FP16 /
BF16 storage, the unweighted, Katsevich (with and without the PI window) and FDK modes, a
projection pointer the TMA path cannot take (the general kernel runs), and a geometry whose
reference-compatible windows would need a device table (refused with FCB_ERR_INVALID).  It
is named to be collected last and must pass alone or after the others."""
import ctypes
import dataclasses
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case, smooth_projections

pytestmark = pytest.mark.gpu

# tolerances of the backprojection parity tests: FP32 arithmetic, and the storage rounding
# of the 16-bit types on smooth data
TOL = {"float32": 2e-5, "float16": 2e-3, "bfloat16": 1e-2}
CODE = {"float32": 0, "float16": 1, "bfloat16": 2}


def _run_pair(g, mode, proj, ptype, offset_bytes=0):
    """Allocating result, then two no-alloc results (host arrays)."""
    import torch

    from fastcone_b200 import _lib

    L = _lib.lib()
    s = g.struct()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    base = proj
    if offset_bytes:
        # the same values starting `offset_bytes` into a larger buffer (not 16-byte aligned)
        n = proj.numel()
        k = offset_bytes // proj.element_size()
        buf = torch.zeros(n + 16, dtype=proj.dtype, device=proj.device)
        buf[k:k + n] = proj.reshape(-1)
        base = buf[k:]
    dp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    want = torch.zeros(g.vol_shape, device="cuda")
    _lib.check(L.fcb_backproject_device(ctypes.byref(s), mode, dp(base), ptype, dp(want), stream))
    _lib.check(L.fcb_sync_status(stream))
    out = []
    for _ in range(2):
        got = torch.zeros(g.vol_shape, device="cuda")
        _lib.check(L.fcb_backproject_device_noalloc(ctypes.byref(s), mode, dp(base), ptype, dp(got), stream))
        out.append(got.cpu().numpy())
    return want.cpu().numpy(), out


@pytest.mark.parametrize("dtype_name", ["float32", "float16", "bfloat16"])
@pytest.mark.parametrize("mode", [2, 1, 0])
def test_noalloc_matches_allocating_entry_point(dtype_name, mode):
    import torch

    g, pb = make_case(vol_xyz=(56, 48, 40), det_wh=(72, 56), nviews=50, D=150.0, pw=0.7)
    proj_np, _ = smooth_projections(pb)
    proj = torch.from_numpy(proj_np).cuda().to(getattr(torch, dtype_name))
    want, got = _run_pair(g, mode, proj, CODE[dtype_name])
    for call in range(2):
        # identical work through the same kernels: equal to FP32 rounding of the summation
        assert O.rel_l2(got[call], want) < 2e-5, (call, O.rel_l2(got[call], want))
    ref = O.backproject_f64(pb, proj_np, kernel_mode=mode)
    assert O.rel_l2(got[1], ref) < TOL[dtype_name], O.rel_l2(got[1], ref)


def test_noalloc_pi_window():
    import torch

    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.helical((48, 48, 40), 1.0, (128, 32), 1.0, 150.0, 300.0, 3, 120, 24.0, pi_window=True)
    dlam = float(g.angles[-1] - g.angles[0]) / (g.nviews - 1)
    g = dataclasses.replace(g, norm=np.full(g.nviews, dlam / (2 * math.pi * g.D), np.float32))
    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid,
                        norm=g.norm)
    proj_np = np.random.default_rng(6).random(g.proj_shape, dtype=np.float32)
    want, got = _run_pair(g, 1, torch.from_numpy(proj_np).cuda(), 0)
    for call in range(2):
        assert O.rel_l2(got[call], want) < 2e-5, (call, O.rel_l2(got[call], want))
    ref, _ = O.katsevich_piwin_f64(pb, proj_np, g.helical_pitch)
    assert O.rel_l2(got[1], ref) < 2e-5, O.rel_l2(got[1], ref)


def test_noalloc_unaligned_projection_runs_general_kernel():
    import torch

    g, pb = make_case(vol_xyz=(40, 36, 32), det_wh=(64, 48), nviews=30)
    proj_np, _ = smooth_projections(pb)
    want, got = _run_pair(g, 2, torch.from_numpy(proj_np).cuda(), 0, offset_bytes=4)
    for call in range(2):
        assert O.rel_l2(got[call], want) < 2e-5, (call, O.rel_l2(got[call], want))
    ref = O.backproject_f64(pb, proj_np, kernel_mode=2)
    assert O.rel_l2(got[1], ref) < 2e-5, O.rel_l2(got[1], ref)


def test_noalloc_refuses_reference_windows_that_matter():
    import torch

    from fastcone_b200 import _lib, ops
    from fastcone_b200.geometry import ConeGeometry

    # the 48^3 / 72-pixel geometry whose reference windows change the FDK result
    g = ConeGeometry((48, 48, 48), (72, 48), np.arange(36) * (2 * np.pi / 36), 200.0, 0.5,
                     reference_windows=True)
    assert ops.reference_windows(g)["bp_matters"]
    s = g.struct()
    proj = torch.ones(g.proj_shape, device="cuda")
    vol = torch.zeros(g.vol_shape, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = _lib.lib().fcb_backproject_device_noalloc(ctypes.byref(s), 2, ctypes.c_void_p(proj.data_ptr()), 0,
                                                   ctypes.c_void_p(vol.data_ptr()), stream)
    assert rc == _lib.FCB_ERR_INVALID
    assert float(vol.abs().sum()) == 0.0
