"""fcb_backproject_device_noalloc: the backprojection entry point for callers that cannot
allocate device memory while they run (GPU memory owned by another allocator or a fixed
budget, or a timing-critical loop that must not stop for an allocation).  Its scratch is a
static device array shared by all calls, so this file checks it through the C ABI against
the allocating entry point, twice in a row (the second call must not see the first one's
leftovers).  It is named to be collected last and must pass alone or after the others."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case, smooth_projections

pytestmark = pytest.mark.gpu

# the tolerance of the backprojection parity tests (FP32 arithmetic)
TOL = 2e-5


def test_noalloc_backprojection_matches_allocating_entry_point():
    import torch

    from fastcone_b200 import _lib

    L = _lib.lib()
    g, pb = make_case(vol_xyz=(56, 48, 40), det_wh=(72, 56), nviews=50, D=150.0, pw=0.7)
    proj_np, _ = smooth_projections(pb)
    proj = torch.from_numpy(proj_np).cuda()
    s = g.struct()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dp = lambda t: ctypes.c_void_p(t.data_ptr())

    want = torch.zeros(g.vol_shape, device="cuda")
    _lib.check(L.fcb_backproject_device(ctypes.byref(s), _lib.MODE_FDK, dp(proj), _lib.FCB_F32, dp(want), stream))
    _lib.check(L.fcb_sync_status(stream))
    want_np = want.cpu().numpy()

    for call in range(2):
        got = torch.zeros(g.vol_shape, device="cuda")
        _lib.check(L.fcb_backproject_device_noalloc(ctypes.byref(s), _lib.MODE_FDK, dp(proj), _lib.FCB_F32,
                                                    dp(got), stream))
        got_np = got.cpu().numpy()
        assert O.rel_l2(got_np, want_np) < TOL, (call, O.rel_l2(got_np, want_np))
    # and both agree with the FP64 oracle
    assert O.rel_l2(got_np, O.backproject_f64(pb, proj_np, kernel_mode=2)) < TOL
