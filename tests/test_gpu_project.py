"""GPU parity of the forward projector and its adjoint against the CPU oracle.

Explicit-FP32 projector vs the FP64 oracle: rel-L2 <= 2e-5.  Texture projector (8-bit
hardware interpolation weights, like the reference) vs the FP64 oracle: rel-L2 <= 1e-3,
and vs the texture-emulating reference path: rel-L2 <= 1e-3.  Adjoint: dot-product test
<Ax, y> = <x, A^T y> to 1e-5 relative, and vs the FP64 transpose at rel-L2 <= 2e-5.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case

pytestmark = pytest.mark.gpu


def _phantom(pb, seed=2):
    from fastcone_b200.phantom import random_ellipsoids

    return O.phantom_voxelize(pb.volDim, random_ellipsoids(8, pb.volDim, seed))


def _proj(g, vol, method):
    import torch

    from fastcone_b200 import ops

    return ops.project(torch.from_numpy(vol).cuda(), g, method=method).cpu().numpy()


@pytest.mark.parametrize("method,tol", [(1, 2e-5), (0, 1e-3)])
def test_project_vs_f64(method, tol):
    g, pb = make_case(vol_xyz=(48, 44, 40), det_wh=(72, 60), nviews=24, D=150.0, pw=0.9)
    vol = _phantom(pb)
    got = _proj(g, vol, method)
    ref64 = O.project_f64(pb, vol)
    assert O.rel_l2(got, ref64) < tol, O.rel_l2(got, ref64)


def test_texture_projector_vs_reference_path():
    g, pb = make_case(vol_xyz=(64, 64, 64), det_wh=(96, 64), nviews=18, D=250.0, pw=0.5)
    vol = _phantom(pb)
    got = _proj(g, vol, 0)
    refpath = O.ref_project(pb, vol, texq=1)
    assert O.rel_l2(got, refpath) < 1e-3


def test_project_subvolume_windows_misaligned():
    g, pb = make_case(vol_xyz=(40, 40, 40), vol_start=(4, 2, 6), vol_end=(36, 39, 33), det_wh=(64, 56),
                      nviews=11, window_wh=(44, 38), woff=np.arange(11) % 4 + 6, hoff=np.arange(11) % 3 + 5)
    vol = np.random.default_rng(4).random(g.vol_shape, dtype=np.float32)
    mis = np.array([0.8, -1.2, 2.0, 0.03, 0.01, -0.02], np.float32)
    import dataclasses

    gm = dataclasses.replace(g, misalignments=mis)
    got = _proj(gm, vol, 1)
    ref64 = O.project_f64(pb, vol, mis=mis)
    assert O.rel_l2(got, ref64) < 2e-5


def test_adjoint_dot_and_f64():
    import torch

    from fastcone_b200 import ops

    g, pb = make_case(vol_xyz=(40, 36, 32), det_wh=(56, 44), nviews=20, D=120.0, pw=0.8)
    rng = np.random.default_rng(7)
    x = rng.random(g.vol_shape, dtype=np.float32)
    y = rng.random(g.proj_shape, dtype=np.float32)
    Ax = ops.project(torch.from_numpy(x).cuda(), g, method=1).double()
    ATy = ops.project_adjoint(torch.from_numpy(y).cuda(), g).double()
    lhs = float((Ax * torch.from_numpy(y).cuda().double()).sum())
    rhs = float((torch.from_numpy(x).cuda().double() * ATy).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    ref = O.project_adjoint_f64(pb, y)
    assert O.rel_l2(ATy.cpu().numpy(), ref) < 2e-5


def test_projector_known_answer_ellipsoid():
    """Analytic line integrals of the continuous phantom vs the projector of its voxelisation
    (discretisation error only)."""
    from fastcone_b200.phantom import random_ellipsoids

    g, pb = make_case(vol_xyz=(96, 96, 96), det_wh=(128, 96), nviews=6, D=300.0, pw=0.9,
                      norm=np.ones(6, np.float32))
    params = random_ellipsoids(5, pb.volDim, 11, axes=(0.15, 0.4), centre_radius=0.45)
    vol = O.phantom_voxelize(pb.volDim, params)
    got = _proj(g, vol, 1)
    # analytic: ray from the source through pixel centres
    ana = np.zeros_like(got)
    for t in range(6):
        ca, sa = math.cos(float(pb.angles[t])), math.sin(float(pb.angles[t]))
        hmp = float(pb.hMid[t]) - 48
        S = np.array([-ca * pb.D, -sa * pb.D, hmp])
        for hh in range(0, 96, 3):
            for ww in range(0, 128, 3):
                P = np.array([-(ww - 64) * pb.pw * sa, (ww - 64) * pb.pw * ca, hmp + (hh - 48) * pb.pw])
                d = (P - S) / np.linalg.norm(P - S)
                ana[t, hh, ww] = O.phantom_line_integral(params, S, d)
    m = np.zeros_like(got, bool)
    m[:, ::3, ::3] = True
    # binary voxelisation error only: a few % per ray, no bias
    assert O.rel_l2(got[m], ana[m]) < 0.05
    assert abs(float(np.sum(got[m] - ana[m]))) / float(np.sum(ana[m])) < 0.01


def test_sample_counter_matches_oracle():
    import torch

    from fastcone_b200 import ops

    g, pb = make_case(vol_xyz=(40, 40, 40), det_wh=(64, 48), nviews=9, D=150.0)
    ctr = torch.zeros(1, dtype=torch.int64, device="cuda")
    ops.project(torch.zeros(g.vol_shape, device="cuda"), g, method=1, sample_counter=ctr)
    n_gpu = int(ctr.item())
    n_orc = O.projector_sample_count(pb)
    assert abs(n_gpu - n_orc) <= max(2, n_orc * 1e-5)


def test_reference_abi_project_zeroes_column0():
    from fastcone_b200 import fastcone as fc

    g, pb = make_case(vol_xyz=(40, 40, 40), det_wh=(56, 48), nviews=8, D=150.0, pw=0.8)
    vol = _phantom(pb)
    proj = np.full(pb.proj_shape, 0.5, np.float32)
    fc.project(vol, proj, pb.angles, pb.D, pb.hMid, norm=pb.norm, pixelWidth=pb.pw)
    # reference-compatible: the sub-problem windows of this geometry drop detector rows
    want = 0.5 + O.ref_project(pb, vol, texq=0)
    want[:, :, 0] = 0.0
    assert np.all(proj[:, :, 0] == 0.0)
    assert O.rel_l2(proj, want) < 1e-3


BRICK_CASES = {
    # name: make_case kwargs
    "cube64": dict(vol_xyz=(64, 64, 64), det_wh=(96, 64), nviews=24, D=200.0, pw=1.0),
    # views at and near 45 degrees: bundles switch dominant axis inside one view
    "diag": dict(vol_xyz=(48, 40, 36), det_wh=(80, 50), nviews=8, D=150.0, pw=0.9,
                 angles=np.deg2rad([45, 135, 225, 315, 44.5, 45.5, 0, 90]).astype(np.float32)),
    # sub-volume, window offsets, detector smaller than a bundle in h
    "windows": dict(vol_xyz=(64, 56, 40), det_wh=(80, 64), nviews=10, D=180.0, pw=0.7,
                    vol_start=(8, 4, 2), vol_end=(56, 52, 38), window_wh=(70, 6),
                    woff=np.arange(10) % 5 + 3, hoff=np.arange(10) % 4 + 20),
    # wide fan, strong magnification: large bricks, many samples near their edges
    "wide": dict(vol_xyz=(64, 64, 64), det_wh=(128, 96), nviews=6, D=60.0, pw=0.4),
    # rows not a multiple of 4 voxels: the unstaged kernel runs
    "odd": dict(vol_xyz=(45, 38, 30), det_wh=(64, 48), nviews=7, D=120.0, pw=0.75),
}


@pytest.mark.parametrize("name", sorted(BRICK_CASES))
def test_brick_projector_bitwise_equals_unstaged(name):
    """The TMA-brick projector takes the same samples with the same FP32 operations as the
    unstaged explicit kernel: identical results, identical sample counts; and the FP64
    oracle agrees."""
    import torch

    from fastcone_b200 import _lib, ops
    from fastcone_b200.phantom import random_ellipsoids

    g, pb = make_case(**BRICK_CASES[name])
    e, s = pb.volEnd, pb.volStart
    full = O.phantom_voxelize(pb.volDim, random_ellipsoids(8, pb.volDim, 11))
    vol = np.ascontiguousarray(full[s[2]:e[2], s[1]:e[1], s[0]:e[0]])
    vol += np.random.default_rng(5).normal(0, 0.01, vol.shape).astype(np.float32)
    v = torch.from_numpy(vol).cuda()
    c1 = torch.zeros(1, dtype=torch.int64, device="cuda")
    c2 = torch.zeros(1, dtype=torch.int64, device="cuda")
    a = ops.project(v, g, method=_lib.PROJ_EXPLICIT, sample_counter=c1)
    b = ops.project(v, g, method=_lib.PROJ_EXPLICIT_GLOBAL, sample_counter=c2)
    plan = ops.ProjectPlan(g, _lib.PROJ_EXPLICIT)
    c = plan(v)
    ops.sync_status()
    info = plan.info()
    if name == "odd":
        assert not info["staged"]
    elif name != "wide":
        assert info["staged"], info
    assert torch.equal(a, b)
    assert torch.equal(c, b)
    assert int(c1.item()) == int(c2.item())
    assert O.rel_l2(a.cpu().numpy(), O.project_f64(pb, vol)) < 2e-5


def test_brick_plan_adjoint_still_exact():
    """The plan's adjoint (unchanged scatter kernel) stays the transpose of the staged
    forward projector: dot-product test."""
    import torch

    from fastcone_b200 import _lib, ops

    g, pb = make_case(**BRICK_CASES["cube64"])
    plan = ops.ProjectPlan(g, _lib.PROJ_EXPLICIT)
    assert plan.info()["staged"]
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(g.vol_shape, device="cuda", generator=gen, dtype=torch.float32)
    y = torch.rand(g.proj_shape, device="cuda", generator=gen, dtype=torch.float32)
    ax = plan(x)
    aty = plan.adjoint(y)
    lhs = float(torch.sum(ax.double() * y.double()))
    rhs = float(torch.sum(x.double() * aty.double()))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


@pytest.mark.parametrize("name", sorted(BRICK_CASES))
def test_brick_adjoint_matches_direct_scatter(name):
    """A^T through shared-memory brick accumulation equals the direct scatter kernel up to
    the order of floating-point additions, and is the transpose of the staged forward
    projector (dot-product test)."""
    import torch

    from fastcone_b200 import _lib, ops

    g, pb = make_case(**BRICK_CASES[name])
    gen = torch.Generator(device="cuda").manual_seed(7)
    y = torch.rand(g.proj_shape, device="cuda", generator=gen, dtype=torch.float32)
    x = torch.rand(g.vol_shape, device="cuda", generator=gen, dtype=torch.float32)
    staged = ops.ProjectPlan(g, _lib.PROJ_EXPLICIT)
    direct = ops.ProjectPlan(g, _lib.PROJ_EXPLICIT_GLOBAL)
    a = staged.adjoint(y)
    b = direct.adjoint(y)
    c = ops.project_adjoint(y, g)
    ops.sync_status()
    rel = float((a - b).norm() / b.norm())
    assert rel < 2e-6, rel
    assert float((c - b).norm() / b.norm()) < 2e-6
    ax = staged(x)
    lhs = float(torch.sum(ax.double() * y.double()))
    rhs = float(torch.sum(x.double() * a.double()))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
