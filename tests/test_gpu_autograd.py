"""Differentiable projector: the matched adjoint through torch.autograd.

Small case: the gradient of ||Ax - y||^2 vs the FP64 oracle gradient 2 A^T (Ax - y)
(rel-L2 <= 1e-4).  Differentiable-batch configuration (8 x 256^3 ellipsoid phantoms plus
N(0, 0.01) texture, 360 views, 384 x 256 detector): dot-product test to 1e-5 relative and
central finite differences (eps = 1e-3) on 64 random voxels (FP32 projections bound the
finite-difference accuracy at ~1e-2 relative).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import make_case

pytestmark = pytest.mark.gpu


def test_gradient_vs_fp64_oracle():
    import torch

    from fastcone_b200 import autograd

    g, pb = make_case(vol_xyz=(40, 36, 32), det_wh=(56, 44), nviews=24, D=120.0, pw=0.8)
    rng = np.random.default_rng(3)
    x = rng.random(g.vol_shape, dtype=np.float32)
    y = rng.random(g.proj_shape, dtype=np.float32) * 10
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    loss = ((autograd.project(xt, g) - torch.from_numpy(y).cuda()) ** 2).sum()
    loss.backward()
    r64 = O.project_f64(pb, x) - y
    g64 = 2.0 * O.project_adjoint_f64(pb, r64.astype(np.float32))
    assert O.rel_l2(xt.grad.cpu().numpy(), g64) < 1e-4


def _cfg4():
    from fastcone_b200 import configs

    return configs.diff_batch()


def _batch(B=8, seed=0):
    import torch

    from fastcone_b200 import ops
    from fastcone_b200.phantom import random_ellipsoids

    g = _cfg4()
    gen = torch.Generator(device="cuda").manual_seed(seed)
    vols = torch.empty((B,) + g.vol_shape, device="cuda")
    for b in range(B):
        ops.phantom(g.vol_xyz, random_ellipsoids(10, g.vol_xyz, seed + b), out=vols[b])
        vols[b] += 0.01 * torch.randn(g.vol_shape, device="cuda", generator=gen)
    return g, vols


def test_dot_product_batch():
    import torch

    from fastcone_b200 import autograd

    g, x = _batch()
    y = torch.rand((x.shape[0],) + g.proj_shape, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    Ax = autograd.project(x, g)
    ATy = autograd.adjoint(y, g)
    lhs = float((Ax.double() * y.double()).sum())
    rhs = float((x.double() * ATy.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-5


def test_finite_differences_batch():
    import torch

    from fastcone_b200 import autograd, ops, _lib

    g, x0 = _batch(seed=10)
    B = x0.shape[0]
    with torch.no_grad():
        y = autograd.project(x0, g) + 0.5 * torch.randn((B,) + g.proj_shape, device="cuda",
                                                       generator=torch.Generator(device="cuda").manual_seed(2))
    x = x0.clone().requires_grad_(True)
    loss = ((autograd.project(x, g) - y) ** 2).double().sum()
    loss.backward()
    grad = x.grad
    rng = np.random.default_rng(0)
    eps = 1e-3
    fd, an = [], []
    nz, ny, nx = g.vol_shape
    for _ in range(64):
        b, k, j, i = int(rng.integers(B)), int(rng.integers(nz // 4, 3 * nz // 4)), \
            int(rng.integers(ny // 4, 3 * ny // 4)), int(rng.integers(nx // 4, 3 * nx // 4))
        vals = []
        for s in (+1, -1):
            xb = x0[b].clone()
            xb[k, j, i] += s * eps
            p = ops.project(xb, g, method=_lib.PROJ_EXPLICIT)
            vals.append(float(((p - y[b]).double() ** 2).sum()))
        fd.append((vals[0] - vals[1]) / (2 * eps))
        an.append(float(grad[b, k, j, i]))
    fd, an = np.array(fd), np.array(an)
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 2e-2
