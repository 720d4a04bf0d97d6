"""Differentiable cone-beam projector.

``ConeProject.apply(vol, geom)`` is the explicit-FP32 ray-driven projector A; its backward
is the hand-written exact transpose A^T (``project_adjoint_kernel``: the same sample
positions and trilinear weights, scattered).  A is linear, so nothing is saved for
backward except the geometry: batched volumes are projected, and their gradients
back-projected, one volume at a time and never stored twice.
"""
from __future__ import annotations

import torch

from . import _lib, ops
from .geometry import ConeGeometry


class ConeProject(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vol: torch.Tensor, geom: ConeGeometry):
        ctx.geom = geom
        vol = vol.contiguous()
        if vol.dim() == 3:
            return ops.project(vol, geom, method=_lib.PROJ_EXPLICIT)
        out = torch.zeros((vol.shape[0],) + geom.proj_shape, device=vol.device, dtype=torch.float32)
        for b in range(vol.shape[0]):
            ops.project(vol[b], geom, method=_lib.PROJ_EXPLICIT, proj=out[b])
        return out

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        geom = ctx.geom
        grad = grad.contiguous().float()
        if grad.dim() == 3:
            return ops.project_adjoint(grad, geom), None
        out = torch.zeros((grad.shape[0],) + geom.vol_shape, device=grad.device, dtype=torch.float32)
        for b in range(grad.shape[0]):
            ops.project_adjoint(grad[b], geom, vol=out[b])
        return out, None


class ConeBackprojectAdjoint(torch.autograd.Function):
    """A^T as a differentiable op (its backward is A), for data terms A^T(Ax - y)."""

    @staticmethod
    def forward(ctx, proj: torch.Tensor, geom: ConeGeometry):
        ctx.geom = geom
        return ConeProject.backward(_Ctx(geom), proj)[0]

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        return ConeProject.forward(_Ctx(ctx.geom), grad, ctx.geom), None


class _Ctx:
    def __init__(self, geom):
        self.geom = geom


def project(vol: torch.Tensor, geom: ConeGeometry) -> torch.Tensor:
    """Differentiable A vol for (nz, ny, nx) or batched (B, nz, ny, nx) volumes."""
    return ConeProject.apply(vol, geom)


def adjoint(proj: torch.Tensor, geom: ConeGeometry) -> torch.Tensor:
    """Differentiable A^T proj."""
    return ConeBackprojectAdjoint.apply(proj, geom)
