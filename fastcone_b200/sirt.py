"""SIRT on the GPU operators.

    x <- x + C * B(R * (y - A x)),   R = 1 / (A 1),   C = 1 / (B 1)

A is the explicit-FP32 ray-driven projector.  B is either its exact transpose
(``backprojector="adjoint"``) or the voxel-driven unweighted backprojector the reference
recommends for iterative reconstruction (kernelMode 0, fastcone.py:166;
``backprojector="voxel"``, the faster one).  Per-ray and per-voxel normalisations are
computed once.  Nothing is stored per iteration.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from . import _lib, ops
from .geometry import ConeGeometry


class SIRT:
    def __init__(self, geom: ConeGeometry, backprojector: str = "voxel", nonneg: bool = True):
        self.g = dataclasses.replace(geom, norm=np.ones(geom.nviews, np.float32))
        self.kind = backprojector
        self.nonneg = nonneg
        self.plan = (ops.BackprojectPlan(self.g, mode=_lib.MODE_UNWEIGHTED)
                     if backprojector == "voxel" else None)
        dev = torch.device("cuda", torch.cuda.current_device())
        ones_v = torch.ones(self.g.vol_shape, device=dev)
        ones_p = torch.ones(self.g.proj_shape, device=dev)
        self.R = self._safe_inv(self.A(ones_v))
        self.C = self._safe_inv(self.B(ones_p))

    @staticmethod
    def _safe_inv(t, eps=1e-6):
        return torch.where(t > eps, 1.0 / t.clamp_min(eps), torch.zeros_like(t))

    def A(self, x):
        return ops.project(x, self.g, method=_lib.PROJ_EXPLICIT)

    def B(self, p):
        if self.kind == "voxel":
            v = torch.zeros(self.g.vol_shape, device=p.device)
            return self.plan(p.contiguous(), v)
        return ops.project_adjoint(p.contiguous(), self.g)

    def step(self, x, y):
        r = (y - self.A(x)) * self.R
        x = x + self.C * self.B(r)
        if self.nonneg:
            x.clamp_(min=0.0)
        return x

    def run(self, y, iters=100, x0=None, callback=None):
        x = torch.zeros(self.g.vol_shape, device=y.device) if x0 is None else x0.clone()
        for k in range(iters):
            x = self.step(x, y)
            if callback is not None:
                callback(k, x)
        return x


def sirt(y, geom, iters=100, backprojector="voxel", x0=None, nonneg=True, callback=None):
    return SIRT(geom, backprojector, nonneg).run(y, iters, x0, callback)
