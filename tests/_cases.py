"""Shared problem builders: the same geometry as an oracle.Problem (ABI arrays) and as a
fastcone_b200.ConeGeometry, plus seeded inputs."""
from __future__ import annotations

import math

import numpy as np

from oracle import oracle as O


def make_case(vol_xyz=(48, 40, 36), det_wh=(64, 48), nviews=45, D=120.0, pw=0.75, arc=2 * math.pi,
              vol_start=(0, 0, 0), vol_end=None, woff=None, hoff=None, window_wh=None, hmid=None,
              norm=None, seed=0, angles=None):
    from fastcone_b200.geometry import ConeGeometry

    rng = np.random.default_rng(seed)
    if angles is None:
        angles = (np.arange(nviews) * (arc / nviews)).astype(np.float32)
    if hmid is None:
        hmid = np.full(nviews, vol_xyz[2] / 2.0, np.float32)
    if norm is None:
        norm = (1.0 + 0.1 * rng.random(nviews)).astype(np.float32)
    g = ConeGeometry(tuple(vol_xyz), tuple(det_wh), angles, D, pw, hmid=hmid, norm=norm,
                     vol_start=tuple(vol_start), vol_end=None if vol_end is None else tuple(vol_end),
                     woff=woff, hoff=hoff, window_wh=window_wh)
    pb = O.Problem(volDim=O._i3(vol_xyz), volStart=O._i3(g.vol_start), volEnd=O._i3(g.vol_end),
                   projDim=O._i3([det_wh[0], det_wh[1], nviews]), projWHSize=O._i3(g.window_wh),
                   projWOffset=O._i3(g.woff), projHOffset=O._i3(g.hoff), angles=g.angles, hMid=g.hmid,
                   D=float(D), pw=float(pw), norm=g.norm)
    return g, pb


def smooth_projections(pb, seed=1):
    """Projections of a random ellipsoid phantom (smooth, realistic data)."""
    from fastcone_b200.phantom import random_ellipsoids

    vol = O.phantom_voxelize(pb.volDim, random_ellipsoids(6, pb.volDim, seed))
    full = O.make_problem(pb.volDim, (int(pb.projDim[0]), int(pb.projDim[1])), int(pb.projDim[2]),
                          D=pb.D, pw=pb.pw, hmid=pb.hMid, angles=pb.angles, norm=np.ones_like(pb.norm),
                          woff=pb.projWOffset, hoff=pb.projHOffset, whsize=pb.projWHSize)
    return O.project_f64(full, vol).astype(np.float32), vol
