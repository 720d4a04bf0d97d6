"""The five workload configurations, as ConeGeometry constructors.

Parameters the workload descriptions leave open are fixed here once:
  * large circular FDK: source-axis / source-detector distances 500 / 1000 mm (those of the
    small configuration) -> D = 2000 voxels, pw = 0.8 voxel;
  * differentiable batch and learned reconstruction (256^3, 384 x 256 detector): voxel
    0.5 mm, pitch 1.0 mm, 500 / 1000 mm -> D = 1000 voxels, pw = 1.0 voxel, so the
    magnified detector (384 x 256 voxels at the axis) covers the volume's 362-voxel
    diagonal in-plane and its full height;
  * helical: 4 turns x 1160 views, pitch 40 mm = 80 voxels per turn, the source rising
    through the volume centre.
"""
from __future__ import annotations

import math

import numpy as np

from .geometry import ConeGeometry


def small_fdk() -> ConeGeometry:
    """128^3 x 1.0 mm, 192x128 detector at 1.0 mm, 500/1000 mm, 180 views over 360 deg."""
    return ConeGeometry.circular((128, 128, 128), 1.0, (192, 128), 1.0, 500.0, 1000.0, 180)


def large_fdk() -> ConeGeometry:
    """1024^3 x 0.25 mm, 1536x1024 detector at 0.4 mm, 1440 views over 360 deg."""
    return ConeGeometry.circular((1024, 1024, 1024), 0.25, (1536, 1024), 0.4, 500.0, 1000.0, 1440)


def helical_katsevich(pi_window: bool = True) -> ConeGeometry:
    """512x512x384 x 0.5 mm, helix radius 570 mm, SDD 1040 mm, pitch 40 mm/turn, 4 turns x
    1160 views, 736x64 detector at 1.0 mm."""
    return ConeGeometry.helical((512, 512, 384), 0.5, (736, 64), 1.0, 570.0, 1040.0, 4, 1160, 40.0,
                                pi_window=pi_window)


def diff_batch(nviews: int = 360) -> ConeGeometry:
    """256^3 x 0.5 mm, 384x256 detector at 1.0 mm, 500/1000 mm, views over 360 deg."""
    return ConeGeometry.circular((256, 256, 256), 0.5, (384, 256), 1.0, 500.0, 1000.0, nviews)


def learned_sparse() -> ConeGeometry:
    """The learned-reconstruction geometry: diff_batch with 90 sparse views."""
    return diff_batch(90)


def with_fdk_norm(g: ConeGeometry) -> ConeGeometry:
    """norm = 1 / nviews, the reference's backprojection default (fastcone.py:190-191)."""
    return g.with_norm(np.full(g.nviews, 1.0 / g.nviews, np.float32))
