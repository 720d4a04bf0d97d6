"""Cone-beam geometry in the reference's units, and conversion from physical set-ups.

Units follow Fastcone (fastcone.py:52-74, coneBeamGPU.cu:1672-1700): lengths in voxels,
the rotation axis through voxel volDim/2 (integer division), a virtual detector through
the axis whose pixel pitch ``pw`` is the physical pitch demagnified to the axis
(pitch * SOD / SDD / voxel), detector pixel g centred at (g - W/2) * pw, the source of view t
at distance ``D`` = SOD / voxel from the axis at angle ``angles[t]`` and height
``hmid[t]`` (a z index counted from volume element 0).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
from typing import Optional

import numpy as np

from ._lib import FcbGeometry, arr_f32, arr_i32, c_float_p, c_int_p, ptr


@dataclasses.dataclass
class ConeGeometry:
    vol_xyz: tuple                 # (nx, ny, nz) of the whole volume grid (volDim)
    det_wh: tuple                  # (W, H) detector pixels
    angles: np.ndarray             # radians, one per view
    D: float                       # source-to-axis distance, voxels
    pw: float                      # detector pitch at the axis, voxels
    hmid: Optional[np.ndarray] = None   # per-view source z index (default volDim_z / 2)
    norm: Optional[np.ndarray] = None   # per-view normalisation (default 1)
    vol_start: tuple = (0, 0, 0)   # sub-volume handled (volStart..volEnd)
    vol_end: Optional[tuple] = None
    woff: Optional[np.ndarray] = None   # per-view window offsets (default 0)
    hoff: Optional[np.ndarray] = None
    window_wh: Optional[tuple] = None   # per-view window size (default det_wh)
    misalignments: Optional[np.ndarray] = None  # Dw, Dh, Dl (pixels), Dphi, Dtheta, Dpsi (rad)
    helical_pitch: float = 0.0     # source z advance per turn, voxels (Katsevich window)
    pi_window: bool = False
    reference_windows: bool = False  # reproduce the reference's sub-problem windows/sweeps

    def __post_init__(self):
        self.angles = arr_f32(self.angles)
        n = len(self.angles)
        if self.hmid is None:
            self.hmid = np.full(n, self.vol_xyz[2] / 2.0, np.float32)
        self.hmid = arr_f32(self.hmid)
        self.norm = arr_f32(np.ones(n) if self.norm is None else self.norm)
        self.woff = arr_i32(np.zeros(n) if self.woff is None else self.woff)
        self.hoff = arr_i32(np.zeros(n) if self.hoff is None else self.hoff)
        if self.vol_end is None:
            self.vol_end = tuple(self.vol_xyz)
        if self.window_wh is None:
            self.window_wh = tuple(self.det_wh)
        if self.misalignments is not None:
            self.misalignments = arr_f32(self.misalignments)
        for a in (self.hmid, self.norm, self.woff, self.hoff):
            if len(a) != n:
                raise ValueError("per-view arrays must have one entry per angle")

    # ------------------------------------------------------------------ shapes
    @property
    def nviews(self):
        return len(self.angles)

    @property
    def vol_shape(self):
        """(nz, ny, nx) of the sub-volume this geometry addresses."""
        s, e = self.vol_start, self.vol_end
        return (e[2] - s[2], e[1] - s[1], e[0] - s[0])

    @property
    def proj_shape(self):
        """(nviews, h, w) of the projection windows."""
        return (self.nviews, self.window_wh[1], self.window_wh[0])

    def with_norm(self, norm):
        return dataclasses.replace(self, norm=arr_f32(norm))

    # ------------------------------------------------------------------ ctypes
    def struct(self):
        """FcbGeometry for the C ABI; keep the returned object alive during the call."""
        g = FcbGeometry()
        for i in range(3):
            g.volDim[i] = int(self.vol_xyz[i])
            g.volStart[i] = int(self.vol_start[i])
            g.volEnd[i] = int(self.vol_end[i])
        g.projDim[0] = int(self.det_wh[0])
        g.projDim[1] = int(self.det_wh[1])
        g.projDim[2] = self.nviews
        g.projWHSize[0] = int(self.window_wh[0])
        g.projWHSize[1] = int(self.window_wh[1])
        g.projWOffset = ptr(self.woff, c_int_p)
        g.projHOffset = ptr(self.hoff, c_int_p)
        g.angles = ptr(self.angles, c_float_p)
        g.hMidPlane = ptr(self.hmid, c_float_p)
        g.sourceSampleDistance = float(self.D)
        g.pixelWidth = float(self.pw)
        g.normalizationFactor = ptr(self.norm, c_float_p)
        g.misAlignments = (ptr(self.misalignments, c_float_p) if self.misalignments is not None
                           else ctypes.cast(None, c_float_p))
        g.helicalPitch = float(self.helical_pitch)
        g.piWindow = 1 if self.pi_window else 0
        g.referenceWindows = 1 if self.reference_windows else 0
        g._keep = (self.woff, self.hoff, self.angles, self.hmid, self.norm, self.misalignments)
        return g

    # ------------------------------------------------------------------ constructors
    @classmethod
    def circular(cls, vol_xyz, voxel_mm, det_wh, pitch_mm, sod_mm, sdd_mm, nviews,
                 arc=2 * math.pi, **kw):
        """Circular trajectory from a physical description (mm)."""
        D = sod_mm / voxel_mm
        pw = pitch_mm * sod_mm / sdd_mm / voxel_mm
        angles = (np.arange(nviews, dtype=np.float64) * (arc / nviews)).astype(np.float32)
        return cls(tuple(vol_xyz), tuple(det_wh), angles, D, pw, **kw)

    @classmethod
    def helical(cls, vol_xyz, voxel_mm, det_wh, pitch_mm, radius_mm, sdd_mm, turns,
                views_per_turn, helix_pitch_mm, z_start=None, **kw):
        """Helical trajectory: the source rises helix_pitch_mm per turn.  The source z index
        starts at ``z_start`` (default: centred so the helix spans the volume midpoint)."""
        D = radius_mm / voxel_mm
        pw = pitch_mm * radius_mm / sdd_mm / voxel_mm
        n = turns * views_per_turn
        t = np.arange(n, dtype=np.float64)
        angles = (t * (2 * math.pi / views_per_turn)).astype(np.float32)
        P = helix_pitch_mm / voxel_mm
        dz = P / views_per_turn
        if z_start is None:
            z_start = vol_xyz[2] / 2.0 - 0.5 * (n - 1) * dz
        hmid = (z_start + t * dz).astype(np.float32)
        return cls(tuple(vol_xyz), tuple(det_wh), angles, D, pw, hmid=hmid, helical_pitch=P, **kw)
