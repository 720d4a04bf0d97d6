"""CPU oracle for the Fastcone operators -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module, as the checker (or the timed CPU baseline); the product package never does.

Contents
  * ctypes bindings of ``liborc.so`` (fc_oracle.c): the reference-path restatement
    (``ref_*``: FP32, tiling, windows, texture emulation) and the FP64 oracle (``*_f64``);
  * ctypes bindings of the reference's own host code built from its sources
    (``oracle/_ref/libfastcone_ref.so``, see Makefile) -- used to pin the restatement;
  * numpy restatements of the Python-layer pre-processing of fastcone.py
    (``rampfilter`` fastcone.py:272-292, the ``fbp`` cosine weight fastcone.py:260-270)
    and of the Shepp-Logan variant this project adds.

All ABI-level arrays follow the reference C ABI (wrapper.c:112-249): dimensions in
[x, y, z] / [w, h, t] order, volumes x-fastest, projections [t][h][w].
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REFLIB = None

_i32p = ctypes.POINTER(ctypes.c_int)
_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liborc.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liborc.so is not built (make -C oracle)")
        _LIB = ctypes.CDLL(path)
        _LIB.orc_projector_sample_count.restype = ctypes.c_int64
        _LIB.orc_phantom_line_integral.restype = ctypes.c_double
    return _LIB


def reflib():
    """The reference's own code (oracle/_ref), or None when it was not built."""
    global _REFLIB
    if _REFLIB is None:
        path = os.path.join(_HERE, "_ref", "libfastcone_ref.so")
        if not os.path.exists(path):
            return None
        _REFLIB = ctypes.CDLL(path)
    return _REFLIB


def _p(a, kind):
    return a.ctypes.data_as(kind)


def _i3(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


@dataclasses.dataclass
class Problem:
    """One call's worth of ABI arguments (reference units: voxels / detector pixels)."""
    volDim: np.ndarray          # [x, y, z] of the whole volume
    volStart: np.ndarray        # sub-volume handled by this call
    volEnd: np.ndarray
    projDim: np.ndarray         # [W, H, nviews]
    projWHSize: np.ndarray      # [w, h] of each view's data window
    projWOffset: np.ndarray     # per view
    projHOffset: np.ndarray
    angles: np.ndarray          # float32 radians
    hMid: np.ndarray            # float32, source z index from volume element 0
    D: float                    # source-to-axis distance, voxels
    pw: float                   # detector pixel pitch at the axis, voxels
    norm: np.ndarray            # float32 per view

    @property
    def vol_shape_zyx(self):
        e, s = self.volEnd, self.volStart
        return (int(e[2] - s[2]), int(e[1] - s[1]), int(e[0] - s[0]))

    @property
    def proj_shape(self):
        return (int(self.projDim[2]), int(self.projWHSize[1]), int(self.projWHSize[0]))

    def args(self):
        return (_p(self.volDim, _i32p), _p(self.volStart, _i32p), _p(self.volEnd, _i32p),
                _p(self.projDim, _i32p), _p(self.projWHSize, _i32p),
                _p(self.projWOffset, _i32p), _p(self.projHOffset, _i32p),
                _p(self.angles, _f32p), _p(self.hMid, _f32p))


def make_problem(vol_xyz, det_wh, nviews, D, pw, hmid=None, angles=None, norm=None,
                 volStart=(0, 0, 0), volEnd=None, woff=None, hoff=None, whsize=None,
                 arc=2 * math.pi):
    vol_xyz = _i3(vol_xyz)
    volStart = _i3(volStart)
    volEnd = _i3(vol_xyz if volEnd is None else volEnd)
    if angles is None:
        angles = (np.arange(nviews, dtype=np.float64) * (arc / nviews)).astype(np.float32)
    if hmid is None:
        hmid = np.full(nviews, float(vol_xyz[2]) / 2.0, dtype=np.float32)
    if norm is None:
        norm = np.ones(nviews, dtype=np.float32)
    whsize = _i3(det_wh if whsize is None else whsize)
    return Problem(
        volDim=vol_xyz, volStart=volStart, volEnd=volEnd,
        projDim=_i3([det_wh[0], det_wh[1], nviews]), projWHSize=whsize,
        projWOffset=_i3(np.zeros(nviews) if woff is None else woff),
        projHOffset=_i3(np.zeros(nviews) if hoff is None else hoff),
        angles=np.ascontiguousarray(angles, dtype=np.float32),
        hMid=np.ascontiguousarray(hmid, dtype=np.float32),
        D=float(D), pw=float(pw), norm=np.ascontiguousarray(norm, dtype=np.float32))


# ---------------------------------------------------------------- reference path (FP32)

def ref_backproject(pb: Problem, proj, kernel_mode=2, texq=1, mis=None, vol=None):
    """Reference-path backprojection (coneBeamBackproject / RayTrace, texture-emulated).
    Returns vol (z, y, x) float32 with the result ADDED."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    if vol is None:
        vol = np.zeros(pb.vol_shape_zyx, dtype=np.float32)
    misp = None if mis is None else _p(np.ascontiguousarray(mis, dtype=np.float32), _f32p)
    rc = lib().orc_ref_backproject(_p(vol, _f32p), _p(proj, _f32p), *pb.args()[:7],
                                   _p(pb.angles, _f32p), _p(pb.hMid, _f32p), ctypes.c_float(pb.D),
                                   _p(pb.norm, _f32p), ctypes.c_float(pb.pw), ctypes.c_int(kernel_mode),
                                   misp, ctypes.c_int(texq))
    assert rc == 0
    return vol


def ref_project(pb: Problem, vol, texq=1, mis=None, proj=None):
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    if proj is None:
        proj = np.zeros(pb.proj_shape, dtype=np.float32)
    misp = None if mis is None else _p(np.ascontiguousarray(mis, dtype=np.float32), _f32p)
    rc = lib().orc_ref_project(_p(vol, _f32p), _p(proj, _f32p), *pb.args()[:7],
                               _p(pb.angles, _f32p), _p(pb.hMid, _f32p), ctypes.c_float(pb.D),
                               _p(pb.norm, _f32p), misp, ctypes.c_float(pb.pw), ctypes.c_int(texq))
    assert rc == 0
    return proj


def ref_backproject_points(pb: Problem, proj, pts, kernel_mode=2, texq=1):
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    pts = np.ascontiguousarray(pts, dtype=np.int32)
    out = np.zeros(len(pts), dtype=np.float32)
    rc = lib().orc_ref_backproject_points(_p(pts, _i32p), ctypes.c_int(len(pts)), _p(out, _f32p),
                                          _p(proj, _f32p), *pb.args()[:7], _p(pb.angles, _f32p),
                                          _p(pb.hMid, _f32p), ctypes.c_float(pb.D), _p(pb.norm, _f32p),
                                          ctypes.c_float(pb.pw), ctypes.c_int(kernel_mode),
                                          ctypes.c_int(texq))
    assert rc == 0
    return out


class _TilingInfo(ctypes.Structure):
    _fields_ = [("subVolDim", ctypes.c_int * 3), ("subProjDim", ctypes.c_int * 3),
                ("numSubProblems", ctypes.c_int), ("nsp", ctypes.c_int)]


def ref_geometry(pb: Problem, mis=None):
    """The restated coneBeamGeometry: dict of tiling sizes, windows, sweeps, vectors."""
    info = _TilingInfo()
    misp = None if mis is None else _p(np.ascontiguousarray(mis, dtype=np.float32), _f32p)
    args = (*pb.args()[:7], _p(pb.angles, _f32p), _p(pb.hMid, _f32p), ctypes.c_float(pb.D), misp,
            ctypes.c_float(pb.pw))
    rc = lib().orc_ref_geometry(*args, ctypes.byref(info), *([None] * 15))
    assert rc == 0
    ns, n2 = info.numSubProblems, info.subProjDim[2]
    npad = info.nsp * n2
    out = {k: np.zeros(ns, np.int32) for k in ("xxStart", "yyStart", "zzStart", "ttStart")}
    for k in ("wwStart", "hhStart", "sweepStart", "sweepNumSteps"):
        out[k] = np.zeros(ns * n2, np.int32)
    for k in ("src", "det", "hstep", "wstep"):
        out[k] = np.zeros(3 * npad, np.float32)
    for k in ("hMidPlane", "sina", "cosa"):
        out[k] = np.zeros(npad, np.float32)
    order = ["xxStart", "yyStart", "zzStart", "ttStart", "wwStart", "hhStart", "sweepStart",
             "sweepNumSteps", "src", "det", "hstep", "wstep", "hMidPlane", "sina", "cosa"]
    ptrs = [_p(out[k], _i32p if out[k].dtype == np.int32 else _f32p) for k in order]
    rc = lib().orc_ref_geometry(*args, ctypes.byref(info), *ptrs)
    assert rc == 0
    out["subVolDim"] = np.array(info.subVolDim[:], np.int32)
    out["subProjDim"] = np.array(info.subProjDim[:], np.int32)
    out["numSubProblems"] = ns
    return out


def reflib_geometry(pb: Problem, mis=None):
    """The same quantities from the reference's OWN coneBeamGeometry (oracle/_ref)."""
    rl = reflib()
    if rl is None:
        return None
    mine = ref_geometry(pb, mis)
    ns, n2 = mine["numSubProblems"], int(mine["subProjDim"][2])
    npad = len(mine["hMidPlane"])
    sizes = np.zeros(7, np.int32)
    out = {k: np.zeros(ns, np.int32) for k in ("xxStart", "yyStart", "zzStart", "ttStart")}
    for k in ("wwStart", "hhStart", "sweepStart", "sweepNumSteps"):
        out[k] = np.zeros(ns * n2, np.int32)
    for k in ("src", "det", "hstep", "wstep"):
        out[k] = np.zeros(3 * npad, np.float32)
    for k in ("hMidPlane", "sina", "cosa"):
        out[k] = np.zeros(npad, np.float32)
    order = ["xxStart", "yyStart", "zzStart", "ttStart", "wwStart", "hhStart", "sweepStart",
             "sweepNumSteps", "src", "det", "hstep", "wstep", "hMidPlane", "sina", "cosa"]
    ptrs = [_p(out[k], _i32p if out[k].dtype == np.int32 else _f32p) for k in order]
    # the reference takes non-const pointers; pass copies
    c = {k: np.array(getattr(pb, k), copy=True) for k in
         ("volDim", "volStart", "volEnd", "projDim", "projWHSize", "projWOffset", "projHOffset",
          "angles", "hMid")}
    misa = np.zeros(6, np.float32) if mis is None else np.array(mis, np.float32)
    rc = rl.fcref_geometry(_p(c["volDim"], _i32p), _p(c["volStart"], _i32p), _p(c["volEnd"], _i32p),
                           _p(c["projDim"], _i32p), _p(c["projWHSize"], _i32p),
                           _p(c["projWOffset"], _i32p), _p(c["projHOffset"], _i32p),
                           _p(c["angles"], _f32p), _p(c["hMid"], _f32p), ctypes.c_float(pb.D),
                           _p(misa, _f32p), ctypes.c_float(pb.pw), _p(sizes, _i32p), *ptrs,
                           ctypes.c_int(ns), ctypes.c_int(npad))
    assert rc == 0
    out["subVolDim"] = sizes[:3].copy()
    out["subProjDim"] = sizes[3:6].copy()
    out["numSubProblems"] = int(sizes[6])
    return out


def reflib_backproject(pb: Problem, proj, kernel_mode=2, vol=None):
    """The reference's own CUDA path (needs a GPU): returns vol with the result added."""
    rl = reflib()
    proj = np.array(proj, dtype=np.float32, copy=True)
    if vol is None:
        vol = np.zeros(pb.vol_shape_zyx, dtype=np.float32)
    c = {k: np.array(getattr(pb, k), copy=True) for k in
         ("volDim", "volStart", "volEnd", "projDim", "projWHSize", "projWOffset", "projHOffset",
          "angles", "hMid", "norm")}
    rc = rl.fcref_backproject(_p(vol, _f32p), _p(proj, _f32p), _p(c["angles"], _f32p),
                              _p(c["hMid"], _f32p), ctypes.c_float(pb.D), ctypes.c_float(pb.pw),
                              _p(c["volDim"], _i32p), _p(c["volStart"], _i32p), _p(c["volEnd"], _i32p),
                              _p(c["projDim"], _i32p), _p(c["projWHSize"], _i32p),
                              _p(c["projWOffset"], _i32p), _p(c["projHOffset"], _i32p),
                              _p(c["norm"], _f32p), ctypes.c_int(kernel_mode))
    if rc < 0:
        raise RuntimeError(f"reference backproject failed: cuda error {-rc}")
    return vol


def reflib_project(pb: Problem, vol, proj=None, mis=None):
    rl = reflib()
    vol = np.array(vol, dtype=np.float32, copy=True)
    if proj is None:
        proj = np.zeros(pb.proj_shape, dtype=np.float32)
    c = {k: np.array(getattr(pb, k), copy=True) for k in
         ("volDim", "volStart", "volEnd", "projDim", "projWHSize", "projWOffset", "projHOffset",
          "angles", "hMid", "norm")}
    misa = np.zeros(6, np.float32) if mis is None else np.array(mis, np.float32)
    rc = rl.fcref_project(_p(vol, _f32p), _p(proj, _f32p), _p(c["angles"], _f32p), _p(c["hMid"], _f32p),
                          ctypes.c_float(pb.D), ctypes.c_float(pb.pw), _p(c["volDim"], _i32p),
                          _p(c["volStart"], _i32p), _p(c["volEnd"], _i32p), _p(c["projDim"], _i32p),
                          _p(c["projWHSize"], _i32p), _p(c["projWOffset"], _i32p),
                          _p(c["projHOffset"], _i32p), _p(c["norm"], _f32p), _p(misa, _f32p))
    if rc < 0:
        raise RuntimeError(f"reference project failed: cuda error {-rc}")
    return proj


# ---------------------------------------------------------------- FP64 oracle

def backproject_f64(pb: Problem, proj, kernel_mode=2, mis=None):
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    vol = np.zeros(pb.vol_shape_zyx, dtype=np.float64)
    misp = None if mis is None else _p(np.ascontiguousarray(mis, dtype=np.float32), _f32p)
    rc = lib().orc_backproject_f64(_p(vol, _f64p), _p(proj, _f32p), *pb.args()[:7],
                                   _p(pb.angles, _f32p), _p(pb.hMid, _f32p), ctypes.c_double(pb.D),
                                   _p(pb.norm, _f32p), ctypes.c_double(pb.pw),
                                   ctypes.c_int(kernel_mode), misp)
    assert rc == 0
    return vol


def katsevich_piwin_f64(pb: Problem, proj, pitch):
    """Katsevich backprojection (weight U) over each voxel's PI interval, FP64; returns
    (volume, number of voxel-view pairs inside the window)."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    vol = np.zeros(pb.vol_shape_zyx, dtype=np.float64)
    pairs = ctypes.c_int64(0)
    rc = lib().orc_katsevich_piwin_f64(_p(vol, _f64p), _p(proj, _f32p), *pb.args()[:7],
                                       _p(pb.angles, _f32p), _p(pb.hMid, _f32p), ctypes.c_double(pb.D),
                                       _p(pb.norm, _f32p), ctypes.c_double(pb.pw), ctypes.c_double(pitch),
                                       ctypes.byref(pairs))
    assert rc == 0
    return vol, int(pairs.value)


def katsevich_piwin_points_f64(pb: Problem, proj, pts, pitch):
    """katsevich_piwin_f64 at listed voxels (rows of global [x, y, z] indices); returns
    (values, number of voxel-view pairs of those voxels inside the window)."""
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    pts = np.ascontiguousarray(pts, dtype=np.int32)
    out = np.zeros(len(pts), dtype=np.float64)
    pairs = ctypes.c_int64(0)
    rc = lib().orc_katsevich_piwin_points_f64(_p(pts, _i32p), ctypes.c_int(len(pts)), _p(out, _f64p),
                                              _p(proj, _f32p), _p(pb.volDim, _i32p), _p(pb.projDim, _i32p),
                                              _p(pb.projWHSize, _i32p), _p(pb.projWOffset, _i32p),
                                              _p(pb.projHOffset, _i32p), _p(pb.angles, _f32p),
                                              _p(pb.hMid, _f32p), ctypes.c_double(pb.D), _p(pb.norm, _f32p),
                                              ctypes.c_double(pb.pw), ctypes.c_double(pitch),
                                              ctypes.byref(pairs))
    assert rc == 0
    return out, int(pairs.value)


def column_points(vol_xyz, vol_start, vol_end, ncols, seed=0):
    """`ncols` random full-z voxel columns of the sub-volume vol_start..vol_end: rows of
    global [x, y, z] indices, column-major (all z of column 0 first)."""
    rng = np.random.default_rng(seed)
    x = rng.integers(vol_start[0], vol_end[0], ncols)
    y = rng.integers(vol_start[1], vol_end[1], ncols)
    z = np.arange(vol_start[2], vol_end[2])
    nz = len(z)
    return np.stack([np.repeat(x, nz), np.repeat(y, nz), np.tile(z, ncols)], 1).astype(np.int32)


def backproject_points_f64(pb: Problem, proj, pts, kernel_mode=2):
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    pts = np.ascontiguousarray(pts, dtype=np.int32)
    out = np.zeros(len(pts), dtype=np.float64)
    rc = lib().orc_backproject_points_f64(_p(pts, _i32p), ctypes.c_int(len(pts)), _p(out, _f64p),
                                          _p(proj, _f32p), *pb.args()[:7], _p(pb.angles, _f32p),
                                          _p(pb.hMid, _f32p), ctypes.c_double(pb.D), _p(pb.norm, _f32p),
                                          ctypes.c_double(pb.pw), ctypes.c_int(kernel_mode))
    assert rc == 0
    return out


def project_f64(pb: Problem, vol, mis=None):
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    proj = np.zeros(pb.proj_shape, dtype=np.float64)
    misp = None if mis is None else _p(np.ascontiguousarray(mis, dtype=np.float32), _f32p)
    rc = lib().orc_project_f64(_p(vol, _f32p), _p(proj, _f64p), *pb.args()[:7], _p(pb.angles, _f32p),
                               _p(pb.hMid, _f32p), ctypes.c_double(pb.D), _p(pb.norm, _f32p), misp,
                               ctypes.c_double(pb.pw))
    assert rc == 0
    return proj


def project_adjoint_f64(pb: Problem, proj, mis=None):
    proj = np.ascontiguousarray(proj, dtype=np.float32)
    vol = np.zeros(pb.vol_shape_zyx, dtype=np.float64)
    misp = None if mis is None else _p(np.ascontiguousarray(mis, dtype=np.float32), _f32p)
    rc = lib().orc_project_adjoint_f64(_p(vol, _f64p), _p(proj, _f32p), *pb.args()[:7],
                                       _p(pb.angles, _f32p), _p(pb.hMid, _f32p), ctypes.c_double(pb.D),
                                       _p(pb.norm, _f32p), misp, ctypes.c_double(pb.pw))
    assert rc == 0
    return vol


def projector_sample_count(pb: Problem):
    return int(lib().orc_projector_sample_count(*pb.args()[:7], _p(pb.angles, _f32p),
                                                _p(pb.hMid, _f32p), ctypes.c_double(pb.D),
                                                ctypes.c_double(pb.pw)))


def phantom_voxelize(vol_xyz, params):
    vol_xyz = _i3(vol_xyz)
    params = np.ascontiguousarray(params, dtype=np.float64)
    vol = np.zeros((int(vol_xyz[2]), int(vol_xyz[1]), int(vol_xyz[0])), dtype=np.float32)
    lib().orc_phantom_voxelize(_p(vol, _f32p), _p(vol_xyz, _i32p), _p(params, _f64p),
                               ctypes.c_int(len(params)))
    return vol


def phantom_line_integral(params, p0, d):
    params = np.ascontiguousarray(params, dtype=np.float64)
    p0 = np.ascontiguousarray(p0, dtype=np.float64)
    d = np.ascontiguousarray(d, dtype=np.float64)
    return float(lib().orc_phantom_line_integral(_p(params, _f64p), ctypes.c_int(len(params)),
                                                 _p(p0, _f64p), _p(d, _f64p)))


# ---------------------------------------------------------------- Python-layer pre-processing

def rampfilter(proj, window="ramlak"):
    """fastcone.rampfilter (fastcone.py:272-292), restated for numpy >= 1.12: zero-pad each
    row to 2W (data at [0, W), not centred), multiply the rfft by pi*|fftfreq(2W)| with the
    DC bin set to 1/8 of the first bin, irfft, keep [0, W).  ``window='shepplogan'``
    additionally multiplies by sinc(fftfreq) (this project's Shepp-Logan)."""
    proj = np.asarray(proj)
    n, h, w = proj.shape
    filt = ramp_filter_response(w, window)
    out = np.empty_like(proj)
    for t in range(n):
        padded = np.zeros((h, 2 * w))
        padded[:, :w] = proj[t]
        spec = np.fft.rfft(padded, axis=1) * filt
        out[t] = np.fft.irfft(spec, axis=1)[:, :w]
    return out


def ramp_filter_response(w, window="ramlak"):
    f = np.abs(np.fft.fftfreq(2 * w))
    f[0] = 0.125 * f[1]
    if window == "shepplogan":
        f = f * np.sinc(np.fft.fftfreq(2 * w))
    elif window != "ramlak":
        raise ValueError(window)
    f = f * np.pi
    return f[: w + 1]


def apodised_ramp_response(w, window="cosramp", scale=0.125):
    """Response of fastcone.cosrampfilter / gaussrampfilter (fastcone.py:294-319) on the
    w//2 + 1 bins of an unpadded length-w rfft: a_k = |fftfreq(w)[k]| = k/w, times
    cos(0.5 a_k pi / w) (cosine, as written there), or times the Gaussian window of
    sigma = scale*w centred at (w-1)/2 and shifted by -w/2 samples with zeros beyond the
    last sample (scipy.ndimage.shift of scipy.signal gaussian; for an even w the shift is a
    whole number of samples and this is that window exactly; for an odd w the reference
    raises before filtering, and the Gaussian is sampled at the shifted position)."""
    k = np.arange(w // 2 + 1, dtype=np.float64)
    a = k / w
    if window == "cosramp":
        return a * np.cos(0.5 * a * np.pi / w)
    if window == "gaussramp":
        g = np.exp(-0.5 * ((k + 0.5) / (scale * w)) ** 2)
        return a * np.where(k + 0.5 * w <= w - 1, g, 0.0)
    raise ValueError(window)


def apodised_rampfilter(proj, window="cosramp", scale=0.125):
    """fastcone.cosrampfilter / gaussrampfilter (fastcone.py:294-319) applied to every view
    (the reference's store sits after its loop, so it writes only the last view) with an
    inverse transform of length w (numpy's default length, 2*(w//2), is w - 1 for odd w)."""
    proj = np.asarray(proj)
    n, h, w = proj.shape
    filt = apodised_ramp_response(w, window, scale)
    out = np.empty_like(proj)
    for t in range(n):
        out[t] = np.fft.irfft(np.fft.rfft(proj[t], axis=1) * filt, n=w, axis=1)
    return out


def fbp_cosine_weight(proj, D, zOrigin):
    """Cosine pre-weight of fastcone.fbp (fastcone.py:261-267): D / sqrt(D^2 + h^2 + w^2)
    with h measured from zOrigin[t] and w from W/2, both in detector pixels."""
    proj = np.asarray(proj)
    n, H, W = proj.shape
    ww = (np.arange(0.0, W, 1.0) - W / 2.0)[None, :]
    out = np.empty_like(proj)
    for t in range(n):
        hh = (np.arange(0.0, H, 1.0) - float(zOrigin[t]))[:, None]
        out[t] = proj[t] * (D / np.sqrt(D * D + hh * hh + ww * ww))
    return out


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))


# ---------------------------------------------------------------- Katsevich filtering (FP64)

def katsevich_filter(proj, angles, D, pw, pitch, n_kappa=None):
    """Katsevich filtering for a flat detector (Noo, Pack & Heuscher, Phys. Med. Biol. 48
    (2003) 3787-3818, sections 3-4), FP64, on this project's virtual detector through the
    rotation axis (source-detector distance = source-axis distance D).

    proj: [n][H][W], detector pixel (i, j) at w = (i - W//2) pw, v = (j - H//2) pw (voxel
    units, v relative to the source height).  The published formulas use the detector
    coordinate u along the source's direction of travel; for the right-handed helix of
    ConeGeometry.helical that is u = -w.  Steps: derivative at fixed ray direction
    g1 = dg/dlam + (u^2+D^2)/D dg/du + u v / D dg/dv; length correction
    g2 = D / sqrt(u^2+D^2+v^2) g1; forward height rebinning onto kappa-lines
    v_k(u, psi) = P/(2 pi) (psi + psi/tan(psi) u/D); Hilbert transform along u with the
    band-limited kernel (1 - cos(pi n)) / (pi n); backward rebinning through the kappa-line
    of smallest |psi|.  Returns g_F in the input layout."""
    proj = np.asarray(proj, np.float64)
    n, H, W = proj.shape
    angles = np.asarray(angles, np.float64)
    dlam = float(angles[-1] - angles[0]) / (n - 1)      # mean step of the float32 angles
    # NPH orientation: u increasing along the flipped w axis
    g = proj[:, :, ::-1]
    u = -((W - 1 - np.arange(W)) - W // 2) * pw          # u of flipped column i
    v = (np.arange(H) - H // 2) * pw
    # 1. derivative at constant ray direction
    dgl = np.gradient(g, dlam, axis=0)
    dgu = np.gradient(g, u, axis=2)
    dgv = np.gradient(g, v, axis=1)
    U = u[None, None, :]
    V = v[None, :, None]
    g1 = dgl + ((U * U + D * D) / D) * dgu + (U * V / D) * dgv
    # 2. length correction
    g2 = g1 * (D / np.sqrt(U * U + D * D + V * V))
    # 3. forward height rebinning
    alpha_m = math.atan(np.max(np.abs(u)) / D)
    K = n_kappa or 2 * H
    psi = np.linspace(-math.pi / 2 - alpha_m, math.pi / 2 + alpha_m, K)
    with np.errstate(divide="ignore", invalid="ignore"):
        cot = np.where(np.abs(psi) < 1e-12, 1.0, psi / np.tan(psi))
    vk = (pitch / (2 * math.pi)) * (psi[:, None] + cot[:, None] * u[None, :] / D)   # [K][W]
    g3 = np.zeros((n, K, W))
    for i in range(W):
        for t in range(n):
            g3[t, :, i] = np.interp(vk[:, i], v, g2[t, :, i], left=0.0, right=0.0)
    # 4. Hilbert transform along u
    m = np.arange(-(W - 1), W)
    with np.errstate(divide="ignore", invalid="ignore"):
        hd = np.where(m == 0, 0.0, (1.0 - np.cos(math.pi * m)) / (math.pi * m))
    g4 = np.zeros_like(g3)
    for t in range(n):
        for k in range(K):
            g4[t, k] = np.convolve(g3[t, k], hd, mode="full")[W - 1:2 * W - 1]
    # 5. backward rebinning: v_k(u, psi) is increasing in psi here, so the kappa-line
    #    through (u, v) is found by interpolating psi's index at height v
    gF = np.zeros((n, H, W))
    idx = np.arange(K, dtype=np.float64)
    for i in range(W):
        kf = np.interp(v, vk[:, i], idx)      # fractional kappa index for every row
        k0 = np.clip(np.floor(kf).astype(int), 0, K - 2)
        a = kf - k0
        gF[:, :, i] = (1 - a)[None, :] * g4[:, k0, i] + a[None, :] * g4[:, k0 + 1, i]
    return gF[:, :, ::-1]
