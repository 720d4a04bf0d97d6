"""Drop-in for the reference's ``fastcone`` module (fastcone.py:52-319).

Same functions, argument names, defaults, array conventions and side effects:

  * ``project(vol, proj, angle, sourceDistance, zOrigin, ...)``  (fastcone.py:52-144)
  * ``backproject(vol, proj, angle, sourceDistance, zOrigin, ...)``  (fastcone.py:147-256)
  * ``fbp(vol, proj, projAngles, specimenLength, zOrigin, ...)``  (fastcone.py:260-270)
  * ``rampfilter(proj)``  (fastcone.py:272-292)

Arrays are numpy: ``vol[z, y, x]`` and ``proj[theta, h, w]`` float32, results ADDED into
them.  Invalid arguments raise ``FastconeArgumentError``, a SystemExit subclass carrying the
reference's own message (the reference calls ``sys.exit`` with it).  Calls reach
libfastcone_b200.so (loaded once, not per call as the reference does at :123/:218) through
the same five C entry points the reference's wrapper.c exports; a failed call raises
``FastconeError`` instead of silently leaving the output untouched.

Differences that are deliberate fixes, not behaviour changes: optional array arguments are
tested with ``is None`` (the reference's ``== None`` raises on arrays, :85-93), and
``rampfilter`` works on numpy >= 1.12 (the reference builds ``np.zeros`` with a float shape,
:274).  ``fbp`` and ``rampfilter`` run their filtering on the GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import FastconeError, c_float_p, c_int_p, lib

FLOAT_TYPE = np.float32
INT_TYPE = np.int32


class FastconeArgumentError(SystemExit):
    """Argument validation failure; the reference reports these with sys.exit(message)."""


def _fp(a):
    return a.ctypes.data_as(c_float_p)


def _ip(a):
    return a.ctypes.data_as(c_int_p)


def _check_common(vol, proj, angle, zOrigin, fname="project"):
    if vol.dtype != FLOAT_TYPE:
        raise FastconeArgumentError(f"Volume array supplied to function '{fname}' does not have data type np.float32")
    if proj.dtype != FLOAT_TYPE:
        raise FastconeArgumentError(f"Projection array supplied to function '{fname}' does not have data type np.float32")
    if angle.size != proj.shape[0]:
        raise FastconeArgumentError("Number of angles supplied does not match number of projections in proj array")
    if zOrigin.size != proj.shape[0]:
        raise FastconeArgumentError("Number of zOrigin elements does not match number of projections in proj array")
    if not (vol.flags.c_contiguous and proj.flags.c_contiguous):
        raise FastconeArgumentError("vol and proj must be C-contiguous arrays")


def _prepare(vol, proj, angle, zOrigin, volStart, volDims, projWOffset, projHOffset, projDims, norm,
             default_norm, vol_dims_default_end):
    volStart = np.asarray(volStart)
    volEnd = np.array([vol.shape[0] + volStart[0], vol.shape[1] + volStart[1], vol.shape[2] + volStart[2]],
                      dtype=INT_TYPE)
    if volDims is None:
        volDims = volEnd.copy() if vol_dims_default_end else np.array(vol.shape, dtype=INT_TYPE)
    if projWOffset is None:
        projWOffset = np.zeros(angle.size, dtype=INT_TYPE)
    if projHOffset is None:
        projHOffset = np.zeros(angle.size, dtype=INT_TYPE)
    projWOffset = np.ascontiguousarray(projWOffset, dtype=INT_TYPE)
    projHOffset = np.ascontiguousarray(projHOffset, dtype=INT_TYPE)
    if projDims is None:
        projDims = np.array([proj.shape[0], proj.shape[1] + projHOffset.max(), proj.shape[2] + projWOffset.max()],
                            dtype=INT_TYPE)
    if norm is None:
        norm = default_norm(projDims)
    projDims = np.array(projDims, dtype=INT_TYPE).copy()
    projDims[0] = proj.shape[0]
    projWHSize = np.array([proj.shape[1], proj.shape[2]], dtype=INT_TYPE)
    hMidplane = np.ascontiguousarray(zOrigin, dtype=FLOAT_TYPE)
    angle = np.ascontiguousarray(angle, dtype=FLOAT_TYPE)
    norm = np.ascontiguousarray(norm, dtype=FLOAT_TYPE)
    # reverse to the C code's [x, y, z] / [w, h, t] order
    rev = lambda a: np.ascontiguousarray(np.asarray(a, dtype=INT_TYPE)[::-1])
    return (angle, hMidplane, rev(volDims), rev(volStart), rev(volEnd), rev(projDims), rev(projWHSize),
            projWOffset, projHOffset, norm)


def project(vol, proj, angle, sourceDistance, zOrigin, volStart=np.array([0, 0, 0], dtype=INT_TYPE),
            volDims=None, projWOffset=None, projHOffset=None, projDims=None, norm=None, GPUID=0,
            misAlignments=np.array([0, 0, 0, 0, 0, 0], dtype=FLOAT_TYPE), pixelWidth=1.0):
    """Cone-beam forward projection; ADDS norm[t] * (A vol) into proj (fastcone.py:52-144).
    Afterwards zeroes detector column 0 of views whose window starts at w <= 0, as the
    reference does (fastcone.py:140-143)."""
    angle = np.asarray(angle)
    zOrigin = np.asarray(zOrigin)
    _check_common(vol, proj, angle, zOrigin, "project")
    (angle, hmid, volDims, volStart_r, volEnd, projDims, projWHSize, projWOffset, projHOffset,
     norm) = _prepare(vol, proj, angle, zOrigin, volStart, volDims, projWOffset, projHOffset, projDims,
                      norm, lambda pd: np.ones(angle.size, dtype=FLOAT_TYPE), False)
    mis = np.ascontiguousarray(misAlignments if misAlignments is not None else np.zeros(6), dtype=FLOAT_TYPE)
    lib().GPU_CB_misalign_project(ctypes.c_int(GPUID), _fp(vol), _fp(proj), _fp(angle), _fp(hmid),
                                  ctypes.c_float(sourceDistance), ctypes.c_float(pixelWidth), _ip(volDims),
                                  _ip(volStart_r), _ip(volEnd), _ip(projDims), _ip(projWHSize),
                                  _ip(projWOffset), _ip(projHOffset), _fp(norm), _fp(mis))
    _lib.check_last()
    for tt in range(proj.shape[0]):
        if projWOffset[tt] <= 0:
            proj[tt, :, 0:(1 + projWOffset[tt])] = 0.0
    return 1


def backproject(vol, proj, angle, sourceDistance, zOrigin, volStart=np.array([0, 0, 0], dtype=INT_TYPE),
                volDims=None, projWOffset=None, projHOffset=None, projDims=None, norm=None, GPUID=0,
                kernelMode=2, misAlignments=None, pixelWidth=1.0):
    """Voxel-driven backprojection; ADDS into vol (fastcone.py:147-256).  kernelMode 2 FDK
    (weight U^2), 1 Katsevich (U), 0 unweighted; misAlignments only with kernelMode 0."""
    angle = np.asarray(angle)
    zOrigin = np.asarray(zOrigin)
    _check_common(vol, proj, angle, zOrigin, "project")
    if (misAlignments is not None) and (kernelMode != 0):
        raise FastconeArgumentError("Cannot conduct misaligned backprojection unless kernel mode is set to 0 "
                                    "(i.e. unweighted, not Feldkamp or Katsevich).")
    (angle, hmid, volDims, volStart_r, volEnd, projDims, projWHSize, projWOffset, projHOffset,
     norm) = _prepare(vol, proj, angle, zOrigin, volStart, volDims, projWOffset, projHOffset, projDims,
                      norm, lambda pd: np.ones(angle.size, dtype=FLOAT_TYPE) / pd[0], True)
    args = (ctypes.c_int(GPUID), _fp(vol), _fp(proj), _fp(angle), _fp(hmid), ctypes.c_float(sourceDistance),
            ctypes.c_float(pixelWidth), _ip(volDims), _ip(volStart_r), _ip(volEnd), _ip(projDims),
            _ip(projWHSize), _ip(projWOffset), _ip(projHOffset), _fp(norm))
    if misAlignments is None:
        lib().GPU_CB_K_backproject(*args, ctypes.c_int(kernelMode))
    else:
        mis = np.ascontiguousarray(misAlignments, dtype=FLOAT_TYPE)
        lib().GPU_CB_misalign_backproject(*args, _fp(mis))
    _lib.check_last()
    return 1


def fbp(vol, proj, projAngles, specimenLength, zOrigin, volStart=np.array([0, 0, 0], dtype=INT_TYPE),
        volDims=None, GPUID=0, pixelWidth=1.0, window="ramlak"):
    """FDK: cosine pre-weight, ramp filter, FDK backprojection with norm 1/nviews
    (fastcone.py:260-270).  Like the reference, overwrites ``proj`` with the weighted,
    filtered projections and returns the last view's cosine-weight array.  One library call
    (fcb_fbp_host) streams the views to the GPU, filters them there, returns them into
    ``proj`` and backprojects them while the next views are in flight."""
    zOrigin = np.asarray(zOrigin)
    if proj.dtype != FLOAT_TYPE or not proj.flags.c_contiguous:
        raise FastconeArgumentError("Projection array must be C-contiguous np.float32")
    projAngles = np.asarray(projAngles)
    _check_common(vol, proj, projAngles, zOrigin, "project")
    (angle, hmid, volDims, volStart_r, volEnd, projDims, projWHSize, projWOffset, projHOffset,
     norm) = _prepare(vol, proj, projAngles, zOrigin, volStart, volDims, None, None, None, None,
                      lambda pd: np.ones(projAngles.size, dtype=FLOAT_TYPE) / pd[0], True)
    g = _lib.FcbGeometry()
    for i in range(3):
        g.volDim[i], g.volStart[i], g.volEnd[i], g.projDim[i] = (int(volDims[i]), int(volStart_r[i]),
                                                                 int(volEnd[i]), int(projDims[i]))
    g.projWHSize[0], g.projWHSize[1] = int(projWHSize[0]), int(projWHSize[1])
    g.projWOffset, g.projHOffset = _ip(projWOffset), _ip(projHOffset)
    g.angles, g.hMidPlane, g.normalizationFactor = _fp(angle), _fp(hmid), _fp(norm)
    g.sourceSampleDistance = float(specimenLength)
    g.pixelWidth = float(pixelWidth)
    g.referenceWindows = 1  # as the GPU_CB_* entry points: the reference's windows where they matter
    _lib.check(lib().fcb_fbp_host(int(GPUID), ctypes.byref(g), _WINDOWS[window], float(specimenLength), _fp(hmid),
                                  1, proj.ctypes.data_as(ctypes.c_void_p), vol.ctypes.data_as(ctypes.c_void_p)))
    W, H = proj.shape[2], proj.shape[1]
    ww = (np.arange(0.0, W, 1.0) - W / 2.0)[None, :]
    hh = (np.arange(0.0, H, 1.0) - float(zOrigin[proj.shape[0] - 1]))[:, None]
    return specimenLength / np.sqrt(specimenLength * specimenLength + hh * hh + ww * ww)


def rampfilter(proj, window="ramlak", GPUID=0):
    """Ramp filter of fastcone.py:272-292 (rows zero-padded to 2W, pi*|f|, DC = f1/8), in
    place, on the GPU.  ``window='shepplogan'`` adds the sinc apodisation."""
    _filter_inplace(proj, 0.0, None, cosine=False, window=window, GPUID=GPUID)


def cosrampfilter(proj, GPUID=0):
    """Cosine-apodised ramp filter of fastcone.py:294-304 (rows of length W, unpadded,
    response |f| * cos(0.5 |f| pi / W)), in place, on the GPU.  Every view is filtered (the
    reference's loop stores only the last view, and its inverse FFT has length W - 1 for an
    odd W; here the inverse has length W)."""
    _filter_inplace(proj, 0.0, None, cosine=False, window="cosramp", GPUID=GPUID)


def gaussrampfilter(proj, scale=0.125, GPUID=0):
    """Gaussian-apodised ramp filter of fastcone.py:306-319 (rows of length W, unpadded;
    |f| times the Gaussian of sigma = scale * W shifted by -W/2 samples), in place, on the
    GPU, every view filtered."""
    _filter_inplace(proj, 0.0, None, cosine=False, window="gaussramp", GPUID=GPUID, gauss_scale=scale)


_WINDOWS = {"ramlak": _lib.FILTER_RAMLAK, "shepplogan": _lib.FILTER_SHEPPLOGAN,
            "cosramp": _lib.FILTER_COSRAMP, "gaussramp": _lib.FILTER_GAUSSRAMP}


def _filter_inplace(proj, D, zOrigin, cosine, window, GPUID, gauss_scale=0.125):
    import torch  # plumbing for device memory and the stream

    if proj.dtype != FLOAT_TYPE or not proj.flags.c_contiguous:
        raise FastconeArgumentError("Projection array must be C-contiguous np.float32")
    win = _WINDOWS[window]
    n, H, W = proj.shape
    dev = torch.device("cuda", GPUID)
    with torch.cuda.device(dev):
        t = torch.from_numpy(proj).to(dev)
        z = np.ascontiguousarray(zOrigin if zOrigin is not None else np.zeros(n), dtype=FLOAT_TYPE)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        plan = ctypes.c_void_p()
        _lib.check(lib().fcb_filter_plan_create_ex(n, H, W, _lib.FCB_F32, win, float(gauss_scale),
                                                   ctypes.byref(plan)))
        try:
            _lib.check(lib().fcb_filter_plan_execute(plan, ctypes.c_void_p(t.data_ptr()),
                                                     ctypes.c_void_p(t.data_ptr()), float(D),
                                                     z.ctypes.data_as(c_float_p), 1 if cosine else 0, st))
            proj[...] = t.cpu().numpy()
        finally:
            torch.cuda.current_stream().synchronize()
            lib().fcb_filter_plan_destroy(plan)


__all__ = ["project", "backproject", "fbp", "rampfilter", "cosrampfilter", "gaussrampfilter", "FastconeArgumentError", "FastconeError",
           "FLOAT_TYPE", "INT_TYPE"]
