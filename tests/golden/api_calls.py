"""Calls of the Python module's project / backproject whose C-ABI arguments are recorded:
the reference's fastcone.py (fastcone.py:52-256) marshals them into the GPU_CB_* entry
points (wrapper.c:112-249) in a fixed order, and the drop-in must pass the same values
(dimension arrays reversed to [x,y,z] / [w,h,t], defaults, normalisation) and point at the
caller's own vol / proj arrays.  Used by make_golden.py (reference side, through a
recording stand-in for ctypes.CDLL) and tests/test_api_cpu.py (this library's side).

Only calls the reference can still run under numpy >= 1.12 are listed: it compares
optional arrays with ``== None`` (fastcone.py:85-93, :182-190), which raises for arrays, so
the optional array arguments other than volStart / misAlignments of ``project`` stay at
their None defaults."""
import ctypes

import numpy as np

N = 3  # views per call


def calls():
    """(function name, keyword arguments) of each recorded call; vol and proj come from
    ``arrays()``."""
    ang64 = np.linspace(0.0, 1.0, N)
    z = np.array([2.5, 3.0, 3.5])
    return [
        ("project", dict(angle=ang64, sourceDistance=50.0, zOrigin=z)),
        ("project", dict(angle=ang64.astype(np.float32), sourceDistance=60.0, zOrigin=z.astype(np.float32),
                         pixelWidth=0.8, volStart=np.array([1, 2, 3]))),
        ("project", dict(angle=ang64, sourceDistance=70.0, zOrigin=z, GPUID=0,
                         misAlignments=np.array([0.5, -0.5, 1.0, 0.01, 0.02, -0.03]))),
        ("backproject", dict(angle=ang64, sourceDistance=50.0, zOrigin=z)),
        ("backproject", dict(angle=ang64, sourceDistance=55.0, zOrigin=z, kernelMode=0,
                             volStart=np.array([0, 1, 2], np.int32))),
        ("backproject", dict(angle=ang64, sourceDistance=45.0, zOrigin=z, kernelMode=1, pixelWidth=1.2)),
    ]


def arrays():
    vol = np.full((5, 6, 7), 0.25, np.float32)
    proj = np.ones((N, 8, 9), np.float32)
    return vol, proj


class Recorder:
    """Stands in for the loaded library: records every GPU_CB_* call."""

    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        if name.startswith("GPU_CB_"):
            return lambda *args: self.calls.append((name, args))
        raise AttributeError(name)


def _values(p, ctype, n):
    q = ctypes.cast(p, ctypes.POINTER(ctype))
    return [q[i] for i in range(n)]


def decode(name, args, vol, proj):
    """JSON form of one recorded call: scalars by value, vol / proj as whether they point at
    the caller's arrays, every other pointer as the values it points at."""
    f, i = ctypes.c_float, ctypes.c_int
    addr = lambda p: ctypes.cast(p, ctypes.c_void_p).value
    out = {"name": name, "GPUID": args[0].value,
           "vol_is_callers": addr(args[1]) == vol.ctypes.data, "proj_is_callers": addr(args[2]) == proj.ctypes.data,
           "angles": _values(args[3], f, N), "hMidPlane": _values(args[4], f, N),
           "sourceSampleDistance": args[5].value, "pixelWidth": args[6].value,
           "volDim": _values(args[7], i, 3), "volStart": _values(args[8], i, 3), "volEnd": _values(args[9], i, 3),
           "projDim": _values(args[10], i, 3), "projWHSize": _values(args[11], i, 2),
           "projWOffset": _values(args[12], i, N), "projHOffset": _values(args[13], i, N),
           "normalizationFactor": _values(args[14], f, N)}
    if name == "GPU_CB_K_backproject":
        out["kernelMode"] = args[15].value
    else:
        out["misAlignments"] = _values(args[15], f, 6)
    return out
