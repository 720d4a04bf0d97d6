"""ctypes binding of libfastcone_b200.so (the C ABI declared in include/fastcone_b200.h).

The library is the product: there is no CPU fallback.  Loading fails loudly when the
shared object has not been built (``python -m fastcone_b200.build``).
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfastcone_b200.so")

c_int_p = ctypes.POINTER(ctypes.c_int)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)

FCB_OK = 0
FCB_ERR_INVALID = 1
FCB_ERR_CUDA = 2
FCB_ERR_NOMEM = 3
FCB_ERR_TIMEOUT = 4
FCB_ERR_NODEVICE = 5
FCB_ERR_RANGE = 6
FCB_ERR_HOST = 7

FCB_F32, FCB_F16, FCB_BF16 = 0, 1, 2
MODE_UNWEIGHTED, MODE_KATSEVICH, MODE_FDK = 0, 1, 2
PROJ_TEXTURE, PROJ_EXPLICIT, PROJ_EXPLICIT_GLOBAL = 0, 1, 2
FILTER_RAMLAK, FILTER_SHEPPLOGAN, FILTER_COSRAMP, FILTER_GAUSSRAMP = 0, 1, 2, 3

# Every symbol include/fastcone_b200.h declares (checked by the CPU test suite).
EXPORTED_SYMBOLS = [
    "fcb_version", "fcb_last_status", "fcb_last_error",
    "GPU_CB_K_backproject", "GPU_CB_backproject", "GPU_CB_misalign_backproject",
    "GPU_CB_misalign_project", "GPU_CB_project",
    "fcb_backproject_host", "fcb_project_host",
    "fcb_backproject_device", "fcb_project_device", "fcb_project_adjoint_device",
    "fcb_project_device_counted",
    "fcb_bp_plan_create", "fcb_bp_plan_execute", "fcb_bp_plan_info", "fcb_bp_plan_destroy",
    "fcb_sync_status", "fcb_fdk_filter_device", "fcb_phantom_device",
    "fcb_backproject_device_noalloc", "fcb_katsevich_filter_device",
    "fcb_conv3d16_device", "fcb_conv3d16_wgrad_device",
    "fcb_proj_plan_create", "fcb_proj_plan_execute", "fcb_proj_plan_destroy",
    "fcb_reference_windows", "fcb_proj_plan_info",
    "fcb_filter_plan_create", "fcb_filter_plan_create_ex", "fcb_filter_plan_execute",
    "fcb_filter_plan_destroy",
    "fcb_katsevich_plan_create", "fcb_katsevich_plan_execute", "fcb_katsevich_plan_destroy",
    "fcb_detector_rows",
    "fcb_bp_plan_set_test_stall", "fcb_katsevich_pi_pairs", "fcb_smem_bandwidth", "fcb_fbp_host",
    "fcb_release_device_cache",
]


class FcbGeometry(ctypes.Structure):
    _fields_ = [
        ("volDim", ctypes.c_int * 3),
        ("volStart", ctypes.c_int * 3),
        ("volEnd", ctypes.c_int * 3),
        ("projDim", ctypes.c_int * 3),
        ("projWHSize", ctypes.c_int * 2),
        ("projWOffset", c_int_p),
        ("projHOffset", c_int_p),
        ("angles", c_float_p),
        ("hMidPlane", c_float_p),
        ("sourceSampleDistance", ctypes.c_float),
        ("pixelWidth", ctypes.c_float),
        ("normalizationFactor", c_float_p),
        ("misAlignments", c_float_p),
        ("helicalPitch", ctypes.c_float),
        ("piWindow", ctypes.c_int),
        ("referenceWindows", ctypes.c_int),
    ]


class FastconeError(RuntimeError):
    """A failed library call; ``status`` is one of the FCB_ERR_* codes."""

    def __init__(self, status, msg):
        super().__init__(f"fastcone_b200 error {status}: {msg}")
        self.status = status


_lock = threading.Lock()
_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FastconeError(FCB_ERR_INVALID,
                                    f"{LIB_PATH} is not built; run python -m fastcone_b200.build")
            L = ctypes.CDLL(LIB_PATH)
            L.fcb_last_error.restype = ctypes.c_char_p
            vp = ctypes.c_void_p
            gp = ctypes.POINTER(FcbGeometry)
            L.fcb_backproject_host.argtypes = [ctypes.c_int, gp, ctypes.c_int, vp, vp]
            L.fcb_project_host.argtypes = [ctypes.c_int, gp, ctypes.c_int, vp, vp]
            L.fcb_backproject_device.argtypes = [gp, ctypes.c_int, vp, ctypes.c_int, vp, vp]
            L.fcb_project_device.argtypes = [gp, ctypes.c_int, vp, vp, vp]
            L.fcb_backproject_device_noalloc.argtypes = [gp, ctypes.c_int, vp, ctypes.c_int, vp, vp]
            L.fcb_project_device_counted.argtypes = [gp, ctypes.c_int, vp, vp, vp, vp]
            L.fcb_project_adjoint_device.argtypes = [gp, vp, vp, vp]
            L.fcb_bp_plan_create.argtypes = [gp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
            L.fcb_bp_plan_execute.argtypes = [vp, vp, vp, vp]
            L.fcb_bp_plan_info.argtypes = [vp, c_int_p, c_int_p, c_int_p,
                                           ctypes.POINTER(ctypes.c_longlong)]
            L.fcb_bp_plan_destroy.argtypes = [vp]
            L.fcb_sync_status.argtypes = [vp]
            L.fcb_release_device_cache.argtypes = []
            L.fcb_fdk_filter_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_float, c_float_p,
                                                ctypes.c_int, ctypes.c_int, vp]
            L.fcb_phantom_device.argtypes = [vp, c_int_p, c_double_p, ctypes.c_int, vp]
            L.fcb_proj_plan_create.argtypes = [gp, ctypes.c_int, ctypes.POINTER(vp)]
            L.fcb_proj_plan_execute.argtypes = [vp, vp, vp, ctypes.c_int, vp]
            L.fcb_proj_plan_destroy.argtypes = [vp]
            L.fcb_conv3d16_device.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, vp]
            L.fcb_conv3d16_wgrad_device.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, vp]
            L.fcb_katsevich_filter_device.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                      c_float_p, ctypes.c_float, ctypes.c_float,
                                                      ctypes.c_float, ctypes.c_int, vp]
            L.fcb_reference_windows.argtypes = [gp] + [c_int_p] * 8
            L.fcb_proj_plan_info.argtypes = [vp] + [c_int_p] * 4
            L.fcb_filter_plan_create.argtypes = [ctypes.c_int] * 5 + [ctypes.POINTER(vp)]
            L.fcb_filter_plan_create_ex.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.POINTER(vp)]
            L.fcb_filter_plan_execute.argtypes = [vp, vp, vp, ctypes.c_float, c_float_p, ctypes.c_int, vp]
            L.fcb_filter_plan_destroy.argtypes = [vp]
            L.fcb_katsevich_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_float_p,
                                                    ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                                    ctypes.c_int, ctypes.POINTER(vp)]
            L.fcb_katsevich_plan_execute.argtypes = [vp, vp, vp, vp]
            L.fcb_katsevich_plan_destroy.argtypes = [vp]
            L.fcb_detector_rows.argtypes = [gp, ctypes.c_int, c_int_p, c_int_p]
            L.fcb_bp_plan_set_test_stall.argtypes = [vp, ctypes.c_int, ctypes.c_ulonglong]
            L.fcb_katsevich_pi_pairs.argtypes = [gp, ctypes.POINTER(ctypes.c_longlong), vp]
            L.fcb_smem_bandwidth.argtypes = [ctypes.c_int, ctypes.c_longlong, c_float_p, c_double_p, vp]
            L.fcb_fbp_host.argtypes = [ctypes.c_int, gp, ctypes.c_int, ctypes.c_float, c_float_p, ctypes.c_int,
                                       vp, vp]
            _lib = L
    return _lib


def check(status):
    """Raise FastconeError for a non-zero status (message from fcb_last_error)."""
    if status != FCB_OK:
        msg = lib().fcb_last_error()
        raise FastconeError(status, msg.decode() if msg else "")
    return status


def last_status():
    return int(lib().fcb_last_status())


def check_last():
    st = last_status()
    if st != FCB_OK:
        check(st)


def arr_i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def arr_f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def ptr(a, kind):
    return a.ctypes.data_as(kind)
