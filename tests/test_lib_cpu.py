"""CPU checks of the product library: it loads, exports every symbol the public header
declares, and reports errors as status codes (never exiting the process)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    with open(os.path.join(ROOT, "include", "fastcone_b200.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\**\s+\**([A-Za-z_][A-Za-z0-9_]*)\s*\(", src, re.M)
    return sorted(set(names))


def test_library_loads_and_exports_header_symbols():
    from fastcone_b200 import _lib

    L = _lib.lib()
    declared = _header_symbols()
    assert "GPU_CB_K_backproject" in declared and "fcb_bp_plan_create" in declared
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared) <= set(_lib.EXPORTED_SYMBOLS)
    assert L.fcb_version() >= 10000


def test_release_device_cache_without_blocks():
    """With no host call made there is nothing cached: releasing touches no device."""
    from fastcone_b200 import _lib

    assert _lib.lib().fcb_release_device_cache() == 0


def test_invalid_arguments_return_status():
    from fastcone_b200 import _lib
    from tests._cases import make_case

    L = _lib.lib()
    g, _ = make_case()
    s = g.struct()
    assert L.fcb_backproject_host(0, ctypes.byref(s), 2, None, None) == _lib.FCB_ERR_INVALID
    bad = g.struct()
    bad.volEnd[0] = bad.volStart[0]
    plan = ctypes.c_void_p()
    assert L.fcb_bp_plan_create(ctypes.byref(bad), 2, 0, ctypes.byref(plan)) == _lib.FCB_ERR_INVALID
    assert b"dimension" in L.fcb_last_error()
    bad = g.struct()
    bad.sourceSampleDistance = 0.0
    assert L.fcb_bp_plan_create(ctypes.byref(bad), 2, 0, ctypes.byref(plan)) == _lib.FCB_ERR_INVALID
    assert L.fcb_bp_plan_create(ctypes.byref(s), 2, 7, ctypes.byref(plan)) == _lib.FCB_ERR_INVALID
    assert L.fcb_fdk_filter_device(None, None, 0, 1, 1, 1, 1.0, None, 0, 0, None) == _lib.FCB_ERR_INVALID
    # filter windows are checked before any device work
    assert L.fcb_filter_plan_create(2, 3, 8, 0, 9, ctypes.byref(plan)) == _lib.FCB_ERR_INVALID
    assert b"window" in L.fcb_last_error()
    assert L.fcb_filter_plan_create_ex(2, 3, 8, 0, _lib.FILTER_GAUSSRAMP, 0.0,
                                       ctypes.byref(plan)) == _lib.FCB_ERR_INVALID
    assert b"gaussScale" in L.fcb_last_error()


def test_reference_entry_point_bad_device_sets_status():
    """The reference exits the process on a bad GPUID (coneBeamGPU.cu:472-475); here the
    void entry point records FCB_ERR_NODEVICE and returns."""
    from fastcone_b200 import _lib
    from tests._cases import make_case

    L = _lib.lib()
    g, pb = make_case(vol_xyz=(8, 8, 8), det_wh=(8, 8), nviews=2, D=50.0)
    vol = np.zeros(g.vol_shape, np.float32)
    proj = np.zeros(g.proj_shape, np.float32)
    fp = lambda a: a.ctypes.data_as(_lib.c_float_p)
    ip = lambda a: a.ctypes.data_as(_lib.c_int_p)
    L.GPU_CB_K_backproject(9999, fp(vol), fp(proj), fp(pb.angles), fp(pb.hMid), ctypes.c_float(50.0),
                           ctypes.c_float(1.0), ip(pb.volDim), ip(pb.volStart), ip(pb.volEnd), ip(pb.projDim),
                           ip(pb.projWHSize), ip(pb.projWOffset), ip(pb.projHOffset), fp(pb.norm), 2)
    assert L.fcb_last_status() == _lib.FCB_ERR_NODEVICE


def test_python_api_argument_errors():
    from fastcone_b200 import fastcone as fc

    vol = np.zeros((4, 4, 4), np.float32)
    proj = np.zeros((3, 4, 4), np.float32)
    with pytest.raises(fc.FastconeArgumentError, match="np.float32"):
        fc.project(vol.astype(np.float64), proj, np.zeros(3), 10.0, np.zeros(3))
    with pytest.raises(fc.FastconeArgumentError, match="angles"):
        fc.backproject(vol, proj, np.zeros(2), 10.0, np.zeros(3))
    with pytest.raises(fc.FastconeArgumentError, match="kernel mode"):
        fc.backproject(vol, proj, np.zeros(3), 10.0, np.zeros(3), kernelMode=2, misAlignments=np.zeros(6))
    assert issubclass(fc.FastconeArgumentError, SystemExit)


def test_geometry_helpers():
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.circular((1024,) * 3, 0.25, (1536, 1024), 0.4, 500.0, 1000.0, 1440)
    assert g.D == pytest.approx(2000.0) and g.pw == pytest.approx(0.8)
    h = ConeGeometry.helical((512, 512, 384), 0.5, (736, 64), 1.0, 570.0, 1040.0, 4, 1160, 40.0)
    assert h.nviews == 4640 and h.helical_pitch == pytest.approx(80.0)
    assert h.pw == pytest.approx(1.0 * 570 / 1040 / 0.5)
    assert np.allclose(np.diff(h.hmid.astype(np.float64)), 80.0 / 1160, atol=1e-3)


def test_new_entry_points_refuse_bad_arguments_before_device_work():
    """fcb_fbp_host, fcb_smem_bandwidth, fcb_bp_plan_set_test_stall and
    fcb_katsevich_pi_pairs check their arguments first and return FCB_ERR_INVALID."""
    from fastcone_b200 import _lib
    from tests._cases import make_case

    L = _lib.lib()
    g, _ = make_case()
    s = g.struct()
    proj = np.zeros(g.proj_shape, np.float32)
    vol = np.zeros(g.vol_shape, np.float32)
    z = np.zeros(g.nviews, np.float32)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    fz = z.ctypes.data_as(_lib.c_float_p)
    assert L.fcb_fbp_host(0, ctypes.byref(s), 9, 100.0, fz, 1, vp(proj), vp(vol)) == _lib.FCB_ERR_INVALID
    assert b"window" in L.fcb_last_error()
    assert L.fcb_fbp_host(0, ctypes.byref(s), 0, 0.0, fz, 1, vp(proj), vp(vol)) == _lib.FCB_ERR_INVALID
    assert L.fcb_fbp_host(0, ctypes.byref(s), 0, 100.0, fz, 1, None, vp(vol)) == _lib.FCB_ERR_INVALID
    ms, nb = ctypes.c_float(), ctypes.c_double()
    assert L.fcb_smem_bandwidth(3, 10, ctypes.byref(ms), ctypes.byref(nb), None) == _lib.FCB_ERR_INVALID
    assert L.fcb_smem_bandwidth(4, 0, ctypes.byref(ms), ctypes.byref(nb), None) == _lib.FCB_ERR_INVALID
    assert L.fcb_bp_plan_set_test_stall(None, 1, 1000) == _lib.FCB_ERR_INVALID
    n = ctypes.c_longlong()
    assert L.fcb_katsevich_pi_pairs(None, ctypes.byref(n), None) == _lib.FCB_ERR_INVALID
    # a circular geometry has no PI window
    assert L.fcb_katsevich_pi_pairs(ctypes.byref(s), ctypes.byref(n), None) == _lib.FCB_ERR_INVALID
    assert b"pitch" in L.fcb_last_error()
