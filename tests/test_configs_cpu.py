"""The five workload configurations as geometries (fastcone_b200.configs): shapes and the
voxel-unit distances derived from their physical descriptions, and the C struct the
library receives for them (dimension order [x,y,z] / [w,h,t], fastcone.py:117-121)."""
import ctypes

import numpy as np
import pytest


def _configs():
    from fastcone_b200 import configs

    return {
        # name: (geometry, vol_xyz, det_wh, nviews, D, pw)
        "small_fdk": (configs.small_fdk(), (128, 128, 128), (192, 128), 180, 500.0, 0.5),
        "large_fdk": (configs.large_fdk(), (1024, 1024, 1024), (1536, 1024), 1440, 2000.0, 0.8),
        "helical": (configs.helical_katsevich(), (512, 512, 384), (736, 64), 4640, 1140.0, 1.0 * 570 / 1040 / 0.5),
        "diff_batch": (configs.diff_batch(), (256, 256, 256), (384, 256), 360, 1000.0, 1.0),
        "learned": (configs.learned_sparse(), (256, 256, 256), (384, 256), 90, 1000.0, 1.0),
    }


@pytest.mark.parametrize("name", ["small_fdk", "large_fdk", "helical", "diff_batch", "learned"])
def test_configuration_shapes_and_units(name):
    g, vol, det, n, D, pw = _configs()[name]
    assert g.vol_xyz == vol and g.det_wh == det and g.nviews == n
    assert g.vol_shape == vol[::-1] and g.proj_shape == (n, det[1], det[0])
    assert g.D == pytest.approx(D) and g.pw == pytest.approx(pw)
    turn = 2 * np.pi if name != "helical" else 4 * 2 * np.pi
    step = np.diff(g.angles.astype(np.float64))
    assert np.allclose(step, turn / n, rtol=0, atol=4e-6)  # FP32 angles up to 8 pi
    assert float(g.angles[0]) == 0.0


def test_helical_source_rises_through_the_volume_centre():
    g = _configs()["helical"][0]
    assert g.helical_pitch == pytest.approx(80.0) and g.pi_window
    hm = g.hmid.astype(np.float64)
    assert np.allclose(np.diff(hm), 80.0 / 1160, atol=1e-4)
    assert 0.5 * (hm[0] + hm[-1]) == pytest.approx(384 / 2.0, abs=1e-3)
    # four turns of 80 voxels: the helix spans the 384-plane volume minus about one turn
    assert hm[-1] - hm[0] == pytest.approx(80.0 * (4640 - 1) / 1160, abs=1e-2)


def test_fdk_norm_is_reciprocal_view_count():
    from fastcone_b200 import configs

    g = configs.with_fdk_norm(configs.small_fdk())
    assert np.all(g.norm == np.float32(1.0 / 180))


def test_struct_carries_the_geometry_in_reference_order():
    from fastcone_b200.geometry import ConeGeometry

    n = 5
    g = ConeGeometry((40, 36, 32), (64, 48), np.linspace(0, 1, n), 150.0, 0.75,
                     hmid=np.arange(n) + 10.0, norm=np.arange(n) + 1.0, vol_start=(2, 3, 4),
                     vol_end=(30, 33, 31), woff=np.arange(n), hoff=2 * np.arange(n), window_wh=(50, 40),
                     misalignments=[1, 2, 3, 0.1, 0.2, 0.3], helical_pitch=12.5, pi_window=True)
    s = g.struct()
    assert list(s.volDim) == [40, 36, 32]
    assert list(s.volStart) == [2, 3, 4] and list(s.volEnd) == [30, 33, 31]
    assert list(s.projDim) == [64, 48, n] and list(s.projWHSize) == [50, 40]
    assert s.sourceSampleDistance == pytest.approx(150.0) and s.pixelWidth == pytest.approx(0.75)
    assert s.helicalPitch == pytest.approx(12.5) and s.piWindow == 1 and s.referenceWindows == 0
    for field, want in (("angles", g.angles), ("hMidPlane", g.hmid), ("normalizationFactor", g.norm),
                        ("misAlignments", g.misalignments)):
        got = np.ctypeslib.as_array(getattr(s, field), shape=(len(want),))
        assert np.array_equal(got, want), field
    for field, want in (("projWOffset", g.woff), ("projHOffset", g.hoff)):
        got = np.ctypeslib.as_array(getattr(s, field), shape=(n,))
        assert np.array_equal(got, want), field
    assert g.vol_shape == (27, 30, 28) and g.proj_shape == (n, 40, 50)
    plain = ConeGeometry((8, 8, 8), (8, 8), np.zeros(2), 50.0, 1.0).struct()
    assert not ctypes.cast(plain.misAlignments, ctypes.c_void_p).value


def test_per_view_arrays_must_match_the_angles():
    from fastcone_b200.geometry import ConeGeometry

    with pytest.raises(ValueError, match="one entry per angle"):
        ConeGeometry((8, 8, 8), (8, 8), np.zeros(3), 50.0, 1.0, norm=np.ones(2))
