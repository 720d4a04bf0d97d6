"""The library's restatement of the reference's sub-problem windows (used when
referenceWindows = 1) against the oracle's, which is pinned bit-exact to the reference's
own coneBeamGeometry (test_oracle_cpu).  Host computation only -- no GPU."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_cpu import GEOMETRY_CASES, _helical_case


def _geom(pb, mis=None):
    from fastcone_b200.geometry import ConeGeometry

    return ConeGeometry(tuple(int(v) for v in pb.volDim), (int(pb.projDim[0]), int(pb.projDim[1])), pb.angles,
                        pb.D, pb.pw, hmid=pb.hMid, norm=pb.norm, vol_start=tuple(int(v) for v in pb.volStart),
                        vol_end=tuple(int(v) for v in pb.volEnd), woff=pb.projWOffset, hoff=pb.projHOffset,
                        window_wh=(int(pb.projWHSize[0]), int(pb.projWHSize[1])), misalignments=mis,
                        reference_windows=True)


def _cases():
    out = [(O.make_problem(**kw), None) for kw in GEOMETRY_CASES]
    out.append((_helical_case(), None))
    out.append((O.make_problem((48, 48, 48), (64, 64), 20, D=150, pw=0.8),
                np.array([1.5, -0.5, 2.0, 0.02, -0.01, 0.03], np.float32)))
    # several tiles in x and z, two view chunks
    out.append((O.make_problem((1100, 40, 600), (1200, 700), 300, D=3000, pw=1.0,
                               volStart=(20, 0, 30), volEnd=(1090, 40, 590)), None))
    # the 48^3 / 72-pixel case whose windows cut the detector
    out.append((O.make_problem((48, 48, 48), (72, 48), 36, D=200.0, pw=0.5), None))
    return out


CASES = _cases()


@pytest.mark.parametrize("idx", range(len(CASES)))
def test_windows_match_oracle(idx):
    pb, mis = CASES[idx]
    _compare_windows(pb, mis)


def test_windows_match_oracle_on_random_geometries():
    """Random volumes, sub-volumes, detectors, windows, distances, pitches and
    misalignments: the library's windows, tiles and sweeps equal the oracle's bit for bit."""
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies

    @hyp.settings(max_examples=60, deadline=None, derandomize=True)
    @hyp.given(vol=st.tuples(st.integers(4, 90), st.integers(4, 90), st.integers(4, 90)),
               det=st.tuples(st.integers(8, 200), st.integers(8, 160)), nviews=st.integers(1, 40),
               D=st.floats(30.0, 600.0), pw=st.floats(0.3, 1.6), sub=st.booleans(), mis=st.booleans(),
               seed=st.integers(0, 2 ** 16))
    def check(vol, det, nviews, D, pw, sub, mis, seed):
        rng = np.random.default_rng(seed)
        kw = {}
        if sub:
            lo = [int(rng.integers(0, max(1, v // 3))) for v in vol]
            hi = [int(rng.integers(l + 1, v + 1)) for l, v in zip(lo, vol)]
            kw = dict(volStart=tuple(lo), volEnd=tuple(hi))
        pb = O.make_problem(vol, det, nviews, D=D, pw=pw, **kw)
        m = rng.uniform(-1, 1, 6).astype(np.float32) * np.array([2, 2, 2, 0.03, 0.03, 0.03], np.float32) if mis else None
        _compare_windows(pb, m)

    check()


def _compare_windows(pb, mis):
    from fastcone_b200 import ops

    a = O.ref_geometry(pb, mis)
    b = ops.reference_windows(_geom(pb, mis))
    assert np.array_equal(b["subVolDim"], a["subVolDim"])
    assert np.array_equal(b["subProjDim"], a["subProjDim"][:2])
    spd2 = int(a["subProjDim"][2])
    nsx, nsy, nsz = (int(v) for v in b["tiles"])
    nsp = a["numSubProblems"] // (nsx * nsy * nsz)
    n = pb.projDim[2]
    tg = np.arange(n)
    pp, t = tg // spd2, tg % spd2
    for kk in range(nsz):
        for jj in range(nsy):
            for ii in range(nsx):
                tile = (kk * nsy + jj) * nsx + ii
                idx_ss = ((kk * nsy + jj) * nsx + ii) * nsp + pp
                o = idx_ss * spd2 + t
                assert np.array_equal(b["ws"][tile], a["wwStart"][o]), (tile, "ws")
                assert np.array_equal(b["hs"][tile], a["hhStart"][o]), (tile, "hs")
                assert np.array_equal(b["sweepStart"][tile], a["sweepStart"][o]), (tile, "sweep")
                assert np.array_equal(b["sweepSteps"][tile], a["sweepNumSteps"][o]), (tile, "steps")


@pytest.mark.parametrize("name,kw", [
    ("quirk", dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5)),
    ("clean", dict(vol_xyz=(48, 48, 48), det_wh=(64, 48), nviews=36, D=200.0, pw=0.5)),
    ("windows", dict(vol_xyz=(64, 56, 40), det_wh=(80, 64), nviews=30, D=180.0, pw=0.7,
                     volStart=(6, 4, 3), volEnd=(58, 50, 37), whsize=(60, 48),
                     woff=np.arange(30) % 5 + 6, hoff=np.arange(30) % 4 + 7)),
])
def test_bp_matters_flag_agrees_with_oracle_difference(name, kw):
    """bp_matters is set exactly when the reference's windowed backprojection (exact
    weights) differs from the ideal one on a random detector."""
    from fastcone_b200 import ops

    pb = O.make_problem(**kw)
    proj = np.random.default_rng(3).random(pb.proj_shape, dtype=np.float32)
    flags = ops.reference_windows(_geom(pb))
    for mode in (2, 0):
        diff = O.rel_l2(O.ref_backproject(pb, proj, kernel_mode=mode, texq=0),
                        O.backproject_f64(pb, proj, kernel_mode=mode))
        assert (diff > 1e-5) == flags["bp_matters"], (mode, diff, flags["bp_matters"])


@pytest.mark.parametrize("kw", [
    dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5),
    dict(vol_xyz=(48, 48, 48), det_wh=(64, 48), nviews=36, D=200.0, pw=0.5),
    dict(vol_xyz=(40, 40, 24), det_wh=(90, 40), nviews=20, D=120.0, pw=0.5),
])
def test_proj_matters_flag_covers_every_difference(kw):
    """proj_matters may be conservative but never misses a case where the reference's
    windows or sweeps change the projection."""
    from fastcone_b200 import ops

    pb = O.make_problem(**kw)
    s, e = pb.volStart, pb.volEnd
    vol = np.random.default_rng(1).random((e[2] - s[2], e[1] - s[1], e[0] - s[0]), dtype=np.float32)
    diff = O.rel_l2(O.ref_project(pb, vol, texq=0), O.project_f64(pb, vol))
    if diff > 1e-5:
        assert ops.reference_windows(_geom(pb))["proj_matters"], diff


def test_flags_never_miss_a_difference_on_random_geometries():
    """Random small geometries: whenever the reference's windows or sweeps change the
    backprojection or the projection (oracle, exact weights), the library's bp_matters /
    proj_matters flag is set, so the reference-compatible kernels run exactly where they
    are needed or more often, never less."""
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies

    from fastcone_b200 import ops

    @hyp.settings(max_examples=30, deadline=None, derandomize=True)
    @hyp.given(vol=st.tuples(st.integers(4, 28), st.integers(4, 28), st.integers(4, 28)),
               det=st.tuples(st.integers(8, 72), st.integers(8, 56)), nviews=st.integers(1, 10),
               D=st.floats(30.0, 300.0), pw=st.floats(0.3, 1.5), seed=st.integers(0, 2 ** 16))
    def check(vol, det, nviews, D, pw, seed):
        pb = O.make_problem(vol, det, nviews, D=D, pw=pw)
        rng = np.random.default_rng(seed)
        flags = ops.reference_windows(_geom(pb))
        proj = rng.random(pb.proj_shape, dtype=np.float32)
        for mode in (2, 0):
            diff = O.rel_l2(O.ref_backproject(pb, proj, kernel_mode=mode, texq=0),
                            O.backproject_f64(pb, proj, kernel_mode=mode))
            assert diff <= 1e-5 or flags["bp_matters"], (mode, diff)
        v = rng.random(vol[::-1], dtype=np.float32)
        diff = O.rel_l2(O.ref_project(pb, v, texq=0), O.project_f64(pb, v))
        assert diff <= 1e-5 or flags["proj_matters"], diff

    check()
