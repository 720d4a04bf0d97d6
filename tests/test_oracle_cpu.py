"""CPU checks of the oracle itself: the geometry/tiling restatement against the reference's
own host code (built from its sources into oracle/_ref), the Python-layer restatements
against golden vectors produced by the reference's fastcone.py, and internal consistency
of the FP64 oracle (adjoint, analytic phantom projections)."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

GEOMETRY_CASES = [
    dict(vol_xyz=(128, 128, 128), det_wh=(192, 128), nviews=180, D=500, pw=0.5),
    dict(vol_xyz=(1024, 1024, 1024), det_wh=(1536, 1024), nviews=1440, D=2000, pw=0.8),
    dict(vol_xyz=(256, 256, 256), det_wh=(384, 256), nviews=360, D=500, pw=1.0),
    dict(vol_xyz=(40, 36, 50), det_wh=(60, 44), nviews=33, D=90, pw=0.9, volStart=(3, 2, 5),
         volEnd=(37, 30, 47)),
    dict(vol_xyz=(64, 64, 64), det_wh=(80, 70), nviews=300, D=200, pw=0.7, whsize=(50, 40),
         woff=np.arange(300) % 7 + 5, hoff=np.arange(300) % 5 + 10),
]


def _helical_case():
    n = 4640
    pb = O.make_problem((512, 512, 384), (736, 64), n, D=1140, pw=1.096)
    pb.hMid[:] = (192 - 160 + np.arange(n) * 80 / 1160).astype(np.float32)
    return pb


@pytest.mark.parametrize("idx", range(len(GEOMETRY_CASES) + 2))
def test_geometry_restatement_matches_reference_host_code(idx):
    """coneBeamGeometry (coneBeamGPU.cu:1360-1849) restated in C vs the reference's own
    compiled class: tiling, detector windows, sweeps and per-view vectors, bit for bit."""
    if O.reflib() is None:
        pytest.skip("oracle/_ref not built (reference sources unavailable at build time)")
    mis = None
    if idx < len(GEOMETRY_CASES):
        pb = O.make_problem(**GEOMETRY_CASES[idx])
    elif idx == len(GEOMETRY_CASES):
        pb = _helical_case()
    else:
        pb = O.make_problem((48, 48, 48), (64, 64), 20, D=150, pw=0.8)
        mis = np.array([1.5, -0.5, 2.0, 0.02, -0.01, 0.03], np.float32)
    a = O.ref_geometry(pb, mis)
    b = O.reflib_geometry(pb, mis)
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_geometry_restatement_matches_reference_on_random_geometries():
    """The same comparison on random volumes, sub-volumes, detectors, data windows,
    distances, pitches, source heights and misalignments."""
    if O.reflib() is None:
        pytest.skip("oracle/_ref not built (reference sources unavailable at build time)")
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies

    @hyp.settings(max_examples=40, deadline=None, derandomize=True)
    @hyp.given(vol=st.tuples(st.integers(4, 120), st.integers(4, 120), st.integers(4, 120)),
               det=st.tuples(st.integers(8, 240), st.integers(8, 200)), nviews=st.integers(1, 60),
               D=st.floats(30.0, 3000.0), pw=st.floats(0.3, 1.6), sub=st.booleans(), win=st.booleans(),
               mis=st.booleans(), seed=st.integers(0, 2 ** 16))
    def check(vol, det, nviews, D, pw, sub, win, mis, seed):
        rng = np.random.default_rng(seed)
        kw = {}
        if sub:
            lo = [int(rng.integers(0, max(1, v // 3))) for v in vol]
            kw.update(volStart=tuple(lo), volEnd=tuple(int(rng.integers(l + 1, v + 1)) for l, v in zip(lo, vol)))
        if win:
            ww, wh = int(rng.integers(4, det[0] + 1)), int(rng.integers(4, det[1] + 1))
            kw.update(whsize=(ww, wh), woff=rng.integers(0, det[0] - ww + 1, nviews),
                      hoff=rng.integers(0, det[1] - wh + 1, nviews))
        pb = O.make_problem(vol, det, nviews, D=D, pw=pw, **kw)
        pb.hMid[:] = (vol[2] / 2 + rng.uniform(-0.3, 0.3, nviews) * vol[2]).astype(np.float32)
        m = (rng.uniform(-1, 1, 6) * np.array([2, 2, 2, 0.03, 0.03, 0.03])).astype(np.float32) if mis else None
        a = O.ref_geometry(pb, m)
        b = O.reflib_geometry(pb, m)
        for k in a:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k

    check()


def test_fp32_exact_weight_path_agrees_with_fp64():
    rng = np.random.default_rng(0)
    pb = O.make_problem((40, 40, 40), (64, 48), 30, D=150, pw=0.6)
    proj = rng.random(pb.proj_shape, dtype=np.float32)
    for mode in (2, 1, 0):
        a = O.ref_backproject(pb, proj, kernel_mode=mode, texq=0)
        b = O.backproject_f64(pb, proj, kernel_mode=mode)
        assert O.rel_l2(a, b) < 2e-5
    vol = rng.random(pb.vol_shape_zyx, dtype=np.float32)
    assert O.rel_l2(O.ref_project(pb, vol, texq=0), O.project_f64(pb, vol)) < 2e-5


def test_points_equal_full_volume():
    rng = np.random.default_rng(1)
    pb = O.make_problem((32, 32, 32), (48, 40), 12, D=100, pw=0.7)
    proj = rng.random(pb.proj_shape, dtype=np.float32)
    pts = rng.integers(0, 32, size=(40, 3)).astype(np.int32)
    full = O.ref_backproject(pb, proj, 2, texq=1)
    assert np.array_equal(O.ref_backproject_points(pb, proj, pts, 2, 1), full[pts[:, 2], pts[:, 1], pts[:, 0]])
    f64 = O.backproject_f64(pb, proj, 2)
    assert np.array_equal(O.backproject_points_f64(pb, proj, pts, 2), f64[pts[:, 2], pts[:, 1], pts[:, 0]])


def test_adjoint_f64_is_transpose():
    rng = np.random.default_rng(2)
    pb = O.make_problem((24, 20, 16), (32, 28), 9, D=80, pw=0.9)
    x = rng.random(pb.vol_shape_zyx, dtype=np.float32)
    y = rng.random(pb.proj_shape, dtype=np.float32)
    lhs = np.sum(O.project_f64(pb, x) * y)
    rhs = np.sum(x * O.project_adjoint_f64(pb, y))
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_projector_f64_known_answer():
    from fastcone_b200.phantom import random_ellipsoids

    pb = O.make_problem((64, 64, 64), (80, 64), 4, D=200, pw=1.0)
    params = random_ellipsoids(4, pb.volDim, 3, axes=(0.2, 0.4), centre_radius=0.45)
    vol = O.phantom_voxelize(pb.volDim, params)
    p = O.project_f64(pb, vol)
    errs, refs = [], []
    for t in range(4):
        ca, sa = math.cos(float(pb.angles[t])), math.sin(float(pb.angles[t]))
        S = np.array([-ca * pb.D, -sa * pb.D, 0.0])
        for hh in range(0, 64, 4):
            for ww in range(0, 80, 4):
                P = np.array([-(ww - 40) * sa, (ww - 40) * ca, hh - 32.0])
                d = (P - S) / np.linalg.norm(P - S)
                refs.append(O.phantom_line_integral(params, S, d))
                errs.append(p[t, hh, ww] - refs[-1])
    # binary voxelisation of 6-13 voxel semi-axes: a few % per ray, no bias
    assert np.linalg.norm(errs) / np.linalg.norm(refs) < 0.05
    assert abs(np.sum(errs)) / np.sum(refs) < 0.01


def test_texture_weights_are_8bit():
    """Emulated texture weights are multiples of 1/256 (CUDA Programming Guide, texture
    fetching: 9-bit fixed point with 8 fractional bits)."""
    pb = O.make_problem((8, 8, 8), (16, 16), 1, D=100, pw=1.0)
    proj = np.zeros(pb.proj_shape, np.float32)
    proj[0, :, 9] = 1.0
    pts = np.array([[4, y, 4] for y in range(8)], np.int32)
    v = O.ref_backproject_points(pb, proj, pts, 0, texq=1)
    # unweighted mode, one view: value = interpolation weight of column 9
    assert np.allclose(v * 256, np.round(v * 256), atol=1e-4)


@pytest.mark.parametrize("name", ["rampfilter_a", "rampfilter_b"])
def test_rampfilter_restatement_matches_reference_golden(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("golden vectors not generated")
    d = np.load(path)
    got = O.rampfilter(d["input"].astype(np.float64))
    assert O.rel_l2(got, d["output"]) < 1e-6


@pytest.mark.parametrize("name,window,scale", [("cosramp_a", "cosramp", 0.125),
                                                ("gaussramp_a", "gaussramp", 0.125),
                                                ("gaussramp_b", "gaussramp", 0.3)])
def test_apodised_ramp_restatement_matches_reference_golden(name, window, scale):
    """cosrampfilter / gaussrampfilter (fastcone.py:294-319), run view by view by the
    reference itself (tests/golden/make_golden.py), against the oracle's restatement."""
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.skip("golden vectors not generated")
    d = np.load(path)
    got = O.apodised_rampfilter(d["input"].astype(np.float64), window, scale)
    assert O.rel_l2(got, d["output"]) < 1e-6


@pytest.mark.parametrize("w", [24, 38, 736, 1536])
@pytest.mark.parametrize("scale", [0.05, 0.125, 0.3])
def test_gauss_window_is_the_shifted_scipy_window_for_even_rows(w, scale):
    """For an even row length the reference's window, scipy.ndimage.shift of a Gaussian by
    -w/2 samples (fastcone.py:310-311), is the closed form the oracle and the library use."""
    import scipy.ndimage
    import scipy.signal

    g = scipy.ndimage.shift(scipy.signal.windows.gaussian(w, scale * w), -0.5 * w)
    want = np.abs(np.fft.fftfreq(w))[: w // 2 + 1] * g[: w // 2 + 1]
    assert np.allclose(O.apodised_ramp_response(w, "gaussramp", scale), want, rtol=0, atol=1e-15)


def test_fbp_weight_restatement_matches_reference_golden():
    path = os.path.join(GOLDEN, "fbp_weight.npz")
    if not os.path.exists(path):
        pytest.skip("golden vectors not generated")
    d = np.load(path)
    w = O.fbp_cosine_weight(d["input"].astype(np.float64), float(d["D"]), d["zOrigin"])
    assert O.rel_l2(w, d["weighted"]) < 1e-7  # golden stored in float32, like the reference
    assert O.rel_l2(O.rampfilter(w), d["filtered"]) < 1e-6


def _fixture(name):
    path = os.path.join(GOLDEN, f"refgpu_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("reference-output fixture missing")
    return np.load(path)


def _compare_fixture(d, arr):
    if "output" in d:
        return O.rel_l2(arr, d["output"])
    s = int(d["sub"])
    assert tuple(arr.shape) == tuple(d["shape"])
    assert abs(arr.sum(dtype=np.float64) - float(d["sum"])) <= 5e-4 * abs(float(d["sum"])) + 1e-3
    return O.rel_l2(arr[::s, ::s, ::s], d["output_sub"])


@pytest.mark.parametrize("name", ["fdk_small", "kats_small", "unw_small", "fdk_windows", "fdk_cfg1",
                                  "proj_small", "proj_cfg1"])
def test_reference_path_matches_reference_gpu_outputs(name):
    """The texture-emulating restatement vs outputs of the reference's own CUDA build
    recorded on a B200 (tests/golden/make_golden_gpu.py).  Bound 5e-4 rel-L2: the 8-bit
    weight rounding is reproduced; the texture unit's remaining internal arithmetic is not
    public."""
    from tests.golden.ref_cases import build_case

    d = _fixture(name)
    pb, proj, vol, kind, mode = build_case(name)
    emu = O.ref_backproject(pb, proj, kernel_mode=mode, texq=1) if kind == "bp" else O.ref_project(pb, vol, texq=1)
    assert _compare_fixture(d, emu) < 5e-4


def test_reference_window_quirk_is_what_the_reference_does():
    """On the 48^3 / 72-pixel case the reference's detector window (16*(1+maxW/16) wide,
    shifted left by 8: coneBeamGPU.cu:1597-1605) ends at column 67 of 72, and clamp
    addressing repeats column 67 beyond it.  The ideal operator differs by ~30%; the
    restatement (with the same windows) reproduces the reference."""
    from tests.golden.ref_cases import build_case

    d = _fixture("fdk_small")
    pb, proj, vol, kind, mode = build_case("fdk_small")
    g = O.ref_geometry(pb)
    assert g["wwStart"][0] + g["subProjDim"][0] < pb.projDim[0]   # window truncates the detector
    ideal = O.backproject_f64(pb, proj, kernel_mode=2)
    assert O.rel_l2(ideal, d["output"]) > 0.1
    assert O.rel_l2(O.ref_backproject(pb, proj, kernel_mode=2, texq=0), d["output"]) < 1e-3


def test_katsevich_oracle_reconstructs_a_phantom():
    """Known answer for the oracle's Katsevich pipeline (Noo-Pack-Heuscher filtering and the
    FP64 PI-window backprojection), independent of the GPU: a seeded ellipsoid phantom,
    projected on a 3-turn helix, is recovered in the central region to the accuracy its
    discretisation allows (rel-L2 <= 0.2, mean within 2 %)."""
    from fastcone_b200.geometry import ConeGeometry
    from fastcone_b200.phantom import random_ellipsoids

    g = ConeGeometry.helical((48, 48, 40), 1.0, (128, 32), 1.0, 150.0, 300.0, 3, 120, 24.0, pi_window=True)
    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid)
    vol = O.phantom_voxelize(g.vol_xyz, random_ellipsoids(4, g.vol_xyz, 5, axes=(0.25, 0.45), centre_radius=0.4))
    proj = O.project_f64(pb, vol).astype(np.float32)
    gF = O.katsevich_filter(proj, g.angles, g.D, g.pw, g.helical_pitch)
    dlam = float(g.angles[-1] - g.angles[0]) / (g.nviews - 1)
    pb.norm[:] = dlam / (2 * math.pi * g.D)
    rec, pairs = O.katsevich_piwin_f64(pb, gF.astype(np.float32), g.helical_pitch)
    c = (slice(12, 28), slice(10, 38), slice(10, 38))
    assert O.rel_l2(rec[c], vol[c]) < 0.2, O.rel_l2(rec[c], vol[c])
    assert abs(rec[c].mean() / vol[c].mean() - 1.0) < 0.02
    assert 0 < pairs < vol.size * g.nviews


def test_fdk_oracle_reconstructs_a_phantom():
    """Known answer for the oracle's FDK chain (the fbp cosine weight and ramp filter of
    fastcone.py:260-292, then the FDK backprojection with norm 1/nviews): a seeded ellipsoid
    phantom is recovered near the mid-plane, where the circular orbit's data are complete
    (rel-L2 <= 0.2, mean within 3 %)."""
    from fastcone_b200.phantom import random_ellipsoids

    n, pw = 180, 0.8
    pa = O.make_problem((48, 48, 32), (96, 48), n, D=400.0, pw=pw, norm=np.ones(n, np.float32))
    pb = O.make_problem((48, 48, 32), (96, 48), n, D=400.0, pw=pw, norm=np.full(n, 1.0 / n, np.float32))
    vol = O.phantom_voxelize((48, 48, 32), random_ellipsoids(4, (48, 48, 32), 3, axes=(0.25, 0.45),
                                                             centre_radius=0.4))
    proj = O.project_f64(pa, vol)
    filt = O.rampfilter(O.fbp_cosine_weight(proj, pb.D, pb.hMid)).astype(np.float32)
    # the reference's FDK result is pw times the attenuation (its filter works in pixels)
    rec = O.backproject_f64(pb, filt, kernel_mode=2) / pw
    c = (slice(12, 20), slice(10, 38), slice(10, 38))
    assert O.rel_l2(rec[c], vol[c]) < 0.2, O.rel_l2(rec[c], vol[c])
    assert abs(rec[c].mean() / vol[c].mean() - 1.0) < 0.03, rec[c].mean() / vol[c].mean()


def test_piwin_points_equal_whole_volume_oracle():
    """The FP64 PI-window backprojection at listed voxels (katsevich_piwin_points_f64, used on
    sampled columns at the full helical size) equals the whole-volume function at those voxels,
    values and in-window pair counts alike; column_points lists whole z columns."""
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.helical((20, 18, 16), 1.0, (40, 12), 1.0, 60.0, 120.0, 2, 40, 8.0, pi_window=True)
    pb = O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid)
    proj = np.random.default_rng(2).random(g.proj_shape, dtype=np.float32)
    vol, pairs = O.katsevich_piwin_f64(pb, proj, g.helical_pitch)
    pts = O.column_points(g.vol_xyz, (0, 0, 0), g.vol_xyz, 5, seed=3)
    assert pts.shape == (5 * 16, 3) and np.array_equal(pts[:16, 2], np.arange(16))
    got, npairs = O.katsevich_piwin_points_f64(pb, proj, pts, g.helical_pitch)
    want = vol[pts[:, 2], pts[:, 1], pts[:, 0]]
    assert np.array_equal(got, want)
    # every voxel listed once: the pair counts add up to the whole volume's
    allpts = np.stack(np.meshgrid(np.arange(20), np.arange(18), np.arange(16), indexing="ij"), -1).reshape(-1, 3)
    _, allpairs = O.katsevich_piwin_points_f64(pb, proj, allpts.astype(np.int32), g.helical_pitch)
    assert allpairs == pairs and 0 < npairs < pairs
