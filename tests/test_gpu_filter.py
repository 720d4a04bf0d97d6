"""GPU FDK pre-processing (cosine weight + ramp / Shepp-Logan filter, the unpadded cosine /
Gaussian apodised ramps) and phantom voxelisation vs the CPU restatements."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("window", ["ramlak", "shepplogan"])
@pytest.mark.parametrize("shape", [(5, 16, 24), (3, 7, 33), (2, 64, 192)])
def test_filter_vs_numpy(window, shape):
    import torch

    from fastcone_b200 import _lib, ops

    rng = np.random.default_rng(0)
    proj = rng.standard_normal(shape).astype(np.float32)
    zorig = (shape[1] / 2 + rng.random(shape[0])).astype(np.float32)
    D = 120.0
    want = O.rampfilter(O.fbp_cosine_weight(proj.astype(np.float64), D, zorig), window=window)
    win = _lib.FILTER_RAMLAK if window == "ramlak" else _lib.FILTER_SHEPPLOGAN
    got = ops.fdk_filter(torch.from_numpy(proj).cuda(), zorigin=zorig, D=D, window=win).cpu().numpy()
    assert O.rel_l2(got, want) < 1e-5
    got16 = ops.fdk_filter(torch.from_numpy(proj).cuda(), zorigin=zorig, D=D, window=win,
                           out_dtype=torch.bfloat16).float().cpu().numpy()
    assert O.rel_l2(got16, want) < 5e-3


def test_rampfilter_api_inplace():
    from fastcone_b200 import fastcone as fc

    proj = np.random.default_rng(1).random((4, 12, 20), dtype=np.float32)
    want = O.rampfilter(proj.astype(np.float64))
    fc.rampfilter(proj)
    assert O.rel_l2(proj, want) < 1e-5


@pytest.mark.parametrize("window,scale", [("cosramp", 0.125), ("gaussramp", 0.125), ("gaussramp", 0.3),
                                          ("gaussramp", 0.05)])
@pytest.mark.parametrize("shape", [(5, 16, 24), (3, 7, 33), (2, 64, 192), (2, 3, 736)])
def test_apodised_filter_vs_oracle(window, scale, shape):
    import torch

    from fastcone_b200 import _lib, ops

    rng = np.random.default_rng(4)
    proj = rng.standard_normal(shape).astype(np.float32)
    want = O.apodised_rampfilter(proj.astype(np.float64), window, scale)
    win = _lib.FILTER_COSRAMP if window == "cosramp" else _lib.FILTER_GAUSSRAMP
    for dt, tol in ((torch.float32, 1e-5), (torch.bfloat16, 5e-3)):
        plan = ops.FilterPlan(shape, out_dtype=dt, window=win, gauss_scale=scale)
        got = plan(torch.from_numpy(proj).cuda(), cosine_weight=False).float().cpu().numpy()
        assert O.rel_l2(got, want) < tol, (dt, O.rel_l2(got, want))


@pytest.mark.parametrize("fn,window,kw", [("cosrampfilter", "cosramp", {}),
                                          ("gaussrampfilter", "gaussramp", {}),
                                          ("gaussrampfilter", "gaussramp", {"scale": 0.2})])
def test_apodised_api_inplace(fn, window, kw):
    """fastcone.cosrampfilter / gaussrampfilter filter every view in place."""
    from fastcone_b200 import fastcone as fc

    proj = np.random.default_rng(6).random((4, 12, 20), dtype=np.float32)
    want = O.apodised_rampfilter(proj.astype(np.float64), window, kw.get("scale", 0.125))
    getattr(fc, fn)(proj, **kw)
    assert O.rel_l2(proj, want) < 1e-5


def test_phantom_matches_oracle():
    from fastcone_b200 import ops
    from fastcone_b200.phantom import random_ellipsoids

    params = random_ellipsoids(12, (40, 36, 30), seed=5)
    got = ops.phantom((40, 36, 30), params).cpu().numpy()
    want = O.phantom_voxelize((40, 36, 30), params)
    assert np.array_equal(got, want)


def test_filter_plan_equals_one_shot():
    """The reusable filter plan gives the one-shot filter's result, call after call, for
    FP32 and BF16 output, ramp and Shepp-Logan, with and without the cosine weight."""
    import numpy as np
    import torch

    from fastcone_b200 import _lib, ops

    gen = torch.Generator(device="cuda").manual_seed(2)
    p = torch.randn((7, 13, 40), device="cuda", generator=gen)
    z = np.linspace(3.0, 9.0, 7).astype(np.float32)
    for dt in (torch.float32, torch.bfloat16):
        for win in (_lib.FILTER_RAMLAK, _lib.FILTER_SHEPPLOGAN):
            plan = ops.FilterPlan(p.shape, out_dtype=dt, window=win)
            for cw in (True, False):
                ref = ops.fdk_filter(p, out_dtype=dt, window=win, cosine_weight=cw, zorigin=z, D=55.0)
                for _ in range(2):
                    got = plan(p, zorigin=z, D=55.0, cosine_weight=cw)
                    torch.cuda.synchronize()
                    assert torch.equal(got, ref)


@pytest.mark.parametrize("window", ["ramlak", "shepplogan"])
@pytest.mark.parametrize("case", [
    dict(vol=(40, 36, 32), det=(64, 48), n=45, pw=0.75),     # rows a multiple of 16 bytes
    dict(vol=(33, 30, 27), det=(71, 48), n=250, pw=0.8),     # odd width (padded rows), 3 view chunks
])
def test_fbp_host_pipeline_vs_oracle(window, case):
    """fastcone.fbp (one fcb_fbp_host call: upload, cosine weight + ramp filter on the GPU,
    filtered views back into proj, FDK backprojection with norm 1/nviews) vs the oracle's
    chain (fastcone.py:260-292 restated in numpy FP64, then the FP64 backprojection): the
    filtered projections <= 1e-5 and the volume <= 2e-5 rel-L2."""
    from fastcone_b200 import fastcone as fc
    from tests._cases import make_case, smooth_projections

    nx, ny, nz = case["vol"]
    g, pb = make_case(vol_xyz=case["vol"], det_wh=case["det"], nviews=case["n"], D=130.0, pw=case["pw"],
                      norm=np.full(case["n"], 1.0 / case["n"], np.float32))
    proj, _ = smooth_projections(pb)
    zorig = pb.hMid
    D = 130.0
    filt = O.rampfilter(O.fbp_cosine_weight(proj.astype(np.float64), D, zorig), window=window)
    want = O.backproject_f64(pb, filt.astype(np.float32), kernel_mode=2)
    vol = np.zeros((nz, ny, nx), np.float32)
    p = proj.copy()
    fc.fbp(vol, p, pb.angles, D, zorig, pixelWidth=case["pw"], window=window)
    assert O.rel_l2(p, filt) < 1e-5, O.rel_l2(p, filt)
    assert O.rel_l2(vol, want) < 2e-5, O.rel_l2(vol, want)


def test_fbp_host_kept_filter_plans(monkeypatch):
    """fcb_fbp_host keeps its filter plans between calls (keyed by views per chunk, detector
    size and window): repeated calls, a call with another window in between, and calls with
    the cache released or switched off give the same volume and filtered views."""
    from fastcone_b200 import _lib
    from fastcone_b200 import fastcone as fc
    from tests._cases import make_case, smooth_projections

    # a detector that covers the volume's shadow: the reference's sub-problem windows (which
    # fastcone.fbp reproduces) then equal the ideal operator the oracle computes
    g, pb = make_case(vol_xyz=(40, 36, 32), det_wh=(64, 48), nviews=130, D=130.0, pw=0.75,
                      norm=np.full(130, 1.0 / 130, np.float32))
    proj, _ = smooth_projections(pb)

    def run(window):
        vol = np.zeros((32, 36, 40), np.float32)
        p = proj.copy()
        fc.fbp(vol, p, pb.angles, 130.0, pb.hMid, pixelWidth=0.75, window=window)
        return vol, p

    first = run("shepplogan")
    ramp = run("ramlak")
    again = run("shepplogan")
    _lib.check(_lib.lib().fcb_release_device_cache())
    released = run("shepplogan")
    monkeypatch.setenv("FCB_HOST_CACHE", "0")
    uncached = run("shepplogan")
    for v, p in (again, released, uncached):
        assert np.array_equal(v, first[0]) and np.array_equal(p, first[1])
    assert not np.array_equal(ramp[0], first[0])
    want = O.backproject_f64(pb, O.rampfilter(O.fbp_cosine_weight(proj.astype(np.float64), 130.0, pb.hMid),
                                              window="shepplogan").astype(np.float32), kernel_mode=2)
    assert O.rel_l2(first[0], want) < 2e-5
