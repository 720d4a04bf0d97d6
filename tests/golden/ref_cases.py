"""Deterministic inputs for the reference-output fixtures (refgpu_*.npz).

Each case: geometry in the reference ABI's units, a seeded ellipsoid phantom voxelised by
the oracle, and (for backprojection) its FP64 projections, cosine-weighted and ramp
filtered as fastcone.fbp does.  Everything here is CPU-only and seeded, so the inputs can
be rebuilt anywhere from this file.
"""
import numpy as np

from oracle import oracle as O

CASES = {
    # name: (problem kwargs, kind, kernelMode)
    "fdk_small": (dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5), "bp", 2),
    "kats_small": (dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5), "bp", 1),
    "unw_small": (dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5), "bp", 0),
    "fdk_windows": (dict(vol_xyz=(64, 56, 40), det_wh=(80, 64), nviews=30, D=180.0, pw=0.7,
                         volStart=(6, 4, 3), volEnd=(58, 50, 37), whsize=(60, 48),
                         woff=np.arange(30) % 5 + 6, hoff=np.arange(30) % 4 + 7), "bp", 2),
    "fdk_cfg1": (dict(vol_xyz=(128, 128, 128), det_wh=(192, 128), nviews=180, D=500.0, pw=0.5), "bp", 2),
    "proj_small": (dict(vol_xyz=(48, 48, 48), det_wh=(72, 48), nviews=36, D=200.0, pw=0.5), "proj", None),
    "proj_cfg1": (dict(vol_xyz=(128, 128, 128), det_wh=(192, 128), nviews=180, D=500.0, pw=0.5), "proj", None),
}


def build_case(name):
    from fastcone_b200.phantom import random_ellipsoids

    kw, kind, mode = CASES[name]
    kw = dict(kw)
    pb = O.make_problem(**kw)
    if kind == "bp":
        pb.norm[:] = 1.0 / pb.projDim[2]
    params = random_ellipsoids(10, pb.volDim, seed=sum(map(ord, name)))
    vol = O.phantom_voxelize(pb.volDim, params)
    e, s = pb.volEnd, pb.volStart
    vol_sub = np.ascontiguousarray(vol[s[2]:e[2], s[1]:e[1], s[0]:e[0]])
    proj = None
    if kind == "bp":
        full = O.make_problem(kw["vol_xyz"], kw["det_wh"], kw["nviews"], D=kw["D"], pw=kw["pw"],
                              woff=kw.get("woff"), hoff=kw.get("hoff"), whsize=kw.get("whsize"))
        p = O.project_f64(full, vol)
        proj = O.rampfilter(O.fbp_cosine_weight(p, pb.D, pb.hMid)).astype(np.float32)
    return pb, proj, vol_sub, kind, mode
