"""The slab decomposition with the library's kernels: several ranks' steps driven in one
process on one GPU (pack -> hand the pieces over -> unpack -> single-GPU kernels on the band
geometry), assembled and compared with the FP64 oracle's whole-volume backprojection
(rel-L2 <= 2e-5, FP32 arithmetic; for the helix the PI-window Katsevich backprojection at
<= 1e-3: the window is a sharp cut that the kernels decide in FP32 and the oracle in FP64,
so voxels whose window edge falls within rounding of a view gain or lose that view) and with
the whole-volume kernels' result (<= 1e-6: the same kernels on the same data).  No rank waits
on another (the exchange is a list hand-over), so this runs on one GPU."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _geoms():
    from fastcone_b200.geometry import ConeGeometry

    circ = ConeGeometry((96, 80, 128), (160, 120), np.linspace(0, 2 * np.pi, 90, endpoint=False), 300.0, 0.9)
    hel = ConeGeometry.helical((64, 64, 96), 0.5, (96, 16), 1.0, 80.0, 140.0, 3, 60, 12.0, pi_window=True)
    return {"circular": circ, "helical": hel}


def _emulate_backproject(dec, proj, mode):
    import torch

    from fastcone_b200 import ops, slabs

    sent = [slabs.pack_backproject(dec, r, proj[slice(*dec.views(r))].contiguous()) for r in range(dec.world)]
    out = []
    for d in range(dec.world):
        vol = torch.zeros(dec.slab_shape(d), device="cuda")
        band = slabs.unpack_backproject(dec, d, [sent[s][d] for s in range(dec.world)])
        g = dec.band_geometry(d)
        if band is not None and g is not None:
            ops.backproject(band, g, mode, vol)
        out.append(vol)
    return torch.cat(out, 0)


@pytest.mark.parametrize("kind,mode", [("circular", 2), ("circular", 0), ("helical", 1)])
@pytest.mark.parametrize("world", [2, 3, 5])
def test_slab_backprojection_equals_whole_volume(kind, mode, world):
    import torch

    from fastcone_b200 import ops, slabs

    import bench

    g = _geoms()[kind]
    proj = torch.rand(g.proj_shape, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    want = ops.backproject(proj, g, mode)
    dec = slabs.SlabDecomposition(g, world)
    got = _emulate_backproject(dec, proj, mode).cpu().numpy()
    torch.cuda.synchronize()
    assert O.rel_l2(got, want.cpu().numpy()) < 1e-6
    pb, ph = bench.oracle_problem(g), proj.cpu().numpy()
    if kind == "helical":
        ref, _ = O.katsevich_piwin_f64(pb, ph, g.helical_pitch)
        tol = 1e-3
    else:
        ref = O.backproject_f64(pb, ph, kernel_mode=mode)
        tol = 2e-5
    assert O.rel_l2(got, ref) < tol, O.rel_l2(got, ref)
    if kind == "helical":
        assert all(len(b.views) < g.nviews for b in dec.bands if b.z1 > b.z0)


def test_slab_backprojection_moves_bf16_rows():
    """BF16-stored projections travel as BF16 and give the whole-volume BF16 result."""
    import torch

    from fastcone_b200 import ops, slabs

    g = _geoms()["circular"]
    proj = torch.rand(g.proj_shape, device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    p16 = proj.to(torch.bfloat16)
    want = ops.backproject(p16, g, 2)
    dec = slabs.SlabDecomposition(g, 3)
    got = _emulate_backproject(dec, p16, 2)
    torch.cuda.synchronize()
    assert O.rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("kind", ["circular", "helical"])
@pytest.mark.parametrize("world", [2, 3])
def test_slab_projection_equals_whole_volume(kind, world):
    import torch

    from fastcone_b200 import _lib, ops, slabs

    g = _geoms()[kind]
    vol = torch.rand(g.vol_shape, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    want = ops.project(vol, g, _lib.PROJ_EXPLICIT)
    dec = slabs.SlabDecomposition(g, world)
    zs = g.vol_start[2]
    sent = []
    for d in range(world):
        z0, z1 = dec.slab(d)
        bg = dec.band_geometry(d)
        band = None
        if bg is not None:
            band = ops.project(vol[z0 - zs:z1 - zs].contiguous(), bg, _lib.PROJ_EXPLICIT)
        sent.append(slabs.pack_project(dec, d, band)[0])
    parts = []
    for s in range(world):
        v0, v1 = dec.views(s)
        p = torch.zeros((v1 - v0,) + g.proj_shape[1:], device="cuda")
        parts.append(slabs.unpack_project(dec, s, [sent[d][s] for d in range(world)], p))
    got = torch.cat(parts, 0)
    torch.cuda.synchronize()
    assert O.rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-5
