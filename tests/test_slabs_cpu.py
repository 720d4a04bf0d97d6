"""One volume split into z-slabs over ranks (fastcone_b200.slabs, the replacement for
mpi_fastcone.project / backproject): the decomposition, the detector-row bands, and the
all-to-all exchange run by 2 and 3 gloo ranks on CPU.  Each rank's single-device operator is
the FP64 oracle here (the GPU kernels take its place in tests/test_gpu_slabs.py), so the
assembled slabs and view runs must equal the oracle's whole-volume result: a band that
missed a row a slab reads, or a piece sent to the wrong rank, shows up as a difference."""
import os
import socket

import numpy as np
import pytest

from oracle import oracle as O


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _geom(kind="circular"):
    from fastcone_b200.geometry import ConeGeometry

    if kind == "circular":
        return ConeGeometry((24, 20, 40), (40, 34), np.linspace(0, 2 * np.pi, 18, endpoint=False), 60.0, 0.8)
    if kind == "subvolume":
        return ConeGeometry((28, 24, 48), (44, 40), np.linspace(0, 2 * np.pi, 14, endpoint=False), 70.0, 0.9,
                            vol_start=(2, 3, 5), vol_end=(26, 21, 45), norm=np.linspace(0.5, 1.5, 14))
    # helical: the source rises through the volume, so most views reach only some slabs
    n = 40
    return ConeGeometry((20, 20, 48), (36, 12), np.arange(n) * (2 * np.pi / 20), 50.0, 0.9,
                        hmid=np.linspace(4.0, 44.0, n))


def _pb(g):
    return O.make_problem(g.vol_xyz, g.det_wh, g.nviews, g.D, g.pw, hmid=g.hmid, angles=g.angles, norm=g.norm,
                          volStart=g.vol_start, volEnd=g.vol_end, woff=g.woff, hoff=g.hoff, whsize=g.window_wh)


def _oracle_bp(band, g, mode, vol):
    import torch

    vol += torch.from_numpy(O.backproject_f64(_pb(g), band.numpy().astype(np.float32), kernel_mode=mode)
                            .astype(np.float32))
    return vol


def _oracle_proj(vol, g, method, proj):
    import torch

    proj += torch.from_numpy(O.project_f64(_pb(g), vol.numpy()).astype(np.float32))
    return proj


def _inputs(g):
    rng = np.random.default_rng(11)
    proj = rng.random(g.proj_shape, dtype=np.float32)
    vol = rng.random(g.vol_shape, dtype=np.float32)
    return proj, vol


def _worker(rank, world, port, kind, align, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as tdist

    from fastcone_b200 import dist as fd
    from fastcone_b200 import slabs

    fd.init("gloo", timeout_s=60)
    g = _geom(kind)
    proj, vol = _inputs(g)
    dec = slabs.SlabDecomposition(g, world, align=align)
    v0, v1 = dec.views(rank)
    z0, z1 = dec.slab(rank)
    zs = g.vol_start[2]
    res = {}
    for mode in (2, 0):
        got = slabs.backproject(torch.from_numpy(proj[v0:v1].copy()), dec, rank, mode=mode, local_op=_oracle_bp)
        want = O.backproject_f64(_pb(g), proj, kernel_mode=mode)[z0 - zs:z1 - zs]
        res[f"bp{mode}"] = (O.rel_l2(got.numpy(), want) if want.size else 0.0, got.shape == want.shape)
    got = slabs.project(torch.from_numpy(vol[z0 - zs:z1 - zs].copy()), dec, rank, local_op=_oracle_proj)
    want = O.project_f64(_pb(g), vol)[v0:v1]
    res["proj"] = (O.rel_l2(got.numpy(), want), got.shape == want.shape)
    tdist.barrier()
    out.put((rank, res))
    tdist.destroy_process_group()


@pytest.mark.parametrize("world,kind,align", [(2, "circular", 8), (3, "subvolume", 8), (3, "helical", 8),
                                              (2, "helical", 32)])
def test_gloo_ranks_assemble_the_whole_volume_result(world, kind, align):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, align, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, r in res:
        for key, (err, shape_ok) in r.items():
            assert shape_ok, (rank, key)
            assert err < 1e-6, (rank, key, err)


@pytest.mark.parametrize("kind", ["circular", "subvolume", "helical"])
@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_decomposition_covers_volume_and_views(kind, world):
    from fastcone_b200 import slabs

    g = _geom(kind)
    dec = slabs.SlabDecomposition(g, world, align=8)
    zs, ze = g.vol_start[2], g.vol_end[2]
    planes, views = [], []
    for r in range(world):
        z0, z1 = dec.slab(r)
        planes.extend(range(z0, z1))
        views.extend(range(*dec.views(r)))
        b = dec.bands[r]
        assert b.rows <= g.det_wh[1]
        assert np.all(b.lo >= 0) and np.all(b.lo + b.rows <= g.det_wh[1])
        # what rank s sends r in a backprojection is what r sends s in a projection
        assert sum(dec.split_sizes(s, r) for s in range(world)) == len(b.views) * b.rows * g.det_wh[0]
    assert planes == list(range(zs, ze))
    assert views == list(range(g.nviews))


def test_helical_slabs_receive_only_the_views_that_reach_them():
    """On the helix each slab's band list holds only the views whose footprint reaches
    it; the exchange moves far less than every view to every rank."""
    from fastcone_b200 import slabs

    g = _geom("helical")
    dec = slabs.SlabDecomposition(g, 3, align=8)
    moved = sum(dec.split_sizes(s, r) for s in range(3) for r in range(3))
    everything = 3 * g.nviews * g.det_wh[1] * g.det_wh[0]
    assert all(len(b.views) < g.nviews for b in dec.bands)
    assert moved < 0.7 * everything


def test_detector_rows_bound_the_voxel_footprints():
    """Every voxel centre of a slab projects strictly inside its view's band (FP64
    projective map of the oracle's geometry), with the margin to spare."""
    from fastcone_b200 import slabs
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry((16, 16, 32), (30, 26), np.linspace(0, 2 * np.pi, 9, endpoint=False), 40.0, 0.7,
                     vol_start=(0, 0, 10), vol_end=(16, 16, 18))
    lo, hi = slabs.detector_rows(g, margin=0)
    zz, yy, xx = np.meshgrid(np.arange(10, 18), np.arange(16), np.arange(16), indexing="ij")
    pts = np.stack([xx.ravel() - 8.0, yy.ravel() - 8.0, zz.ravel() - 16.0], 1)
    for t in range(g.nviews):
        a = float(g.angles[t])
        ca, sa = np.cos(a), np.sin(a)
        src = np.array([-ca * g.D, -sa * g.D, float(g.hmid[t]) - 16.0])
        ray = pts - src
        depth = ray @ np.array([ca, sa, 0.0])
        s = g.D / depth  # magnification onto the detector plane through the axis
        h = (src[2] + ray[:, 2] * s) / g.pw + g.det_wh[1] // 2
        assert lo[t] <= np.floor(h.min()) and np.floor(h.max()) + 1 < hi[t], t


def test_windowed_or_reference_geometries_are_refused():
    from fastcone_b200 import slabs
    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry((8, 8, 8), (10, 10), np.zeros(2), 30.0, 1.0, window_wh=(10, 6), hoff=np.array([1, 2]))
    with pytest.raises(ValueError):
        slabs.SlabDecomposition(g, 2)
    g = ConeGeometry((8, 8, 8), (10, 10), np.zeros(2), 30.0, 1.0, reference_windows=True)
    with pytest.raises(ValueError):
        slabs.SlabDecomposition(g, 2)


def _footprint_rows(g, t, z0, z1):
    """Floor of the lowest and highest detector row that the voxel centres of planes
    [z0, z1) reach in view t (FP64 projective map; the 8 corners of the slab's box bound the
    rows, since h is monotone in z and in the in-plane depth)."""
    zc = g.vol_xyz[2] // 2
    xs = np.array([g.vol_start[0], g.vol_end[0] - 1], float) - g.vol_xyz[0] // 2
    ys = np.array([g.vol_start[1], g.vol_end[1] - 1], float) - g.vol_xyz[1] // 2
    zs = np.array([z0, z1 - 1], float) - zc
    a = float(g.angles[t])
    ca, sa = np.cos(a), np.sin(a)
    src_z = float(g.hmid[t]) - zc
    hs = []
    for x in xs:
        for y in ys:
            depth = g.D + x * ca + y * sa
            for z in zs:
                # the detector centre rides with the source (row H // 2 at the source's height)
                hs.append((z - src_z) * g.D / depth / g.pw + g.det_wh[1] // 2)
    return np.floor(min(hs)), np.floor(max(hs))


def test_decomposition_properties_on_random_geometries():
    """Random circular and helical geometries, sub-volumes and world sizes (more ranks than
    z tiles included): the slabs partition the sub-volume's planes in rank order in multiples
    of the alignment, the view runs partition the views, every band lies on the detector,
    both directions of the exchange agree in size, and every view a slab keeps covers the
    rows its voxels reach."""
    hyp = pytest.importorskip("hypothesis")
    st = hyp.strategies

    from fastcone_b200 import slabs
    from fastcone_b200.geometry import ConeGeometry

    @hyp.settings(max_examples=40, deadline=None, derandomize=True)
    @hyp.given(nx=st.integers(4, 24), nz=st.integers(1, 70), zlo=st.integers(0, 10), nviews=st.integers(1, 24),
               world=st.integers(1, 7), align=st.sampled_from([1, 8, 32]), helical=st.booleans(),
               D=st.floats(40.0, 400.0), pw=st.floats(0.5, 1.5))
    def check(nx, nz, zlo, nviews, world, align, helical, D, pw):
        nzv = nz + zlo + 3
        H = int(np.ceil(nzv * 1.6 / pw)) + 4
        W = int(np.ceil(nx * 2.2 / pw)) + 4
        angles = np.arange(nviews) * (2 * np.pi / max(1, min(nviews, 12)))
        hmid = np.linspace(0.0, nzv, nviews) if helical else None
        g = ConeGeometry((nx, nx, nzv), (W, H), angles, D, pw, hmid=hmid, vol_start=(0, 0, zlo),
                         vol_end=(nx, nx, zlo + nz))
        dec = slabs.SlabDecomposition(g, world, align=align)
        planes, views = [], []
        for r in range(world):
            z0, z1 = dec.slab(r)
            assert (z0 - zlo) % align == 0 or z0 == z1
            planes.extend(range(z0, z1))
            views.extend(range(*dec.views(r)))
            b = dec.bands[r]
            assert np.all(b.lo >= 0) and np.all(b.lo + b.rows <= H)
            assert sum(dec.split_sizes(s, r) for s in range(world)) == len(b.views) * b.rows * W
            for i, t in enumerate(b.views):
                lo, hi = _footprint_rows(g, int(t), z0, z1)
                # rows the bilinear taps read: floor(h) and floor(h) + 1, clipped to the detector
                need_lo, need_hi = max(0.0, lo), min(H - 1.0, hi + 1)
                if need_lo <= need_hi:
                    assert b.lo[i] <= need_lo and need_hi < b.lo[i] + b.rows, (r, t)
        assert planes == list(range(zlo, zlo + nz))
        assert views == list(range(nviews))

    check()
