"""One volume over several GPUs: z-slab ownership with the views spread over the ranks -- the
replacement for mpi_fastcone.project / backproject (mpi_fastcone.py:371-526).

Each of ``world`` ranks owns a z-slab of the volume (whole xy planes, like mpi_fastcone's
volume chunks) and a contiguous run of views (its projection images).  A slab needs, of
each view, only the detector rows its interpolation support projects to
(``fcb_detector_rows``, FP64), so

* ``backproject``: every rank sends every other rank those rows of its own views in one
  all-to-all (NCCL over NVLink between GPUs; views a slab never reaches are not sent), then
  backprojects its slab from that windowed projection set (per-view window offset = the
  band's first row) with the single-GPU kernels;
* ``project``: every rank projects its slab onto the same per-view row bands (projection is
  linear in the volume, and the kernels sample a sub-volume exactly as its zero-extended
  volume), sends each band back to the view's owner in the reverse all-to-all, and the
  owners add them in rank order.

mpi_fastcone moves per-chunk detector windows with point-to-point pickled messages in loops
ordered to avoid deadlock (mpi_fastcone.py:379-447, :458-526); here one collective per call
moves them, and the bands are the rows each slab reads rather than whole chunk windows.
Every rank computes the whole decomposition itself from the same FP64 geometry, so all
ranks agree on every message size without exchanging them.

The steps are separate functions (``pack_*`` / ``unpack_*``) so that a test can drive
several ranks' steps in one process; ``backproject`` / ``project`` chain them around
``torch.distributed.all_to_all_single``.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .dist import z_slab
from .geometry import ConeGeometry


@dataclasses.dataclass
class _Band:
    z0: int
    z1: int
    views: np.ndarray   # global indices of the views whose footprint reaches the slab
    lo: np.ndarray      # first detector row of each of those views' bands
    rows: int           # band height (the same for every view of this slab)


class SlabDecomposition:
    """z-slabs and view runs of ``geom`` over ``world`` ranks, and the row band each slab
    needs from each view.

    ``geom`` must address the whole detector (no per-view windows) and must not use the
    reference's sub-problem windows.  Slabs are multiples of ``align`` planes (the
    backprojector's z tile) except the last; views are split into ``world`` contiguous runs
    of nearly equal length.
    """

    def __init__(self, geom: ConeGeometry, world: int, align: int = 32, margin: int = 1):
        if world < 1:
            raise ValueError("world must be >= 1")
        W, H = (int(v) for v in geom.det_wh)
        if tuple(geom.window_wh) != (W, H) or np.any(geom.woff) or np.any(geom.hoff):
            raise ValueError("the slab decomposition needs whole-detector projections (no windows)")
        if geom.reference_windows:
            raise ValueError("the reference's sub-problem windows do not split into slabs")
        self.geom, self.world, self.W, self.H = geom, int(world), W, H
        n = geom.nviews
        cuts = [(n * r) // world for r in range(world + 1)]
        self.view_runs = [(cuts[r], cuts[r + 1]) for r in range(world)]
        zs, ze = int(geom.vol_start[2]), int(geom.vol_end[2])
        self.bands = []
        for r in range(world):
            a, b = z_slab(ze - zs, world, r, align)
            z0, z1 = zs + a, zs + b
            if z1 <= z0:
                self.bands.append(_Band(z0, z0, np.zeros(0, np.int64), np.zeros(0, np.int64), 0))
                continue
            lo, hi = detector_rows(dataclasses.replace(geom, vol_start=(geom.vol_start[0], geom.vol_start[1], z0),
                                                       vol_end=(geom.vol_end[0], geom.vol_end[1], z1)), margin)
            act = np.nonzero(hi > lo)[0]
            if geom.pi_window and len(act) == 1 and geom.nviews > 1:
                # the kernels read the helix's handedness from the first and last view of a
                # set; a neighbour that misses the slab adds nothing but that direction
                v = act[0]
                nb = v + 1 if v + 1 < geom.nviews else v - 1
                lo[nb], hi[nb] = lo[v], lo[v] + 1
                act = np.sort(np.array([v, nb]))
            rows = int((hi[act] - lo[act]).max()) if len(act) else 0
            # one band height per slab: widen short bands (real rows, kept inside the detector)
            l = np.clip(lo[act], 0, H - rows).astype(np.int64)
            self.bands.append(_Band(z0, z1, act.astype(np.int64), l, rows))

    # ----------------------------------------------------------------- layout
    def slab(self, r: int):
        """[z0, z1) of rank r's slab in the global grid."""
        return self.bands[r].z0, self.bands[r].z1

    def views(self, r: int):
        """[v0, v1) of the views rank r holds."""
        return self.view_runs[r]

    def slab_shape(self, r: int):
        z0, z1 = self.slab(r)
        g = self.geom
        return (z1 - z0, g.vol_end[1] - g.vol_start[1], g.vol_end[0] - g.vol_start[0])

    def band_geometry(self, r: int) -> ConeGeometry | None:
        """The geometry rank r computes with: its slab, the views that reach it, each as a
        window of ``rows`` detector rows starting at the band's first row; None when the
        slab is empty or no view reaches it."""
        b, g = self.bands[r], self.geom
        if b.z1 <= b.z0 or len(b.views) == 0:
            return None
        v = b.views
        return dataclasses.replace(
            g, angles=g.angles[v], hmid=g.hmid[v], norm=g.norm[v], woff=np.zeros(len(v), np.int32),
            hoff=b.lo.astype(np.int32), window_wh=(self.W, b.rows),
            vol_start=(g.vol_start[0], g.vol_start[1], b.z0), vol_end=(g.vol_end[0], g.vol_end[1], b.z1))

    def _sel(self, src: int, dst: int):
        """Positions, within dst's band list, of the views src holds."""
        v0, v1 = self.view_runs[src]
        vv = self.bands[dst].views
        return np.nonzero((vv >= v0) & (vv < v1))[0]

    def split_sizes(self, src: int, dst: int) -> int:
        """Elements src sends dst in a backprojection (dst sends src in a projection)."""
        return len(self._sel(src, dst)) * self.bands[dst].rows * self.W


def detector_rows(geom: ConeGeometry, margin: int = 1):
    """Per view, the global detector rows [lo, hi) ``geom``'s sub-volume projects to
    (``fcb_detector_rows``); lo == hi where it misses the detector."""
    n = geom.nviews
    lo, hi = np.zeros(n, np.int32), np.zeros(n, np.int32)
    g = geom.struct()
    _lib.check(_lib.lib().fcb_detector_rows(ctypes.byref(g), int(margin), lo.ctypes.data_as(_lib.c_int_p),
                                            hi.ctypes.data_as(_lib.c_int_p)))
    return lo.astype(np.int64), hi.astype(np.int64)


# --------------------------------------------------------------------- backprojection
def pack_backproject(dec: SlabDecomposition, rank: int, proj_local):
    """The pieces rank sends each destination: [n, rows_dst, W] blocks of its own views'
    bands, in view order."""
    import torch

    v0, _ = dec.views(rank)
    out = []
    for d in range(dec.world):
        sel = dec._sel(rank, d)
        b = dec.bands[d]
        if len(sel) == 0 or b.rows == 0:
            out.append(proj_local.new_empty((0, b.rows, dec.W)))
            continue
        dev = proj_local.device
        t = torch.as_tensor(b.views[sel] - v0, device=dev)
        rows = torch.as_tensor(b.lo[sel], device=dev)[:, None] + torch.arange(b.rows, device=dev)[None, :]
        out.append(proj_local[t[:, None], rows])
    return out


def unpack_backproject(dec: SlabDecomposition, rank: int, pieces):
    """Rank's windowed projection set [n_views_reaching, rows, W] from the pieces each
    source sent it (source order is view order)."""
    import torch

    b = dec.bands[rank]
    parts = [p.reshape(-1, b.rows, dec.W) for p in pieces if p.numel()]
    if not parts:
        return None
    return torch.cat(parts, 0).contiguous()


def backproject(proj_local, dec: SlabDecomposition, rank: int, mode: int = _lib.MODE_FDK,
                vol_slab=None, group=None, local_op=None):
    """vol_slab += the backprojection of all ranks' views onto rank's slab.

    ``proj_local`` holds this rank's views [v1 - v0, H, W] (float32, float16 or bfloat16:
    the exchange moves the stored type).  ``local_op(band_proj, band_geom, mode, vol)`` is
    the single-GPU backprojection (default: the library's kernels through ``ops``)."""
    import torch
    import torch.distributed as tdist

    if vol_slab is None:
        vol_slab = torch.zeros(dec.slab_shape(rank), device=proj_local.device, dtype=torch.float32)
    send = pack_backproject(dec, rank, proj_local)
    sendbuf = torch.cat([p.reshape(-1) for p in send]) if send else proj_local.new_empty(0)
    in_sizes = [dec.split_sizes(rank, d) for d in range(dec.world)]
    out_sizes = [dec.split_sizes(s, rank) for s in range(dec.world)]
    recvbuf = proj_local.new_empty(sum(out_sizes))
    if dec.world > 1:
        tdist.all_to_all_single(recvbuf, sendbuf.contiguous(), out_sizes, in_sizes, group=group)
    else:
        recvbuf.copy_(sendbuf)
    band = unpack_backproject(dec, rank, list(torch.split(recvbuf, out_sizes)))
    g = dec.band_geometry(rank)
    if band is not None and g is not None:
        (local_op or _ops_backproject)(band, g, mode, vol_slab)
    return vol_slab


def _ops_backproject(band, geom, mode, vol):
    from . import ops

    return ops.backproject(band, geom, mode, vol)


# --------------------------------------------------------------------- projection
def pack_project(dec: SlabDecomposition, rank: int, band_proj):
    """Rank's projected bands [n_views_reaching, rows, W] cut into the pieces each view
    owner receives."""
    b = dec.bands[rank]
    out = []
    for s in range(dec.world):
        sel = dec._sel(s, rank)
        if len(sel) == 0 or band_proj is None:
            out.append(None)
            continue
        out.append(band_proj[int(sel[0]):int(sel[-1]) + 1])  # a source's views are contiguous
    return out, b.rows


def unpack_project(dec: SlabDecomposition, rank: int, pieces, proj_local):
    """proj_local += every slab's band contribution to rank's views, sources in rank order."""
    import torch

    v0, _ = dec.views(rank)
    dev = proj_local.device
    for d, p in enumerate(pieces):
        sel = dec._sel(rank, d)
        b = dec.bands[d]
        if len(sel) == 0 or p is None or p.numel() == 0:
            continue
        p = p.reshape(len(sel), b.rows, dec.W)
        t = torch.as_tensor(b.views[sel] - v0, device=dev)
        rows = torch.as_tensor(b.lo[sel], device=dev)[:, None] + torch.arange(b.rows, device=dev)[None, :]
        proj_local.index_put_((t[:, None], rows), p.to(proj_local.dtype), accumulate=True)
    return proj_local


def project(vol_slab, dec: SlabDecomposition, rank: int, proj_local=None, group=None, local_op=None,
            method: int = _lib.PROJ_EXPLICIT):
    """proj_local += the projection of the whole (distributed) volume for rank's views.

    ``vol_slab`` is rank's slab (float32).  ``local_op(vol, band_geom, method, proj)`` is the
    single-GPU projection (default: the library's kernels through ``ops``)."""
    import torch
    import torch.distributed as tdist

    v0, v1 = dec.views(rank)
    if proj_local is None:
        proj_local = torch.zeros((v1 - v0, dec.H, dec.W), device=vol_slab.device, dtype=torch.float32)
    g = dec.band_geometry(rank)
    band = None
    if g is not None:
        band = torch.zeros(g.proj_shape, device=vol_slab.device, dtype=torch.float32)
        (local_op or _ops_project)(vol_slab, g, method, band)
    pieces, _ = pack_project(dec, rank, band)
    in_sizes = [dec.split_sizes(s, rank) for s in range(dec.world)]
    out_sizes = [dec.split_sizes(rank, d) for d in range(dec.world)]
    sendbuf = torch.cat([p.reshape(-1) for p in pieces if p is not None] or
                        [torch.zeros(0, device=vol_slab.device)])
    recvbuf = torch.empty(sum(out_sizes), device=vol_slab.device, dtype=torch.float32)
    if dec.world > 1:
        tdist.all_to_all_single(recvbuf, sendbuf.contiguous(), out_sizes, in_sizes, group=group)
    else:
        recvbuf.copy_(sendbuf)
    return unpack_project(dec, rank, list(torch.split(recvbuf, out_sizes)), proj_local)


def _ops_project(vol, geom, method, proj):
    from . import ops

    return ops.project(vol, geom, method, proj)


__all__ = ["SlabDecomposition", "detector_rows", "backproject", "project", "pack_backproject",
           "unpack_backproject", "pack_project", "unpack_project"]
