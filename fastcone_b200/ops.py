"""Device-side operators on torch CUDA tensors, stream-ordered on torch's current stream.

torch is only the plumbing here (device memory, streams); every operator is a kernel of
libfastcone_b200.so reached through its C ABI.  There is no CPU fallback: tensors must live
on a CUDA device.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib
from .geometry import ConeGeometry

_DTYPES = {torch.float32: _lib.FCB_F32, torch.float16: _lib.FCB_F16, torch.bfloat16: _lib.FCB_BF16}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(t: torch.Tensor, name: str, dtype=None):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (there is no CPU path)")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}")
    return ctypes.c_void_p(t.data_ptr())


def backproject(proj: torch.Tensor, geom: ConeGeometry, mode: int = _lib.MODE_FDK,
                vol: torch.Tensor | None = None) -> torch.Tensor:
    """vol += sum_t norm[t] * w_mode(U) * bilinear(proj[t]); proj (n, h, w) float32/16/bf16."""
    if proj.dtype not in _DTYPES:
        raise ValueError("projection dtype must be float32, float16 or bfloat16")
    if tuple(proj.shape) != geom.proj_shape:
        raise ValueError(f"projection shape {tuple(proj.shape)} != {geom.proj_shape}")
    if vol is None:
        vol = torch.zeros(geom.vol_shape, device=proj.device, dtype=torch.float32)
    g = geom.struct()
    check(lib().fcb_backproject_device(ctypes.byref(g), mode, _dev(proj, "proj"), _DTYPES[proj.dtype],
                                       _dev(vol, "vol", torch.float32), _stream()))
    return vol


class BackprojectPlan:
    """Geometry digested once; ``__call__`` queues the kernels and allocates nothing."""

    def __init__(self, geom: ConeGeometry, mode: int = _lib.MODE_FDK, dtype=torch.float32):
        self.geom = geom
        self.mode = mode
        self.dtype = dtype
        self._h = ctypes.c_void_p()
        g = geom.struct()
        check(lib().fcb_bp_plan_create(ctypes.byref(g), mode, _DTYPES[dtype], ctypes.byref(self._h)))

    def info(self):
        bw, bh, nl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        upd = ctypes.c_longlong()
        check(lib().fcb_bp_plan_info(self._h, ctypes.byref(bw), ctypes.byref(bh), ctypes.byref(nl),
                                     ctypes.byref(upd)))
        return {"box_w": bw.value, "box_h": bh.value, "launches": nl.value, "updates": upd.value}

    def __call__(self, proj: torch.Tensor, vol: torch.Tensor) -> torch.Tensor:
        if proj.dtype != self.dtype or tuple(proj.shape) != self.geom.proj_shape:
            raise ValueError("projection dtype/shape does not match the plan")
        if tuple(vol.shape) != self.geom.vol_shape:
            raise ValueError("volume shape does not match the plan")
        check(lib().fcb_bp_plan_execute(self._h, _dev(proj, "proj"), _dev(vol, "vol", torch.float32),
                                        _stream()))
        return vol

    def __del__(self):
        # also runs at interpreter exit, when module globals may already be gone
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._h = None
            try:
                lib().fcb_bp_plan_destroy(h)
            except Exception:
                pass


def project(vol: torch.Tensor, geom: ConeGeometry, method: int = _lib.PROJ_EXPLICIT,
            proj: torch.Tensor | None = None, sample_counter: torch.Tensor | None = None) -> torch.Tensor:
    """proj += norm[t] * sum_m trilinear(vol, S + m d) over integer-distance samples."""
    if tuple(vol.shape) != geom.vol_shape:
        raise ValueError(f"volume shape {tuple(vol.shape)} != {geom.vol_shape}")
    if proj is None:
        proj = torch.zeros(geom.proj_shape, device=vol.device, dtype=torch.float32)
    g = geom.struct()
    if sample_counter is not None:
        check(lib().fcb_project_device_counted(ctypes.byref(g), method, _dev(vol, "vol", torch.float32),
                                               _dev(proj, "proj", torch.float32),
                                               _dev(sample_counter, "counter", torch.int64), _stream()))
    else:
        check(lib().fcb_project_device(ctypes.byref(g), method, _dev(vol, "vol", torch.float32),
                                       _dev(proj, "proj", torch.float32), _stream()))
    return proj


class ProjectPlan:
    """Reusable projector (and, for the explicit method, its exact adjoint); calls are
    stream-ordered and allocate nothing."""

    def __init__(self, geom: ConeGeometry, method: int = _lib.PROJ_EXPLICIT):
        self.geom = geom
        self.method = method
        self._h = ctypes.c_void_p()
        g = geom.struct()
        check(lib().fcb_proj_plan_create(ctypes.byref(g), method, ctypes.byref(self._h)))

    def __call__(self, vol: torch.Tensor, proj: torch.Tensor | None = None) -> torch.Tensor:
        if tuple(vol.shape) != self.geom.vol_shape:
            raise ValueError("volume shape does not match the plan")
        if proj is None:
            proj = torch.zeros(self.geom.proj_shape, device=vol.device, dtype=torch.float32)
        check(lib().fcb_proj_plan_execute(self._h, _dev(vol, "vol", torch.float32), _dev(proj, "proj", torch.float32),
                                          0, _stream()))
        return proj

    def info(self) -> dict:
        """Whether the explicit projector runs on TMA-staged bricks, and their shape."""
        v = [ctypes.c_int() for _ in range(4)]
        check(lib().fcb_proj_plan_info(self._h, *[ctypes.byref(x) for x in v]))
        return {"staged": bool(v[0].value), "brick_c": v[1].value, "brick_z": v[2].value,
                "stages": v[3].value}

    def adjoint(self, proj: torch.Tensor, vol: torch.Tensor | None = None) -> torch.Tensor:
        if tuple(proj.shape) != self.geom.proj_shape:
            raise ValueError("projection shape does not match the plan")
        if vol is None:
            vol = torch.zeros(self.geom.vol_shape, device=proj.device, dtype=torch.float32)
        check(lib().fcb_proj_plan_execute(self._h, _dev(vol, "vol", torch.float32), _dev(proj, "proj", torch.float32),
                                          1, _stream()))
        return vol

    def __del__(self):
        # also runs at interpreter exit, when module globals may already be gone
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._h = None
            try:
                lib().fcb_proj_plan_destroy(h)
            except Exception:
                pass


def project_adjoint(proj: torch.Tensor, geom: ConeGeometry, vol: torch.Tensor | None = None) -> torch.Tensor:
    """vol += A^T (norm * proj), the exact transpose of project(method=PROJ_EXPLICIT)."""
    if tuple(proj.shape) != geom.proj_shape:
        raise ValueError(f"projection shape {tuple(proj.shape)} != {geom.proj_shape}")
    if vol is None:
        vol = torch.zeros(geom.vol_shape, device=proj.device, dtype=torch.float32)
    g = geom.struct()
    check(lib().fcb_project_adjoint_device(ctypes.byref(g), _dev(proj, "proj", torch.float32),
                                           _dev(vol, "vol", torch.float32), _stream()))
    return vol


def fdk_filter(proj: torch.Tensor, geom: ConeGeometry | None = None, out_dtype=torch.float32,
               window: int = _lib.FILTER_RAMLAK, cosine_weight: bool = True,
               zorigin=None, D: float | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
    """Cosine weight (fastcone.fbp's) + ramp filter (fastcone.rampfilter's) on the GPU."""
    n, H, W = proj.shape
    if out is None:
        out = torch.empty((n, H, W), device=proj.device, dtype=out_dtype)
    if cosine_weight:
        if zorigin is None:
            zorigin = geom.hmid
        if D is None:
            D = geom.D
    z = np.ascontiguousarray(np.asarray(zorigin if zorigin is not None else np.zeros(n), np.float32))
    check(lib().fcb_fdk_filter_device(_dev(proj, "proj", torch.float32), _dev(out, "out"),
                                      _DTYPES[out.dtype], n, H, W, float(D or 0.0),
                                      z.ctypes.data_as(_lib.c_float_p), 1 if cosine_weight else 0,
                                      window, _stream()))
    return out


class FilterPlan:
    """Reusable FDK filter (cosine weight + ramp / Shepp-Logan, or the unpadded cosine /
    Gaussian apodised ramps with ``window=FILTER_COSRAMP / FILTER_GAUSSRAMP``) for projections of shape
    (nviews, H, W): cuFFT plans and scratch made once; calls are stream-ordered, allocate
    nothing and do not synchronise."""

    def __init__(self, shape, out_dtype=torch.float32, window: int = _lib.FILTER_RAMLAK,
                 gauss_scale: float = 0.125):
        self.shape = tuple(int(v) for v in shape)
        self.out_dtype = out_dtype
        self._h = ctypes.c_void_p()
        n, H, W = self.shape
        check(lib().fcb_filter_plan_create_ex(n, H, W, _DTYPES[out_dtype], int(window), float(gauss_scale),
                                              ctypes.byref(self._h)))

    def __call__(self, proj: torch.Tensor, zorigin=None, D: float | None = None, cosine_weight: bool = True,
                 out: torch.Tensor | None = None) -> torch.Tensor:
        if tuple(proj.shape) != self.shape:
            raise ValueError("projection shape does not match the plan")
        if out is None:
            out = torch.empty(self.shape, device=proj.device, dtype=self.out_dtype)
        z = np.ascontiguousarray(np.asarray(zorigin if zorigin is not None else np.zeros(self.shape[0]), np.float32))
        check(lib().fcb_filter_plan_execute(self._h, _dev(proj, "proj", torch.float32), _dev(out, "out"),
                                            float(D or 0.0), z.ctypes.data_as(_lib.c_float_p),
                                            1 if cosine_weight else 0, _stream()))
        return out

    def __del__(self):
        # also runs at interpreter exit, when module globals may already be gone
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._h = None
            try:
                lib().fcb_filter_plan_destroy(h)
            except Exception:
                pass


def katsevich_filter(proj: torch.Tensor, geom: ConeGeometry, n_kappa: int = 0,
                     out: torch.Tensor | None = None) -> torch.Tensor:
    """Katsevich filtering of helical projections (float32 (n, H, W)) for geom's helix."""
    if geom.helical_pitch == 0.0:
        raise ValueError("Katsevich filtering needs a helical geometry (helical_pitch != 0)")
    n, H, W = proj.shape
    if out is None:
        out = torch.empty_like(proj)
    check(lib().fcb_katsevich_filter_device(_dev(proj, "proj", torch.float32), _dev(out, "out", torch.float32),
                                            n, H, W, geom.angles.ctypes.data_as(_lib.c_float_p), float(geom.D),
                                            float(geom.pw), float(geom.helical_pitch), int(n_kappa), _stream()))
    return out


class KatsevichPlan:
    """Reusable Katsevich filter for geom's helix and detector (tables, cuFFT plans and
    intermediate buffers made once); calls are stream-ordered and allocate nothing."""

    def __init__(self, geom: ConeGeometry, n_kappa: int = 0):
        if geom.helical_pitch == 0.0:
            raise ValueError("Katsevich filtering needs a helical geometry (helical_pitch != 0)")
        self.shape = geom.proj_shape
        self._h = ctypes.c_void_p()
        n, H, W = self.shape
        check(lib().fcb_katsevich_plan_create(n, H, W, geom.angles.ctypes.data_as(_lib.c_float_p), float(geom.D),
                                              float(geom.pw), float(geom.helical_pitch), int(n_kappa),
                                              ctypes.byref(self._h)))

    def __call__(self, proj: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        if tuple(proj.shape) != self.shape:
            raise ValueError("projection shape does not match the plan")
        if out is None:
            out = torch.empty_like(proj)
        check(lib().fcb_katsevich_plan_execute(self._h, _dev(proj, "proj", torch.float32),
                                               _dev(out, "out", torch.float32), _stream()))
        return out

    def __del__(self):
        # also runs at interpreter exit, when module globals may already be gone
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._h = None
            try:
                lib().fcb_katsevich_plan_destroy(h)
            except Exception:
                pass


def katsevich_reconstruct(proj: torch.Tensor, geom: ConeGeometry, n_kappa: int = 0,
                          dtype=torch.float32) -> torch.Tensor:
    """Exact helical reconstruction: Katsevich filtering, then backprojection with weight U
    over each voxel's PI interval, norm = (angle step) / (2 pi D)."""
    import dataclasses
    import math

    gF = katsevich_filter(proj, geom, n_kappa)
    dlam = (float(geom.angles[-1]) - float(geom.angles[0])) / (geom.nviews - 1)
    g = dataclasses.replace(geom, pi_window=True,
                            norm=np.full(geom.nviews, abs(dlam) / (2 * math.pi * geom.D), np.float32))
    return backproject(gF.to(dtype), g, mode=_lib.MODE_KATSEVICH)


def phantom(vol_xyz, params: np.ndarray, device="cuda", out: torch.Tensor | None = None) -> torch.Tensor:
    """Voxelise an ellipsoid phantom (n x 16 parameter rows) on the GPU."""
    nx, ny, nz = (int(v) for v in vol_xyz)
    if out is None:
        out = torch.empty((nz, ny, nx), device=device, dtype=torch.float32)
    dims = np.array([nx, ny, nz], np.int32)
    p = np.ascontiguousarray(params, dtype=np.float64)
    check(lib().fcb_phantom_device(_dev(out, "out", torch.float32), dims.ctypes.data_as(_lib.c_int_p),
                                   p.ctypes.data_as(_lib.c_double_p), len(p), _stream()))
    return out


def sync_status():
    """Synchronise the current stream; raise if a kernel recorded a device-side failure."""
    check(lib().fcb_sync_status(_stream()))


def reference_windows(geom: ConeGeometry) -> dict:
    """The reference's sub-problem decomposition of ``geom`` (host computation): tile and
    window sizes, per [tile, view] window starts and projector sweeps, and whether the
    windows change the backprojection / projection (``bp_matters`` / ``proj_matters``)."""
    L = lib()
    g = geom.struct()
    sv, sp, tiles, m = (np.zeros(k, np.int32) for k in (3, 2, 3, 2))
    ip = lambda a: a.ctypes.data_as(_lib.c_int_p)  # noqa: E731
    null = ctypes.cast(None, _lib.c_int_p)
    check(L.fcb_reference_windows(ctypes.byref(g), ip(sv), ip(sp), ip(tiles), null, null, null, null, ip(m)))
    n = int(np.prod(tiles)) * geom.nviews
    ws, hs, s0, sn = (np.zeros(n, np.int32) for _ in range(4))
    check(L.fcb_reference_windows(ctypes.byref(g), null, null, null, ip(ws), ip(hs), ip(s0), ip(sn), null))
    shp = (int(np.prod(tiles)), geom.nviews)
    return dict(subVolDim=sv, subProjDim=sp, tiles=tiles, ws=ws.reshape(shp), hs=hs.reshape(shp),
                sweepStart=s0.reshape(shp), sweepSteps=sn.reshape(shp), bp_matters=bool(m[0]),
                proj_matters=bool(m[1]))
