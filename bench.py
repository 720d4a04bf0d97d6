"""Benchmark: FDK backprojection GUPS on the large circular configuration
(1024^3 voxels of 0.25 mm, 1440 views over 360 deg, 1536 x 1024 detector at 0.4 mm,
source-axis 500 mm, source-detector 1000 mm -> D = 2000 voxels, pw = 0.8 voxel), plus the
forward projector's Gsamples/s on the differentiable-batch geometry (256^3, 360 views,
384 x 256) as a secondary figure.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` = voxel-view updates per second over the whole job with
filtered projections (FP32) already in HBM; `e2e` = the same through the reference-facing
C entry point GPU_CB_K_backproject with pinned host buffers (H2D of projections + volume and
D2H of the volume inside the timed region).  Inputs (9.06 GB + 4.3 GB) exceed L2, so no
flush is needed between steps.  Multi-GPU: every rank backprojects its own copy of the
workload (independent reconstructions, weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FDK backproj GUPS"
UNIT = "GUPS"

VOL = (1024, 1024, 1024)
DET = (1536, 1024)
NVIEWS = 1440
VOXEL_MM, PITCH_MM, SOD_MM, SDD_MM = 0.25, 0.4, 500.0, 1000.0
FDK_BYTES_PER_UPDATE = {"f32": 16, "bf16": 8}  # bilinear gather: 4 detector samples
WORKLOAD = "circular FDK backprojection 1024^3 voxels, 1440 views, 1536x1024 detector, FP32 filtered projections"


# DRAM bytes per FDK launch (1024^3, 180 views per launch): ncu dram__bytes_read.sum +
# dram__bytes_write.sum of every launch of one step of this benchmark, mean over the step's 8
# launches; they range from 14.9 to 16.7 GB (the volume's read-modify-write, 8.6 GB, plus the
# detector rows), 125.5 GB per step, since each launch runs its tiles along the axis that
# moves the detector column less.
FDK_TRAFFIC_PER_LAUNCH = 15.69e9
FDK_TRAFFIC_NOTE = "measured by ncu on the 8 launches of one step (mean; 14.9-16.7 GB per launch)"


def smem_probe(stream, target_s=0.4):
    """Measured shared-memory load bandwidth of this GPU (fcb_smem_bandwidth: conflict-free
    ld.shared by every resident thread), for 4-, 8- and 16-byte loads: GB/s of each, from a
    region of about `target_s` seconds timed with CUDA events."""
    from fastcone_b200 import _lib

    L = _lib.lib()
    out = {}
    for nb in (4, 8, 16):
        ms, nbytes = ctypes.c_float(), ctypes.c_double()
        _lib.check(L.fcb_smem_bandwidth(nb, 2000, ctypes.byref(ms), ctypes.byref(nbytes), stream))
        iters = max(2000, int(2000 * target_s * 1e3 / max(ms.value, 1e-3)))
        _lib.check(L.fcb_smem_bandwidth(nb, iters, ctypes.byref(ms), ctypes.byref(nbytes), stream))
        out[f"ld{8 * nb}_GBs"] = nbytes.value / (ms.value / 1e3) / 1e9
        out[f"ld{8 * nb}_ms"] = ms.value
    return out


def err_stats(got, ref):
    """Relative L2 and max-abs error of `got` against the FP64 `ref` (the same points), with
    the largest reference magnitude beside them."""
    import numpy as np

    from oracle import oracle as O

    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return {"rel_l2": O.rel_l2(got, ref), "max_abs": O.max_abs(got, ref), "ref_max_abs": float(np.abs(ref).max())}


def _gather(vol, pts, g):
    """GPU volume values at global voxel indices pts (rows x, y, z) of geometry g's sub-volume."""
    import torch

    s = g.vol_start
    t = torch.from_numpy(pts.astype("int64")).to(vol.device)
    return vol[t[:, 2] - s[2], t[:, 1] - s[1], t[:, 0] - s[0]].double().cpu().numpy()


def oracle_problem(g):
    """The oracle's description of geometry g, with the same FP32 distances the library gets."""
    import numpy as np

    from oracle import oracle as O

    return O.make_problem(g.vol_xyz, g.det_wh, g.nviews, D=float(np.float32(g.D)), pw=float(np.float32(g.pw)),
                          angles=g.angles, hmid=g.hmid, norm=g.norm, volStart=g.vol_start, volEnd=g.vol_end,
                          woff=g.woff, hoff=g.hoff, whsize=g.window_wh)


def fdk_parity(dev, ncols=256, seed=11, nellip=50):
    """Error of the large circular FDK backprojection (1024^3, 1440 views, 1536x1024) against
    the FP64 oracle, with FP32-, BF16- and FP16-stored filtered projections (FP32 accumulation
    all): a seeded 50-ellipsoid phantom projected by the explicit projector, cosine-weighted
    and Shepp-Logan filtered on the GPU, backprojected over the whole volume; `ncols` random
    full-z voxel columns are compared with the oracle's FP64 backprojection of the same FP32
    filtered projections."""
    import numpy as np
    import torch

    from fastcone_b200 import _lib, ops
    from fastcone_b200.phantom import random_ellipsoids
    from oracle import oracle as O

    g = geometry()
    vol = ops.phantom(g.vol_xyz, random_ellipsoids(nellip, g.vol_xyz, seed), device=dev)
    proj = ops.ProjectPlan(g.with_norm(np.ones(g.nviews, np.float32)), _lib.PROJ_EXPLICIT)(vol)
    del vol
    ops.FilterPlan(g.proj_shape, window=_lib.FILTER_SHEPPLOGAN)(proj, zorigin=g.hmid, D=g.D, out=proj)
    pts = O.column_points(g.vol_xyz, g.vol_start, g.vol_end, ncols, seed)
    res = {"workload": f"{WORKLOAD}; seeded {nellip}-ellipsoid phantom, explicit projector, cosine weight + "
                       f"Shepp-Logan filter; {ncols} random full-z voxel columns vs the FP64 oracle",
           "points": int(len(pts))}
    got = {}
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        p = proj if dt == torch.float32 else proj.to(dt)
        v = torch.zeros(g.vol_shape, device=dev)
        ops.BackprojectPlan(g, mode=_lib.MODE_FDK, dtype=dt)(p, v)
        ops.sync_status()
        got[name] = _gather(v, pts, g)
        del v, p
    proj_h = proj.cpu().numpy()
    del proj
    torch.cuda.empty_cache()
    ref = O.backproject_points_f64(oracle_problem(g), proj_h, pts, kernel_mode=2)
    for name in got:
        res[name] = err_stats(got[name], ref)
    return res


def helix_parity(dev, ncols=128, seed=12, nellip=20):
    """Error of the helical Katsevich reconstruction's PI-window backprojection (512x512x384,
    4 turns x 1160 views, 736x64) against the FP64 oracle: a seeded phantom projected by the
    explicit projector along the helix, Katsevich-filtered on the GPU, backprojected with
    weight U over each voxel's PI interval; `ncols` random full-z columns compared with the
    oracle's FP64 PI-window backprojection of the same filtered projections, and their
    in-window voxel-view pairs counted by the oracle and by fcb_katsevich_pi_pairs."""
    import dataclasses

    import numpy as np
    import torch

    from fastcone_b200 import _lib, configs, ops
    from fastcone_b200.phantom import random_ellipsoids
    from oracle import oracle as O

    gk = configs.helical_katsevich(pi_window=True)
    vol = ops.phantom(gk.vol_xyz, random_ellipsoids(nellip, gk.vol_xyz, seed), device=dev)
    proj = ops.ProjectPlan(gk, _lib.PROJ_EXPLICIT)(vol)
    del vol
    pf = ops.KatsevichPlan(gk)(proj)
    del proj
    dlam = (float(gk.angles[-1]) - float(gk.angles[0])) / (gk.nviews - 1)
    g = dataclasses.replace(gk, norm=np.full(gk.nviews, abs(dlam) / (2 * math.pi * gk.D), np.float32))
    v = torch.zeros(g.vol_shape, device=dev)
    ops.BackprojectPlan(g, mode=_lib.MODE_KATSEVICH)(pf, v)
    ops.sync_status()
    pts = O.column_points(g.vol_xyz, g.vol_start, g.vol_end, ncols, seed)
    got = _gather(v, pts, g)
    ref, pairs = O.katsevich_piwin_points_f64(oracle_problem(g), pf.cpu().numpy(), pts, g.helical_pitch)
    # the same columns' pairs counted on the GPU, one single-column sub-volume at a time
    nz = g.vol_xyz[2]
    gpu_pairs = 0
    for c in range(ncols):
        x, y = int(pts[c * nz, 0]), int(pts[c * nz, 1])
        gpu_pairs += pi_pairs(dataclasses.replace(g, vol_start=(x, y, 0), vol_end=(x + 1, y + 1, nz)))
    # the largest contribution one view can make to a voxel (U at the volume's widest radius):
    # the kernel decides the window edge in FP32, the oracle in FP64, so a voxel whose edge
    # falls within rounding of a view may gain or lose that view at its entry and its exit
    nx, ny = g.vol_xyz[0], g.vol_xyz[1]
    umax = g.D / (g.D - math.hypot(nx / 2, ny / 2))
    one_view = float(np.abs(g.norm).max()) * umax * float(pf.abs().max())
    return {"workload": f"helical 512x512x384, 4 turns x 1160 views, 736x64; seeded {nellip}-ellipsoid "
                        f"phantom, explicit projector, Katsevich filter, PI-window backprojection; {ncols} "
                        f"random full-z voxel columns vs the FP64 oracle",
            "points": int(len(pts)), "f32": err_stats(got, ref), "one_view_max": one_view,
            "pi_pairs_oracle": pairs, "pi_pairs_gpu": gpu_pairs}


def pi_pairs(g):
    """Exact number of voxel-view pairs of geometry g inside the PI window (on the GPU)."""
    import torch

    from fastcone_b200 import _lib

    s = g.struct()
    n = ctypes.c_longlong()
    _lib.check(_lib.lib().fcb_katsevich_pi_pairs(ctypes.byref(s), ctypes.byref(n),
                                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return int(n.value)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the error measurement against the FP64 oracle at the headline and helical sizes")
    ap.add_argument("--shard", default=None, choices=["replicas", "z", "slabs"],
                    help="replicas: every rank reconstructs its own volume (weak scaling; the default "
                         "for one GPU); slabs: one volume in z-slabs, the views spread over the ranks and "
                         "exchanged as detector-row bands by an NCCL all-to-all (strong scaling; the "
                         "default for N > 1); z: one volume in z-slabs, every rank holding all views")
    ap.add_argument("--case", default=None,
                    choices=["fdk-slab", "fdk-slab-bf16", "proj-512", "proj-256", "conv-256", "katsevich",
                             "pipeline", "misaligned-256", "fdk-filter"],
                    help="profiling case: run only this kernel on a reduced workload (no JSON line)")
    return ap.parse_args()


def run_case(args):
    """Reduced single-kernel workloads for ncu captures (a few GB on the device):
    fdk-slab[-bf16]: the 1024^3 geometry restricted to a 1024x1024x128 z-slab (z 448..575),
    64 views (0.5 GB volume + 0.4 GB projections);
    proj-512: the staged, unstaged and texture projectors on 512^3, 90 views, 768x512
    detector (0.5 GB volume); proj-256: the same on 256^3, 360 views, 384x256;
    conv-256: one unrolled step's convolutions at 256^3 x 16 BF16 channels (0.54 GB per
    activation): forward (three kernel forms) and weight gradient (tensor cores and the
    CUDA-core kernel), all on tcgen05 except the last;
    katsevich: the helical PI-window backprojection (512x512x384, 4640 views; 1.3 GB);
    fdk-filter: the FDK filter (cosine weight + Shepp-Logan) of the 1440 x 1024 x 1536
    projections of the 1024^3 workload through a filter plan, in place (9.06 GB);
    misaligned-256: the general-matrix backprojector (a misaligned detector, unweighted) on
    256^3 / 360 views / 384x256 through a plan, CUDA events over the timed calls;
    pipeline: every other kernel once at a moderate size, inputs above L2 where the workload
    allows: phantom, FDK filter (ramp + Shepp-Logan), Katsevich filter, projector adjoint,
    misaligned (generic) backprojection, reference-window backprojection and projection,
    brick-size and footprint pre-passes, volume transpose."""
    import numpy as np
    import torch

    from fastcone_b200 import _lib, ops
    from fastcone_b200.geometry import ConeGeometry

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if args.case.startswith("fdk-slab"):
        n = 64
        g = ConeGeometry.circular(VOL, VOXEL_MM, DET, PITCH_MM, SOD_MM, SDD_MM, NVIEWS)
        import dataclasses

        g = dataclasses.replace(g, angles=g.angles[:n], hmid=g.hmid[:n], norm=np.full(n, 1.0 / NVIEWS, np.float32),
                                woff=g.woff[:n], hoff=g.hoff[:n], vol_start=(0, 0, 448), vol_end=(1024, 1024, 576))
        dt = torch.bfloat16 if args.case.endswith("bf16") else torch.float32
        proj = torch.randn((n, DET[1], DET[0]), device=dev).to(dt)
        vol = torch.zeros(g.vol_shape, device=dev)
        plan = ops.BackprojectPlan(g, mode=_lib.MODE_FDK, dtype=dt)
        for _ in range(args.warmup):
            plan(proj, vol)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            plan(proj, vol)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        upd = 1024 * 1024 * 128 * n
        print(json.dumps({"case": args.case, "ms": ms, "GUPS": upd / ms / 1e6, "box": plan.info()}))
    elif args.case == "fdk-filter":
        p = torch.randn((NVIEWS, DET[1], DET[0]), device=dev)
        zorig = np.full(NVIEWS, DET[1] / 2.0, np.float32)
        plan = ops.FilterPlan(tuple(p.shape), window=_lib.FILTER_SHEPPLOGAN)
        for _ in range(args.warmup):
            plan(p, zorigin=zorig, D=2500.0, out=p)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            plan(p, zorigin=zorig, D=2500.0, out=p)
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"case": args.case, "ms": e0.elapsed_time(e1) / args.steps, "views": NVIEWS}))
    elif args.case == "katsevich":
        from fastcone_b200 import configs

        gk = configs.helical_katsevich(pi_window=True)
        pk = torch.randn(gk.proj_shape, device=dev)
        vk = torch.zeros(gk.vol_shape, device=dev)
        plan = ops.BackprojectPlan(gk, mode=_lib.MODE_KATSEVICH, dtype=torch.float32)
        for _ in range(args.warmup):
            plan(pk, vk)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            plan(pk, vk)
        e1.record()
        torch.cuda.synchronize()
        res = {"case": args.case, "ms": e0.elapsed_time(e1) / args.steps, **plan.info()}
        # the Katsevich filter on the same projections: FFT Hilbert transform vs the direct sum
        for name, direct in (("filter_fft_ms", "0"), ("filter_direct_ms", "1")):
            os.environ["FCB_KATS_DIRECT_HILBERT"] = direct
            ops.katsevich_filter(pk, gk)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ops.katsevich_filter(pk, gk)
            torch.cuda.synchronize()
            res[name] = (time.perf_counter() - t0) * 1e3
        os.environ.pop("FCB_KATS_DIRECT_HILBERT", None)
        print(json.dumps(res))
    elif args.case == "misaligned-256":
        import dataclasses

        from fastcone_b200 import configs

        gd = configs.diff_batch()
        gm = dataclasses.replace(gd, misalignments=np.array([1.5, -0.5, 2.0, 0.01, -0.01, 0.02], np.float32))
        proj = torch.randn(gd.proj_shape, device=dev)
        plan = ops.BackprojectPlan(gm, mode=_lib.MODE_UNWEIGHTED)
        vol = torch.zeros(gm.vol_shape, device=dev)
        for _ in range(args.warmup):
            plan(proj, vol)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            plan(proj, vol)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        print(json.dumps({"case": args.case, "ms": ms, "GUPS": 256 ** 3 * 360 / ms / 1e6}))
    elif args.case == "pipeline":
        import dataclasses

        from fastcone_b200 import configs
        from fastcone_b200.phantom import random_ellipsoids

        gd = configs.diff_batch()                        # 256^3, 360 views, 384x256
        vol = ops.phantom(gd.vol_xyz, random_ellipsoids(10, gd.vol_xyz, 3), device=dev)
        proj = torch.randn(gd.proj_shape, device=dev)    # 141 MB
        for _ in range(args.warmup + args.steps):
            ops.fdk_filter(proj, gd)
            ops.fdk_filter(proj, gd, window=_lib.FILTER_SHEPPLOGAN)
            ops.project_adjoint(proj, gd)
            ops.project(vol, gd, method=_lib.PROJ_EXPLICIT)   # includes pre-pass + transpose
            gm = dataclasses.replace(gd, misalignments=np.array([1.5, -0.5, 2.0, 0.01, -0.01, 0.02], np.float32))
            ops.backproject(proj, gm, mode=_lib.MODE_UNWEIGHTED)
        gk = configs.helical_katsevich(pi_window=True)
        pk = torch.randn(gk.proj_shape, device=dev)      # 874 MB
        for _ in range(args.warmup + args.steps):
            ops.katsevich_filter(pk, gk)
        # reference-compatible windows on the 48^3 / 72-pixel geometry they change
        gq = ConeGeometry((48, 48, 48), (72, 48), np.arange(36) * (2 * np.pi / 36), 200.0, 0.5,
                          reference_windows=True)
        vq = ops.phantom(gq.vol_xyz, random_ellipsoids(5, gq.vol_xyz, 4), device=dev)
        for _ in range(args.warmup + args.steps):
            pq = ops.project(vq, gq, method=_lib.PROJ_EXPLICIT)
            ops.backproject(pq, gq, mode=_lib.MODE_FDK)
        print(json.dumps({"case": args.case}))
    elif args.case == "conv-256":
        from fastcone_b200 import nn

        gen = torch.Generator(device=dev).manual_seed(0)
        x = torch.randn((256, 256, 2, 256, 8), device=dev, generator=gen).to(torch.bfloat16)
        wk = (0.05 * torch.randn((27, 16, 16), device=dev, generator=gen)).to(torch.bfloat16)
        b = torch.zeros(16, device=dev)
        res = {}

        def fwd_variant(v):
            def run():
                os.environ["FCB_CONV_SIMPLE"] = v
                try:
                    return nn.conv3d16(x, wk, b, relu=True)
                finally:
                    os.environ.pop("FCB_CONV_SIMPLE", None)
            return run

        def wgrad_simt():
            os.environ["FCB_WGRAD_SIMT"] = "1"
            try:
                return nn.conv3d16_wgrad(x, x)
            finally:
                os.environ.pop("FCB_WGRAD_SIMT", None)

        for name, fn in (("fwd", lambda: nn.conv3d16(x, wk, b, relu=True)),
                         ("fwd_one_tile_per_cta", fwd_variant("1")),
                         ("fwd_persistent_no_row_reuse", fwd_variant("2")),
                         ("wgrad", lambda: nn.conv3d16_wgrad(x, x)),
                         ("wgrad_cuda_cores", wgrad_simt)):
            for _ in range(args.warmup):
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            flop = 2.0 * 16 * 27 * 16 * 256 ** 3
            res[name] = {"ms": ms, "TFLOP/s": flop / ms / 1e9}
        print(json.dumps({"case": args.case, **res}))
    else:
        if args.case == "proj-256":
            from fastcone_b200 import configs

            g = configs.diff_batch()  # 256^3, 360 views, 384x256
        else:
            g = ConeGeometry.circular((512, 512, 512), 1.0, (768, 512), 1.0, 1000.0, 2000.0, 90)
        from fastcone_b200.phantom import random_ellipsoids

        v = ops.phantom(g.vol_xyz, random_ellipsoids(10, g.vol_xyz, 1), device=dev)
        res = {}
        for name, meth in (("explicit", _lib.PROJ_EXPLICIT), ("explicit_unstaged", _lib.PROJ_EXPLICIT_GLOBAL),
                           ("texture", _lib.PROJ_TEXTURE)):
            plan = ops.ProjectPlan(g, meth)
            p = plan(v)
            for _ in range(args.warmup):
                plan(v, p)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                plan(v, p)
            e1.record()
            torch.cuda.synchronize()
            res[name] = {"ms": e0.elapsed_time(e1) / args.steps, **(plan.info() if meth == _lib.PROJ_EXPLICIT else {})}
            if meth != _lib.PROJ_TEXTURE:
                # the transpose of the same plan
                vt = plan.adjoint(p)
                e0.record()
                for _ in range(args.steps):
                    plan.adjoint(p, vt)
                e1.record()
                torch.cuda.synchronize()
                res[name]["adjoint_ms"] = e0.elapsed_time(e1) / args.steps
        print(json.dumps({"case": args.case, **res}))
    ops.sync_status()
    torch.cuda.synchronize()
    print("case", args.case, "done")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def geometry():
    import numpy as np

    from fastcone_b200.geometry import ConeGeometry

    g = ConeGeometry.circular(VOL, VOXEL_MM, DET, PITCH_MM, SOD_MM, SDD_MM, NVIEWS)
    return g.with_norm(np.full(NVIEWS, 1.0 / NVIEWS, np.float32))


class CpuReferencePath:
    """Reference path (texture-emulating restatement of Fastcone's FDK kernel, sub-problem
    tiling and windows) on this host's cores, over bounded samples of the workload: whole
    columns of voxels (all z, all views) at random (x, y).  `calibrate` sizes one sample for a
    target duration; `sample` times one."""

    def __init__(self, g, seed=0):
        import numpy as np

        from oracle import oracle as O

        self.O = O
        self.vol, self.det, self.nviews = tuple(g.vol_xyz), tuple(g.det_wh), g.nviews
        self.pb = O.make_problem(self.vol, self.det, self.nviews, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid,
                                 norm=g.norm)
        self.rng = np.random.default_rng(seed)
        self.proj = self.rng.standard_normal((self.nviews, self.det[1], self.det[0]), dtype=np.float32)
        self.cores = os.cpu_count() or 1
        self.ncols = 2

    def sample(self, ncols=None):
        """Backproject `ncols` random voxel columns; returns (seconds, voxel-view updates)."""
        import numpy as np

        ncols = ncols or self.ncols
        nx, ny, nz = self.vol
        xy = np.stack([self.rng.integers(0, nx, ncols), self.rng.integers(0, ny, ncols)], 1)
        z = np.arange(nz)
        pts = np.stack([np.repeat(xy[:, 0], nz), np.repeat(xy[:, 1], nz), np.tile(z, ncols)], 1)
        pts = pts.astype(np.int32)
        t0 = time.perf_counter()
        self.O.ref_backproject_points(self.pb, self.proj, pts, kernel_mode=2, texq=1)
        return time.perf_counter() - t0, len(pts) * self.nviews

    def calibrate(self, target_s):
        dt, _ = self.sample(2)
        self.ncols = max(2, int(2 * target_s / max(dt, 1e-3)))
        return self.ncols

    def describe(self, dt, upd, nsamples=1):
        nx, ny, nz = self.vol
        return (f"{nsamples} x {self.ncols} random (x,y) columns x {nz} z x {self.nviews} views = {upd:.3g} "
                f"updates of the {nx}x{ny}x{nz} / {self.nviews}-view FDK, texture-emulating reference path "
                f"(oracle/fc_oracle.c, {self.cores} threads), {dt:.1f} s")


def cpu_baseline(g, target_s=6.0, runs=2):
    """The best of `runs` bounded samples of the CPU reference path (about `target_s` seconds
    each, different random columns); returns the cpu_baseline object of the JSON line."""
    ref = CpuReferencePath(g)
    ref.calibrate(target_s)
    best = None
    for _ in range(runs):
        dt, upd = ref.sample()
        if best is None or upd / dt > best[1] / best[0]:
            best = (dt, upd)
    dt, upd = best
    return {"value": upd / dt / 1e9, "unit": UNIT, "cores": ref.cores, "kind": "port",
            "sample": f"best of {runs}: " + ref.describe(dt, upd)}


def reference_line(args, g, budget_s=150.0):
    """The reference arm: W untimed and K timed steps, each step one bounded sample of the
    workload on the CPU reference path (all host threads), sized so the whole run stays within
    about `budget_s` seconds; value = the K samples' updates / their total time."""
    ref = CpuReferencePath(g)
    per_step = min(12.0, max(1.0, budget_s / max(1, args.steps + args.warmup)))
    ref.calibrate(per_step)
    for _ in range(args.warmup):
        ref.sample()
    times, upd = [], 0
    for _ in range(max(1, args.steps)):
        dt, u = ref.sample()
        times.append(dt)
        upd += u
    total = sum(times)
    value = upd / total / 1e9
    sample = ref.describe(total, upd, len(times))
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "inputs": "host memory (the reference path has no device copy)",
                       "parallelism": "host threads", "step": "one bounded sample of the workload",
                       "sample": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference(args, rank, world):
    if rank != 0:
        return
    print(json.dumps(reference_line(args, geometry())), flush=True)


def run_slabs(args, rank, world, local):
    """One 1024^3 volume over `world` GPUs (fastcone_b200.slabs, the mpi_fastcone.backproject
    replacement): rank r holds views [1440 r / N, 1440 (r + 1) / N) and owns z-slab r; a step
    is one slabs.backproject -- pack every view's detector-row bands for the slabs they
    reach, one NCCL all-to-all, unpack, backproject the slab (a plan made once per rank).
    value = the volume's voxel-view updates / the slowest rank's step time (strong scaling)."""
    import numpy as np
    import torch

    from fastcone_b200 import _lib, ops, slabs
    from fastcone_b200 import dist as fd

    # NCCL's communicator log (one line per rank with nranks) on stderr, so that stdout
    # carries only the JSON line
    os.environ.setdefault("NCCL_DEBUG", "INFO")
    os.environ.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    os.environ.setdefault("NCCL_DEBUG_FILE", "/dev/stderr")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    fd.init("nccl", device=dev)
    g = geometry()
    dec = slabs.SlabDecomposition(g, world)
    v0, v1 = dec.views(rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    proj = torch.randn((v1 - v0, DET[1], DET[0]), device=dev, generator=gen)
    vol = torch.zeros(dec.slab_shape(rank), device=dev)
    gb = dec.band_geometry(rank)
    plan = ops.BackprojectPlan(gb, mode=_lib.MODE_FDK) if gb is not None else None
    local_op = lambda band, geom, mode, v: plan(band, v)  # noqa: E731

    def step():
        slabs.backproject(proj, dec, rank, _lib.MODE_FDK, vol, local_op=local_op)

    for _ in range(args.warmup):
        step()
    ops.sync_status()
    torch.cuda.synchronize()
    fd.barrier()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        fd.barrier()
        e0.record(st)
        for _ in range(args.steps):
            step()
        e1.record(st)
        torch.cuda.synchronize()
        fd.barrier()
    ops.sync_status()
    ms_step = fd.max_over_ranks(e0.elapsed_time(e1), dev) / args.steps
    updates = VOL[0] * VOL[1] * VOL[2] * NVIEWS
    value = updates / (ms_step / 1e3) / 1e9
    band_bytes = sum(dec.split_sizes(s_, d) for s_ in range(world) for d in range(world) if s_ != d) * 4
    launches = plan.info()["launches"] if plan is not None else 0
    my_updates = int(np.prod(dec.slab_shape(rank))) * (len(dec.bands[rank].views))

    # end to end: this rank's views from pinned host memory, the slab back to the host
    hproj = torch.empty(proj.shape, dtype=torch.float32, pin_memory=True)
    hproj.copy_(proj)
    hvol = torch.zeros(vol.shape, dtype=torch.float32, pin_memory=True)
    times = []
    for _ in range(max(3, args.steps // 2)):
        fd.barrier()
        t0 = time.perf_counter()
        proj.copy_(hproj, non_blocking=True)
        step()
        hvol.copy_(vol, non_blocking=True)
        torch.cuda.synchronize()
        fd.barrier()
        times.append(time.perf_counter() - t0)
    dt = fd.max_over_ranks(float(np.median(times)), dev)
    e2e = {"value": updates / dt / 1e9, "unit": UNIT, "h2d_bytes_per_step": hproj.numel() * 4,
           "d2h_bytes_per_step": hvol.numel() * 4, "ms_per_step": dt * 1e3,
           "statistic": f"median of {len(times)} steps, slowest rank",
           "path": "slabs.backproject with this rank's views copied in from pinned host memory and its slab "
                   "copied out (sizes per rank)"}
    cpu = cpu_baseline(g) if rank == 0 and world == 1 and not args.no_cpu else None
    hbm, _ = measured_peaks()
    ach = FDK_BYTES_PER_UPDATE["f32"] * my_updates / (ms_step / 1e3) / 1e9
    clocks = clk.summary()
    del plan
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": f"z-slabs x{world}, views spread over the ranks, one "
                                                        f"NCCL all-to-all of detector-row bands per step",
                   "inputs": "each rank's views resident in HBM (value); pinned host buffers (e2e)",
                   "band_bytes_exchanged_per_step": band_bytes,
                   "l2": "inputs larger than L2; no flush"},
        "gpu_launches": launches * args.steps,
        "roofline": {"bound": "smem", "achieved": ach, "peak": None, "unit": "GB/s", "frac": None,
                     "traffic": None, "note": "rank 0's gather bytes (16 B/update) / step time; the "
                                              "single-GPU line measures the peak and the fraction"},
        "hbm_peak": hbm, "clocks": clocks, "e2e": e2e, "cpu_baseline": cpu}), flush=True)


def main():
    args = parse()
    from fastcone_b200.dist import env_ranks

    rank, world, local = env_ranks()
    if args.case:
        run_case(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.shard is None:
        args.shard = "slabs" if world > 1 else "replicas"
    if args.shard == "slabs":
        run_slabs(args, rank, world, local)
        return
    import numpy as np
    import torch

    from fastcone_b200 import _lib, ops
    from fastcone_b200.geometry import ConeGeometry

    from fastcone_b200 import dist as fd

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    fd.init("nccl", device=dev)

    def barrier_max(x):
        return fd.max_over_ranks(x, dev)

    barrier = fd.barrier

    g = geometry()
    if args.shard == "z":
        # one volume split into z-slabs, one per rank (strong scaling): each rank owns the
        # planes [z0, z1) and backprojects them from all projections
        import dataclasses

        z0, z1 = fd.z_slab(VOL[2], world, rank)
        g = dataclasses.replace(g, vol_start=(0, 0, z0), vol_end=(VOL[0], VOL[1], max(z1, z0 + 1)))
    # work of the whole job per step: every rank's volume (replicas) or the one volume (z)
    updates = VOL[0] * VOL[1] * VOL[2] * NVIEWS
    job_updates = updates * (world if args.shard == "replicas" else 1)
    updates = g.vol_shape[0] * g.vol_shape[1] * g.vol_shape[2] * NVIEWS  # this rank's
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    proj = torch.randn((NVIEWS, DET[1], DET[0]), device=dev, dtype=torch.float32, generator=gen)
    vol = torch.zeros(g.vol_shape, device=dev, dtype=torch.float32)
    plan = ops.BackprojectPlan(g, mode=_lib.MODE_FDK, dtype=torch.float32)
    info = plan.info()
    launches_per_step = info["launches"]

    for _ in range(args.warmup):
        plan(proj, vol)
    ops.sync_status()
    torch.cuda.synchronize()
    barrier()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        e0.record(st)
        for _ in range(args.steps):
            plan(proj, vol)
        e1.record(st)
        torch.cuda.synchronize()
        barrier()
    ops.sync_status()
    clk_summary = clk.summary()
    ms = e0.elapsed_time(e1)
    ms = barrier_max(ms)
    ms_step = ms / args.steps
    value = job_updates / (ms_step / 1e3) / 1e9

    hbm, peak_kind = measured_peaks()
    # per launch: the step's launches split the views; bytes and time both scale with views
    achieved = FDK_BYTES_PER_UPDATE["f32"] * updates / (ms_step / 1e3) / 1e9
    ms_launch = ms_step / launches_per_step

    # the binding ceiling, measured on this GPU: conflict-free 32-bit shared-memory loads
    with ClockSampler(local) as clk_probe:
        probe = smem_probe(ctypes.c_void_p(st.cuda_stream))
    probe["clocks"] = clk_probe.summary()
    smem_peak = probe["ld32_GBs"]

    # BF16-stored filtered projections (same kernel family; taps read as 32-bit pairs)
    proj16 = proj.to(torch.bfloat16)
    plan16 = ops.BackprojectPlan(g, mode=_lib.MODE_FDK, dtype=torch.bfloat16)
    for _ in range(max(2, args.warmup)):
        plan16(proj16, vol)
    torch.cuda.synchronize()
    e0.record(st)
    k16 = max(2, args.steps // 2)
    for _ in range(k16):
        plan16(proj16, vol)
    e1.record(st)
    torch.cuda.synchronize()
    ops.sync_status()
    ms16 = barrier_max(e0.elapsed_time(e1)) / k16
    ach16 = FDK_BYTES_PER_UPDATE["bf16"] * updates / (ms16 / 1e3) / 1e9
    del proj16, plan16

    # secondary: forward projector Gsamples/s on 256^3, 360 views, 384 x 256
    from fastcone_b200 import configs

    gp = configs.diff_batch()
    from fastcone_b200.phantom import random_ellipsoids

    pv = ops.phantom(gp.vol_xyz, random_ellipsoids(10, gp.vol_xyz, 1), device=dev)
    ctr = torch.zeros(1, dtype=torch.int64, device=dev)
    pp = ops.project(pv, gp, method=_lib.PROJ_EXPLICIT, sample_counter=ctr)
    torch.cuda.synchronize()
    nsamp = int(ctr.item())
    # the reference's own sample count: its per-(tile, view) sweep x every window pixel
    import dataclasses

    rw = ops.reference_windows(dataclasses.replace(gp, reference_windows=True))
    ref_sweep = int(rw["sweepSteps"].astype(np.int64).sum()) * int(rw["subProjDim"][0]) * int(rw["subProjDim"][1])
    proj_res = {}
    for name, meth in (("explicit", _lib.PROJ_EXPLICIT), ("explicit_unstaged", _lib.PROJ_EXPLICIT_GLOBAL),
                       ("texture", _lib.PROJ_TEXTURE)):
        pplan = ops.ProjectPlan(gp, meth)  # geometry, brick sizing, buffers: once
        for _ in range(2):
            pplan(pv, pp)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(3):
            pplan(pv, pp)
        e1.record(st)
        torch.cuda.synchronize()
        proj_res[name] = nsamp / (e0.elapsed_time(e1) / 3 / 1e3) / 1e9
        if meth != _lib.PROJ_TEXTURE:
            # the matched transpose of the same plan (the autograd backward), same samples
            av = torch.zeros_like(pv)
            pplan.adjoint(pp, av)
            torch.cuda.synchronize()
            e0.record(st)
            for _ in range(3):
                pplan.adjoint(pp, av)
            e1.record(st)
            torch.cuda.synchronize()
            proj_res[name + "_adjoint"] = nsamp / (e0.elapsed_time(e1) / 3 / 1e3) / 1e9
            del av
        del pplan
    del pv, pp

    # helical Katsevich backprojection with the PI window (512x512x384, 4 turns x 1160 views)
    gk = configs.helical_katsevich(pi_window=True)
    pk = torch.randn(gk.proj_shape, device=dev, generator=gen)
    vk = torch.zeros(gk.vol_shape, device=dev)
    kplan = ops.BackprojectPlan(gk, mode=_lib.MODE_KATSEVICH, dtype=torch.float32)
    for _ in range(2):
        kplan(pk, vk)
    torch.cuda.synchronize()
    e0.record(st)
    kk = 3
    for _ in range(kk):
        kplan(pk, vk)
    e1.record(st)
    torch.cuda.synchronize()
    ops.sync_status()
    ms_k = barrier_max(e0.elapsed_time(e1)) / kk
    # Katsevich filtering of the same projections through a filter plan (CUDA events)
    kfp = ops.KatsevichPlan(gk)
    fk = kfp(pk)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(kk):
        kfp(pk, fk)
    e1.record(st)
    torch.cuda.synchronize()
    ms_kf = barrier_max(e0.elapsed_time(e1)) / kk
    del fk, kfp
    dense = gk.vol_shape[0] * gk.vol_shape[1] * gk.vol_shape[2] * gk.nviews
    pairs = pi_pairs(gk)  # exact, FP64, on the GPU (fcb_katsevich_pi_pairs)
    katsevich = {"workload": "helical 512x512x384, 4 turns x 1160 views, 736x64 detector, PI window",
                 "ms_per_pass": ms_k, "filter_ms": ms_kf, "dense_pairs": dense,
                 "dense_equivalent_GUPS": dense / (ms_k / 1e3) / 1e9, "pi_window_pairs": pairs,
                 "pi_window_GUPS": pairs / (ms_k / 1e3) / 1e9, "launches": kplan.info()["launches"]}
    del pk, vk, kplan

    # parity at the headline and helical configurations (after every timed region): the
    # oracle is only the checker here
    parity = None
    if rank == 0 and not args.no_parity:
        del proj, vol
        torch.cuda.empty_cache()
        parity = {"fdk_1024": fdk_parity(dev), "katsevich_helix": helix_parity(dev)}
        torch.cuda.empty_cache()

    # learned unrolled reconstruction vs SIRT-100 (committed weights), two held-out phantoms
    learned_res = None
    wpath = os.path.join(ROOT, "fastcone_b200", "weights", "unrolled8.pt")
    if not args.no_learned and rank == 0 and os.path.exists(wpath):
        from fastcone_b200 import learned

        net = learned.UnrolledNet().to(dev)
        net.load_state_dict(torch.load(wpath, map_location=dev)["model"])

        def summary(r, what):
            mean = lambda k: sum(x[k] for x in r) / len(r)  # noqa: E731
            return {
                "phantoms": what,
                "sirt100_psnr": mean("sirt_psnr"), "sirt100_ssim": mean("sirt_ssim"), "sirt100_s": mean("sirt_time_s"),
                "learned_psnr": mean("learned_psnr"), "learned_ssim": mean("learned_ssim"),
                "learned_s": mean("learned_time_s"), "fdk_psnr": mean("fdk_psnr"),
                "fallback_psnr": mean("no_net_psnr"),
                "time_to_sirt100_psnr_s": [x["time_to_sirt_psnr_s"] for x in r],
                "speedup_to_sirt100_psnr": [x["speedup_to_sirt_psnr"] for x in r],
            }

        gl = configs.learned_sparse()
        r_in = learned.evaluate(net, gl, seeds=[1, 2], sirt_iters=100)
        r_shift = learned.evaluate(net, gl, seeds=[3, 4], sirt_iters=100, dist=learned.OUT_OF_DISTRIBUTION)
        r_far = learned.evaluate(net, gl, seeds=[5, 6], sirt_iters=100, dist=learned.FAR_OUT_OF_DISTRIBUTION)
        learned_res = {
            "workload": "256^3, 90 views, 384x256; 8 unrolled steps vs SIRT-100 from zero; each method timed "
                        "as the median of 3 passes after one untimed pass (CUDA events)",
            "training": "2000 seeded phantoms, each with 5-30 ellipsoids, densities U(lo, lo + 0.5..1.0) with "
                        "lo in 0.05..0.6, Poisson I0 log-uniform in 4e3..2e4 (learned.mixed_params)",
            "in_distribution": summary(r_in, "held-out seeds 1, 2: 10 ellipsoids, densities U(0.1, 1), "
                                             "Poisson I0 = 1e4 (inside the training ranges)"),
            "shifted": summary(r_shift, "seeds 3, 4: 30 ellipsoids, densities U(0.5, 1.5), Poisson I0 = 5e3 "
                                        "(at the edge of the training ranges)"),
            "out_of_distribution": summary(r_far, "seeds 5, 6: 40 ellipsoids, densities U(1.0, 2.2), Poisson "
                                                  "I0 = 2.5e3 (outside every training range)"),
        }
        del net
        torch.cuda.empty_cache()

    # end to end through the reference-facing C entry point, pinned host buffers
    e2e = None
    if parity is None:
        del proj, vol
    torch.cuda.empty_cache()
    if not args.no_e2e:
        hproj = torch.empty((NVIEWS, DET[1], DET[0]), dtype=torch.float32, pin_memory=True)
        hproj.normal_(generator=torch.Generator().manual_seed(7))
        hvol = torch.zeros(g.vol_shape, dtype=torch.float32, pin_memory=True)
        L = _lib.lib()
        i32 = lambda a: np.ascontiguousarray(np.asarray(a, np.int32))
        volDim, volStart, volEnd = i32(VOL), i32(g.vol_start), i32(g.vol_end)
        projDim, whs = i32([DET[0], DET[1], NVIEWS]), i32(DET)
        woff = i32(np.zeros(NVIEWS)); hoff = i32(np.zeros(NVIEWS))
        fp = lambda a: a.ctypes.data_as(_lib.c_float_p)
        ip = lambda a: a.ctypes.data_as(_lib.c_int_p)

        def call():
            L.GPU_CB_K_backproject(local, ctypes.c_void_p(hvol.data_ptr()), ctypes.c_void_p(hproj.data_ptr()),
                                   fp(g.angles), fp(g.hmid), ctypes.c_float(g.D), ctypes.c_float(g.pw),
                                   ip(volDim), ip(volStart), ip(volEnd), ip(projDim), ip(whs), ip(woff),
                                   ip(hoff), fp(g.norm), 2)
            _lib.check_last()

        call()
        barrier()
        # each call timed on its own (host clock around the whole call: copies in, kernels,
        # copies out); the median of the calls, since a single host-side stall (paging,
        # another process on the host) otherwise moves a two-call mean by a third
        ke = max(3, args.steps // 2)
        times = []
        for _ in range(ke):
            t0 = time.perf_counter()
            call()
            times.append(time.perf_counter() - t0)
        dt = barrier_max(float(np.median(times)))
        e2e = {"value": job_updates / dt / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": hproj.numel() * 4 + hvol.numel() * 4,
               "d2h_bytes_per_step": hvol.numel() * 4, "ms_per_step": dt * 1e3,
               "calls_ms": [round(t * 1e3, 1) for t in times], "statistic": f"median of {ke} calls",
               "path": "GPU_CB_K_backproject (C ABI), pinned host buffers"}

        # the reference's whole FDK path, fastcone.fbp (cosine weight + Shepp-Logan filter +
        # backprojection, the filtered projections returned into the caller's array), through
        # the C entry point fcb_fbp_host with the same pinned buffers
        gs = g.struct()

        def fbp_call():
            _lib.check(L.fcb_fbp_host(local, ctypes.byref(gs), _lib.FILTER_SHEPPLOGAN, ctypes.c_float(g.D),
                                      fp(g.hmid), 1, ctypes.c_void_p(hproj.data_ptr()),
                                      ctypes.c_void_p(hvol.data_ptr())))

        fbp_call()
        barrier()
        times = []
        for _ in range(ke):
            t0 = time.perf_counter()
            fbp_call()
            times.append(time.perf_counter() - t0)
        dt = barrier_max(float(np.median(times)))
        e2e["fbp"] = {"value": job_updates / dt / 1e9, "unit": UNIT,
                      "h2d_bytes_per_step": hproj.numel() * 4 + hvol.numel() * 4,
                      "d2h_bytes_per_step": hproj.numel() * 4 + hvol.numel() * 4, "ms_per_step": dt * 1e3,
                      "calls_ms": [round(t * 1e3, 1) for t in times], "statistic": f"median of {ke} calls",
                      "path": "fcb_fbp_host (C ABI; fastcone.fbp): cosine weight + Shepp-Logan filter on the GPU, "
                              "filtered views back into the host array, FDK backprojection; pinned host buffers"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(g)

    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    scaling = "weak" if args.shard == "replicas" else "strong"
    parallelism = f"replicas x{world}" if args.shard == "replicas" else f"z-slabs x{world}"
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": scaling,
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "inputs": "resident in HBM (value); pinned host buffers (e2e)",
                   "voxel_view_updates_per_step": updates, "D_voxels": g.D, "pw_voxels": g.pw,
                   "l2": "inputs (13.4 GB) larger than L2; no flush", "box": [info["box_w"], info["box_h"]],
                   "parallelism": parallelism},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                     "frac": achieved / smem_peak, "traffic": round(FDK_TRAFFIC_PER_LAUNCH),
                     "kernel": "fdk_tma_kernel<float,32,0,1,3>",
                     "note": f"achieved = 16 B/update (4 FP32 taps, each a 32-bit ld.shared from the "
                             f"TMA-staged box) x {updates // launches_per_step} updates per launch / the "
                             f"launch's mean CUDA-event time ({ms_launch:.1f} ms, {launches_per_step} "
                             f"launches per step); peak = 32-bit shared-memory load bandwidth measured "
                             f"in this run (fcb_smem_bandwidth, see smem_probe); traffic = DRAM bytes per "
                             f"launch, {FDK_TRAFFIC_NOTE}"},
        "hbm": {"achieved": FDK_TRAFFIC_PER_LAUNCH / (ms_launch / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": FDK_TRAFFIC_PER_LAUNCH / (ms_launch / 1e3) / 1e9 / hbm,
                "compulsory_bytes_per_step": (NVIEWS * DET[0] * DET[1] + 2 * launches_per_step * updates // NVIEWS) * 4,
                "note": f"DRAM bytes per launch (ncu) / launch time against the {peak_kind} HBM copy "
                        f"bandwidth; the gathers are served from shared memory, HBM is not the bound"},
        "smem_probe": probe,
        "bf16_storage": {"value": job_updates / (ms16 / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms16,
                         "roofline": {"bound": "smem", "achieved": ach16, "peak": smem_peak, "unit": "GB/s",
                                      "frac": ach16 / smem_peak,
                                      "note": "8 B/update: two 32-bit ld.shared of tap pairs (BF16 (w, w+1) "
                                              "per row)"}},
        "error_vs_fp64": parity,
        "fwd_proj": {"unit": "Gsamples/s", "samples_per_pass": nsamp,
                     "reference_sweep_samples_per_pass": ref_sweep,
                     "workload": "256^3, 360 views, 384x256 detector",
                     "note": "rates count the samples taken (rays clipped to the interpolant's support); the "
                             "reference marches a fixed sphere sweep per ray and window pixel "
                             "(reference_sweep_samples_per_pass, fcb_reference_windows), about 2.9x as many",
                     **{k: v for k, v in proj_res.items()}},
        "clocks": clk_summary,
        "katsevich": katsevich,
        "learned": learned_res,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
