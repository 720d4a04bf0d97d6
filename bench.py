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
# dram__bytes_write.sum of every launch of one step of this benchmark (a one-pass capture of
# `bench.py --steps 1 --warmup 1`), mean over the step's 8 launches; they range from 15.2 GB
# (views near 0 and 180 degrees) to 68.3 GB (near 90 and 270 degrees), 326 GB per step
# (profiles/fdk_tma_kernel_fdk-slab.md).
FDK_TRAFFIC_PER_LAUNCH = 40.72e9
FDK_TRAFFIC_NOTE = "measured by ncu on the 8 launches of one step (mean; 15.2-68.3 GB per launch)"


def pi_window_fraction(g, nvox=4096, seed=0):
    """Fraction of voxel-view pairs inside the Tam-Danielsson window, estimated on random
    voxels with the window test of the FP64 Katsevich reference (u = sign * w / D, bounds
    q (pi/2 -+ atan u), q = P / (2 pi) (1 + u^2), lengths in voxels)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    nz, ny, nx = g.vol_shape
    xyz = rng.integers(0, [nx, ny, nz], size=(nvox, 3)).astype(np.float64)
    x = xyz[:, 0:1] - g.vol_xyz[0] // 2
    y = xyz[:, 1:2] - g.vol_xyz[1] // 2
    z = xyz[:, 2:3] - g.vol_xyz[2] // 2
    a = g.angles.astype(np.float64)[None, :]
    hm = g.hmid.astype(np.float64)[None, :] - g.vol_xyz[2] // 2
    U = g.D / (g.D + x * np.cos(a) + y * np.sin(a))
    w = (y * np.cos(a) - x * np.sin(a)) * U
    h = (z - hm) * U
    turn = float(g.angles[-1]) - float(g.angles[0])
    sgn = -1.0 if (turn >= 0) == (g.helical_pitch >= 0) else 1.0
    u = sgn * w / g.D
    q = g.helical_pitch / (2 * np.pi) * (1 + u * u)
    inside = (h <= q * (np.pi / 2 - np.arctan(u))) & (h >= -q * (np.pi / 2 + np.arctan(u)))
    return float(inside.mean())


def smem_roofline(gather_gbs, clocks):
    """The binding ceiling of the FDK kernel: 4 ld.shared per voxel-view update, one 128-byte
    wavefront per warp instruction -> 128 B/clk/SM of gather bytes on 148 SMs."""
    mhz = clocks.get("sm_mhz") or 1965.0
    peak = 128.0 * 148 * mhz * 1e6 / 1e9
    return {"bound": "smem", "achieved": gather_gbs, "peak": peak, "unit": "GB/s", "frac": gather_gbs / peak,
            "clock_mhz": mhz, "note": "peak = 128 B/clk/SM x 148 SMs x median sampled SM clock"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--shard", default="replicas", choices=["replicas", "z"],
                    help="N>1: independent volumes per rank (weak scaling) or one volume in z-slabs "
                         "(strong scaling)")
    ap.add_argument("--case", default=None,
                    choices=["fdk-slab", "fdk-slab-bf16", "proj-512", "conv-256", "katsevich", "pipeline",
                             "misaligned-256"],
                    help="profiling case: run only this kernel on a reduced workload (no JSON line)")
    return ap.parse_args()


def run_case(args):
    """Reduced single-kernel workloads for ncu captures (a few GB on the device):
    fdk-slab[-bf16]: the 1024^3 geometry restricted to a 1024x1024x128 z-slab (z 448..575),
    64 views (0.5 GB volume + 0.4 GB projections);
    proj-512: the staged, unstaged and texture projectors on 512^3, 90 views, 768x512
    detector (0.5 GB volume);
    conv-256: one unrolled step's convolutions at 256^3 x 16 BF16 channels (0.54 GB per
    activation): forward (three kernel forms) and weight gradient (tensor cores and the
    CUDA-core kernel), all on tcgen05 except the last;
    katsevich: the helical PI-window backprojection (512x512x384, 4640 views; 1.3 GB);
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


def cpu_baseline(g, target_s=12.0):
    """One bounded sample of the CPU reference path (about `target_s` seconds); returns the
    cpu_baseline object of the JSON line."""
    ref = CpuReferencePath(g)
    ref.calibrate(target_s)
    dt, upd = ref.sample()
    return {"value": upd / dt / 1e9, "unit": UNIT, "cores": ref.cores, "kind": "port",
            "sample": ref.describe(dt, upd)}


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

    # BF16-stored filtered projections (same kernel family, 2-byte gathers)
    proj16 = proj.to(torch.bfloat16)
    plan16 = ops.BackprojectPlan(g, mode=_lib.MODE_FDK, dtype=torch.bfloat16)
    for _ in range(2):
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
    frac = pi_window_fraction(gk)
    katsevich = {"workload": "helical 512x512x384, 4 turns x 1160 views, 736x64 detector, PI window",
                 "ms_per_pass": ms_k, "filter_ms": ms_kf, "dense_GUPS": dense / (ms_k / 1e3) / 1e9,
                 "pi_window_pairs_fraction": frac, "pi_window_GUPS": frac * dense / (ms_k / 1e3) / 1e9,
                 "launches": kplan.info()["launches"]}
    del pk, vk, kplan

    # learned unrolled reconstruction vs SIRT-100 (committed weights), two held-out phantoms
    learned_res = None
    wpath = os.path.join(ROOT, "fastcone_b200", "weights", "unrolled8.pt")
    if not args.no_learned and rank == 0 and os.path.exists(wpath):
        from fastcone_b200 import learned

        net = learned.UnrolledNet().to(dev)
        net.load_state_dict(torch.load(wpath, map_location=dev)["model"])
        r = learned.evaluate(net, configs.learned_sparse(), seeds=[1, 2], sirt_iters=100)
        mean = lambda k: sum(x[k] for x in r) / len(r)  # noqa: E731
        sp = [x["speedup_to_sirt_psnr"] for x in r]
        learned_res = {
            "workload": "256^3, 90 views, 384x256, Poisson I0=1e4; 8 unrolled steps vs SIRT-100 from zero",
            "sirt100_psnr": mean("sirt_psnr"), "sirt100_ssim": mean("sirt_ssim"), "sirt100_s": mean("sirt_time_s"),
            "learned_psnr": mean("learned_psnr"), "learned_ssim": mean("learned_ssim"),
            "learned_s": mean("learned_time_s"), "fdk_psnr": mean("fdk_psnr"),
            "fallback_psnr": mean("no_net_psnr"),
            "time_to_sirt100_psnr_s": [x["time_to_sirt_psnr_s"] for x in r],
            "speedup_to_sirt100_psnr": sp,
        }
        del net
        torch.cuda.empty_cache()

    # end to end through the reference-facing C entry point, pinned host buffers
    e2e = None
    if not args.no_e2e:
        del proj
        torch.cuda.empty_cache()
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
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": round(FDK_TRAFFIC_PER_LAUNCH),
                     "note": f"achieved = 16 B/update bilinear gather bytes per launch / launch time "
                             f"(CUDA events); peak = {peak_kind} HBM copy bandwidth. frac > 1: the gathers "
                             f"are served from shared memory (TMA-staged boxes), see smem_roofline; "
                             f"traffic = DRAM bytes per launch, {FDK_TRAFFIC_NOTE}"},
        "smem_roofline": smem_roofline(achieved, clk_summary),
        "bf16_storage": {"value": job_updates / (ms16 / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms16},
        "fwd_proj": {"unit": "Gsamples/s", "samples_per_pass": nsamp,
                     "workload": "256^3, 360 views, 384x256 detector",
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
