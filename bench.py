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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--case", default=None, choices=["fdk-slab", "fdk-slab-bf16", "proj-512"],
                    help="profiling case: run only this kernel on a reduced workload (no JSON line)")
    return ap.parse_args()


def run_case(args):
    """Reduced single-kernel workloads for ncu captures (a few GB on the device):
    fdk-slab[-bf16]: the 1024^3 geometry restricted to a 1024x1024x128 z-slab (z 448..575),
    64 views (0.5 GB volume + 0.4 GB projections);
    proj-512: both projectors on 512^3, 90 views, 768x512 detector (0.5 GB volume)."""
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
    else:
        g = ConeGeometry.circular((512, 512, 512), 1.0, (768, 512), 1.0, 1000.0, 2000.0, 90)
        from fastcone_b200.phantom import random_ellipsoids

        v = ops.phantom(g.vol_xyz, random_ellipsoids(10, g.vol_xyz, 1), device=dev)
        for _ in range(args.warmup + args.steps):
            ops.project(v, g, method=_lib.PROJ_EXPLICIT)
            ops.project(v, g, method=_lib.PROJ_TEXTURE)
    ops.sync_status()
    torch.cuda.synchronize()
    print("case", args.case, "done")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


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


def cpu_baseline(g, target_s=12.0):
    """Reference path (texture-emulating restatement of Fastcone's FDK kernel, sub-problem
    tiling and windows) on this host's cores, on a bounded sample: whole detector-height
    columns of voxels (all z, all views) at random (x, y); returns GUPS and the sample."""
    import numpy as np

    from oracle import oracle as O

    pb = O.make_problem(VOL, DET, NVIEWS, D=g.D, pw=g.pw, angles=g.angles, hmid=g.hmid, norm=g.norm)
    rng = np.random.default_rng(0)
    proj = rng.standard_normal((NVIEWS, DET[1], DET[0]), dtype=np.float32)
    cores = os.cpu_count() or 1

    def run(ncols):
        xy = rng.integers(0, VOL[0], size=(ncols, 2))
        z = np.arange(VOL[2])
        pts = np.stack([np.repeat(xy[:, 0], VOL[2]), np.repeat(xy[:, 1], VOL[2]), np.tile(z, ncols)], 1)
        t0 = time.perf_counter()
        O.ref_backproject_points(pb, proj, pts.astype(np.int32), kernel_mode=2, texq=1)
        return time.perf_counter() - t0, len(pts) * NVIEWS

    dt, upd = run(2)
    ncols = max(2, int(2 * target_s / max(dt, 1e-3)))
    dt, upd = run(ncols)
    return {"value": upd / dt / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{ncols} random (x,y) columns x {VOL[2]} z x {NVIEWS} views = {upd:.3g} updates "
                      f"of the 1024^3 / 1440-view FDK, texture-emulating reference path "
                      f"(oracle/fc_oracle.c), {dt:.1f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    g = geometry()
    cb = cpu_baseline(g)
    out = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "circular FDK 1024^3, 1440 views, 1536x1024 detector (bounded sample)",
                      "sample": cb["sample"]},
           "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
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

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    def barrier_max(x):
        if world == 1:
            return x
        import torch.distributed as dist

        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    g = geometry()
    updates = VOL[0] * VOL[1] * VOL[2] * NVIEWS
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
    ms = e0.elapsed_time(e1)
    ms = barrier_max(ms)
    ms_step = ms / args.steps
    value = world * updates / (ms_step / 1e3) / 1e9

    hbm, peak_kind = measured_peaks()
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
    for name, meth in (("explicit", _lib.PROJ_EXPLICIT), ("texture", _lib.PROJ_TEXTURE)):
        for _ in range(2):
            pp.zero_()
            ops.project(pv, gp, method=meth, proj=pp)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(3):
            ops.project(pv, gp, method=meth, proj=pp)
        e1.record(st)
        torch.cuda.synchronize()
        proj_res[name] = nsamp / (e0.elapsed_time(e1) / 3 / 1e3) / 1e9
    del pv, pp

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
        volDim, volStart, volEnd = i32(VOL), i32([0, 0, 0]), i32(VOL)
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
        t0 = time.perf_counter()
        ke = max(2, args.steps // 2)
        for _ in range(ke):
            call()
        dt = barrier_max(time.perf_counter() - t0) / ke
        e2e = {"value": world * updates / dt / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": hproj.numel() * 4 + hvol.numel() * 4,
               "d2h_bytes_per_step": hvol.numel() * 4, "ms_per_step": dt * 1e3,
               "path": "GPU_CB_K_backproject (C ABI), pinned host buffers"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(g)

    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "circular FDK backprojection 1024^3 voxels, 1440 views, 1536x1024 detector, "
                               "FP32 filtered projections in HBM",
                   "voxel_view_updates_per_step": updates, "D_voxels": g.D, "pw_voxels": g.pw,
                   "l2": "inputs (13.4 GB) larger than L2; no flush", "box": [info["box_w"], info["box_h"]],
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "note": f"achieved = 16 B/update bilinear gather bytes / kernel time; peak {peak_kind} "
                             f"HBM copy bandwidth; the gathers are served from shared memory"},
        "bf16_storage": {"value": world * updates / (ms16 / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms16},
        "fwd_proj": {"unit": "Gsamples/s", "samples_per_pass": nsamp,
                     "workload": "256^3, 360 views, 384x256 detector",
                     **{k: v for k, v in proj_res.items()}},
        "clocks": clk.summary(),
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
