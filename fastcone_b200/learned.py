"""Learned unrolled reconstruction for sparse-view, noisy cone-beam data.

Workload: 256^3 volumes from 90 views on a 384 x 256 detector (configs.learned_sparse),
transmission data with Poisson noise at I0 = 1e4 photons.

    x_0     = FDK(y)                                        (GPU filter + backprojection)
    g_k     = C * B(R * (y - A x_k))                        (the SIRT step)
    x_{k+1} = max(0, x_k + g_k + CNN_k([x_k, g_k]))         k = 0..7

A is the projector (texture trilinear, this project's kernel), B the voxel-driven unweighted
backprojector (kernelMode 0, the reference's iterative-reconstruction backprojector),
R = 1/(A 1), C = 1/(B 1).  Each CNN_k has 3 layers (2->16->16->1 channels, 3^3 kernels,
ReLU between) on the tcgen05 convolution kernels with BF16 weights/activations and FP32
accumulation; its last layer starts at zero, so the untrained network is exactly FDK + 8
SIRT steps (the fallback it is compared with).  The SIRT step g_k enters the network as
data: training back-propagates through the CNNs and the x_k path, not through A and B.

Attenuation: phantom densities U(0.1, 1.0) scaled by MU_PER_VOXEL = 0.025 per voxel, which
puts the longest line integrals of the 10-ellipsoid phantoms near 3.
"""
from __future__ import annotations

import dataclasses
import math
import statistics
import time

import numpy as np
import torch

from . import _lib, configs, ops
from .geometry import ConeGeometry
from .nn import Conv3d
from .phantom import random_ellipsoids

MU_PER_VOXEL = 0.025
I0 = 1.0e4
N_ELLIPSOIDS = 10
STEPS = 8
X_SCALE = 1.0 / 0.05   # network input scaling of attenuation values (per voxel)


class Operators:
    """A, B, R, C and the FDK initialiser for one geometry (plans built once)."""

    def __init__(self, geom: ConeGeometry):
        self.g = dataclasses.replace(geom, norm=np.ones(geom.nviews, np.float32))
        self.A = ops.ProjectPlan(self.g, _lib.PROJ_TEXTURE)
        self.Aexact = ops.ProjectPlan(self.g, _lib.PROJ_EXPLICIT)
        self.Bplan = ops.BackprojectPlan(self.g, mode=_lib.MODE_UNWEIGHTED)
        gf = configs.with_fdk_norm(self.g)
        self.fdk_plan = ops.BackprojectPlan(gf, mode=_lib.MODE_FDK)
        self.filter_plan = ops.FilterPlan(self.g.proj_shape)
        dev = torch.device("cuda", torch.cuda.current_device())
        ones_v = torch.ones(self.g.vol_shape, device=dev)
        ones_p = torch.ones(self.g.proj_shape, device=dev)
        self.R = _safe_inv(self.A(ones_v))
        self.C = _safe_inv(self.B(ones_p))

    def B(self, p):
        v = torch.zeros(self.g.vol_shape, device=p.device)
        return self.Bplan(p.contiguous(), v)

    def sirt_step_dir(self, x, y):
        return self.C * self.B((y - self.A(x)) * self.R)

    def fdk(self, y):
        f = self.filter_plan(y, zorigin=self.g.hmid, D=self.g.D)
        v = torch.zeros(self.g.vol_shape, device=y.device)
        # the reference's FDK scale is pw times the attenuation (pw = 1 voxel here)
        return self.fdk_plan(f, v).mul_(1.0 / self.g.pw).clamp_(min=0.0)


def _safe_inv(t, eps=1e-6):
    return torch.where(t > eps, 1.0 / t.clamp_min(eps), torch.zeros_like(t))


# The training distribution, and a shifted one for out-of-distribution evaluation: three
# times the ellipsoids, denser material (mean density x 1.8) and half the photons.
IN_DISTRIBUTION = {"n_ellipsoids": None, "density": (0.1, 1.0), "i0": None}
OUT_OF_DISTRIBUTION = {"n_ellipsoids": 30, "density": (0.5, 1.5), "i0": 5e3}
# beyond every range of the mixed training distribution below (more ellipsoids, denser,
# fewer photons)
FAR_OUT_OF_DISTRIBUTION = {"n_ellipsoids": 40, "density": (1.0, 2.2), "i0": 2.5e3}


def mixed_params(seed: int) -> dict:
    """Phantom and noise parameters of the mixed training distribution, drawn per phantom from
    its seed: 5-30 ellipsoids, densities U(lo, hi) with lo ~ U(0.05, 0.6) and hi - lo ~
    U(0.5, 1.0), I0 log-uniform in [4e3, 2e4] photons."""
    rng = np.random.default_rng(seed + 7919)
    k = int(rng.integers(5, 31))
    lo = float(rng.uniform(0.05, 0.6))
    hi = lo + float(rng.uniform(0.5, 1.0))
    i0 = float(10.0 ** rng.uniform(math.log10(4e3), math.log10(2e4)))
    return {"n_ellipsoids": k, "density": (lo, hi), "i0": i0}


def make_sample(ops_: Operators, seed: int, device="cuda", n_ellipsoids=None, density=(0.1, 1.0), i0=None):
    """Seeded phantom (attenuation per voxel) and its noisy log-transformed projections; the
    defaults are the training distribution (N_ELLIPSOIDS ellipsoids, densities U(0.1, 1),
    I0 photons)."""
    g = ops_.g
    n_ellipsoids = n_ellipsoids or N_ELLIPSOIDS
    i0 = i0 or I0
    mu = ops.phantom(g.vol_xyz, random_ellipsoids(n_ellipsoids, g.vol_xyz, seed, density=density), device=device)
    mu.mul_(MU_PER_VOXEL)
    p = ops_.Aexact(mu)
    gen = torch.Generator(device=device).manual_seed(seed)
    counts = torch.poisson(i0 * torch.exp(-p), generator=gen)
    y = -torch.log(counts.clamp_min(1.0) / i0)
    return mu, y


class UnrolledNet(torch.nn.Module):
    def __init__(self, steps: int = STEPS):
        super().__init__()
        self.steps = steps
        self.blocks = torch.nn.ModuleList()
        for _ in range(steps):
            l3 = Conv3d(16, 1, relu=False)
            torch.nn.init.zeros_(l3.weight)
            self.blocks.append(torch.nn.ModuleList([Conv3d(2, 16, relu=True), Conv3d(16, 16, relu=True), l3]))

    @staticmethod
    def pack(x, g):
        """[x, g] -> BF16 activations of 16 channels (14 zero) in the convolution layout
        [nz, ny, 2, nx, 8]."""
        nz, ny, nx = x.shape
        t = torch.zeros((nz, ny, 2, nx, 8), device=x.device, dtype=torch.bfloat16)
        t[:, :, 0, :, 0] = (x * X_SCALE).to(torch.bfloat16)
        t[:, :, 0, :, 1] = (g * X_SCALE).to(torch.bfloat16)
        return t

    def step(self, k, x, g):
        h = self.pack(x, g)
        for layer in self.blocks[k]:
            h = layer(h)
        return h[:, :, 0, :, 0].float() / X_SCALE

    def forward(self, x0, y, ops_: Operators, callback=None):
        x = x0
        for k in range(self.steps):
            with torch.no_grad():
                g = ops_.sirt_step_dir(x.detach(), y)
            x = torch.relu(x + g + self.step(k, x, g))
            if callback is not None:
                callback(k, x)
        return x


def fov_mask(geom: ConeGeometry, device="cuda"):
    """Voxels every view sees: inside the inscribed cylinder of the detector's fan and
    within the central slab the cone covers at its narrowest."""
    nz, ny, nx = geom.vol_shape
    W, H = geom.det_wh
    D, pw = geom.D, geom.pw
    r = 0.5 * W * pw * D / math.sqrt(D * D + (0.5 * W * pw) ** 2)
    rfov = r * D / (D + r)
    zi = torch.arange(nz, device=device) - nz // 2
    yi = torch.arange(ny, device=device) - ny // 2
    xi = torch.arange(nx, device=device) - nx // 2
    rr = torch.sqrt(yi[:, None].float() ** 2 + xi[None, :].float() ** 2)
    hz = 0.5 * H * pw * (D - rfov) / D
    return (rr[None] <= rfov - 1) & (zi.abs()[:, None, None].float() <= hz - 1)


def psnr(x, ref, mask):
    mse = torch.mean((x[mask] - ref[mask]) ** 2)
    return float(10 * torch.log10(ref[mask].max() ** 2 / mse))


def ssim3d(x, ref, mask, sigma=1.5):
    """3-D SSIM (Gaussian window, standard constants) averaged over the mask."""
    import torch.nn.functional as F

    L = float(ref[mask].max())
    c1, c2 = (0.01 * L) ** 2, (0.03 * L) ** 2
    r = int(3 * sigma)
    t = torch.arange(-r, r + 1, device=x.device, dtype=torch.float64)
    g1 = torch.exp(-t * t / (2 * sigma * sigma))
    g1 = g1 / g1.sum()

    def blur(v):
        v = v[None, None]
        v = F.conv3d(v, g1.view(1, 1, -1, 1, 1), padding=(r, 0, 0))
        v = F.conv3d(v, g1.view(1, 1, 1, -1, 1), padding=(0, r, 0))
        v = F.conv3d(v, g1.view(1, 1, 1, 1, -1), padding=(0, 0, r))
        return v[0, 0]

    x, ref = x.double(), ref.double()  # the variance differences below need the precision
    mx, my = blur(x), blur(ref)
    sxx = blur(x * x) - mx * mx
    syy = blur(ref * ref) - my * my
    sxy = blur(x * ref) - mx * my
    s = ((2 * mx * my + c1) * (2 * sxy + c2)) / ((mx * mx + my * my + c1) * (sxx + syy + c2))
    return float(s[mask].mean())


def step_weights(steps: int = STEPS, final: float = 2.0):
    """Loss weight of each unrolled step's output: every step is supervised (so each
    intermediate x_k is already a good reconstruction and the chain can stop early), the
    final output counts `final` times; normalised to sum 1."""
    w = [1.0] * (steps - 1) + [final]
    t = sum(w)
    return [v / t for v in w]


def train(net: UnrolledNet, geom: ConeGeometry, n_phantoms: int = 2000, lr: float = 1e-3, seed0: int = 1000,
          log_every: int = 50, checkpoint: str | None = None, log=print, deep: bool = True,
          mixed: bool = False):
    """Trains on seeded phantoms generated (and projected) on the GPU, one per step.
    deep=True supervises every step's output (step_weights), else only the last.
    mixed=True draws each phantom's parameters from mixed_params (else the fixed training
    distribution: N_ELLIPSOIDS ellipsoids, densities U(0.1, 1), I0 photons)."""
    ops_ = Operators(geom)
    mask = fov_mask(ops_.g)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, n_phantoms)
    wk = step_weights(net.steps) if deep else [0.0] * (net.steps - 1) + [1.0]
    t0 = time.time()
    for i in range(n_phantoms):
        mu, y = make_sample(ops_, seed0 + i, **(mixed_params(seed0 + i) if mixed else {}))
        with torch.no_grad():
            x0 = ops_.fdk(y)
        outs = []
        x = net(x0, y, ops_, callback=lambda k, xk: outs.append(xk))
        m = mu[mask]
        loss = sum(w * torch.mean((xk[mask] - m) ** 2) for w, xk in zip(wk, outs) if w > 0)
        loss = loss / MU_PER_VOXEL ** 2
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        sched.step()
        if (i + 1) % log_every == 0 or i == 0:
            log(f"train {i + 1}/{n_phantoms} loss {loss.item():.4e} psnr {psnr(x.detach(), mu, mask):.2f} "
                f"t {time.time() - t0:.0f}s")
        if checkpoint and (i + 1) % 500 == 0:
            torch.save({"model": net.state_dict(), "optim": opt.state_dict(), "phantoms_seen": i + 1,
                        "seed0": seed0, "deep": deep, "mixed": mixed}, checkpoint)
    return net


@torch.no_grad()
def evaluate(net: UnrolledNet, geom: ConeGeometry, seeds, sirt_iters: int = 100, dist=None, reps: int = 3):
    """Per phantom: SIRT-sirt_iters (from zero) PSNR/SSIM/time; FDK + k SIRT steps without the
    network; the learned steps with their cumulative times; time to reach SIRT's PSNR.
    `dist`: phantom / noise distribution (make_sample's keywords; default: the training one).
    Both methods are timed the same way: one untimed pass (plans, allocator), then `reps`
    timed passes with CUDA events; the median pass time counts (per step for the learned
    steps)."""
    ops_ = Operators(geom)
    mask = fov_mask(ops_.g)
    dist = {k: v for k, v in (dist or {}).items() if v is not None}
    res = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for s in seeds:
        mu, y = make_sample(ops_, s, **dist)
        t_runs = []
        for rep in range(reps + 1):
            x = torch.zeros_like(mu)
            torch.cuda.synchronize()
            ev0.record()
            for _ in range(sirt_iters):
                x = torch.relu(x + ops_.sirt_step_dir(x, y))
            ev1.record()
            torch.cuda.synchronize()
            if rep > 0:
                t_runs.append(ev0.elapsed_time(ev1) / 1e3)
        t_sirt = statistics.median(t_runs)
        p_sirt, s_sirt = psnr(x, mu, mask), ssim3d(x, mu, mask)
        # learned: cumulative time at each step (events between steps, no host sync)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(STEPS + 2)]
        runs = []
        for rep in range(reps + 1):
            states = []
            torch.cuda.synchronize()
            marks[0].record()
            x = ops_.fdk(y)
            marks[1].record()
            states.append(x)
            for k in range(STEPS):
                g = ops_.sirt_step_dir(x, y)
                x = torch.relu(x + g + net.step(k, x, g))
                marks[k + 2].record()
                states.append(x)
            torch.cuda.synchronize()
            if rep > 0:
                runs.append([marks[0].elapsed_time(m) / 1e3 for m in marks[1:]])
        times = [statistics.median(c) for c in zip(*runs)]
        psnrs = [psnr(v, mu, mask) for v in states]
        # the same pipeline without the network (FDK + SIRT steps)
        xb = states[0].clone()
        for k in range(STEPS):
            xb = torch.relu(xb + ops_.sirt_step_dir(xb, y))
        p_base = psnr(xb, mu, mask)
        k_eq = next((k for k, p in enumerate(psnrs) if p >= p_sirt), None)
        res.append({
            "seed": s, "sirt_psnr": p_sirt, "sirt_ssim": s_sirt, "sirt_time_s": t_sirt,
            "learned_psnr": psnrs[-1], "learned_ssim": ssim3d(states[-1], mu, mask),
            "learned_time_s": times[-1], "step_psnr": psnrs, "step_time_s": times,
            "fdk_psnr": psnrs[0], "no_net_psnr": p_base,
            "time_to_sirt_psnr_s": None if k_eq is None else times[k_eq],
            "speedup_to_sirt_psnr": None if k_eq is None else t_sirt / times[k_eq],
        })
    return res


def main():
    import argparse
    import json

    ap = argparse.ArgumentParser(description="train / evaluate the unrolled reconstruction")
    ap.add_argument("--train", type=int, default=0, help="number of training phantoms")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--weights", default=None, help="load weights from / save weights to this file")
    ap.add_argument("--eval", type=int, default=0, help="number of held-out phantoms to evaluate")
    ap.add_argument("--out", default=None, help="write the evaluation JSON here")
    ap.add_argument("--final-only", action="store_true", help="supervise only the last step")
    ap.add_argument("--mixed", action="store_true", help="train on the mixed distribution (mixed_params)")
    a = ap.parse_args()
    torch.manual_seed(0)
    geom = configs.learned_sparse()
    net = UnrolledNet().cuda()
    if a.weights and a.train == 0:
        net.load_state_dict(torch.load(a.weights, map_location="cuda")["model"])
    if a.train:
        train(net, geom, a.train, a.lr, checkpoint=a.weights, deep=not a.final_only, mixed=a.mixed)
        if a.weights:
            torch.save({"model": net.state_dict(), "phantoms_seen": a.train, "deep": not a.final_only,
                        "mixed": a.mixed}, a.weights)
    if a.eval:
        r = evaluate(net, geom, list(range(1, a.eval + 1)))
        s = json.dumps(r)
        print(s)
        if a.out:
            with open(a.out, "w") as f:
                f.write(s)


if __name__ == "__main__":
    main()
