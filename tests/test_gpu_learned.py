"""Learned unrolled reconstruction on a scaled-down sparse-view geometry (64^3, 90 views,
96 x 64 detector, same pixel pitch at the axis as the 256^3 configuration).

* the untrained network (last layers zero) is exactly its fallback, FDK + 8 SIRT steps;
* a short training on seeded phantoms beats that fallback on held-out phantoms.
"""
import pytest

pytestmark = pytest.mark.gpu


def _geom():
    from fastcone_b200.geometry import ConeGeometry

    return ConeGeometry.circular((64, 64, 64), 2.0, (96, 64), 4.0, 500.0, 1000.0, 90)


def test_untrained_network_is_fdk_plus_sirt():
    import torch

    from fastcone_b200 import learned

    g = _geom()
    ops_ = learned.Operators(g)
    net = learned.UnrolledNet().cuda()
    mu, y = learned.make_sample(ops_, 7)
    with torch.no_grad():
        x0 = ops_.fdk(y)
        x = net(x0, y, ops_)
        xb = x0.clone()
        for _ in range(learned.STEPS):
            xb = torch.relu(xb + ops_.sirt_step_dir(xb, y))
    assert torch.equal(x, xb)


def test_training_gains_over_fallback():
    import numpy as np
    import torch

    from fastcone_b200 import learned

    torch.manual_seed(0)
    g = _geom()
    net = learned.UnrolledNet().cuda()
    learned.train(net, g, n_phantoms=60, lr=2e-3, seed0=5000, log_every=1000, log=lambda *a: None)
    res = learned.evaluate(net, g, seeds=[1, 2, 3], sirt_iters=20)
    gain = np.mean([r["learned_psnr"] - r["no_net_psnr"] for r in res])
    assert gain > 0.5, [(r["learned_psnr"], r["no_net_psnr"]) for r in res]
