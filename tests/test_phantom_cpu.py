"""The synthetic-input generator: seeded ellipsoid parameters follow the stated
distributions (centres in the scaled unit ball, semi-axes and densities in their ranges,
proper rotations), and the same seed gives the same phantom."""
import numpy as np


def test_random_ellipsoids_distribution_and_determinism():
    from fastcone_b200.phantom import random_ellipsoids

    vol = (128, 96, 64)
    p = random_ellipsoids(200, vol, seed=7, axes=(0.05, 0.4), density=(0.1, 1.0), centre_radius=0.8)
    assert p.shape == (200, 16)
    assert np.array_equal(p, random_ellipsoids(200, vol, seed=7, axes=(0.05, 0.4), density=(0.1, 1.0),
                                               centre_radius=0.8))
    assert not np.array_equal(p, random_ellipsoids(200, vol, seed=8))
    half = np.array(vol, float) / 2
    assert np.all(np.linalg.norm(p[:, 0:3] / half, axis=1) <= 0.8 + 1e-12)
    hw = half.min()
    assert np.all((p[:, 3:6] >= 0.05 * hw) & (p[:, 3:6] <= 0.4 * hw))
    assert np.all((p[:, 15] >= 0.1) & (p[:, 15] <= 1.0))
    for row in p:
        R = row[6:15].reshape(3, 3)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-12) and np.isclose(np.linalg.det(R), 1.0)


def test_voxelised_phantom_is_the_sum_of_its_ellipsoids():
    """Densities add where ellipsoids overlap (the oracle's voxelisation, which the GPU
    phantom kernel must equal bit for bit)."""
    from oracle import oracle as O

    from fastcone_b200.phantom import random_ellipsoids

    vol = (24, 20, 16)
    p = random_ellipsoids(3, vol, seed=2, axes=(0.3, 0.5), centre_radius=0.3)
    whole = O.phantom_voxelize(vol, p)
    parts = sum(O.phantom_voxelize(vol, p[k:k + 1]) for k in range(3))
    assert np.allclose(whole, parts, atol=1e-6)
    assert whole.max() > 0 and whole.shape == vol[::-1]


def test_mixed_training_distribution():
    """learned.mixed_params: deterministic per seed, inside its stated ranges, and the far
    evaluation set lies outside every one of them."""
    import math

    from fastcone_b200 import learned

    ps = [learned.mixed_params(s) for s in range(1000, 1400)]
    assert ps[0] == learned.mixed_params(1000)
    for p in ps:
        lo, hi = p["density"]
        assert 5 <= p["n_ellipsoids"] <= 30
        assert 0.05 <= lo <= 0.6 and 0.5 <= hi - lo <= 1.0
        assert 4e3 * (1 - 1e-9) <= p["i0"] <= 2e4 * (1 + 1e-9)
    assert len({p["n_ellipsoids"] for p in ps}) > 20
    assert min(math.log10(p["i0"]) for p in ps) < 3.7 and max(math.log10(p["i0"]) for p in ps) > 4.2
    far = learned.FAR_OUT_OF_DISTRIBUTION
    assert far["n_ellipsoids"] > 30 and far["density"][1] > 1.6 and far["i0"] < 4e3
