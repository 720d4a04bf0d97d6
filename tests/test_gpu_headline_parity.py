"""Parity at the full headline sizes, against the FP64 oracle on sampled voxel columns.

* Large circular FDK (1024^3, 1440 views, 1536x1024): a seeded 50-ellipsoid phantom projected
  by the explicit projector, cosine-weighted and Shepp-Logan filtered on the GPU, then
  backprojected over the whole volume from FP32- and from BF16-stored filtered projections
  (FP32 accumulation both).  64 random full-z columns are compared with the oracle's FP64
  backprojection of the same FP32 filtered projections (coneBeamGPU.cu:341-420 restated).
  Bounds: FP32 storage rel-L2 <= 2e-5 and max-abs <= 2e-5 of the largest reference value
  (FP32 arithmetic, as the small-size parity tests); BF16 storage rel-L2 <= 1e-3 and max-abs
  <= 1e-3 of it (BF16 keeps 8 significant bits of each filtered value; the rounding errors of
  the 1440 views average out in the sum); FP16 storage (11 significant bits) <= 2e-4 both.
* Helical Katsevich (512x512x384, 4 turns x 1160 views, 736x64): the projected phantom is
  Katsevich-filtered on the GPU and backprojected with the PI window; 64 random full-z
  columns vs the oracle's FP64 PI-window backprojection (coneBeamGPU.cu:258-338 plus the
  Tam-Danielsson window), rel-L2 <= 1e-3 (the parity bound against the reference) and
  max-abs <= two single-view contributions: the window is a sharp cut that the kernel
  decides in FP32 and the oracle in FP64, so a voxel whose window edge falls within rounding
  of a view gains or loses that view at its entry or exit.  Their in-window voxel-view pairs
  counted on the GPU equal the oracle's count.

Each test states both errors in its failure message."""
import pytest

pytestmark = pytest.mark.gpu


def test_fdk_1024_fp32_bf16_fp16_storage_vs_fp64():
    import torch

    import bench

    r = bench.fdk_parity(torch.device("cuda", 0), ncols=64)
    f32, b16, h16 = r["f32"], r["bf16"], r["f16"]
    assert f32["rel_l2"] <= 2e-5 and f32["max_abs"] <= 2e-5 * f32["ref_max_abs"], r
    assert b16["rel_l2"] <= 1e-3 and b16["max_abs"] <= 1e-3 * b16["ref_max_abs"], r
    assert h16["rel_l2"] <= 2e-4 and h16["max_abs"] <= 2e-4 * h16["ref_max_abs"], r


def test_helix_pi_window_vs_fp64():
    import torch

    import bench

    r = bench.helix_parity(torch.device("cuda", 0), ncols=64)
    e = r["f32"]
    assert e["rel_l2"] <= 1e-3 and e["max_abs"] <= 2.0 * r["one_view_max"], r
    assert r["pi_pairs_gpu"] == r["pi_pairs_oracle"], r
