"""tcgen05 3x3x3 convolution vs torch.nn.functional.conv3d in FP32 on the same BF16-rounded
inputs (FP32 accumulation both sides: rel-L2 <= 1e-5), the tcgen05 weight gradient vs
torch's in FP32 on the same BF16 inputs (rel-L2 <= 2e-4: sums over up to 5e5 voxels in a
different order), input and weight gradients vs torch autograd (rel-L2 <= 1e-2 -- the
gradient flowing in is rounded to BF16 by design)."""
import pytest

pytestmark = pytest.mark.gpu


def _ref(x_l, w, b, relu):
    import torch
    import torch.nn.functional as F

    from fastcone_b200 import nn

    x = nn.from_layout(x_l).float().unsqueeze(0)                 # [1, C, z, y, x]
    y = F.conv3d(x, w.float(), b.float(), padding=1)
    if relu:
        y = torch.relu(y)
    return nn.to_layout(y.squeeze(0))                            # [z, y, 2, x, 8]


def _act(shape, g, dtype=None):
    import torch

    from fastcone_b200 import nn

    t = nn.to_layout(torch.randn((16,) + tuple(shape), device="cuda", generator=g))
    return t.to(dtype) if dtype is not None else t


def _rel(a, b):
    return float((a.float() - b.float()).norm() / b.float().norm())


@pytest.mark.parametrize("shape", [(20, 17, 130), (8, 9, 256), (3, 5, 7)])
@pytest.mark.parametrize("relu", [False, True])
def test_conv_forward_vs_torch(shape, relu):
    import torch

    from fastcone_b200 import nn

    g = torch.Generator(device="cuda").manual_seed(0)
    x = _act(shape, g, torch.bfloat16)
    w = (torch.randn(16, 16, 3, 3, 3, device="cuda", generator=g) * 0.1).to(torch.bfloat16).float()
    b = torch.randn(16, device="cuda", generator=g)
    y = nn.conv3d16(x, nn.to_kernel_weights(w).to(torch.bfloat16).contiguous(), b, relu=relu,
                    out_dtype=torch.float32)
    ref = _ref(x, w, b, relu)
    assert _rel(y, ref) < 1e-5, _rel(y, ref)


def test_conv_gradients_vs_torch():
    import torch
    import torch.nn.functional as F

    from fastcone_b200 import nn

    g = torch.Generator(device="cuda").manual_seed(1)
    shape = (12, 10, 140)
    x = _act(shape, g, torch.bfloat16)
    w = (torch.randn(16, 16, 3, 3, 3, device="cuda", generator=g) * 0.1).to(torch.bfloat16).float()
    b = torch.randn(16, device="cuda", generator=g) * 0.1
    gy = _act(shape, g)

    # ours: gradients through the custom function
    xin = x.clone().requires_grad_(True)
    w2 = w.clone().requires_grad_(True)
    b2 = b.clone().requires_grad_(True)
    y2 = nn.Conv3d16Function.apply(xin, w2, b2, True)
    (y2.float() * gy).sum().backward()
    # reference in FP32
    xr = nn.from_layout(x).float().unsqueeze(0).clone().requires_grad_(True)
    wr = w.clone().requires_grad_(True)
    br = b.clone().requires_grad_(True)
    yr = nn.to_layout(torch.relu(F.conv3d(xr, wr, br, padding=1)).squeeze(0))
    (yr * gy).sum().backward()
    gx_ref = nn.to_layout(xr.grad.squeeze(0))
    assert _rel(xin.grad, gx_ref) < 1e-2
    assert _rel(w2.grad, wr.grad) < 1e-2
    assert _rel(b2.grad, br.grad) < 1e-2


@pytest.mark.parametrize("shape", [(20, 17, 130), (4, 3, 512), (1, 1, 5), (37, 41, 300), (6, 70, 128)])
def test_persistent_conv_equals_one_tile_per_cta(shape, monkeypatch):
    """The row-reusing persistent kernel (default), the persistent kernel without reuse and
    the one-tile-per-CTA kernel issue the same MMAs in the same order: identical outputs,
    including chunks of many rows (70 > one chunk of 32), CTAs with many chunks, and fewer
    tiles than SMs."""
    import torch

    from fastcone_b200 import nn

    g = torch.Generator(device="cuda").manual_seed(1)
    x = _act(shape, g, torch.bfloat16)
    wk = (torch.randn(27, 16, 16, device="cuda", generator=g) * 0.1).to(torch.bfloat16)
    b = torch.randn(16, device="cuda", generator=g)
    monkeypatch.delenv("FCB_CONV_SIMPLE", raising=False)
    y1 = nn.conv3d16(x, wk, b, relu=True, out_dtype=torch.float32)      # row reuse
    monkeypatch.setenv("FCB_CONV_SIMPLE", "1")
    y2 = nn.conv3d16(x, wk, b, relu=True, out_dtype=torch.float32)      # one tile per CTA
    monkeypatch.setenv("FCB_CONV_SIMPLE", "2")
    y3 = nn.conv3d16(x, wk, b, relu=True, out_dtype=torch.float32)      # persistent, no reuse
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)
    assert torch.equal(y3, y2)


@pytest.mark.parametrize("shape", [(20, 17, 130), (3, 5, 7), (6, 70, 128), (37, 41, 300), (1, 1, 5), (9, 33, 257)])
def test_wgrad_tensor_cores_vs_torch(shape, monkeypatch):
    """The tcgen05 weight gradient (BF16 x and dY, FP32 accumulation) against torch's FP32
    weight gradient on the same values and against the CUDA-core kernel: odd and even x
    extents (single-voxel and voxel-pair boxes), partial x tiles, chunks longer than 32
    rows, and fewer tiles than SMs."""
    import torch

    from fastcone_b200 import nn, ops

    g = torch.Generator(device="cuda").manual_seed(7)
    x = _act(shape, g, torch.bfloat16)
    gy = _act(shape, g, torch.bfloat16)
    monkeypatch.delenv("FCB_WGRAD_SIMT", raising=False)
    dw = nn.conv3d16_wgrad(x, gy)
    ops.sync_status()
    xr = nn.from_layout(x).float().unsqueeze(0)
    gr = nn.from_layout(gy).float().unsqueeze(0)
    tf32 = torch.backends.cudnn.allow_tf32
    torch.backends.cudnn.allow_tf32 = False
    try:
        ref = torch.nn.grad.conv3d_weight(xr, (16, 16, 3, 3, 3), gr, padding=1)
    finally:
        torch.backends.cudnn.allow_tf32 = tf32
    assert _rel(nn.from_kernel_weights(dw), ref) < 2e-4, _rel(nn.from_kernel_weights(dw), ref)
    monkeypatch.setenv("FCB_WGRAD_SIMT", "1")
    dw2 = nn.conv3d16_wgrad(x, gy)
    torch.cuda.synchronize()
    assert _rel(dw2, dw) < 2e-4


def test_conv_forward_and_gradients_vs_cpu_fp64():
    """Forward, input gradient and weight gradient of the tcgen05 kernels against torch on
    the CPU in FP64, on the same BF16 values (the kernels accumulate in FP32: rel-L2 <= 1e-5).
    The input gradient is the forward kernel with tap-flipped, transposed weights, as the
    autograd function runs it."""
    import torch
    import torch.nn.functional as F

    from fastcone_b200 import nn, ops

    g = torch.Generator(device="cuda").manual_seed(11)
    shape = (10, 12, 70)
    x = _act(shape, g, torch.bfloat16)
    gy = _act(shape, g, torch.bfloat16)
    w = (torch.randn(16, 16, 3, 3, 3, device="cuda", generator=g) * 0.1).to(torch.bfloat16)
    wk = nn.to_kernel_weights(w.float()).to(torch.bfloat16).contiguous()
    y = nn.conv3d16(x, wk, None, relu=False, out_dtype=torch.float32)
    gx = nn.conv3d16(gy, wk.flip(0).transpose(1, 2).contiguous(), None, relu=False, out_dtype=torch.float32)
    dw = nn.conv3d16_wgrad(x, gy)
    ops.sync_status()

    xc = nn.from_layout(x).double().cpu().unsqueeze(0)
    gc = nn.from_layout(gy).double().cpu().unsqueeze(0)
    wc = w.double().cpu()
    y_ref = F.conv3d(xc, wc, padding=1)
    gx_ref = torch.nn.grad.conv3d_input(xc.shape, wc, gc, padding=1)
    dw_ref = torch.nn.grad.conv3d_weight(xc, wc.shape, gc, padding=1)
    assert _rel(nn.from_layout(y).cpu().unsqueeze(0).double(), y_ref) < 1e-5
    assert _rel(nn.from_layout(gx).cpu().unsqueeze(0).double(), gx_ref) < 1e-5
    assert _rel(nn.from_kernel_weights(dw).cpu().double(), dw_ref) < 1e-5
