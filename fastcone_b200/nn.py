"""3x3x3 convolutions on the tcgen05 kernels, as torch autograd functions.

Activations are BF16 volumes of 16 channels in the kernels' channel-half-major layout
``[nz, ny, 2, nx, 8]`` (channel c at ``[:, :, c // 8, :, c % 8]``; ``to_layout`` /
``from_layout`` convert from / to ``[16, nz, ny, nx]``); a layer with fewer channels is
zero-padded to 16 (the kernels' fixed width).  Forward and input gradient run the
tensor-core kernel (``fcb_conv3d16_device``), the weight gradient the tensor-core reduction
over voxels (``fcb_conv3d16_wgrad_device`` with BF16 dY); master weights stay FP32 and are
rounded to BF16 per call.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import check, lib


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def to_kernel_weights(w: torch.Tensor) -> torch.Tensor:
    """torch layout [out, in, 3, 3, 3] -> kernel layout [27 (dz,dy,dx)][out][in]."""
    return w.permute(2, 3, 4, 0, 1).reshape(27, w.shape[0], w.shape[1])


def from_kernel_weights(wk: torch.Tensor) -> torch.Tensor:
    return wk.reshape(3, 3, 3, wk.shape[1], wk.shape[2]).permute(3, 4, 0, 1, 2)


def to_layout(t: torch.Tensor) -> torch.Tensor:
    """[16, nz, ny, nx] -> the kernels' [nz, ny, 2, nx, 8]."""
    c, nz, ny, nx = t.shape
    return t.reshape(2, 8, nz, ny, nx).permute(2, 3, 0, 4, 1).contiguous()


def from_layout(t: torch.Tensor) -> torch.Tensor:
    """[nz, ny, 2, nx, 8] -> [16, nz, ny, nx]."""
    nz, ny, _, nx, _ = t.shape
    return t.permute(2, 4, 0, 1, 3).reshape(16, nz, ny, nx)


def _check_act(x: torch.Tensor, name: str):
    if x.dim() != 5 or x.shape[2] != 2 or x.shape[4] != 8 or not x.is_contiguous():
        raise ValueError(f"{name} must be contiguous [nz, ny, 2, nx, 8]")


def conv3d16(x: torch.Tensor, wk: torch.Tensor, bias: torch.Tensor | None = None, relu: bool = False,
             out_dtype=torch.bfloat16) -> torch.Tensor:
    """y = act(conv3d(x, w) + b); x BF16 [nz, ny, 2, nx, 8], wk BF16 [27, 16, 16]."""
    _check_act(x, "x")
    if x.dtype != torch.bfloat16:
        raise ValueError("x must be BF16")
    wk = wk.to(torch.bfloat16).contiguous()
    nz, ny, _, nx, _ = x.shape
    y = torch.empty(x.shape, device=x.device, dtype=out_dtype)
    b = bias.float().contiguous() if bias is not None else None
    check(lib().fcb_conv3d16_device(_p(x), _p(wk), _p(b) if b is not None else None, _p(y),
                                    _lib.FCB_F32 if out_dtype == torch.float32 else _lib.FCB_BF16,
                                    nx, ny, nz, 1 if relu else 0, _stream()))
    return y


def conv3d16_wgrad(x: torch.Tensor, gy: torch.Tensor) -> torch.Tensor:
    """dW[t][co][ci] = sum_v gy[v][co] x[v + tap t][ci] (FP32); both [nz, ny, 2, nx, 8]."""
    _check_act(x, "x")
    nz, ny, _, nx, _ = x.shape
    dw = torch.zeros((27, 16, 16), device=x.device, dtype=torch.float32)
    gy = gy.contiguous()
    check(lib().fcb_conv3d16_wgrad_device(_p(x), _p(gy), _lib.FCB_F32 if gy.dtype == torch.float32 else _lib.FCB_BF16,
                                          _p(dw), nx, ny, nz, _stream()))
    return dw


class Conv3d16Function(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, w, b, relu):
        wk = to_kernel_weights(w).to(torch.bfloat16).contiguous()
        y = conv3d16(x, wk, b, relu=relu)
        ctx.relu = relu
        ctx.save_for_backward(x, wk, y)
        return y

    @staticmethod
    def backward(ctx, gy):
        x, wk, y = ctx.saved_tensors
        g = gy.float()
        if ctx.relu:
            g = g * (y > 0)
        gb = g.to(torch.bfloat16).contiguous()
        # input gradient: the same convolution with tap-flipped, transposed weights
        wt = wk.flip(0).transpose(1, 2).contiguous()
        gx = conv3d16(gb, wt, None, relu=False, out_dtype=torch.float32).to(torch.bfloat16)
        dwk = conv3d16_wgrad(x, gb)
        dw = from_kernel_weights(dwk)
        db = g.sum(dim=(0, 1, 3)).reshape(16)
        return gx, dw, db, None


class Conv3d(torch.nn.Module):
    """3x3x3 convolution with cin, cout <= 16 channels (padded to 16 in the kernels)."""

    def __init__(self, cin: int, cout: int, relu: bool):
        super().__init__()
        self.cin, self.cout, self.relu = cin, cout, relu
        w = torch.empty(cout, cin, 3, 3, 3)
        torch.nn.init.kaiming_uniform_(w, a=5 ** 0.5)
        self.weight = torch.nn.Parameter(w)
        self.bias = torch.nn.Parameter(torch.zeros(cout))

    def padded(self):
        w = torch.zeros(16, 16, 3, 3, 3, device=self.weight.device, dtype=self.weight.dtype)
        w[: self.cout, : self.cin] = self.weight
        b = torch.zeros(16, device=self.bias.device, dtype=self.bias.dtype)
        b[: self.cout] = self.bias
        return w, b

    def forward(self, x):
        w, b = self.padded()
        return Conv3d16Function.apply(x, w, b, self.relu)
