"""U-Net preconditioner of the FWI update, on this library's BF16 convolutions.

The network maps ``[gradient, source illumination, current vp]`` (each
standardised) to a vp update.  Every 3x3 convolution runs on the tensor cores
through ``sweep_b200_conv3x3_gemm`` / ``sweep_b200_conv3x3_wgrad``: BF16
activations and weights, FP32 accumulation; master weights, biases and the
optimiser state stay FP32.  Pooling, upsampling, concatenation and GELU are
plain tensor operations around them.  The reference has no learned
component; the convolutions are checked against PyTorch's float32 ``conv2d``.

Layout inside the network: NHWC, channel counts multiples of 8 (the 3 input
channels are zero-padded to 8; the output layer has 8 channels of which the
first is the update).
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F

from . import _lib

__all__ = ["conv3x3", "check", "UNet"]


def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


class _Conv3x3(torch.autograd.Function):
    """y = conv3x3(x, w) + b with x (N, H, W, C) bf16, w (Co, 3, 3, C) and b (Co,)
    float32 (cast to bf16 for the tensor cores), y float32 (N, H, W, Co)."""

    @staticmethod
    def forward(ctx, x, w, b):
        if not x.is_cuda:
            raise RuntimeError("sweep_b200 convolutions run on a CUDA device only")
        x = x.contiguous()
        n, h, wd, c = x.shape
        co = w.shape[0]
        wb = w.to(torch.bfloat16).contiguous()
        out = torch.empty((n, h, wd, co), dtype=torch.float32, device=x.device)
        _lib.call("sweep_b200_conv3x3_gemm", x.data_ptr(), wb.data_ptr(), b.contiguous().data_ptr(),
                  out.data_ptr(), n, h, wd, c, co, 1, _stream(x))
        ctx.save_for_backward(x, wb)
        return out

    @staticmethod
    def backward(ctx, gout):
        x, wb = ctx.saved_tensors
        n, h, wd, c = x.shape
        co = wb.shape[0]
        g = gout.to(torch.bfloat16).contiguous()
        gx = gw = gb = None
        if ctx.needs_input_grad[0]:
            wt = wb.permute(3, 1, 2, 0).contiguous()            # (C, 3, 3, Co): per-tap transpose
            gx32 = torch.empty((n, h, wd, c), dtype=torch.float32, device=x.device)
            _lib.call("sweep_b200_conv3x3_gemm", g.data_ptr(), wt.data_ptr(), None, gx32.data_ptr(),
                      n, h, wd, co, c, -1, _stream(x))
            gx = gx32.to(torch.bfloat16)
        if ctx.needs_input_grad[1]:
            gw = torch.empty((co, 3, 3, c), dtype=torch.float32, device=x.device)
            _lib.call("sweep_b200_conv3x3_wgrad", x.data_ptr(), g.data_ptr(), gw.data_ptr(), n, h, wd, c, co,
                      _stream(x))
        if ctx.needs_input_grad[2]:
            gb = gout.sum(dim=(0, 1, 2))
        return gx, gw, gb


def conv3x3(x, w, b):
    """BF16 3x3 convolution (stride 1, zero padding 1), FP32 accumulation."""
    return _Conv3x3.apply(x, w, b)


def check(device=None):
    """Wait for the current stream and raise if a convolution launched since
    the last check timed out on the device (its outputs are then invalid)."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    _lib.call("sweep_b200_conv3x3_status", torch.cuda.current_stream(dev).cuda_stream)


class _Conv(torch.nn.Module):
    def __init__(self, cin, cout, gen):
        super().__init__()
        bound = math.sqrt(6.0 / (9 * cin))                      # He-uniform for GELU
        self.w = torch.nn.Parameter((torch.rand((cout, 3, 3, cin), generator=gen) * 2 - 1) * bound)
        self.b = torch.nn.Parameter(torch.zeros(cout))

    def forward(self, x):
        return conv3x3(x, self.w, self.b)


def _block(x, convs):
    for cv in convs:
        x = F.gelu(cv(x)).to(torch.bfloat16)
    return x


def _pool(x):
    n, h, w, c = x.shape
    return x.float().view(n, h // 2, 2, w // 2, 2, c).mean(dim=(2, 4)).to(torch.bfloat16)


def _up(x):
    return x.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)


class UNet(torch.nn.Module):
    """4 levels, ``base`` channels at the top (32 by default), two 3x3
    convolutions with GELU per level, average-pool down, nearest up, skip
    concatenation.  Input (B, 3, H, W), output (B, 1, H, W); H and W multiples
    of 8."""

    def __init__(self, base=32, levels=4, seed=0):
        super().__init__()
        gen = torch.Generator().manual_seed(seed)
        ch = [base * 2 ** i for i in range(levels)]
        self.levels = levels
        self.enc = torch.nn.ModuleList()
        cin = 8
        for c in ch:
            self.enc.append(torch.nn.ModuleList([_Conv(cin, c, gen), _Conv(c, c, gen)]))
            cin = c
        self.dec = torch.nn.ModuleList()
        for i in range(levels - 2, -1, -1):
            self.dec.append(torch.nn.ModuleList([_Conv(ch[i + 1] + ch[i], ch[i], gen), _Conv(ch[i], ch[i], gen)]))
        self.out = _Conv(ch[0], 8, gen)
        with torch.no_grad():
            self.out.w.mul_(0.1)

    def forward(self, x):
        check(x.device)                  # the previous step's convolutions (forward and backward)
        b, c, h, w = x.shape
        if h % 2 ** (self.levels - 1) or w % 2 ** (self.levels - 1):
            raise ValueError(f"input size {h}x{w} must be a multiple of {2 ** (self.levels - 1)}")
        z = torch.zeros((b, h, w, 8), dtype=torch.bfloat16, device=x.device)
        z[..., :c] = x.permute(0, 2, 3, 1).to(torch.bfloat16)
        skips = []
        for i, blk in enumerate(self.enc):
            z = _block(z, blk)
            if i < self.levels - 1:
                skips.append(z)
                z = _pool(z)
        for blk in self.dec:
            z = torch.cat([_up(z), skips.pop()], dim=-1)
            z = _block(z, blk)
        y = self.out(z)
        return y[..., :1].permute(0, 3, 1, 2).contiguous()
