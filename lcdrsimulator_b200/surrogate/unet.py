"""3-D U-Net warm-start network (4 levels, 32 base channels, 3x3x3 convolutions).

Encoder level l: two convolutions to 32 * 2^l channels (leaky ReLU), then 2x2x2 average
pooling. Decoder level l: nearest 2x upsampling, a convolution to 32 * 2^l channels,
concatenation with the encoder skip (2 * 32 * 2^l channels), two convolutions. Head: one
convolution to 16 channels (the first 5 are the predicted Q components Qxx, Qxy, Qxz, Qyy,
Qyz) with FP32 output. Activations are NDHWC BF16; weights are FP32 master copies cast to BF16
per call; every convolution runs on the tcgen05 kernels.
"""
from __future__ import annotations

import math

import torch
from torch import nn

from .conv import conv3d

IN_CHANNELS = 16
OUT_CHANNELS = 16


def avg_pool2(h: torch.Tensor) -> torch.Tensor:
    N, D, H, W, C = h.shape
    return h.view(N, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(dim=(2, 4, 6)).contiguous()


def upsample2(h: torch.Tensor) -> torch.Tensor:
    N, D, H, W, C = h.shape
    return h[:, :, None, :, None, :, None, :].expand(N, D, 2, H, 2, W, 2, C).reshape(N, 2 * D, 2 * H, 2 * W,
                                                                                        C).contiguous()


class ConvLayer(nn.Module):
    def __init__(self, ci: int, co: int, act: int = 1, out_fp32: bool = False, gen: torch.Generator | None = None):
        super().__init__()
        std = math.sqrt(2.0 / (27 * ci))
        self.weight = nn.Parameter(torch.randn(co, 27, ci, generator=gen) * std)
        self.bias = nn.Parameter(torch.zeros(co))
        self.act = act
        self.out_fp32 = out_fp32

    def forward(self, x):
        return conv3d(x, self.weight, self.bias, self.act, self.out_fp32)


class UNet3D(nn.Module):
    def __init__(self, base: int = 32, levels: int = 4, seed: int = 0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        ch = [base * 2 ** l for l in range(levels)]
        self.levels = levels
        self.enc = nn.ModuleList()
        cin = IN_CHANNELS
        for c in ch:
            self.enc.append(nn.ModuleList([ConvLayer(cin, c, gen=g), ConvLayer(c, c, gen=g)]))
            cin = c
        self.up = nn.ModuleList([ConvLayer(ch[l + 1], ch[l], gen=g) for l in range(levels - 1)])
        self.dec = nn.ModuleList([nn.ModuleList([ConvLayer(2 * ch[l], ch[l], gen=g), ConvLayer(ch[l], ch[l], gen=g)])
                                  for l in range(levels - 1)])
        self.head = ConvLayer(ch[0], OUT_CHANNELS, act=0, out_fp32=True, gen=g)

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: (N, D, H, W, 16) BF16 with D, H, W divisible by 2^(levels-1). Returns FP32 (N, D, H, W, 16)."""
        skips = []
        h = x
        for l in range(self.levels):
            h = self.enc[l][1](self.enc[l][0](h))
            if l < self.levels - 1:
                skips.append(h)
                h = avg_pool2(h)
        for l in reversed(range(self.levels - 1)):
            h = self.up[l](upsample2(h))
            h = torch.cat([skips[l], h], dim=-1).contiguous()
            h = self.dec[l][1](self.dec[l][0](h))
        return self.head(h)
