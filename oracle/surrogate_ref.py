"""CPU reference of the surrogate network and its convolutions (test infrastructure).

The surrogate has no counterpart in the reference project; its CUDA kernels are checked
against torch's CPU conv3d in FP32/FP64 on BF16-representable inputs. Weight layout of the
library: (Co, 27, Ci) with tap t = 9*(dz+1) + 3*(dy+1) + (dx+1); activations NDHWC.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F


def to_torch_weight(w: torch.Tensor) -> torch.Tensor:
    """(Co, 27, Ci) -> torch's (Co, Ci, 3, 3, 3)."""
    Co, _, Ci = w.shape
    return w.reshape(Co, 3, 3, 3, Ci).permute(0, 4, 1, 2, 3).contiguous()


def conv3d_ref(x: torch.Tensor, w: torch.Tensor, bias=None, act=0, dtype=torch.float64) -> torch.Tensor:
    """NDHWC conv on the CPU in `dtype`; x (N, D, H, W, Ci), w (Co, 27, Ci)."""
    xc = x.to("cpu", dtype).permute(0, 4, 1, 2, 3)
    y = F.conv3d(xc, to_torch_weight(w.to("cpu", dtype)), None if bias is None else bias.to("cpu", dtype), padding=1)
    if act == 1:
        y = F.leaky_relu(y, 0.01)
    return y.permute(0, 2, 3, 4, 1).contiguous()


def avg_pool2(h):
    N, D, H, W, C = h.shape
    return h.view(N, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(dim=(2, 4, 6))


def upsample2(h):
    N, D, H, W, C = h.shape
    return h[:, :, None, :, None, :, None, :].expand(N, D, 2, H, 2, W, 2, C).reshape(N, 2 * D, 2 * H, 2 * W, C)


def _bf16(t):
    """Rounds values to BF16; the cast's backward rounds the incoming gradient to BF16 too."""
    return t.to(torch.bfloat16).to(t.dtype)


def unet_ref(net, x: torch.Tensor, dtype=torch.float64, mimic_bf16=False) -> torch.Tensor:
    """The U-Net forward of `net` (a lcdrsimulator_b200.surrogate.UNet3D) on the CPU in `dtype`,
    with the weights rounded to BF16 as the GPU path uses them. Differentiable. With
    mimic_bf16 the activations (and, through the casts, their gradients) are rounded to BF16
    at the points where the GPU path stores them in BF16."""
    rb = _bf16 if mimic_bf16 else (lambda t: t)

    def conv(layer, h):
        w = layer.weight.detach().to(torch.bfloat16).to("cpu", dtype).requires_grad_(True)
        b = layer.bias.detach().to("cpu", dtype).requires_grad_(True)
        conv.params.append((layer, w, b))
        y = F.conv3d(h.permute(0, 4, 1, 2, 3), to_torch_weight(w), b, padding=1).permute(0, 2, 3, 4, 1)
        if layer.act == 1:
            return rb(F.leaky_relu(y, 0.01))
        return y.to(torch.float32).to(dtype) if mimic_bf16 else y
    conv.params = []
    skips = []
    h = x.to("cpu", dtype)
    for l in range(net.levels):
        h = conv(net.enc[l][1], conv(net.enc[l][0], h))
        if l < net.levels - 1:
            skips.append(h)
            h = rb(avg_pool2(h))
    for l in reversed(range(net.levels - 1)):
        h = conv(net.up[l], upsample2(h))
        h = torch.cat([skips[l], h], dim=-1)
        h = conv(net.dec[l][1], conv(net.dec[l][0], h))
    out = conv(net.head, h)
    return out, conv.params
