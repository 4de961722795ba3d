"""GPU parity of the surrogate's tcgen05 BF16 implicit-GEMM convolutions against torch's CPU
conv3d in FP64 on BF16-representable inputs, and of the U-Net's gradients against the CPU
reference network.

Tolerances (relative to the largest magnitude of the reference):
  * FP32-output forward, data and weight gradient: 1e-4 (FP32 accumulation of exact BF16
    products; only the summation order and the tensor core's internal accumulation differ)
  * BF16-output forward: 1e-2 (one BF16 rounding of the output)
  * whole U-Net without activations, against a reference that rounds activations and their
    gradients to BF16 at the same points: output 1e-2, per-layer gradient cosine >= 0.9999 and
    relative L2 <= 1.5e-2
  * whole U-Net with leaky ReLU against the plain FP64 reference: cosine >= 0.98, relative
    L2 <= 0.25 (activation masks flip where the two forwards straddle zero)
"""
import numpy as np
import pytest
import torch

from oracle.surrogate_ref import conv3d_ref, unet_ref

pytestmark = pytest.mark.gpu

FWD_SHAPES = [
    (2, 8, 8, 16, 16, 32),     # Ci 16: 32-byte swizzle, one MMA per K step
    (1, 8, 16, 16, 32, 64),    # Ci 32: 64-byte swizzle
    (1, 16, 16, 16, 64, 32),   # Ci 64: 128-byte swizzle
    (2, 4, 4, 4, 128, 256),    # 64-voxel volumes: one box spans two samples; N = 256
    (1, 4, 4, 4, 256, 128),    # box rows beyond the batch are skipped
    (1, 6, 10, 12, 64, 48),    # dims that are not powers of two: partial boxes
    (3, 2, 2, 2, 32, 16),      # 8-voxel volumes, Co 16
]

WGRAD_SHAPES = [
    (2, 8, 8, 16, 16, 32),
    (1, 8, 16, 16, 32, 64),
    (1, 8, 8, 16, 64, 128),
    (2, 4, 4, 4, 128, 256),
    (1, 8, 8, 8, 256, 64),     # Ci 256: two row tiles per tap
    (1, 6, 10, 12, 64, 16),    # partial K boxes, Co 16
    (2, 8, 8, 8, 32, 32),
]


def bf16_randn(*shape, scale=1.0, gen=None):
    return (torch.randn(*shape, generator=gen) * scale).to(torch.bfloat16)


def rel(a, b):
    a = a.double().cpu()
    b = b.double().cpu()
    return float((a - b).abs().max() / max(b.abs().max(), 1e-300))


@pytest.fixture(scope="module")
def conv():
    from lcdrsimulator_b200.surrogate import conv as C
    return C


@pytest.mark.parametrize("shape", FWD_SHAPES)
def test_conv_forward_matches_cpu(conv, shape):
    N, D, H, W, Ci, Co = shape
    g = torch.Generator().manual_seed(hash(shape) % 1000)
    x = bf16_randn(N, D, H, W, Ci, gen=g)
    w = bf16_randn(Co, 27, Ci, scale=0.1, gen=g)
    b = torch.randn(Co, generator=g)
    want = conv3d_ref(x, w, b, act=0)
    got = conv.conv3d_fwd(x.cuda(), w.cuda(), b.cuda(), act=0, out_fp32=True)
    conv.check()
    assert rel(got, want) <= 1e-4, rel(got, want)
    got16 = conv.conv3d_fwd(x.cuda(), w.cuda(), b.cuda(), act=1)
    want16 = conv3d_ref(x, w, b, act=1)
    assert got16.dtype == torch.bfloat16
    assert rel(got16, want16) <= 1e-2


@pytest.mark.parametrize("shape", WGRAD_SHAPES)
def test_conv_gradients_match_cpu(conv, shape):
    N, D, H, W, Ci, Co = shape
    g = torch.Generator().manual_seed(7 + hash(shape) % 1000)
    x = bf16_randn(N, D, H, W, Ci, gen=g)
    w = bf16_randn(Co, 27, Ci, scale=0.1, gen=g)
    dy = bf16_randn(N, D, H, W, Co, gen=g)
    xr = x.double().requires_grad_(True)
    wr = w.double().requires_grad_(True)
    y = conv3d_ref(xr, wr, None, act=0)
    y.backward(dy.double())
    dw = conv.conv3d_wgrad(x.cuda(), dy.cuda())
    conv.check()
    assert rel(dw, wr.grad) <= 1e-4, ("wgrad", rel(dw, wr.grad))
    if Co in (16, 32, 64, 128, 256):
        wf = conv.flip_weights(w.cuda())
        dx = conv.conv3d_fwd(dy.cuda(), wf, None, act=0, out_fp32=True)
        conv.check()
        assert rel(dx, xr.grad) <= 1e-4, ("dgrad", rel(dx, xr.grad))


def test_flip_weights_layout(conv):
    Co, Ci = 32, 16
    w = bf16_randn(Co, 27, Ci)
    wf = conv.flip_weights(w.cuda()).cpu()
    for co, t, ci in [(0, 0, 0), (5, 13, 7), (31, 26, 15), (17, 3, 9)]:
        assert wf[ci, 26 - t, co] == w[co, t, ci]


def test_conv_rejects_bad_shapes(conv):
    x = torch.zeros(1, 4, 4, 4, 24, dtype=torch.bfloat16, device="cuda")
    w = torch.zeros(16, 27, 24, dtype=torch.bfloat16, device="cuda")
    from lcdrsimulator_b200 import LdgError
    with pytest.raises(LdgError):
        conv.conv3d_fwd(x, w)                       # Ci = 24 is not supported
    with pytest.raises(ValueError):
        conv.conv3d_fwd(x.float(), w)               # wrong dtype
    x = torch.zeros(1, 4, 4, 4, 16, dtype=torch.bfloat16, device="cuda")
    w = torch.zeros(20, 27, 16, dtype=torch.bfloat16, device="cuda")
    with pytest.raises(LdgError):
        conv.conv3d_fwd(x, w)                       # Co = 20 is not a multiple of 16


def _cos_l2(a, b):
    a = a.double().cpu().flatten()
    b = b.double().cpu().flatten()
    return float(torch.nn.functional.cosine_similarity(a, b, dim=0)), float((a - b).norm() / b.norm())


def _unet_grads(act: bool, mimic: bool):
    from lcdrsimulator_b200.surrogate import UNet3D
    torch.manual_seed(0)
    net = UNet3D(seed=3).cuda()
    if not act:
        for m in net.modules():
            if hasattr(m, "act"):
                m.act = 0
    x = bf16_randn(2, 16, 16, 16, 16, scale=0.5)
    r = torch.randn(2, 16, 16, 16, 5)
    out = net(x.cuda())
    (out[..., :5] * r.cuda()).sum().backward()
    ref_out, params = unet_ref(net, x, mimic_bf16=mimic)
    (ref_out[..., :5] * r.double()).sum().backward()
    return out.detach(), ref_out.detach(), params


def test_unet_linear_gradients_match_cpu_reference():
    # Without activations there are no masks that a slightly different forward value can flip,
    # so the whole-network gradients must agree with the BF16-rounding reference closely.
    out, ref, params = _unet_grads(act=False, mimic=True)
    assert rel(out, ref) <= 1e-2
    for layer, w, b in params:
        cos, l2 = _cos_l2(layer.weight.grad, w.grad)
        assert cos >= 0.9999 and l2 <= 1.5e-2, (tuple(w.shape), cos, l2)
        cos, l2 = _cos_l2(layer.bias.grad, b.grad)
        assert cos >= 0.9999 and l2 <= 1.5e-2, (tuple(b.shape), cos, l2)


def test_unet_gradients_match_cpu_reference():
    # With leaky ReLU, pre-activations within the forward's BF16 error of zero take the other
    # slope in one of the two computations; that changes gradients by O(sqrt(fraction flipped)).
    out, ref, params = _unet_grads(act=True, mimic=False)
    assert rel(out, ref) <= 2e-2
    for layer, w, b in params:
        cos, l2 = _cos_l2(layer.weight.grad, w.grad)
        assert cos >= 0.98 and l2 <= 0.25, (tuple(w.shape), cos, l2)


def test_unet_training_reduces_loss():
    from lcdrsimulator_b200.surrogate import UNet3D
    torch.manual_seed(1)
    net = UNet3D(seed=5).cuda()
    x = bf16_randn(2, 16, 16, 16, 16, scale=0.5).cuda()
    target = torch.randn(2, 16, 16, 16, 5, device="cuda") * 0.3
    opt = torch.optim.Adam(net.parameters(), lr=1e-3)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        loss = ((net(x)[..., :5] - target) ** 2).mean()
        loss.backward()
        torch.nn.utils.clip_grad_norm_(net.parameters(), 1.0)
        opt.step()
        losses.append(float(loss.detach()))
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.7 * losses[0], losses
