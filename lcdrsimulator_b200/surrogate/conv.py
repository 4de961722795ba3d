"""ctypes bindings of the sg_conv3d_* kernels for CUDA torch tensors, and the autograd Function.

Layouts: activations (N, D, H, W, C) BF16 contiguous; weights (Co, 27, Ci) with tap
t = 9*(dz+1) + 3*(dy+1) + (dx+1) -- torch's conv3d weight (Co, Ci, kd, kh, kw) is
``w.permute(0, 2, 3, 4, 1).reshape(Co, 27, Ci)``.
"""
from __future__ import annotations

import ctypes as C

import torch

from .. import load_library, _check

CHANNELS_IN = (16, 32, 64, 128, 256)


class SgShape(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("N", "D", "H", "W", "Ci", "Co")]


_bound = False


def _lib():
    global _bound
    L = load_library()
    if not _bound:
        vp = C.c_void_p
        L.sg_conv3d_fwd.argtypes = [C.POINTER(SgShape), vp, vp, vp, vp, C.c_int, C.c_int, vp]
        L.sg_conv3d_wgrad.argtypes = [C.POINTER(SgShape), vp, vp, vp, vp]
        L.sg_conv3d_flip_weights.argtypes = [C.POINTER(SgShape), vp, vp, vp]
        L.sg_check.argtypes = [vp]
        L.sg_launch_count.restype = C.c_longlong
        _bound = True
    return L


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _require(t: torch.Tensor, dtype, shape, name):
    if not t.is_cuda or t.dtype != dtype or tuple(t.shape) != tuple(shape) or not t.is_contiguous():
        raise ValueError(f"{name}: expected contiguous CUDA {dtype} of shape {tuple(shape)}, got "
                         f"{t.dtype} {tuple(t.shape)} on {t.device}")
    if t.data_ptr() % 16:
        raise ValueError(f"{name}: data pointer must be 16-byte aligned")


def conv3d_fwd(x: torch.Tensor, w: torch.Tensor, bias: torch.Tensor | None = None, act: int = 0,
               out_fp32: bool = False) -> torch.Tensor:
    """y = act(conv3d(x, w) + bias) through the tcgen05 kernel."""
    N, D, H, W, Ci = x.shape
    Co = w.shape[0]
    _require(x, torch.bfloat16, (N, D, H, W, Ci), "x")
    _require(w, torch.bfloat16, (Co, 27, Ci), "w")
    if bias is not None:
        _require(bias, torch.float32, (Co,), "bias")
    y = torch.empty((N, D, H, W, Co), dtype=torch.float32 if out_fp32 else torch.bfloat16, device=x.device)
    s = SgShape(N, D, H, W, Ci, Co)
    _check(_lib().sg_conv3d_fwd(C.byref(s), x.data_ptr(), w.data_ptr(),
                                bias.data_ptr() if bias is not None else None, y.data_ptr(), int(act),
                                int(out_fp32), _stream()), "sg_conv3d_fwd")
    return y


def conv3d_wgrad(x: torch.Tensor, dy: torch.Tensor) -> torch.Tensor:
    """dw[Co, 27, Ci] (FP32) of y = conv3d(x, w)."""
    N, D, H, W, Ci = x.shape
    Co = dy.shape[-1]
    _require(x, torch.bfloat16, (N, D, H, W, Ci), "x")
    _require(dy, torch.bfloat16, (N, D, H, W, Co), "dy")
    dw = torch.empty((Co, 27, Ci), dtype=torch.float32, device=x.device)
    s = SgShape(N, D, H, W, Ci, Co)
    _check(_lib().sg_conv3d_wgrad(C.byref(s), x.data_ptr(), dy.data_ptr(), dw.data_ptr(), _stream()),
           "sg_conv3d_wgrad")
    return dw


def flip_weights(w: torch.Tensor) -> torch.Tensor:
    """wf[Ci, 26 - t, Co] = w[Co, t, Ci] (weights of the data-gradient convolution)."""
    Co, _, Ci = w.shape
    _require(w, torch.bfloat16, (Co, 27, Ci), "w")
    wf = torch.empty((Ci, 27, Co), dtype=torch.bfloat16, device=w.device)
    s = SgShape(1, 1, 1, 1, Ci, Co)
    _check(_lib().sg_conv3d_flip_weights(C.byref(s), w.data_ptr(), wf.data_ptr(), _stream()),
           "sg_conv3d_flip_weights")
    return wf


def check(stream=None):
    _check(_lib().sg_check(C.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)),
           "sg_check")


def launch_count() -> int:
    return _lib().sg_launch_count()


class Conv3dFunction(torch.autograd.Function):
    """3x3x3 convolution, stride 1, zero padding 1, with bias and optional leaky ReLU (slope 0.01).

    Forward, data gradient (forward of the flipped weights) and weight gradient all run on the
    tcgen05 kernels; only the activation mask and the bias gradient (a channel sum) use torch.
    """

    @staticmethod
    def forward(ctx, x, w, bias, act, out_fp32):
        wb = w.to(torch.bfloat16).contiguous()
        y = conv3d_fwd(x, wb, bias, act, out_fp32)
        ctx.save_for_backward(x, wb, y)
        ctx.act = act
        ctx.x_grad = x.requires_grad
        return y

    @staticmethod
    def backward(ctx, gy):
        x, wb, y = ctx.saved_tensors
        g = gy
        if ctx.act == 1:
            g = g * torch.where(y > 0, 1.0, 0.01).to(g.dtype)
        g = g.to(torch.bfloat16).contiguous()
        dx = None
        if ctx.x_grad:
            dx = conv3d_fwd(g, flip_weights(wb))
        dw = conv3d_wgrad(x, g)
        db = g.float().sum(dim=(0, 1, 2, 3))
        return dx, dw, db, None, None


def conv3d(x, w, bias, act=1, out_fp32=False):
    return Conv3dFunction.apply(x, w, bias, act, out_fp32)
