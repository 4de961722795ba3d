"""Warm-start surrogate: a 3-D U-Net whose convolutions are the library's BF16 tcgen05
implicit-GEMM kernels (forward, data gradient and weight gradient), trained on equilibria
produced by the ensemble solver. PyTorch is used only for the training loop (optimizer,
pooling, concatenation, loss); the solver path never imports this package.
"""
from .conv import conv3d, conv3d_fwd, conv3d_wgrad, flip_weights, Conv3dFunction
from .unet import UNet3D

__all__ = ["conv3d", "conv3d_fwd", "conv3d_wgrad", "flip_weights", "Conv3dFunction", "UNet3D"]
