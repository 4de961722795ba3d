"""Throughput of the surrogate's tcgen05 convolution kernels and of one U-Net training step.

    python -m lcdrsimulator_b200.surrogate.bench_conv [--iters 20] [--cases N,S,Ci,Co ...] [--unet]

Prints one JSON line per case: forward (bias + leaky ReLU, BF16 out) and weight-gradient
time (CUDA events on the current stream, after 3 warm-up calls) and TFLOP/s counted as
2 * N * S^3 * 27 * Ci * Co per call; with --cudnn also torch's conv3d (cuDNN, channels-last
BF16) on the same shape for context; with --unet the time of one U-Net training step
(forward, backward, Adam) and of one forward.
"""
from __future__ import annotations

import argparse
import json

import torch

from . import UNet3D
from . import conv as C

DEFAULT_CASES = ["4,64,32,32", "4,64,64,32", "4,32,64,64", "4,32,128,64", "4,16,128,128", "4,16,256,128",
                 "8,8,256,256", "4,64,16,32"]


def timeit(fn, iters):
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(iters):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / iters


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--cases", nargs="*", default=DEFAULT_CASES)
    ap.add_argument("--cudnn", action="store_true")
    ap.add_argument("--unet", action="store_true")
    args = ap.parse_args(argv)
    torch.manual_seed(0)
    for case in args.cases:
        N, S, Ci, Co = (int(v) for v in case.split(","))
        x = (torch.randn(N, S, S, S, Ci, device="cuda") * 0.5).to(torch.bfloat16)
        w = (torch.randn(Co, 27, Ci, device="cuda") * 0.05).to(torch.bfloat16)
        b = torch.zeros(Co, device="cuda")
        dy = torch.randn(N, S, S, S, Co, device="cuda").to(torch.bfloat16)
        flops = 2.0 * N * S ** 3 * 27 * Ci * Co
        tf = timeit(lambda: C.conv3d_fwd(x, w, b, 1), args.iters)
        tw = timeit(lambda: C.conv3d_wgrad(x, dy), args.iters)
        C.check()
        line = dict(N=N, S=S, Ci=Ci, Co=Co, fwd_ms=tf, fwd_tflops=flops / tf / 1e9, wgrad_ms=tw,
                    wgrad_tflops=flops / tw / 1e9)
        if args.cudnn:
            xc = x.permute(0, 4, 1, 2, 3).contiguous().to(memory_format=torch.channels_last_3d)
            wc = w.reshape(Co, 3, 3, 3, Ci).permute(0, 4, 1, 2, 3).contiguous().to(
                memory_format=torch.channels_last_3d)
            tc = timeit(lambda: torch.nn.functional.conv3d(xc, wc, padding=1), args.iters)
            line.update(cudnn_fwd_ms=tc, cudnn_fwd_tflops=flops / tc / 1e9)
        print(json.dumps(line), flush=True)
    if args.unet:
        for N, S in [(8, 32), (4, 64)]:
            net = UNet3D(seed=0).cuda()
            opt = torch.optim.Adam(net.parameters(), lr=1e-4)
            x = (torch.randn(N, S, S, S, 16, device="cuda") * 0.5).to(torch.bfloat16)
            y = torch.randn(N, S, S, S, 5, device="cuda")

            def step():
                opt.zero_grad()
                loss = ((net(x)[..., :5] - y) ** 2).mean()
                loss.backward()
                opt.step()
            t_step = timeit(step, 10)
            with torch.no_grad():
                t_fwd = timeit(lambda: net(x), 10)
            print(json.dumps(dict(unet=True, N=N, S=S, train_step_ms=t_step, forward_ms=t_fwd)), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
