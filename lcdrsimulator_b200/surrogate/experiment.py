"""Runs the warm-start experiment end to end and prints one JSON summary.

    python -m lcdrsimulator_b200.surrogate.experiment [--n-coarse 32] [--train 256] [--eval 4]
        [--coarse-tols 1e-7,1e-8] [--save unet.pt | --load unet.pt]

1. training data: `--train` cases relaxed on the coarse grid by the ensemble solver;
2. training: the U-Net on (low-pass random field, parameters) -> relaxed field;
3. evaluation: `--eval` unseen cases on the fine grid, plain relaxation from the fine random
   field against relaxation from the upsampled prediction, to the same convergence criterion;
   with --coarse-tols, also the prediction relaxed on the coarse grid first, and the same coarse
   stage without the network (control).
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np
import torch

from . import UNet3D
from . import warmstart as ws
from .conv import launch_count


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-coarse", type=int, default=32)
    ap.add_argument("--dx", type=float, default=5e-9, help="fine-grid spacing (m); coarse = 2 dx")
    ap.add_argument("--r-min", type=float, default=100e-9)
    ap.add_argument("--r-max", type=float, default=140e-9)
    ap.add_argument("--train", type=int, default=256)
    ap.add_argument("--eval", type=int, default=4)
    ap.add_argument("--train-steps", type=int, default=400000)
    ap.add_argument("--train-check", type=int, default=5000)
    ap.add_argument("--eval-steps", type=int, default=2000000)
    ap.add_argument("--eval-check", type=int, default=5000)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--warmup-epochs", type=float, default=0.0, help="linear learning-rate warm-up before the decay")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--augment", action="store_true", help="random cube-symmetry transform of every batch")
    ap.add_argument("--coarse-tols", default="",
                    help="comma-separated rate tolerances of the coarse-stage arms (unet+coarse, coarse control)")
    ap.add_argument("--save", default=None, help="path for the trained weights (torch.save)")
    ap.add_argument("--load", default=None, help="trained weights to evaluate (skips data generation and training)")
    ap.add_argument("--out", default=None, help="path for the JSON summary")
    args = ap.parse_args(argv)
    R = (args.r_min, args.r_max)
    if 2 * args.n_coarse * args.dx < 2.2 * R[1]:
        raise SystemExit("droplet does not fit the fine grid: need 2 * n_coarse * dx >= 2.2 * r_max")

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    net = UNet3D(seed=args.seed).cuda()
    if args.load:
        net.load_state_dict(torch.load(args.load, map_location="cuda"))
        data = dict(conv=[])
        hist, t_data, t_train, conv_launches = [None], 0.0, 0.0, 0
    else:
        t0 = time.time()
        train_cases = ws.sample_cases(args.train, args.seed, R_range=R)
        data = ws.make_dataset(train_cases, args.n_coarse, args.dx, args.train_steps, args.train_check, args.tol,
                               log=log)
        t_data = time.time() - t0
        l0 = launch_count()
        t1 = time.time()
        hist = ws.train(net, data["X"], data["Y"], data["M"], epochs=args.epochs, batch=args.batch, lr=args.lr,
                        seed=args.seed, log=log, augment=args.augment, warmup_epochs=args.warmup_epochs)
        torch.cuda.synchronize()
        t_train = time.time() - t1
        conv_launches = launch_count() - l0
    if args.save:
        torch.save(net.state_dict(), args.save)
    eval_cases = ws.sample_cases(args.eval, args.seed + 7919, R_range=R)
    coarse_tols = [float(t) for t in args.coarse_tols.split(",") if t]
    t2 = time.time()
    ev = ws.evaluate(net, eval_cases, args.n_coarse, args.dx, args.eval_steps, args.eval_check, args.tol, log=log,
                     coarse_tols=coarse_tols, coarse_max_steps=args.train_steps)
    t_eval = time.time() - t2
    speedups = []
    for r in ev["results"]:
        if r["plain_steps"] and r["warm_steps"]:
            speedups.append(r["plain_steps"] / r["warm_steps"])
    summary = dict(
        grid=dict(coarse=args.n_coarse, fine=2 * args.n_coarse, dx_fine=args.dx, R_range_m=R),
        train=dict(cases=args.train, steps_cap=args.train_steps, converged=sum(c is not None for c in data["conv"]),
                   loaded=args.load,
                   epochs=args.epochs, loss_first=hist[0], loss_last=hist[-1], data_s=t_data, train_s=t_train,
                   conv_kernel_launches=conv_launches),
        eval=dict(cases=args.eval, tol_per_step=args.tol, check_every=args.eval_check, steps_cap=args.eval_steps,
                  dt=ev["dt"], predict_s=ev["predict_s"], eval_s=t_eval,
                  step_us_per_instance=ev["step_us_per_instance"], results=ev["results"],
                  speedup_steps=speedups,
                  speedup_geomean=float(np.exp(np.mean(np.log(speedups)))) if speedups else None,
                  arms=ev["arms"], speedup_geomean_by_arm=ev["speedup_geomean_by_arm"],
                  coarse_us_per_droplet_step=ev["coarse"].get("us_per_droplet_step"),
                  chunk_fine=ev["chunk"], chunk_coarse=ev["coarse"].get("chunk"),
                  coarse_steps_by_arm={k: v for k, v in ev["coarse"].items() if isinstance(v, list)},
                  energy_plain=ev["energy_plain"], energy_warm=ev["energy_warm"]))
    line = json.dumps(summary)
    print(line, flush=True)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
