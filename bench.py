"""Benchmark of the fused LdG step (the QSR_cuda hot path) on B200.

Default workload (one GPU): the anisotropic weak-anchoring relaxation -- 256^3 grid, droplet
R = 120 cells, L1/L2/L3 = 6/3/1e-12 N, W = 1e-5 J/m^2, boundary_S = 0.6, T = 302 K, seeded random
directors S0 = 0.5, explicit Euler at the reference's stable dt. A step is one explicit time
step of the whole grid. ``value`` is box-cell-updates/s with the field resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs N independent replicas (one per GPU, no data-path collective; weak scaling).
``--impl reference`` times the reference's own CPU step chain (QSR.cpp, built from the
reference sources into oracle/_ref/) on the host cores, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LdG cell-updates/s"
UNIT = "cell-updates/s"
BYTES_PER_CELL = 40  # FP32 SoA: 5 components read + 5 written per cell-update

WORKLOADS = {
    "anisotropic_weak_256": dict(
        desc="256^3 droplet R=120 cells, L1/L2/L3=6/3/1e-12 N, W=1e-5 J/m^2 (boundary_S=0.6), T=302 K, "
             "random directors S0=0.5 seed 42, explicit Euler at dt_max",
        params=dict(Nx=256, Ny=256, Nz=256, dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6,
                    T_star=307.0, bulk_modechoice=1, kappa=0.0, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5, gamma=0.1,
                    droplet_radius_cells=120.0),
        T=302.0, S_shell=0.6, S0=0.5, seed=42),
    "plain_relaxation_64": dict(
        desc="64^3 droplet R=28 cells, L1=6e-12 N, strong anchoring (equilibrium S_shell), T=300 K, "
             "random directors S0=0.5 seed 42, explicit Euler at dt_max",
        params=dict(Nx=64, Ny=64, Nz=64, dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6,
                    T_star=307.0, bulk_modechoice=1, kappa=0.0, L1=6e-12, L2=0.0, L3=0.0, W=0.0, gamma=0.1,
                    droplet_radius_cells=28.0),
        T=300.0, S_shell=None, S0=0.5, seed=42),
}
WORKLOADS["imex_relaxation_256"] = dict(
    desc="256^3 droplet R=120 cells, L1=6e-12 N, strong anchoring (equilibrium S_shell), T=300 K, random "
         "directors S0=0.5 seed 42, semi-implicit IMEX step (the reference's sim_mode 3 default): L_stab=L1, "
         "25 Helmholtz-Jacobi sweeps, dt = 4 dt_max",
    params=dict(Nx=256, Ny=256, Nz=256, dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6,
                T_star=307.0, bulk_modechoice=1, kappa=0.0, L1=6e-12, L2=0.0, L3=0.0, W=0.0, gamma=0.1,
                droplet_radius_cells=120.0),
    T=300.0, S_shell=None, S0=0.5, seed=42, imex=dict(L_stab=6e-12, jacobi=25, dt_factor=4.0))
WORKLOADS["periodic_quench_512"] = dict(
    kind="periodic",
    desc="512^3 periodic bulk LdG, kappa=6e-12 N, gamma=0.1, linear ramp 315->295 K over 1e4 steps, "
         "Langevin noise_strength=kT/dx^3 (300 K), init N(0,1e-3) seed 12345",
    N=512, d=1e-8, kappa=6e-12, gamma=0.1, a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0, T_high=315.0,
    T_low=295.0, ramp=10000, amp=1e-3, seed=12345, log_every=100)
WORKLOADS["quench_ensemble_128"] = dict(
    kind="ensemble",
    desc="128 droplets, R ~ U{16..48} cells (seed 2024) on (2R+8)^3 grids, L1=6e-12 N, strong anchoring with "
         "equilibrium shell order, linear ramp 315->295 K over tau_Q in {1e3,3e3,1e4,3e4} steps, Langevin "
         "noise_strength=kT/dx^3 (300 K) with per-droplet Philox seeds, init N(0,1e-3); one persistent launch "
         "per step over all droplets",
    n=128, r_lo=16, r_hi=48, seed=2024, taus=(1000, 3000, 10000, 30000), T_high=315.0, T_low=295.0,
    params=dict(dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0, bulk_modechoice=1,
                kappa=0.0, L1=6e-12, L2=0.0, L3=0.0, W=0.0, gamma=0.1, q_norm_cap=0.0, boundary_custom=0,
                boundary_S=0.0, protocol=2),
    amp=1e-3, log_every=100)
DEFAULT_WORKLOAD = "anisotropic_weak_256"


def ensemble_instances(w, rank=0):
    """The droplet list of the ensemble workload (radii, grids, ramps, seeds)."""
    rng = np.random.default_rng(w["seed"])
    radii = rng.integers(w["r_lo"], w["r_hi"] + 1, size=w["n"])
    out = []
    for n, R in enumerate(radii):
        out.append(dict(N=int(2 * R + 8), droplet_radius_cells=float(R), T_high=w["T_high"], T_low=w["T_low"],
                        pre_equil_iters=0, ramp_iters=int(w["taus"][n % len(w["taus"])]),
                        seed=int(w["seed"] * 1000 + rank * w["n"] + n), noise_sigma=0.0))
    return out


def ensemble_dt_sigma(w):
    from lcdrsimulator_b200.physics import DtRequest, estimate_stable_dt_window
    p = w["params"]
    r = DtRequest(dx=p["dx"], dy=p["dy"], dz=p["dz"], gamma=p["gamma"], a=p["a"], b=p["b"], c=p["c"],
                  T_star=p["T_star"], modechoice=p["bulk_modechoice"], kappa=p["kappa"], L1=p["L1"], L2=p["L2"],
                  L3=p["L3"], S0=0.5, T_a=w["T_high"], T_b=w["T_low"])
    dt = estimate_stable_dt_window(r)["dt_max"]
    kT = 1.380649e-23 * 300.0
    sigma = math.sqrt(2.0 * (1.0 / p["gamma"]) * (kT / p["dx"] ** 3) * dt)
    return dt, sigma


def bench_ensemble(args, w, torch, pg, rank, world, local):
    """Droplet ensemble (sim_mode 3 quench statistics): one persistent launch per step."""
    import lcdrsimulator_b200 as L
    dt, sigma = ensemble_dt_sigma(w)
    if args.droplets:
        w = dict(w, n=args.droplets)
    inst = ensemble_instances(w, rank)
    for d in inst:
        d["noise_sigma"] = sigma
    ens = L.EnsembleSolver(inst, dt=dt, **w["params"])
    ens.initial_fields(init_mode=2, S0=0.5, noise_amplitude=w["amp"])
    fields = [ens.download(n) for n in range(len(inst))]
    stream = torch.cuda.ExternalStream(ens.stream())
    chunk = ens.autotune(trial_steps=10)
    ens.step(args.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    l0 = ens.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rank_barrier(pg)
    e0.record(stream)
    ens.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    rank_barrier(pg)
    clocks = sampler.stop()
    launches = ens.launch_count() - l0
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    c = ens.counts()
    t_step = ms / 1e3 / args.steps
    peak, peak_kind = load_peaks()
    alg = 20 * (c["active_cells"] + c["written_cells"])
    e2e = None
    if not args.no_e2e:
        pinned = [torch.from_numpy(f).pin_memory().numpy() for f in fields]
        outs = [torch.empty(f.size, dtype=torch.float64).pin_memory().numpy() for f in fields]
        ens2 = L.EnsembleSolver(inst, dt=dt, **w["params"])
        ens2.initial_fields(init_mode=2, S0=0.5, noise_amplitude=w["amp"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for n, f in enumerate(pinned):
            ens2.upload(n, f)
        n_obs = 0
        done = 0
        while done < args.steps:
            k = min(w["log_every"], args.steps - done)
            if done % w["log_every"] == 0:
                ens2.observe_all()
                n_obs += 1
            ens2.step(k)
            done += k
        for n, o in enumerate(outs):
            ens2.download(n, out=o)
        t_e2e = max_over_ranks(pg, time.perf_counter() - t0)
        ens2.close()
        e2e = {"value": world * c["cells"] * args.steps / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": 40 * c["cells"] / args.steps,
               "d2h_bytes_per_step": (40 * c["cells"] + n_obs * len(inst) * 136) / args.steps,
               "note": "ens_upload of every droplet + K steps + ens_observe_all every 100 steps + "
                       "ens_download of every droplet; host wall clock around the whole sequence"}
    if rank == 0:
        line = {"metric": METRIC, "value": world * c["cells"] * args.steps / (ms / 1e3), "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": args.workload, "desc": w["desc"], "droplets": len(inst),
                           "box_cells": c["cells"], "active_cells": c["active_cells"],
                           "written_cells": c["written_cells"], "dt_s": dt, "noise_sigma": sigma,
                           "chunk": chunk, "parallelism": f"replicas{world}",
                           "active_cell_updates_per_s": world * c["active_cells"] * args.steps / (ms / 1e3),
                           "l2": "inputs larger than L2 (two FP32 fields per droplet, %.2f GB)" % (
                               40 * c["cells"] / 1e9)},
                "roofline": {"bound": "hbm", "achieved": alg / t_step / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": alg / t_step / 1e9 / peak, "traffic": load_traffic(args.workload, alg),
                             "peak_source": peak_kind, "bytes_per_launch": alg, "kernel_ms": t_step * 1e3},
                "clocks": clocks, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    ens.close()
    return 0


def bench_periodic(args, w, torch, pg, rank, world, local):
    """Periodic bulk quench (the KZM_bulk_ldg path): one kzm_step kernel per step."""
    import lcdrsimulator_b200 as L
    from lcdrsimulator_b200.physics import bulk_ABC, S_eq
    N, d = (args.grid or w["N"]), w["d"]
    # rough explicit limit of the reference (KZM_bulk_ldg.cu:330-349)
    Ah = bulk_ABC(w["a"], w["b"], w["c"], w["T_high"], w["T_star"])[0]
    Al, Bl, Cl = bulk_ABC(w["a"], w["b"], w["c"], w["T_low"], w["T_star"])
    Sl = S_eq(Al, Bl, Cl)
    stiff = (1.0 / w["gamma"]) * (2.0 * w["kappa"] * 3.0 / (d * d) + max(abs(Ah), abs(Al)) + abs(Bl) * abs(Sl) +
                                  abs(Cl) * 2.0 * Sl * Sl / 3.0)
    dt = 0.2 / stiff
    kT = 1.380649e-23 * 300.0
    sigma = math.sqrt(2.0 * (1.0 / w["gamma"]) * (kT / d ** 3) * dt)
    s = L.KZMSolver(N, N, N, d, d, d, w["kappa"], w["gamma"])
    rng = np.random.default_rng(w["seed"])
    q0 = w["amp"] * rng.standard_normal(5 * N ** 3)
    s.upload(q0)
    stream = torch.cuda.ExternalStream(s.stream())

    def T_at(it):
        if it >= w["ramp"]:
            return w["T_low"]
        return w["T_high"] + (w["T_low"] - w["T_high"]) * it / w["ramp"]

    def step(it):
        A, B, C = bulk_ABC(w["a"], w["b"], w["c"], T_at(it), w["T_star"])
        s.step(1, A, B, C, dt, noise_sigma=sigma, seed=w["seed"], step_index=it)

    for it in range(args.warmup):
        step(it)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    l0 = s.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rank_barrier(pg)
    e0.record(stream)
    for it in range(args.warmup, args.warmup + args.steps):
        step(it)
    e1.record(stream)
    e1.synchronize()
    rank_barrier(pg)
    clocks = sampler.stop()
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    launches = s.launch_count() - l0
    sites = N ** 3
    t_step = ms / 1e3 / args.steps
    peak, peak_kind = load_peaks()
    alg = BYTES_PER_CELL * sites
    e2e = None
    if not args.no_e2e:
        q_in = torch.from_numpy(q0).pin_memory().numpy()
        q_out = torch.empty(q0.size, dtype=torch.float64).pin_memory().numpy()
        torch.cuda.synchronize()
        e0.record(stream)
        s.upload(q_in)
        n_obs = 0
        for it in range(args.steps):
            step(it)
            if it % w["log_every"] == 0:
                A, B, C = bulk_ABC(w["a"], w["b"], w["c"], T_at(it), w["T_star"])
                s.observe(A, B, C)
                n_obs += 1
        s.download(q_out)
        e1.record(stream)
        e1.synchronize()
        ems = max_over_ranks(pg, e0.elapsed_time(e1))
        e2e = {"value": world * sites * args.steps / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": (40 * sites + args.steps * 56) / args.steps,
               "d2h_bytes_per_step": (40 * sites + n_obs * 80) / args.steps,
               "note": "kzm_upload + K x kzm_step + kzm_observe every 100 steps + kzm_download"}
    if rank == 0:
        line = {"metric": METRIC, "value": world * sites * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": args.workload, "desc": w["desc"], "grid": [N, N, N], "dt_s": dt,
                           "noise_sigma": sigma, "parallelism": f"replicas{world}",
                           "l2": l2_note(20 * sites)},
                "roofline": {"bound": "hbm", "achieved": alg / t_step / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": alg / t_step / 1e9 / peak, "traffic": load_traffic(args.workload, alg),
                             "peak_source": peak_kind, "bytes_per_launch": alg, "kernel_ms": t_step * 1e3},
                "clocks": clocks, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    s.close()
    return 0


def dt_max(w):
    from lcdrsimulator_b200.physics import DtRequest, estimate_stable_dt_window
    p = w["params"]
    r = DtRequest(dx=p["dx"], dy=p["dy"], dz=p["dz"], gamma=p["gamma"], a=p["a"], b=p["b"], c=p["c"],
                  T_star=p["T_star"], modechoice=p["bulk_modechoice"], kappa=p["kappa"], L1=p["L1"], L2=p["L2"],
                  L3=p["L3"], S0=w["S0"], T_a=w["T"], T_b=w["T"])
    return estimate_stable_dt_window(r)["dt_max"]


def shell_order(w):
    from lcdrsimulator_b200.physics import equilibrium_shell_order
    if w["S_shell"] is not None:
        return w["S_shell"]
    p = w["params"]
    return equilibrium_shell_order(p["a"], p["b"], p["c"], w["T"], p["T_star"], p["bulk_modechoice"])


def max_over_ranks(pg, x, device="cuda"):
    """Maximum of a per-rank scalar over all ranks (identity without a process group)."""
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def rank_barrier(pg, device="cuda"):
    """All ranks meet (an all-reduce), then the device is synchronised."""
    import torch
    if pg is not None:
        t = torch.ones(1, device=device)
        pg.all_reduce(t)
    if device == "cuda":
        torch.cuda.synchronize()


L2_BYTES = 126 * 1024 * 1024


def l2_note(field_bytes):
    """How the timed steps stand against the 126 MB L2: each step reads one field (5 FP32
    components per cell, or 10 with compensated hi + lo storage) and writes the other."""
    if 2 * field_bytes > L2_BYTES:
        return "inputs larger than L2 (two fields of %.0f MB)" % (field_bytes / 1e6)
    return "inputs fit in L2 (two fields of %.1f MB): not an HBM measurement" % (field_bytes / 1e6)


def load_traffic(workload, alg_bytes):
    """DRAM bytes (read + write) per launch of the dominant kernel from the committed ncu
    summary profiles/traffic.json: measured at full size, or measured on a smaller case and
    scaled by algorithmic bytes (traffic grows in proportion)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)[workload]
    except Exception:
        return None
    if "bytes_per_launch" in t:
        return t["bytes_per_launch"]
    if "traffic_per_algorithmic_byte" in t:
        return t["traffic_per_algorithmic_byte"] * alg_bytes
    return None


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _reference_problem(w, grid=0):
    """The workload's own grid, droplet and seeded initial field for the reference's CPU path:
    parameters, the reference's initial field (initializeQTensor, QSR.cu:1841-1880, from the
    reference build) and the step scalars. grid > 0 shrinks the box (CPU tests only)."""
    from oracle.oracle import make_params, ref_initial_field
    p = dict(w["params"])
    if grid:
        scale = grid / p["Nx"]
        p.update(Nx=grid, Ny=grid, Nz=grid, droplet_radius_cells=p.get("droplet_radius_cells", 0.0) * scale)
    op = make_params(**p)
    q = ref_initial_field(op, 0, w["seed"], w["S0"])
    return op, q, dt_max(w), shell_order(w)


def cpu_reference_sample(w, target_s=12.0, max_steps=400):
    """The reference's own CPU step chain (QSR.cpp) on a bounded number of steps of the workload."""
    from oracle.oracle import RefCPU
    ref = RefCPU()
    op, q, dt, S_shell = _reference_problem(w)
    t1 = ref.run_steps(op, q, w["T"], S_shell, dt, 1)  # warm-up and per-step estimate
    n = int(max(2, min(max_steps, target_s / max(t1, 1e-6))))
    t = ref.run_steps(op, q, w["T"], S_shell, dt, n)
    cells = op.Nx * op.Ny * op.Nz
    return {"value": cells * n / t, "unit": UNIT, "cores": ref.max_threads(), "kind": "reference",
            "sample": f"QSR.cpp step chain (computeLaplacian, computeChemicalPotential, applyWeakAnchoringPenalty, "
                      f"updateQTensor, applyBoundaryConditions) on the workload's {op.Nx}x{op.Ny}x{op.Nz} grid, "
                      f"droplet R = {op.droplet_radius_cells:g} cells and seeded initial field, "
                      f"{n} steps, {t:.2f} s"}, t / n


def run_reference_arm(args, w):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle.oracle import RefCPU
    ref = RefCPU()
    op, q, dt, S_shell = _reference_problem(w, args.ref_grid)
    cells = op.Nx * op.Ny * op.Nz
    if args.warmup > 0:
        ref.run_steps(op, q, w["T"], S_shell, dt, args.warmup)
    t = ref.run_steps(op, q, w["T"], S_shell, dt, args.steps)
    value = cells * args.steps / t
    same = not args.ref_grid
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": args.workload, "desc": w["desc"], "grid": [op.Nx, op.Ny, op.Nz],
                       "droplet_radius_cells": op.droplet_radius_cells,
                       "note": "the reference CPU path (QSR.cpp step chain, all host threads) on "
                               + ("the workload's own grid, droplet and seeded initial field" if same else
                                  "a reduced grid of the workload's physics")},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.max_threads(), "kind": "reference",
                             "sample": f"{op.Nx}^3 grid, droplet R = {op.droplet_radius_cells:g} cells, "
                                       f"{args.steps} timed steps"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--ref-grid", type=int, default=0,
                    help="reference arm: box edge of a reduced grid (0 = the workload's own grid)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--compensated", action="store_true",
                    help="confined workloads: compensated (hi + lo) field storage")
    ap.add_argument("--droplets", type=int, default=0,
                    help="ensemble workload: first N droplets of the distribution (small profiling cases)")
    ap.add_argument("--grid", type=int, default=0,
                    help="box edge of a smaller case of the workload (profiling; droplet radius scaled with it)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, w)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    import lcdrsimulator_b200 as L

    if w.get("kind") == "periodic":
        return bench_periodic(args, w, torch, pg, rank, world, local)
    if w.get("kind") == "ensemble":
        return bench_ensemble(args, w, torch, pg, rank, world, local)

    if args.grid:
        # a smaller box of the same physics (profiling cases): droplet radius scaled with the box
        scale = args.grid / w["params"]["Nx"]
        w = dict(w, params=dict(w["params"], Nx=args.grid, Ny=args.grid, Nz=args.grid,
                                droplet_radius_cells=w["params"]["droplet_radius_cells"] * scale))
    solver = L.QSRSolver(**dict(w["params"], compensated=1 if args.compensated else 0))
    geo = solver.geometry()
    q0 = solver.initial_field(0, w["seed"], w["S0"])
    dt = dt_max(w)
    S_shell = shell_order(w)
    T = w["T"]
    solver.upload(q0)
    stream = torch.cuda.ExternalStream(solver.stream())

    def barrier():
        rank_barrier(pg)

    imex = w.get("imex")
    if imex:
        dt = dt * imex["dt_factor"]
        args_step = solver.step_args(T, S_shell, dt, semi_implicit=True, L_stab=imex["L_stab"],
                                     jacobi_iters=imex["jacobi"])
    else:
        args_step = solver.step_args(T, S_shell, dt)
    # work-item length of the tiled kernel chosen by the library's autotuner (field restored)
    chunk = solver.autotune(T, S_shell, dt, trial_steps=10,
                            **({"semi_implicit": True, "L_stab": imex["L_stab"], "jacobi_iters": imex["jacobi"]}
                               if imex else {}))
    geo = solver.geometry()  # visited cells of the work list at the chosen item length
    for s in range(args.warmup):
        args_step.step_index = s
        solver.step_raw(1, args_step)
    solver.sync()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    l0 = solver.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for s in range(args.steps):
        args_step.step_index = args.warmup + s
        solver.step_raw(1, args_step)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    barrier()
    clocks = sampler.stop()
    launches = solver.launch_count() - l0
    ms = max_over_ranks(pg, ms)
    box = geo["box_cells"]
    t_step = ms / 1e3 / args.steps
    value = world * box * args.steps / (ms / 1e3)
    touched = geo["active_cells"]
    written = geo["written_cells"] if os.environ.get("LDG_QSR_KERNEL", "") != "direct" else box
    if os.environ.get("LDG_QSR_KERNEL", "") == "direct":
        touched = box
    peak, peak_kind = load_peaks()
    # algorithmic bytes per launch: each visited cell's 5 FP32 components read once, each
    # changing cell's 5 components written once
    alg_bytes = (BYTES_PER_CELL // 2) * (touched + written)
    if args.compensated and not imex:
        alg_bytes += 40 * written  # low words of the changing cells read and written
    if imex:
        # IMEX step: the RHS kernel (visited cells read, moving cells' RHS written) plus one pass
        # per Jacobi sweep over the changing cells: each reads and writes the field (moving and
        # strongly anchored cells) and reads the RHS of the moving cells
        alg_bytes += imex["jacobi"] * (40 * written + 20 * geo["evolving_cells"])
    achieved = alg_bytes / t_step / 1e9
    # the committed DRAM traffic of each storage mode was captured at the workload's own size
    traffic = None if args.grid else load_traffic(args.workload + ("+compensated" if args.compensated else ""),
                                                  alg_bytes)

    e2e = None
    if not args.no_e2e:
        # Drop-in run through the C ABI with host buffers: upload the field from pinned host
        # memory, K steps with per-step host arguments, observables every 200 steps (the
        # reference's print_freq default), download into pinned host memory.
        q_in = torch.from_numpy(q0).pin_memory().numpy()
        q_out = torch.empty(q0.size, dtype=torch.float64).pin_memory().numpy()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.upload(q_in)
        n_obs = 0
        for s in range(args.steps):
            args_step.step_index = s
            solver.step_raw(1, args_step)
            if s % 200 == 0:
                solver.observe(T, S_shell)
                n_obs += 1
        solver.download(q_out)
        e1.record(stream)
        e1.synchronize()
        ems = max_over_ranks(pg, e0.elapsed_time(e1))
        barrier()
        field_bytes = 5 * 8 * box
        e2e = {"value": world * box * args.steps / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": (field_bytes + args.steps * 72) / args.steps,
               "d2h_bytes_per_step": (field_bytes + n_obs * 136) / args.steps,
               "note": "qsr_upload (AoS FP64, pinned) + K x qsr_step + qsr_observe every 200 steps + qsr_download"}

    comp = None
    if not args.compensated and not imex and not args.grid:
        # The same workload with compensated storage, timed the same way: the storage mode that
        # keeps the free energy within 1e-7 of FP64 over the longest runs (plain FP32 storage is
        # the headline; both are reported).
        s2 = L.QSRSolver(**dict(w["params"], compensated=1))
        s2.upload(q0)
        s2.autotune(T, S_shell, dt, trial_steps=10)
        g2 = s2.geometry()
        a2 = s2.step_args(T, S_shell, dt)
        st2 = torch.cuda.ExternalStream(s2.stream())
        for s in range(args.warmup):
            a2.step_index = s
            s2.step_raw(1, a2)
        s2.sync()
        barrier()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(st2)
        for s in range(args.steps):
            a2.step_index = args.warmup + s
            s2.step_raw(1, a2)
        c1.record(st2)
        c1.synchronize()
        cms = max_over_ranks(pg, c0.elapsed_time(c1))
        barrier()
        s2.close()
        ct = cms / 1e3 / args.steps
        cbytes = (BYTES_PER_CELL // 2) * (g2["active_cells"] + g2["written_cells"]) + 40 * g2["written_cells"]
        comp = {"storage": "compensated hi+lo FP32", "ms_per_step": cms / args.steps,
                "value": world * box * args.steps / (cms / 1e3), "roofline_frac": cbytes / ct / 1e9 / peak,
                "bytes_per_launch": cbytes, "traffic": load_traffic(args.workload + "+compensated", cbytes)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _ = cpu_reference_sample(w)
        except Exception as e:  # the reference build is test infrastructure; report its absence
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "desc": w["desc"], "grid": [w["params"]["Nx"], w["params"]["Ny"],
                                                                            w["params"]["Nz"]],
                       "box_cells": box, "active_cells": touched, "evolving_cells": geo["evolving_cells"],
                       "active_cell_updates_per_s": world * touched * args.steps / (ms / 1e3),
                       "dt_s": dt, "S_shell": S_shell, "parallelism": f"replicas{world}",
                       "storage": "compensated hi+lo FP32" if args.compensated else "FP32", "chunk": chunk,
                       "l2": l2_note((40 if args.compensated else 20) * box)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "bytes_per_launch": alg_bytes, "read_cells": touched, "written_cells": written,
                         "kernel_ms": t_step * 1e3},
            "clocks": clocks,
            "e2e": e2e,
            "gpu_launches": launches,
            "cpu_baseline": cpu,
        }
        if comp is not None:
            line["compensated"] = comp
        print(json.dumps(line), flush=True)
    solver.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
