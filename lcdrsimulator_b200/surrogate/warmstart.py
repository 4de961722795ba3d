"""Warm-start experiment: solver-generated training data, U-Net training, and the
time-to-equilibrium comparison of plain relaxation against relaxation from the network's
prediction.

Scales. A case is one droplet: radius R (physical), temperature T, Rapini-Papoular W and L2/L1
(L1 = 6e-12 N, L3 = 0), relaxed at constant T with the equilibrium shell order S_eq(T) and
explicit Euler steps. The network works on a coarse grid (n_coarse^3, spacing 2*dx); the
evaluation grid is n_fine = 2*n_coarse with spacing dx. The initial field of a case is a seeded
low-pass Gaussian random Q on the fine grid (zero outside the droplet, like the reference's
initialisation); its 2x2x2 average is the coarse field the network sees and from which the
training targets are relaxed.

Convergence criterion (the reference's early-stop form): the relative free-energy change per
step, measured over `check_every` steps as |E(t) - E(t - K)| / |E(t)| / K, below `tol`.
"""
from __future__ import annotations

import dataclasses
import math
import time

import numpy as np
import torch
import torch.nn.functional as F

from .. import EnsembleSolver
from ..physics import DtRequest, estimate_stable_dt_window

L1 = 6e-12
MATERIAL = dict(a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0, bulk_modechoice=1, gamma=0.1, kappa=0.0, L1=L1,
                L2=0.0, L3=0.0, W=0.0, q_norm_cap=0.0, boundary_custom=0, boundary_S=0.0, protocol=1)


@dataclasses.dataclass
class Case:
    R_m: float        # droplet radius (m)
    T: float          # K
    W: float          # J/m^2
    l2_ratio: float   # L2 / L1
    seed: int


def sample_cases(n: int, seed: int, R_range=(100e-9, 140e-9), T_range=(295.0, 306.0), W_range=(1e-6, 1e-4),
                 l2_range=(0.0, 2.0)) -> list[Case]:
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(Case(R_m=float(rng.uniform(*R_range)), T=float(rng.uniform(*T_range)),
                        W=float(10 ** rng.uniform(math.log10(W_range[0]), math.log10(W_range[1]))),
                        l2_ratio=float(rng.uniform(*l2_range)), seed=int(seed * 100003 + i)))
    return out


def lowpass_field(n: int, seed: int, sigma_cells: float = 4.0, amplitude: float = 0.25) -> np.ndarray:
    """Seeded low-pass Gaussian random traceless Q on an n^3 grid: (n, n, n, 5) FP64 with RMS
    Frobenius norm `amplitude` (5 stored components Qxx, Qxy, Qxz, Qyy, Qyz)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((5, n, n, n))
    k = np.fft.fftfreq(n)
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    filt = np.exp(-2.0 * (math.pi * sigma_cells) ** 2 * kk)
    q = np.real(np.fft.ifftn(np.fft.fftn(g, axes=(1, 2, 3)) * filt, axes=(1, 2, 3)))
    q = np.moveaxis(q, 0, -1)
    xx, xy, xz, yy, yz = (q[..., i] for i in range(5))
    fro2 = xx ** 2 + yy ** 2 + (xx + yy) ** 2 + 2 * (xy ** 2 + xz ** 2 + yz ** 2)
    return q * (amplitude / math.sqrt(fro2.mean()))


def pool2(q: np.ndarray) -> np.ndarray:
    n = q.shape[0] // 2
    return q.reshape(n, 2, n, 2, n, 2, -1).mean(axis=(1, 3, 5))


def droplet_mask(geo: dict, n: int, dx: float) -> np.ndarray:
    i = np.arange(n) * dx
    X = (i[:, None, None] - geo["center_x"]) / geo["radius_x"]
    Y = (i[None, :, None] - geo["center_y"]) / geo["radius_y"]
    Z = (i[None, None, :] - geo["center_z"]) / geo["radius_z"]
    return (X ** 2 + Y ** 2 + Z ** 2) <= 1.0


def stable_dt(dx: float, cases: list[Case]) -> float:
    dts = []
    for c in cases:
        r = DtRequest(dx=dx, dy=dx, dz=dx, gamma=MATERIAL["gamma"], a=MATERIAL["a"], b=MATERIAL["b"],
                      c=MATERIAL["c"], T_star=MATERIAL["T_star"], modechoice=1, kappa=0.0, L1=L1,
                      L2=c.l2_ratio * L1, L3=0.0, S0=0.5, T_a=c.T, T_b=c.T)
        dts.append(estimate_stable_dt_window(r)["dt_max"])
    return min(dts)


def instances(cases: list[Case], n: int, dx: float) -> list[dict]:
    return [dict(N=n, droplet_radius_cells=c.R_m / dx, T_high=c.T, T_low=c.T, pre_equil_iters=0, ramp_iters=0,
                 seed=c.seed, noise_sigma=0.0, own_material=1, W=c.W, L2=c.l2_ratio * L1, L3=0.0) for c in cases]


def geometries(cases: list[Case], n: int, dx: float) -> list[dict]:
    """The library's droplet geometry of every case (no stepping)."""
    ens = EnsembleSolver(instances(cases, n, dx), dx=dx, dy=dx, dz=dx, dt=1e-12, **MATERIAL)
    out = [ens.geometry(i) for i in range(len(cases))]
    ens.close()
    return out


def relax(cases: list[Case], n: int, dx: float, fields: list[np.ndarray], max_steps: int, check_every: int,
          tol: float, dt: float | None = None, snapshot_tols=()) -> dict:
    """Relaxes every case from its field (n^3 x 5, FP64) in one ensemble; returns the final
    fields, the first checked step at which each case met the criterion (None if never), the
    energy histories and the device time of the stepping. For every tolerance in
    `snapshot_tols` the field of each case is also kept at the first check where its rate fell
    below that tolerance (`snapshots[t][i]`, step in `snapshot_step[t][i]`; a case that never
    got there keeps its final field and the last step)."""
    dt = stable_dt(dx, cases) if dt is None else dt
    ens = EnsembleSolver(instances(cases, n, dx), dx=dx, dy=dx, dz=dx, dt=dt, **MATERIAL)
    for i, f in enumerate(fields):
        ens.upload(i, np.ascontiguousarray(f, dtype=np.float64).ravel())
    chunk = ens.autotune()   # small droplets want short work items; the fields are restored
    stream = torch.cuda.ExternalStream(ens.stream())
    energy = [[o["total"]] for o in ens.observe_all()]
    conv_step = [None] * len(cases)
    snaps = {t: [None] * len(cases) for t in snapshot_tols}
    snap_step = {t: [None] * len(cases) for t in snapshot_tols}
    steps = 0
    dev_ms = 0.0
    while steps < max_steps:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(check_every)
        e1.record(stream)
        e1.synchronize()
        dev_ms += e0.elapsed_time(e1)
        steps += check_every
        obs_now = ens.observe_all()
        for i in range(len(cases)):
            E = obs_now[i]["total"]
            rate = abs(E - energy[i][-1]) / max(abs(E), 1e-300) / check_every
            if conv_step[i] is None and rate < tol:
                conv_step[i] = steps
            for t in snapshot_tols:
                if snaps[t][i] is None and rate < t:
                    snaps[t][i] = ens.download(i).reshape(n, n, n, 5)
                    snap_step[t][i] = steps
            energy[i].append(E)
        if all(s is not None for s in conv_step):
            break
    out = [ens.download(i).reshape(n, n, n, 5) for i in range(len(cases))]
    obs = ens.observe_all()
    ens.close()
    for t in snapshot_tols:
        for i in range(len(cases)):
            if snaps[t][i] is None:
                snaps[t][i], snap_step[t][i] = out[i], steps
    return dict(fields=out, conv_step=conv_step, energy=energy, steps=steps, dt=dt, device_ms=dev_ms, obs=obs,
                snapshots=snaps, snapshot_step=snap_step, chunk=chunk)


# ---------------------------------------------------------------------------------------
# Network input / output
# ---------------------------------------------------------------------------------------
Q_SCALE = 2.5   # network Q channels are Q * Q_SCALE (|Q| ~ 0.4 -> ~1)


def network_input(q_coarse: np.ndarray, mask: np.ndarray, c: Case) -> np.ndarray:
    """16-channel input: mask, 5 scaled Q components, T, R, log10 W, L2/L1 (normalised), zeros."""
    n = q_coarse.shape[0]
    x = np.zeros((n, n, n, 16), np.float32)
    x[..., 0] = mask
    x[..., 1:6] = q_coarse * Q_SCALE * mask[..., None]
    x[..., 6] = (c.T - 300.5) / 5.5
    x[..., 7] = (c.R_m - 120e-9) / 20e-9
    x[..., 8] = math.log10(c.W) + 5.0
    x[..., 9] = c.l2_ratio - 1.0
    return x


# Cube symmetries: the droplet is a sphere centred in a cubic box and every term of the free
# energy is rotation invariant, so a relaxed pair (input, target) maps to another valid pair under
# any of the 48 axis permutations with sign flips R, with Q transformed as Q' = R Q R^T.
def _q5_to_mat(q):
    xx, xy, xz, yy, yz = (q[..., i] for i in range(5))
    zz = -(xx + yy)
    return torch.stack([torch.stack([xx, xy, xz], -1), torch.stack([xy, yy, yz], -1),
                        torch.stack([xz, yz, zz], -1)], -2)


def _mat_to_q5(m):
    return torch.stack([m[..., 0, 0], m[..., 0, 1], m[..., 0, 2], m[..., 1, 1], m[..., 1, 2]], -1)


def cube_symmetry(x: torch.Tensor, perm, flips, q_slices):
    """Applies the symmetry (axis permutation `perm`, then sign flips `flips` of the new axes) to
    a (N, X, Y, Z, C) tensor whose channel slices in `q_slices` hold Q components (5 each)."""
    y = x.permute(0, 1 + perm[0], 1 + perm[1], 1 + perm[2], 4)
    dims = [1 + a for a in range(3) if flips[a] < 0]
    if dims:
        y = y.flip(dims)
    R = torch.zeros(3, 3, dtype=torch.float32, device=x.device)
    for a in range(3):
        R[a, perm[a]] = float(flips[a])
    y = y.clone()
    for sl in q_slices:
        m = _q5_to_mat(y[..., sl].float())
        m = torch.einsum("ai,...ij,bj->...ab", R, m, R)
        y[..., sl] = _mat_to_q5(m).to(y.dtype)
    return y.contiguous()


def masked_loss(net, inputs: np.ndarray, targets: np.ndarray, masks: np.ndarray, batch: int = 8) -> float:
    """The training loss (masked MSE on the 5 scaled Q components) over a data set, no gradients."""
    tot, cnt = 0.0, 0.0
    with torch.no_grad():
        for s in range(0, len(inputs), batch):
            X = torch.from_numpy(inputs[s:s + batch]).to("cuda", torch.bfloat16)
            Y = torch.from_numpy(targets[s:s + batch] * Q_SCALE).to("cuda", torch.float32)
            M = torch.from_numpy(masks[s:s + batch].astype(np.float32)).to("cuda")[..., None]
            tot += float((((net(X)[..., :5] - Y) ** 2) * M).sum())
            cnt += float(M.sum()) * 5
    return tot / max(cnt, 1.0)


def train(net, inputs: np.ndarray, targets: np.ndarray, masks: np.ndarray, epochs: int = 40, batch: int = 8,
          lr: float = 1e-3, seed: int = 0, log=None, augment: bool = False, warmup_epochs: float = 0.0) -> list[float]:
    """Masked MSE on the 5 scaled Q components; Adam with gradient clipping, a linear learning-rate
    warm-up over `warmup_epochs` and cosine decay after it; each batch transformed by a random
    cube symmetry when `augment` (at 512 training droplets and 80 epochs this under-fits: 2.0x
    instead of 2.55x time-to-equilibrium speed-up)."""
    dev = torch.device("cuda")
    X = torch.from_numpy(inputs).to(dev, torch.bfloat16)
    Y = torch.from_numpy(targets * Q_SCALE).to(dev, torch.float32)
    M = torch.from_numpy(masks.astype(np.float32)).to(dev)[..., None]
    n = X.shape[0]
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    total = epochs * ((n + batch - 1) // batch)
    warm = int(round(warmup_epochs * ((n + batch - 1) // batch)))

    def lr_factor(step):
        if step < warm:
            return (step + 1) / warm
        return 0.5 * (1.0 + math.cos(math.pi * (step - warm) / max(total - warm, 1)))

    sched = torch.optim.lr_scheduler.LambdaLR(opt, lr_factor)
    g = torch.Generator().manual_seed(seed)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g)
        acc = 0.0
        for s in range(0, n, batch):
            idx = perm[s:s + batch].to(dev)
            xb, yb, m = X[idx], Y[idx], M[idx]
            if augment:
                ax = torch.randperm(3, generator=g).tolist()
                fl = [1 if v else -1 for v in (torch.rand(3, generator=g) < 0.5).tolist()]
                xb = cube_symmetry(xb, ax, fl, [slice(1, 6)])
                yb = cube_symmetry(yb, ax, fl, [slice(0, 5)])
                m = cube_symmetry(m, ax, fl, [])
            opt.zero_grad()
            out = net(xb)[..., :5]
            loss = (((out - yb) ** 2) * m).sum() / (m.sum() * 5)
            loss.backward()
            torch.nn.utils.clip_grad_norm_(net.parameters(), 1.0)
            opt.step()
            sched.step()
            acc += float(loss.detach()) * len(idx)
        hist.append(acc / n)
        if log:
            log(f"epoch {ep} loss {hist[-1]:.5f}")
    return hist


@torch.no_grad()
def predict(net, inputs: np.ndarray) -> np.ndarray:
    X = torch.from_numpy(inputs).to("cuda", torch.bfloat16)
    out = net(X)[..., :5].float() / Q_SCALE
    return out.cpu().numpy().astype(np.float64)


def upsample2(q: np.ndarray) -> np.ndarray:
    """Trilinear 2x upsampling of an (n, n, n, 5) field; fine cell f sits at coarse coordinate
    f/2 - 1/4, which is torch's align_corners=False convention."""
    t = torch.from_numpy(np.moveaxis(q, -1, 0)[None]).double()
    u = F.interpolate(t, scale_factor=2, mode="trilinear", align_corners=False)
    return np.moveaxis(u[0].numpy(), 0, -1)


# ---------------------------------------------------------------------------------------
# The experiment
# ---------------------------------------------------------------------------------------
def make_dataset(cases: list[Case], n_coarse: int, dx_fine: float, max_steps: int, check_every: int, tol: float,
                 batch: int = 128, log=None) -> dict:
    dxc = 2.0 * dx_fine
    X, Y, Mk, conv = [], [], [], []
    t0 = time.time()
    for s in range(0, len(cases), batch):
        part = cases[s:s + batch]
        masks = [droplet_mask(g, n_coarse, dxc) for g in geometries(part, n_coarse, dxc)]
        q0 = [pool2(lowpass_field(2 * n_coarse, c.seed)) * m[..., None] for c, m in zip(part, masks)]
        r = relax(part, n_coarse, dxc, q0, max_steps, check_every, tol)
        for c, q, m, f, cs in zip(part, q0, masks, r["fields"], r["conv_step"]):
            X.append(network_input(q, m, c))
            Y.append(f)
            Mk.append(m)
            conv.append(cs)
        if log:
            log(f"dataset {s + len(part)}/{len(cases)}: {r['steps']} steps, {r['device_ms'] / 1e3:.1f} s device, "
                f"converged {sum(x is not None for x in r['conv_step'])}/{len(part)}, wall {time.time() - t0:.0f} s")
    return dict(X=np.stack(X), Y=np.stack(Y), M=np.stack(Mk), conv=conv)


def _geomean(xs):
    xs = [x for x in xs if x]
    return float(np.exp(np.mean(np.log(xs)))) if xs else None


def evaluate(net, cases: list[Case], n_coarse: int, dx_fine: float, max_steps: int, check_every: int, tol: float,
             log=None, coarse_tols=(), coarse_max_steps: int = 600000) -> dict:
    """Plain relaxation from the fine low-pass field against relaxation from the upsampled
    prediction, all cases and all arms in one ensemble with one dt.

    With `coarse_tols`, two more arms per tolerance t run a coarse stage first (both on the
    n_coarse grid, same dt): "unet+coarse@t" relaxes the network's prediction and "coarse@t"
    (the control without the network) relaxes the 2x2x2 average of the fine initial field, each
    until its rate per step falls below t; the upsampled coarse field then starts a fine
    relaxation to `tol`. Cost of an arm = coarse steps x device time per coarse droplet-step +
    fine steps x device time per fine droplet-step (both measured here, in ensembles of the same
    kind); its speed-up is the plain arm's cost over that."""
    nf = 2 * n_coarse
    dxc = 2.0 * dx_fine
    gcs = geometries(cases, n_coarse, dxc)
    gfs = geometries(cases, nf, dx_fine)
    fine0, inputs, warm, mfs, mcs = [], [], [], [], []
    for c, gc, gf in zip(cases, gcs, gfs):
        mf = droplet_mask(gf, nf, dx_fine)
        mc = droplet_mask(gc, n_coarse, dxc)
        q = lowpass_field(nf, c.seed) * mf[..., None]
        fine0.append(q)
        mfs.append(mf)
        mcs.append(mc)
        inputs.append(network_input(pool2(q) * mc[..., None], mc, c))
    t0 = time.perf_counter()
    pred = predict(net, np.stack(inputs))
    torch.cuda.synchronize()
    t_pred = time.perf_counter() - t0
    for p, mf in zip(pred, mfs):
        warm.append(upsample2(p) * mf[..., None])
    dt = stable_dt(dx_fine, cases)
    k = len(cases)
    arms = {"plain": fine0, "unet": warm}
    coarse = {}
    if coarse_tols:
        starts = [p * mc[..., None] for p, mc in zip(pred, mcs)] + \
                 [pool2(q) * mc[..., None] for q, mc in zip(fine0, mcs)]
        rc = relax(cases + cases, n_coarse, dxc, starts, coarse_max_steps, check_every, min(coarse_tols), dt=dt,
                   snapshot_tols=tuple(coarse_tols))
        coarse["us_per_droplet_step"] = rc["device_ms"] * 1e3 / max(rc["steps"], 1) / (2 * k)
        coarse["steps"] = rc["steps"]
        coarse["chunk"] = rc["chunk"]
        for t in coarse_tols:
            for a, name in enumerate((f"unet+coarse@{t:g}", f"coarse@{t:g}")):
                arms[name] = [upsample2(rc["snapshots"][t][a * k + i]) * mfs[i][..., None] for i in range(k)]
                coarse[name] = [rc["snapshot_step"][t][a * k + i] for i in range(k)]
    names = list(arms)
    r = relax(cases * len(names), nf, dx_fine, [f for nm in names for f in arms[nm]], max_steps, check_every, tol,
              dt=dt)
    t_f = r["device_ms"] * 1e3 / max(r["steps"], 1) / (len(names) * k)
    t_c = coarse.get("us_per_droplet_step", 0.0)
    res = []
    for i, c in enumerate(cases):
        row = dict(case=dataclasses.asdict(c), arms={})
        for a, nm in enumerate(names):
            j = a * k + i
            fs = r["conv_step"][j]
            cs = coarse[nm][i] if nm in coarse else 0
            row["arms"][nm] = dict(coarse_steps=cs, fine_steps=fs, E=r["obs"][j]["total"], E0=r["energy"][j][0],
                                   defects=r["obs"][j]["defect_count"],
                                   cost_us=(cs * t_c + fs * t_f) if fs is not None else None)
        base = row["arms"]["plain"]["cost_us"]
        for nm in names:
            cu = row["arms"][nm]["cost_us"]
            row["arms"][nm]["speedup"] = base / cu if (base and cu) else None
        # fields kept for the plain/warm summary
        row.update(plain_steps=row["arms"]["plain"]["fine_steps"], warm_steps=row["arms"]["unet"]["fine_steps"],
                   plain_E=row["arms"]["plain"]["E"], warm_E=row["arms"]["unet"]["E"],
                   plain_defects=row["arms"]["plain"]["defects"], warm_defects=row["arms"]["unet"]["defects"],
                   plain_E0=row["arms"]["plain"]["E0"], warm_E0=row["arms"]["unet"]["E0"])
        res.append(row)
        if log:
            log(f"case {i}: " + ", ".join(f"{nm} {row['arms'][nm]['coarse_steps']}+{row['arms'][nm]['fine_steps']} "
                                          f"x{row['arms'][nm]['speedup'] or 0:.2f}" for nm in names))
    summary = {nm: _geomean([row["arms"][nm]["speedup"] for row in res]) for nm in names}
    return dict(results=res, dt=dt, steps=r["steps"], device_ms=r["device_ms"], predict_s=t_pred, chunk=r["chunk"],
                step_us_per_instance=t_f, coarse=coarse, arms=names, speedup_geomean_by_arm=summary,
                energy_plain=[r["energy"][i] for i in range(k)], energy_warm=[r["energy"][k + i] for i in range(k)])
