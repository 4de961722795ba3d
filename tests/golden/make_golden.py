"""Generate golden fixtures from the reference's own FP64 CUDA code (needs a GPU).

Runs the reference kernels of QSR.cu and KZM_bulk_ldg.cu, compiled from the reference
sources into oracle/_ref/ by oracle/Makefile, on seeded small inputs, and stores the
resulting fields and observables as .npz files next to this script. The initial fields are
produced by the oracle's restatement of the reference initialisation and stored by hash.

    python tests/golden/make_golden.py [outdir]
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Oracle, RefCUDA, RefKZM, make_params, OrcBulkParams  # noqa: E402

QSR_CASES = {
    "l1_strong": dict(grid=(16, 16, 16), p=dict(L1=6e-12), T=300.0, S=None, steps=10, imex=False),
    "kappa_strong": dict(grid=(16, 16, 16), p=dict(L1=0.0, kappa=6.5e-12), T=300.0, S=None, steps=10, imex=False),
    "l123_weak": dict(grid=(16, 16, 24), p=dict(L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5), T=302.0, S=0.6, steps=10,
                      imex=False),
    "ravnik_l3_weak": dict(grid=(16, 16, 16), p=dict(bulk_modechoice=2, L1=6e-12, L3=2e-12, W=1e-5), T=301.0,
                           S=0.6, steps=8, imex=False),
    "aniso_l2_weak": dict(grid=(16, 24, 16), p=dict(L1=6e-12, L2=2e-12, W=2e-5, dy=1.2e-8, dz=0.9e-8), T=302.0,
                          S=0.5, steps=8, imex=False),
    "imex_l1_strong": dict(grid=(16, 16, 16), p=dict(L1=6e-12), T=305.0, S=None, steps=3, imex=True),
}


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def main(outdir=HERE):
    orc = Oracle()
    ref = RefCUDA()
    for name, c in QSR_CASES.items():
        Nx, Ny, Nz = c["grid"]
        op = make_params(Nx=Nx, Ny=Ny, Nz=Nz, T_star=307.0, **c["p"])
        g, fl = orc.geometry(op)
        q0 = orc.init(op, g, 0, 42, 0.5)
        A, B, C = orc.bulk_ABC(op.a, op.b, op.c, c["T"], op.T_star, op.bulk_modechoice)
        S_shell = c["S"] if c["S"] is not None else max(orc.S_eq(A, B, C), 0.0)
        dt = 1.5e-10
        ref.create(op)
        ref.upload(q0)
        for _ in range(c["steps"]):
            if c["imex"]:
                ref.step(c["T"], S_shell, 4 * dt, imex=True, L_stab=op.L1, jacobi_iters=25)
            else:
                ref.step(c["T"], S_shell, dt)
        q1 = ref.download()
        obs = ref.observe(c["T"], S_shell, Nz // 2)
        delta_eff = ref.L.qref_delta_eff()
        ref.destroy()
        np.savez_compressed(os.path.join(outdir, f"qsr_{name}.npz"), q_final=q1, init_sha=_sha(q0),
                            grid=np.array(c["grid"]), T=c["T"], S_shell=S_shell, dt=dt, steps=c["steps"],
                            imex=int(c["imex"]), params=repr(c["p"]), delta_eff=delta_eff,
                            **{f"obs_{k}": v for k, v in obs.items()})
        print("wrote", name, obs["bulk"], obs["elastic"], obs["anchoring"])
    kref = RefKZM()
    bp = OrcBulkParams(16, 8, 24, 1e-8, 1.1e-8, 0.9e-8, 6e-12, 0.1, 1e-10, 0.0, 0.1, 0.25)
    q0 = orc.bulk_init(bp, 12345, 0.2)
    A, B, C = orc.bulk_ABC(0.044e6, 1.413e6, 1.153e6, 296.0, 307.0, 1)
    q1 = kref.run(bp, q0, 40, A, B, C)
    obs = kref.observe(bp, q1, A, B, C)
    np.savez_compressed(os.path.join(outdir, "kzm_periodic.npz"), q_final=q1, init_sha=_sha(q0), steps=40,
                        A=A, B=B, C=C, **{f"obs_{k}": v for k, v in obs.items()})
    print("wrote kzm_periodic", obs)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
