"""End-to-end warm-start pipeline at a small scale: solver-generated training data (ensemble),
U-Net training on the tcgen05 convolution kernels, and plain against warm-started relaxation on
the 2x finer grid.

What must hold even at this scale: the data are finite relaxed fields, training reduces the
loss, the warm start begins far closer to equilibrium than the random initial field (lower
free energy), and both arms end at the same free energy within 2 % when both converged.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_COARSE = 16
DX = 5e-9
R_RANGE = (0.3 * 2 * N_COARSE * DX, 0.42 * 2 * N_COARSE * DX)


def test_warmstart_pipeline_small():
    from lcdrsimulator_b200.surrogate import UNet3D
    from lcdrsimulator_b200.surrogate import warmstart as ws
    cases = ws.sample_cases(24, seed=3, R_range=R_RANGE)
    data = ws.make_dataset(cases, N_COARSE, DX, max_steps=30000, check_every=1000, tol=1e-8)
    assert data["X"].shape == (24, N_COARSE, N_COARSE, N_COARSE, 16)
    assert np.isfinite(data["Y"]).all()
    # relaxed fields are ordered nematics inside the droplet
    assert np.abs(data["Y"][data["M"]]).max() > 0.1
    net = UNet3D(seed=0).cuda()
    hist = ws.train(net, data["X"], data["Y"], data["M"], epochs=40, batch=8, lr=1e-3)
    assert hist[-1] < 0.5 * hist[0], hist
    ev = ws.evaluate(net, ws.sample_cases(2, seed=99, R_range=R_RANGE), N_COARSE, DX, max_steps=400000,
                     check_every=2000, tol=1e-8, coarse_tols=(1e-7,), coarse_max_steps=100000)
    assert ev["arms"] == ["plain", "unet", "unet+coarse@1e-07", "coarse@1e-07"]
    assert ev["coarse"]["us_per_droplet_step"] > 0
    for r in ev["results"]:
        assert np.isfinite([r["plain_E"], r["warm_E"], r["plain_E0"], r["warm_E0"]]).all()
        assert r["warm_E0"] < r["plain_E0"], r
        if r["plain_steps"] and r["warm_steps"]:
            assert abs(r["warm_E"] - r["plain_E"]) <= 0.02 * abs(r["plain_E"]), r
        for nm in ("unet+coarse@1e-07", "coarse@1e-07"):
            a = r["arms"][nm]
            assert a["coarse_steps"] > 0 and np.isfinite([a["E"], a["E0"]]).all(), a
            # a coarse-relaxed start is closer to equilibrium than the random field
            assert a["E0"] < r["plain_E0"], a
            if a["fine_steps"] and r["plain_steps"]:
                assert abs(a["E"] - r["plain_E"]) <= 0.02 * abs(r["plain_E"]), a
