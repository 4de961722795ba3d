"""The benchmark's reference arm runs on the CPU (the reference's own QSR.cpp step chain built
under oracle/_ref) and prints one JSON line with the keys the benchmark contract names."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_contract_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libqsr_cpu_ref.so")):
        pytest.skip("reference CPU build absent")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--ref-grid", "16"], cwd=ROOT, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, RANK="0", WORLD_SIZE="1"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"] == "anisotropic_weak_256"


def test_l2_note_follows_the_field_size():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    # 256^3 and 512^3 fields (20 B per cell) exceed the 126 MB L2 twice over; 64^3 fits
    assert bench.l2_note(20 * 256 ** 3).startswith("inputs larger than L2")
    assert bench.l2_note(20 * 512 ** 3).startswith("inputs larger than L2")
    assert bench.l2_note(20 * 64 ** 3).startswith("inputs fit in L2")
