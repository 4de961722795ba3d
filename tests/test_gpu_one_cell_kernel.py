"""The one-cell-per-thread step kernel (LDG_QSR_PAIR=0) against the oracle (GPU).

The library runs two cells per thread by default and reads LDG_QSR_PAIR once per process, so the
one-cell kernels are checked in a child process: the explicit-step, IMEX, noise, tiled-vs-direct
and compensated-storage cases of tests/test_gpu_qsr.py, and the ensemble cases of
tests/test_gpu_ensemble.py.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_one_cell_kernels_match_oracle():
    env = dict(os.environ, LDG_QSR_PAIR="0")
    cmd = [sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu",
           os.path.join(HERE, "test_gpu_qsr.py"), os.path.join(HERE, "test_gpu_ensemble.py"),
           "-k", "explicit_steps or imex_steps or noise_stream or tiled_matches_direct or compensated or ensemble"]
    r = subprocess.run(cmd, env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and " failed" not in r.stdout
