"""Both confined step kernels against the oracle, whatever the default chooses (GPU).

A single grid takes one cell per thread when its work list is small and two cells per thread
when it fills the GPU at least twice over; the ensemble always takes two. LDG_QSR_PAIR=0 / 1
forces one / two cells per thread, and the library reads it once per process, so each kernel is
checked in a child process on the explicit-step, IMEX, noise, tiled-vs-direct, compensated-storage
and ensemble cases of tests/test_gpu_qsr.py and tests/test_gpu_ensemble.py.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("mode", ["0", "1"])
def test_forced_kernel_matches_oracle(mode):
    env = dict(os.environ, LDG_QSR_PAIR=mode)
    cmd = [sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", "-m", "gpu",
           os.path.join(HERE, "test_gpu_qsr.py"), os.path.join(HERE, "test_gpu_ensemble.py"),
           "-k", "explicit_steps or imex_steps or noise_stream or tiled_matches_direct or compensated or ensemble"]
    r = subprocess.run(cmd, env=env, cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and " failed" not in r.stdout
