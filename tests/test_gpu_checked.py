"""The index-checked library (emopt_b200/FDTD_checked.so, built with
FDTD_BOUNDS_CHECK) runs the parity cases of the production kernels.

In that build every index the vector pair and the serving kernel compute is
checked against its array before the access; a lane out of range records the
site and skips, and the solve, slab and serving calls then return an error.
The selected tests (fp64 golden boxes, every boundary combination, ragged
row tails, converging step counts, fp32 error bounds, z slabs at fixed step
counts, serving) therefore pass only if no index of theirs leaves its array.  They run in a child
process, which loads the checked library through EMOPT_B200_LIB.
"""
import os
import subprocess
import sys

import pytest

from helpers import ROOT

pytestmark = pytest.mark.gpu

SELECT = ("(test_gpu_parity and (vector or split)) or every_bc or test_fixed_steps "
          "or test_gpu_serving or test_split_pair")


def test_parity_cases_pass_with_index_checks():
    lib = os.path.join(ROOT, "emopt_b200", "FDTD_checked.so")
    assert os.path.exists(lib), "build the checked library first (python -m emopt_b200.build)"
    env = dict(os.environ, EMOPT_B200_LIB=lib)
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
           "-k", SELECT, "tests/test_gpu_parity.py", "tests/test_gpu_zslab.py", "tests/test_gpu_serving.py",
           "tests/test_gpu_split.py"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    print(out.stdout[-3000:], out.stderr[-2000:])
    assert out.returncode == 0
    assert " passed" in out.stdout and "deselected" in out.stdout

