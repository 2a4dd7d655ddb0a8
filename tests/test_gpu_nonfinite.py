"""GPU tests of the non-finite stop of FDTD_solve_cw.

The reference treats NaN/Inf probe values as "not converged" and runs on to
Nmax (emopt/fdtd.py:1050-1057); FDTDSolveOptions.stop_nonfinite = 1 (the
solver's ``stop_nonfinite`` attribute) ends the main loop at the first probe
that sees them instead.  Both report FDTD_NONFINITE.  The failure is made on
the host: NaN written into the permittivity array."""
import numpy as np
import pytest

from emopt_b200 import fdtd_ctypes as ct
from emopt_b200 import problems as P

pytestmark = pytest.mark.gpu


def _nan_box():
    p = P.random_box(seed=51, shape=(12, 10, 14), fixed_steps=None, rtol=1e-6)
    eps = [a.copy() for a in p.mats[:3]]
    for a in eps:
        a[:, :, : a.shape[2] // 2] = np.nan
    p.mats = tuple(eps) + tuple(p.mats[3:])
    p.Nmax = 1500
    return p


@pytest.mark.parametrize("stop", [False, True])
def test_nan_permittivity(stop):
    p = _nan_box()
    sim = P.make_solver(p, precision="fp32", kernel="vector")
    sim.stop_nonfinite = stop
    info = sim._solve([sim._Ex_fwd_t0, sim._Ey_fwd_t0, sim._Ez_fwd_t0, sim._Hx_fwd_t0,
                       sim._Hy_fwd_t0, sim._Hz_fwd_t0],
                      [sim._Ex_fwd_t1] * 6, sim._sources)
    Tn = int(np.int64(sim._Ncycle * 3 / 4))
    assert info["status"] == ct.FDTD_NONFINITE
    if stop:
        assert info["nprobes"] == 1 and info["steps"] == 3 * Tn
    else:
        # the reference's loop: every probe up to the step budget
        assert info["n_main"] > p.Nmax and info["steps"] == info["n_main"] + 2 * Tn
