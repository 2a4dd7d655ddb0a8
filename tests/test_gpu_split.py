"""The split vector pair (kernel 6: per half step an interior launch whose
body has no CPML code, over the warp tasks that lie in no CPML slab, and a
rim launch over the tasks of the CPML slabs) against the vector pair (kernel
5) on grids whose interior box holds warp tasks: random media with sources
inside and outside the box, symmetric faces, lossy media, mu arrays, float32
and float64.  Every task is computed by the same body arithmetic as in the
vector pair; the interior body is compiled on its own, so the compiler may
contract its multiply-adds differently, and the fields agree to rounding
(1e-12 relative in float64, 1e-6 in float32; measured 4e-16 and 2e-7)."""
import numpy as np
import pytest

from emopt_b200 import problems as P
from emopt_b200.fdtd_ctypes import libFDTD

pytestmark = pytest.mark.gpu

SHAPE = (14, 12, 200)          # interior box: planes 3..10, rows 3..9, 64-cell blocks 1..2
CASES = {
    "pec": dict(seed=41, bc="000", n_sources=3),
    "sym": dict(seed=42, bc="EH0", n_sources=3),
    "lossy_mu": dict(seed=43, bc="0HE", complex_eps=True, mu_random=True, n_sources=2),
    "edge": dict(seed=44, bc="000", edge_source=True, n_sources=2),
}


def _fields(p, precision, kernel):
    sim = P.make_solver(p, precision=precision, kernel=kernel)
    info = sim._solve([sim._Ex_fwd_t0, sim._Ey_fwd_t0, sim._Ez_fwd_t0, sim._Hx_fwd_t0,
                       sim._Hy_fwd_t0, sim._Hz_fwd_t0],
                      [sim._Ex_fwd_t1, sim._Ey_fwd_t1, sim._Ez_fwd_t1, sim._Hx_fwd_t1,
                       sim._Hy_fwd_t1, sim._Hz_fwd_t1], sim._sources)
    return np.stack([sim._raw(c, False) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")]), info


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(CASES))
def test_split_pair_equals_vector_pair(name, precision):
    p = P.random_box(shape=SHAPE, w_pml=(3, 4, 3, 2, 3, 4), fixed_steps=160, **CASES[name])
    F5, i5 = _fields(p, precision, "vector")
    F6, i6 = _fields(p, precision, "split")
    assert i5["steps"] == i6["steps"]
    tol = 1e-12 if precision == "fp64" else 1e-6
    err = float(np.linalg.norm(F6 - F5) / np.linalg.norm(F5))
    print("%s %s: split vs vector %.2e, identical %s" % (name, precision, err, np.array_equal(F5, F6)))
    assert err <= tol


def test_auto_takes_the_split_pair_only_for_a_large_float32_interior():
    """Kernel 0 (auto) equals the split pair on a float32 grid whose interior
    holds >= 60% of the warp tasks, and the vector pair on the MMI-like grid
    with a thick CPML (float32) and in float64."""
    # interior: 37 of 40 planes, 36 of 40 rows, 8 of 10 blocks: 67% of the tasks
    big = P.random_box(shape=(40, 40, 640), w_pml=(2, 2, 2, 2, 2, 2), fixed_steps=60, seed=45, n_sources=2)
    Fa, _ = _fields(big, "fp32", "auto")
    F6, _ = _fields(big, "fp32", "split")
    assert np.array_equal(Fa, F6)
    Fa64, _ = _fields(big, "fp64", "auto")
    F5, _ = _fields(big, "fp64", "vector")
    assert np.array_equal(Fa64, F5)
    thick = P.random_box(shape=SHAPE, w_pml=(3, 4, 3, 2, 3, 4), fixed_steps=60, seed=46)
    Fa, _ = _fields(thick, "fp32", "auto")
    F5, _ = _fields(thick, "fp32", "vector")
    assert np.array_equal(Fa, F5)
