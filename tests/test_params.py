"""CPU tests of the host-side logic: parameter derivation against the oracle's
restatement of emopt/fdtd.py:236-437, domain index rules, problem builders."""
import numpy as np
import pytest

from emopt_b200 import problems as P
from emopt_b200.misc import DomainCoordinates
from helpers import oracle_for


@pytest.mark.parametrize("dims", [(4.0, 3.0, 2.56, 0.04, 0.04, 0.04, 1.55),
                                  (8.0, 4.0, 2.5, 0.025, 0.025, 0.025, 1.55),
                                  (1.3, 0.7, 0.9, 0.02, 0.025, 0.04, 1.31)])
def test_parameters_match_driver(dims):
    from emopt_b200.fdtd import derive_parameters
    from oracle.driver import OracleFDTD
    X, Y, Z, dx, dy, dz, wl = dims
    prm = derive_parameters(X, Y, Z, dx, dy, dz, wl)
    o = OracleFDTD(X, Y, Z, dx, dy, dz, wl, lib="oracle")
    assert (prm["Nx"], prm["Ny"], prm["Nz"]) == (o.Nx, o.Ny, o.Nz)
    for key, val in (("dt", o.dt), ("src_T", o.src_T), ("Nmax", o.Nmax), ("Ncycle", o.Ncycle)):
        assert prm[key] == val, key
    assert prm["Tn"] == int(np.int64(o.Ncycle * 3 / 4))
    np.testing.assert_array_equal(prm["conv_pts"], o.conv_pts)


def test_benchmark_grid_sizes():
    assert P.waveguide().shape == (65, 76, 101)
    assert P.mmi_block().shape == (101, 161, 321)


def test_domain_index_rule():
    d = DomainCoordinates(0.6, 0.6, 0.0, 3.0, 0.0, 2.56, 0.04, 0.04, 0.04)
    assert (d.k1, d.k2) == (int(0.6 / 0.04), int(0.6 / 0.04) + 1)
    e = DomainCoordinates.from_indices(15, 16, 0, 76, 0, 65, 0.04, 0.04, 0.04)
    assert e.shape == (65, 76, 1)


def test_mmi_design_density_projection():
    p = P.mmi_block()
    rho = p.design_density
    assert rho.shape == (120, 80) and rho.min() >= 0 and rho.max() <= 1
    eps = p.mats[2].real
    assert eps.min() == pytest.approx(2.085) and eps.max() <= 12.25 + 1e-12


def test_oracle_config_from_problem():
    p = P.random_box(3, bc="EH0")
    o = oracle_for(p, "oracle")
    assert o.bc == "EH0" and o.w_pml_cells == list(p.w_pml)
