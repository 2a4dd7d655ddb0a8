"""Host-side tables of the device field kernels (emopt_b200/fieldops.py), on
the CPU: the source-power planes, their signs and the (E1, H2, E2, H1)
components of each plane's flux reproduce FDTD.get_source_power (the host
restatement of emopt/fdtd.py:1555-1667) term for term, on grids where every
plane holds cells."""
import numpy as np
import pytest
from types import SimpleNamespace

from emopt_b200 import adjoint as A
from emopt_b200 import fieldops as FO
from emopt_b200.fdtd import FDTD


def _host_sim(shape, w_cells, bc, d=0.04, seed=0):
    """An FDTD object with only what get_field_interp / get_source_power read:
    lengths, cell sizes, CPML widths, boundary letters and the t0 phasors."""
    Nz, Ny, Nx = shape
    s = FDTD.__new__(FDTD)
    s._dx = s._dy = s._dz = d
    s._Nx, s._Ny, s._Nz = Nx, Ny, Nz
    s._X, s._Y, s._Z = (Nx - 1) * d, (Ny - 1) * d, (Nz - 1) * d
    s._w_pml = [w * d for w in w_cells]
    s._bc = bc
    rng = np.random.default_rng(seed)
    for c in FO.COMPONENTS:
        setattr(s, "_%s_fwd_t0" % c, rng.standard_normal(Nx * Ny * Nz) + 1j * rng.standard_normal(Nx * Ny * Nz))
    view = SimpleNamespace(dx=d, dy=d, dz=d, _w_pml=s._w_pml, X=s._X, Y=s._Y, Z=s._Z, bc=bc)
    return s, view


@pytest.mark.parametrize("bc", ["000", "E00", "H00", "0E0", "0H0", "EH0", "HE0"])
def test_flux_table_reproduces_host_source_power(bc):
    s, view = _host_sim((14, 13, 16), (3, 4, 3, 2, 2, 3), bc, seed=len(bc) + ord(bc[0]) + ord(bc[1]))
    planes = A.source_power_planes(view)
    assert len(planes) == 6 - (bc[0] in "EH") - (bc[1] in "EH")
    dA = {0: s._dy * s._dz, 1: s._dx * s._dz, 2: s._dx * s._dy}
    total = 0.0
    axes_seen = set()
    for dom, axis, sign in planes:
        assert dom.i2 > dom.i1 and dom.j2 > dom.j1 and dom.k2 > dom.k1
        e1, h2, e2, h1 = FO._FLUX[axis]
        g = s.get_field_interp
        flux = np.sum(np.real(g(e1, dom) * np.conj(g(h2, dom)) - g(e2, dom) * np.conj(g(h1, dom))))
        assert abs(flux) > 0
        total += sign * 0.5 * dA[axis] * flux
        axes_seen.add(axis)
    assert axes_seen == {0, 1, 2}
    assert total == pytest.approx(s.get_source_power(), rel=1e-13)


def test_flux_components_are_the_normal_poynting_component():
    """Re(E1 H2* - E2 H1*) is the component of E x H* along the plane normal."""
    rng = np.random.default_rng(3)
    E = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    H = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    S = np.cross(E, np.conj(H))
    idx = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 0, "Hy": 1, "Hz": 2}
    for axis in range(3):
        e1, h2, e2, h1 = FO._FLUX[axis]
        v = E[idx[e1]] * np.conj(H[idx[h2]]) - E[idx[e2]] * np.conj(H[idx[h1]])
        assert v.real == pytest.approx(S[axis].real, rel=1e-14)
