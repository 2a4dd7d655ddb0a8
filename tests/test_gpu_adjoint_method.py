"""check_gradient of an AdjointMethodPNF3D subclass over the GPU solver.

A user script written against the reference's adjoint-method classes
(emopt/adjoint_method.py:1329-1486) runs unchanged over emopt_b200: a layered
structure (StructuredMaterial3D) whose two design rectangles carry the
parameters as their permittivities, a current-sheet source, a mode-match
figure of merit on an output plane normalised by the source power
(fomutils.ModeMatch, power_norm_dFdx_3D), and the reference's gradient
protocol: the adjoint gradient from FDTD.calc_ydAx on the updated boxes
against one-sided finite differences of the figure of merit, total relative
error below the reference's 1% warning threshold.  The multi-objective
driver (emopt/adjoint_method.py:723-929) combines two such objectives at two
wavelengths, each on its own GPU solver.  Fixed step counts make the
figures of merit smooth functions of the parameters."""
import numpy as np
import pytest

from emopt_b200 import grid as G
from emopt_b200.adjoint_method import AdjointMethodMO, AdjointMethodPNF3D
from emopt_b200.fdtd import FDTD
from emopt_b200.fomutils import ModeMatch
from emopt_b200.misc import DomainCoordinates

pytestmark = pytest.mark.gpu

COMPS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
X, Y, Z, D = 2.4, 1.4, 1.2, 0.04
RECTS = [(1.0, 0.55, 0.4, 0.5), (1.45, 0.85, 0.4, 0.5)]       # (x0, y0, xspan, yspan)
ZD = (0.4, 0.8)                                                # design layer


class TwoBlocks(AdjointMethodPNF3D):
    def __init__(self, sim, rects, plane, mode):
        super().__init__(sim, step=1e-6)
        self.rects, self.plane, self.mode = rects, plane, mode

    def update_system(self, params):
        for r, p in zip(self.rects, params):
            r.set_material(complex(p))

    def get_update_boxes(self, sim, params):
        return [(r.x0 - r.width / 2 - D, r.x0 + r.width / 2 + D, r.y0 - r.height / 2 - D,
                 r.y0 + r.height / 2 + D, ZD[0] - D, ZD[1] + D) for r in self.rects]

    def _mm(self, sim):
        mm = ModeMatch((1, 0, 0), D, D, **self.mode)
        mm.compute(**{c: sim.get_field_interp(c, self.plane) for c in COMPS})
        return mm

    def calc_f(self, sim, params):
        return self._mm(sim).get_mode_match_forward(1.0)

    def calc_dfdx(self, sim, params):
        mm = self._mm(sim)
        return [[mm.get_dFdEx(), mm.get_dFdEy(), mm.get_dFdEz(), mm.get_dFdHx(), mm.get_dFdHy(),
                 mm.get_dFdHz()]]

    def get_fom_domains(self):
        return [self.plane]

    def calc_grad_p(self, sim, params):
        return np.zeros(len(params))


def _setup(wavelength=1.55):
    sim = FDTD(X, Y, Z, D, D, D, wavelength, rtol=1e-6, precision="fp64")
    sim.set_pml_cells([8, 8, 8, 8, 8, 8])
    sim.fixed_steps = 2500
    eps = G.StructuredMaterial3D(sim.X, sim.Y, sim.Z, D, D, D)
    bg = G.Rectangle(sim.X / 2, sim.Y / 2, 2 * sim.X, 2 * sim.Y)
    bg.set_material(1.444 ** 2)
    bg.layer = 3
    eps.add_primitive(bg, -1.0, 2 * sim.Z)
    core = G.Rectangle(sim.X / 2, sim.Y / 2, 2 * sim.X, 0.5)
    core.set_material(2.9 ** 2)
    core.layer = 2
    eps.add_primitive(core, ZD[0], ZD[1])
    rects = []
    for x0, y0, xs, ys in RECTS:
        r = G.Rectangle(x0, y0, xs, ys)
        r.layer = 1
        eps.add_primitive(r, ZD[0], ZD[1])
        rects.append(r)
    sim.set_materials(eps, G.ConstantMaterial3D(1.0))
    # a Jz current sheet across the core at x = 0.5 um
    src_dom = DomainCoordinates(0.5, 0.5, 0.2, sim.Y - 0.2, 0.2, sim.Z - 0.2, D, D, D)
    J, K = src_dom.shape[1], src_dom.shape[2]
    y = np.linspace(-1, 1, J)[None, :, None]
    z = np.linspace(-1, 1, src_dom.shape[0])[:, None, None]
    Jz = (np.exp(-(y / 0.35) ** 2 - ((z - 0.0) / 0.35) ** 2) * np.ones((1, 1, K))).astype(np.complex128)
    zero = np.zeros_like(Jz)
    sim.set_sources((zero, zero, Jz, zero, zero, zero), src_dom)
    sim.build()
    # the output plane and a smooth synthetic mode on it
    plane = DomainCoordinates(sim.X - 0.5, sim.X - 0.5, 0.2, sim.Y - 0.2, 0.2, sim.Z - 0.2, D, D, D)
    shp = plane.shape
    zz, yy = np.meshgrid(np.linspace(-1, 1, shp[0]), np.linspace(-1, 1, shp[1]), indexing="ij")
    prof = np.exp(-(yy / 0.4) ** 2 - (zz / 0.4) ** 2).reshape(shp).astype(np.complex128)
    mode = {"Ezm": prof, "Hym": -prof / 1.4}
    return sim, rects, plane, mode


def test_check_gradient_of_a_power_normalised_mode_match():
    sim, rects, plane, mode = _setup()
    am = TwoBlocks(sim, rects, plane, mode)
    params = np.array([3.2, 2.6])
    err, g_fd, g_am = am.check_gradient(params, plot=False, verbose=False, return_gradients=True,
                                        fd_step=1e-4)
    print("finite differences", g_fd, "adjoint", g_am, "total relative error %.3e" % err)
    assert np.all(np.abs(g_fd) > 0)
    assert err < 1e-2


class Broadband(AdjointMethodMO):
    """The mean of the objectives at several wavelengths."""

    def calc_total_fom(self, foms):
        return float(np.mean(foms))

    def calc_total_gradient(self, foms, grads):
        return np.mean(np.array(grads), axis=0)


def test_check_gradient_of_a_two_wavelength_objective():
    ams = []
    for wl in (1.50, 1.60):
        sim, rects, plane, mode = _setup(wl)
        ams.append(TwoBlocks(sim, rects, plane, mode))
    mo = Broadband(ams)
    params = np.array([3.2, 2.6])
    f = mo.fom(params.copy())
    assert f == pytest.approx(np.mean([am.calc_fom(am.sim, params) for am in ams]), rel=1e-12)
    err, g_fd, g_am = mo.check_gradient(params, plot=False, verbose=False, return_gradients=True,
                                        fd_step=1e-4)
    print("finite differences", g_fd, "adjoint", g_am, "total relative error %.3e" % err)
    assert np.all(np.abs(g_fd) > 0)
    assert err < 1e-2
