"""GPU tests of the full-vector mode solver (emopt_b200/modes.py over
emopt_b200/csrc/modes.cu) against the oracle restatement of the reference's
ModeFullVector (oracle/modes.py: the reference's A and B, SuperLU + ARPACK
shift-and-invert about n0).

Planes of each orientation, boundary types and both directions: effective
indices to 1e-10 relative, every raw field component, the interpolated fields
and the six source planes of get_source to 1e-8 (relative L2, after aligning
the one free phase of each mode).
"""
import numpy as np
import pytest

from emopt_b200.grid import FunctionMaterial3D
from emopt_b200.misc import DomainCoordinates
from emopt_b200.modes import ModeFullVector
from oracle import modes as O

pytestmark = pytest.mark.gpu
WL = 1.55
D = 0.04


def strip(yc, zc, w=0.5, h=0.22, core=12.25, clad=2.085, axis="x"):
    """A rectangular core along `axis` (the other two coordinates bounded)."""
    def f(x, y, z):
        a, b = {"x": (y, z), "y": (x, z), "z": (x, y)}[axis]
        return np.where((np.abs(a - yc) < w / 2) & (np.abs(b - zc) < h / 2), core, clad) + 0j
    return f


def oracle_modes(f, dom, ndir, M, N, bc, n0, neigs, backwards=False):
    ef = lambda k, j, i: f(k * D, j * D, i * D)
    mf = lambda k, j, i: np.ones(np.shape(k)) + 0j
    planes = O.material_planes(ef, mf, ndir, M, N, dom.k1, dom.j1, dom.i1)
    dx, dy = {"x": (D, D), "y": (D, D), "z": (D, D)}[ndir]
    A, B = O.build_system(planes, M, N, dx, dy, WL, bc=bc, backwards=backwards)
    neff, V = O.solve(A, B, n0, neigs)
    return neff, V, planes


def aligned_err(a, b):
    c = np.vdot(a, b)
    c = c / abs(c) if c != 0 else 1.0
    return np.linalg.norm(a * c - b) / np.linalg.norm(b)


CASES = {
    # name: (material, domain indices (k1, k2, j1, j2, i1, i2), bc, n0, neigs, backwards, sweep)
    "x_strip": (strip(0.7, 0.46), (5, 6, 0, 36, 0, 24), ("0", "0"), 3.0, 3, False, None),
    "x_strip_sweep_x": (strip(0.7, 0.46), (5, 6, 0, 36, 0, 24), ("0", "0"), 3.0, 3, False, "x"),
    "x_strip_sweep_y": (strip(0.7, 0.46), (5, 6, 0, 36, 0, 24), ("0", "0"), 3.0, 3, False, "y"),
    "z_sym_back": (strip(0.0, 0.0, w=0.6, h=0.4, axis="z"), (0, 20, 0, 16, 3, 4), ("E", "H"), 3.2, 2, True, None),
    "y_plane": (strip(0.5, 0.4, w=0.44, h=0.3, axis="y"), (0, 26, 4, 5, 0, 20), ("H", "0"), 3.1, 2, False, None),
}


@pytest.mark.parametrize("name", list(CASES))
def test_modes_match_oracle(name):
    f, idx, bc, n0, neigs, back, sweep = CASES[name]
    dom = DomainCoordinates.from_indices(*idx, D, D, D)
    eps = FunctionMaterial3D(f, D, D, D)
    mu = FunctionMaterial3D(lambda x, y, z: np.ones(np.shape(x)) + 0j, D, D, D)
    m = ModeFullVector(WL, eps, mu, dom, n0=n0, neigs=neigs, backwards=back, device=0, sweep=sweep)
    m.bc = list(bc)
    m.build()
    # the sampled planes are the oracle's
    ndir, M, N = O.plane_orientation(dom.shape)
    neff, V, planes = oracle_modes(f, dom, ndir, M, N, bc, n0, neigs, back)
    for got, want in zip(m._planes, planes):
        np.testing.assert_array_equal(got.cpu().numpy(), want)
    m.solve()
    print(name, m.stats, m.neff)
    np.testing.assert_allclose(m.neff, neff, rtol=1e-10)
    for q in range(neigs):
        for c in O.COMPONENTS:
            want = O.get_field(V[q], c, M, N, ndir)
            got = m.get_field(q, c, squeeze=True)
            if np.linalg.norm(want) > 1e-6 * np.linalg.norm(V[q]):
                assert aligned_err(got, want) < 1e-8, (q, c)
        # one phase per mode: align once on the whole vector, then compare all
        vg = np.concatenate([m.get_field(q, c, permute=False, squeeze=True).ravel() for c in O.COMPONENTS])
        c = np.vdot(vg, V[q])
        c /= abs(c)
        for comp in O.COMPONENTS:
            want = O.get_field_interp(V[q], comp, M, N, ndir, bc)
            got = m.get_field_interp(q, comp, squeeze=True) * c
            assert np.linalg.norm(got - want) <= 1e-8 * np.linalg.norm(V[q]) * np.sqrt(M * N), comp
        ef = lambda k, j, i: f(k * D, j * D, i * D)
        one = lambda *a: np.ones(np.shape(a[0])) + 0j
        kk, jj, ii = np.meshgrid(np.arange(dom.k1, dom.k2), np.arange(dom.j1, dom.j2),
                                 np.arange(dom.i1, dom.i2), indexing="ij")
        eps_plane = np.transpose(ef(kk, jj, ii), (2, 1, 0)).reshape(M, N)
        want_src = O.get_source(V[q], neff[q], M, N, ndir, bc, WL, D, D, D, eps_plane,
                                np.ones((M, N), complex), np.ones((M, N), complex), backwards=back)
        got_src = m.get_source(q, D, D, D)
        # one factor for all six planes: the mode's phase, and the sign of
        # sqrt(S), which for a backward mode (S < 0) follows the rounding of
        # Im S in both the reference and here
        cs = np.vdot(np.concatenate([g.ravel() for g in got_src]),
                     np.concatenate([w.ravel() for w in want_src]))
        cs /= abs(cs)
        if not back:
            assert abs(cs - c) < 1e-8
        total = np.sqrt(sum(np.linalg.norm(w) ** 2 for w in want_src))
        for g, w in zip(got_src, want_src):
            assert g.shape == dom.shape
            assert np.linalg.norm(g.reshape(M, N) * cs - w) <= 1e-8 * max(np.linalg.norm(w), 1e-3 * total)


def test_mode_source_launches_the_mode():
    """The reference's simple_waveguide_mode_3D set-up, smaller: a silicon strip
    in oxide, the mode source of ModeFullVector on a plane across it, one CW
    solve.  The field on a plane downstream is the mode (overlap >= 0.98) and
    almost nothing travels the other way (backward flux < 2% of forward)."""
    from emopt_b200 import grid
    from emopt_b200.fdtd import FDTD
    X, Y, Z, d = 3.0, 2.0, 1.6, 0.04
    sim = FDTD(X, Y, Z, d, d, d, WL, rtol=1e-6)
    w = d * 10
    sim.w_pml = [w] * 6
    X, Y, Z = sim.X, sim.Y, sim.Z
    r1 = grid.Rectangle(X / 2, Y / 2, 2 * X, 0.5)
    r1.layer = 1
    r1.material_value = 3.45 ** 2
    r2 = grid.Rectangle(X / 2, Y / 2, 2 * X, 2 * Y)
    r2.layer = 2
    r2.material_value = 1.444 ** 2
    eps = grid.StructuredMaterial3D(X, Y, Z, d, d, d)
    eps.add_primitive(r2, -Z, Z)
    eps.add_primitive(r1, Z / 2 - 0.11, Z / 2 + 0.11)
    mu = grid.ConstantMaterial3D(1.0)
    sim.set_materials(eps, mu)
    sim.build()
    src = DomainCoordinates(0.8, 0.8, w, Y - w, w, Z - w, d, d, d)
    mode = ModeFullVector(WL, eps, mu, src, n0=3.45, neigs=4, device=0)
    mode.build()
    mode.solve()
    print("neff", mode.neff, mode.stats)
    assert 2.0 < mode.neff[0].real < 3.0 and abs(mode.neff[0].imag) < 1e-9
    sim.set_sources(mode, src)
    sim.solve_forward()

    def fields(x):
        plane = DomainCoordinates(x, x, w, Y - w, w, Z - w, d, d, d)
        return {c: sim.get_field_interp(c, plane) for c in ("Ey", "Ez", "Hy", "Hz")}

    def flux(F):
        return 0.5 * np.sum(F["Ey"] * np.conj(F["Hz"]) - F["Ez"] * np.conj(F["Hy"])).real

    fwd, back = fields(2.2), fields(0.56)
    Pf, Pb = flux(fwd), flux(back)
    Pm_f = {c: mode.get_field_interp(0, c) for c in ("Ey", "Ez", "Hy", "Hz")}
    Pm = flux(Pm_f)
    cross = np.sum(fwd["Ey"] * np.conj(Pm_f["Hz"]) - fwd["Ez"] * np.conj(Pm_f["Hy"])
                   + np.conj(Pm_f["Ey"]) * fwd["Hz"] - np.conj(Pm_f["Ez"]) * fwd["Hy"])
    eta = abs(cross) ** 2 / (16 * Pm * Pf)
    print("forward flux %.4e backward %.4e overlap %.5f" % (Pf, Pb, eta))
    assert Pf > 0 and abs(Pb) < 0.02 * Pf
    assert eta > 0.98
