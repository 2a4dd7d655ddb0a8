"""CPU tests of the mode-solver oracle (oracle/modes.py) and of the host side of
emopt_b200/modes.py.

* known answer: a uniform medium in the PEC box has the discrete dispersion
  relation of the compressed Yee grid, so every nonzero eigenvalue of the
  restated A, B must satisfy it ('0' and 'H' boundaries);
* the shift-and-invert solve (SuperLU + ARPACK, as SLEPc with a target)
  returns the dense QZ solve's eigenpairs closest to n0;
* the product's interpolation onto the plane's Ez points and its component
  permutation equal the oracle's on the same raw fields.
"""
import numpy as np
import pytest

from oracle import modes as O

WL = 1.55


@pytest.mark.parametrize("bc", [("0", "0"), ("H", "0"), ("0", "H"), ("H", "H")])
def test_uniform_box_dispersion(bc):
    M, N, dx, dy, eps = 7, 9, 0.1, 0.12, 2.5
    planes = [np.full((M, N), eps, complex)] * 3 + [np.ones((M, N), complex)] * 3
    A, B = O.build_system(planes, M, N, dx, dy, WL, bc=bc)
    w, _ = O.solve_dense(A, B, 1.5, 6 * M * N)
    n2 = (w ** 2)[np.abs(w) > 1e-6]
    spec = O.discrete_box_spectrum(eps, 1.0, M, N, dx, dy, WL).ravel()
    assert len(n2) > 100
    assert max(np.min(np.abs(spec - v)) for v in n2) < 1e-9
    # the guided end is there: the (p, q) = (1, 0) mode
    assert np.min(np.abs(n2 - spec[1])) < 1e-10


def _layered(M, N, seed):
    rng = np.random.default_rng(seed)
    ex = 2.0 + 10 * (rng.uniform(size=(M, N)) > 0.6)
    return [ex + 0j, np.roll(ex, 1, 0) + 0.01j, np.roll(ex, 1, 1) + 0j] + [np.ones((M, N), complex)] * 3


@pytest.mark.parametrize("bc,back", [(("0", "0"), False), (("E", "H"), True), (("H", "E"), False)])
def test_shift_invert_matches_dense(bc, back):
    M, N = 8, 11
    A, B = O.build_system(_layered(M, N, 1), M, N, 0.05, 0.06, WL, bc=bc, backwards=back)
    w1, V1 = O.solve(A, B, 3.3, 4)
    w2, V2 = O.solve_dense(A, B, 3.3, 4)
    assert np.abs(w1 - w2).max() < 1e-12
    assert np.all(np.abs(w1 - 3.3)[:-1] <= np.abs(w1 - 3.3)[1:])
    for q in range(4):
        assert abs(np.vdot(V1[q], V2[q])) == pytest.approx(1.0, abs=1e-10)


def test_backward_mode_flips_h():
    M, N = 8, 9
    planes = _layered(M, N, 2)
    Af, Bf = O.build_system(planes, M, N, 0.05, 0.05, WL)
    Ab, Bb = O.build_system(planes, M, N, 0.05, 0.05, WL, backwards=True)
    wf, Vf = O.solve(Af, Bf, 3.0, 2)
    wb, Vb = O.solve(Ab, Bb, 3.0, 2)
    assert np.allclose(wf, wb, rtol=1e-12)
    # the mode travelling the other way: Ex, Ey, Hz kept, Ez, Hx, Hy reversed
    MN = M * N
    sign = np.repeat([1, 1, -1, -1, -1, 1], MN)
    for q in range(2):
        c = np.vdot(Vb[q] * sign, Vf[q])
        c /= abs(c)
        assert np.allclose(Vb[q] * sign * c, Vf[q], atol=1e-10)


@pytest.mark.parametrize("ndir,shape", [("x", (6, 5, 1)), ("y", (6, 1, 7)), ("z", (1, 5, 7))])
@pytest.mark.parametrize("bc", [("0", "0"), ("E", "H"), ("H", "E")])
def test_product_interpolation_matches_oracle(ndir, shape, bc):
    torch = pytest.importorskip("torch")
    from emopt_b200.grid import ConstantMaterial3D
    from emopt_b200.misc import DomainCoordinates
    from emopt_b200.modes import ModeFullVector
    Nz, Ny, Nx = shape
    dom = DomainCoordinates.from_indices(3, 3 + Nx, 2, 2 + Ny, 1, 1 + Nz, 0.05, 0.05, 0.05)
    m = ModeFullVector(WL, ConstantMaterial3D(2.0), ConstantMaterial3D(1.0), dom, device=0)
    m.bc = list(bc)
    assert m.ndir == ndir
    M, N = m._M, m._N
    rng = np.random.default_rng(3)
    vec = rng.standard_normal(6 * M * N) + 1j * rng.standard_normal(6 * M * N)
    m._x = torch.as_tensor(vec.reshape(1, 6, M, N))
    for c in O.COMPONENTS:
        np.testing.assert_array_equal(m.get_field(0, c, squeeze=True), O.get_field(vec, c, M, N, ndir))
        assert m.get_field(0, c).shape == shape
        want = O.get_field_interp(vec, c, M, N, ndir, bc)
        np.testing.assert_allclose(m.get_field_interp(0, c, squeeze=True), want, rtol=0, atol=1e-15)
