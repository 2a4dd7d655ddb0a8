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


@pytest.mark.parametrize("bc", [(a, b) for a in "0EH" for b in "0EH"])
def test_uniform_box_dispersion(bc):
    M, N, dx, dy, eps = 7, 9, 0.1, 0.12, 2.5
    planes = [np.full((M, N), eps, complex)] * 3 + [np.ones((M, N), complex)] * 3
    A, B = O.build_system(planes, M, N, dx, dy, WL, bc=bc)
    w, _ = O.solve_dense(A, B, 1.5, 6 * M * N)
    n2 = (w ** 2)[np.abs(w) > 1e-6]
    spec = O.discrete_box_spectrum(eps, 1.0, M, N, dx, dy, WL, bc)
    assert len(n2) > 100
    assert max(np.min(np.abs(spec - v)) for v in n2) < 1e-9
    # the guided end is there: the largest n^2 is one of the two largest of
    # the spectrum (the (0, 0) value eps mu is a mode only with 'H' letters)
    top = np.unique(np.round(spec, 9))[::-1][:2]
    assert np.min(np.abs(np.max(n2.real) - top)) < 1e-8


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


def _line_order(M, N, sweep_y):
    L, NL = (N, M) if sweep_y else (M, N)
    perm = np.empty(NL * 6 * L, dtype=np.int64)
    for l in range(NL):
        for c in range(6):
            for p in range(L):
                y, x = (l, p) if sweep_y else (p, l)
                perm[(l * 6 + c) * L + p] = c * M * N + y * N + x
    return perm, L, NL


def _emulate_device(m, A, B, M, N):
    """Replace the product's device calls (assembly, B v, batched line GEMV,
    couplings) by exact host computations from the oracle's A and B."""
    import torch
    m._dev = torch.device("cpu")
    perm, L, NL = _line_order(M, N, bool(m._lines.sweep_y))
    nb = 6 * L
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    Al, Bl = A.toarray()[np.ix_(perm, perm)], B.toarray()[np.ix_(perm, perm)]
    Acoo = A.tocoo()

    def assemble(sig):
        T = Al - sig * Bl
        D = torch.as_tensor(np.stack([T[l * nb:(l + 1) * nb, l * nb:(l + 1) * nb] for l in range(NL)]))
        pcol, ncol = -torch.ones(NL, nb, dtype=torch.int32), -torch.ones(NL, nb, dtype=torch.int32)
        pval, nval = torch.zeros(NL, nb, dtype=torch.complex128), torch.zeros(NL, nb, dtype=torch.complex128)
        for i, j, v in zip(inv[Acoo.row], inv[Acoo.col], Acoo.data):
            li, lj = i // nb, j // nb
            if lj == li - 1:
                pcol[li, i % nb], pval[li, i % nb] = int(j % nb), v
            elif lj == li + 1:
                ncol[li, i % nb], nval[li, i % nb] = int(j % nb), v
        return D, pcol, pval, ncol, nval

    def gemv(lines32, rows32, rhs, corr, out):
        for l in lines32.tolist():
            r = m._W[l] @ (rhs[l] - (corr[l] if corr is not None else 0))
            if rows32 is None:
                out[l] += r
            else:
                out[l, rows32.long()] += r[rows32.long()]

    def couple(lines32, nbrs32, C, rows32, cols32, src, dst, sign):
        for z, (l, n) in enumerate(zip(lines32.tolist(), nbrs32.tolist())):
            dst[l, rows32.long()] += sign * (C[z] @ src[n, cols32.long()])

    m._assemble, m._gemv, m._couple = assemble, gemv, couple
    m._bmul = lambda v, out: out.view(-1).copy_(torch.as_tensor(Bl) @ v)
    return Al, Bl, perm


@pytest.mark.parametrize("M,N,sweep,bc,back", [
    (6, 7, "y", ("0", "0"), False), (6, 7, "x", ("0", "0"), False), (9, 5, "y", ("E", "H"), True),
    (9, 5, "x", ("H", "E"), False), (2, 3, "y", ("0", "0"), False), (1, 4, "y", ("0", "0"), False),
    (13, 4, "y", ("0", "0"), False), (4, 16, "x", ("E", "0"), True)])
def test_product_cyclic_reduction_solves_the_system(M, N, sweep, bc, back):
    """The product's block cyclic reduction (factor and the application of
    (A - n0 B)^-1 B), run on the CPU with its device calls emulated exactly
    from the oracle's A and B, equals a dense solve of the same system."""
    torch = pytest.importorskip("torch")
    from emopt_b200.grid import ConstantMaterial3D
    from emopt_b200.misc import DomainCoordinates
    from emopt_b200.modes import ModeFullVector
    sigma = 3.1
    A, B = O.build_system(_layered(M, N, 4), M, N, 0.05, 0.06, WL, bc=bc, backwards=back)
    dom = DomainCoordinates.from_indices(0, N, 0, M, 0, 1, 0.05, 0.06, 0.05)
    m = ModeFullVector(WL, ConstantMaterial3D(2.0), ConstantMaterial3D(1.0), dom, device=0, sweep=sweep)
    Al, Bl, _ = _emulate_device(m, A, B, M, N)
    m._factor(sigma)
    n = Al.shape[0]
    rng = np.random.default_rng(0)
    v = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n))
    out = torch.empty_like(v)
    m._apply_direct(v, out)
    want = np.linalg.solve(Al - sigma * Bl, Bl @ v.numpy())
    assert np.linalg.norm(out.numpy() - want) < 1e-12 * np.linalg.norm(want)


@pytest.mark.parametrize("sweep,bc,back", [("y", ("0", "0"), False), ("x", ("E", "H"), True)])
def test_product_solve_matches_oracle_host_emulated(sweep, bc, back):
    """ModeFullVector.solve end to end on the CPU (factor, Krylov-Schur,
    ordering, normalisation, field access, interpolation) with the device
    calls emulated from the oracle's A and B: the oracle's modes."""
    torch = pytest.importorskip("torch")
    from emopt_b200.grid import ConstantMaterial3D
    from emopt_b200.misc import DomainCoordinates
    from emopt_b200.modes import ModeFullVector
    M, N, n0, k = 8, 11, 3.3, 3
    A, B = O.build_system(_layered(M, N, 1), M, N, 0.05, 0.06, WL, bc=bc, backwards=back)
    dom = DomainCoordinates.from_indices(0, N, 0, M, 0, 1, 0.05, 0.06, 0.05)
    m = ModeFullVector(WL, ConstantMaterial3D(2.0), ConstantMaterial3D(1.0), dom, n0=n0, neigs=k,
                       backwards=back, device=0, sweep=sweep)
    m.bc = list(bc)
    _emulate_device(m, A, B, M, N)
    m._planes = []                                   # sampled planes are not used by the emulation
    m.solve()
    neff, V = O.solve(A, B, n0, k)
    np.testing.assert_allclose(m.neff, neff, rtol=1e-10)
    for q in range(k):
        got = np.concatenate([m.get_field(q, c, permute=False, squeeze=True).ravel() for c in O.COMPONENTS])
        assert np.linalg.norm(got) == pytest.approx(1.0, abs=1e-12)
        c = np.vdot(got, V[q])
        c /= abs(c)
        assert np.linalg.norm(got * c - V[q]) < 1e-8
        for comp in O.COMPONENTS:
            want = O.get_field_interp(V[q], comp, M, N, "z", bc)
            assert np.linalg.norm(m.get_field_interp(q, comp, squeeze=True) * c - want) < 1e-8


@pytest.mark.parametrize("k,m", [(1, 16), (4, 24), (6, 14)])
def test_krylov_schur_finds_largest_modulus_eigenpairs(k, m):
    """The product's Krylov-Schur iteration (run on the CPU with a dense
    operator) returns the k eigenvalues of largest modulus of a non-normal
    matrix with a slowly decaying spectrum -- restarts included -- and their
    eigenvectors."""
    torch = pytest.importorskip("torch")
    from emopt_b200.modes import _krylov_schur
    rng = np.random.default_rng(k)
    n = 300
    lam = (0.97 ** np.arange(n)) * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = X @ np.diag(lam) @ np.linalg.inv(X)
    At = torch.as_tensor(A)
    apply = lambda v, out: out.copy_(At @ v)
    v0 = torch.as_tensor(rng.standard_normal(n) + 0j)
    theta, V, nconv, napply = _krylov_schur(apply, n, k, m, 1e-12, 200, v0, torch.device("cpu"))
    assert nconv == k and napply > m            # it had to restart
    want = lam[np.argsort(-np.abs(lam))[:k]]
    np.testing.assert_allclose(np.sort_complex(theta), np.sort_complex(want), rtol=1e-9)
    for q in range(k):
        x = V[q].numpy()
        assert np.linalg.norm(A @ x - theta[q] * x) < 1e-8 * np.linalg.norm(x) * abs(theta[q])


def test_product_component_energy_and_mode_number():
    """component_energy: the energy fractions eps|E|^2, mu|H|^2 of a mode's
    raw components (emopt/modes.py:2054-2097); mode numbering is a stub in the
    reference and raises here."""
    torch = pytest.importorskip("torch")
    from emopt_b200.grid import ConstantMaterial3D
    from emopt_b200.misc import DomainCoordinates
    from emopt_b200.modes import ModeFullVector
    dom = DomainCoordinates.from_indices(4, 5, 0, 7, 0, 6, 0.05, 0.05, 0.05)
    m = ModeFullVector(WL, ConstantMaterial3D(4.0), ConstantMaterial3D(1.0), dom, device=0)
    rng = np.random.default_rng(9)
    vec = rng.standard_normal(6 * 6 * 7) + 1j * rng.standard_normal(6 * 6 * 7)
    m._x = torch.as_tensor(vec.reshape(1, 6, 6, 7))
    W = m.component_energy(0)
    raw = [np.sum(np.abs(vec.reshape(6, 42)[q]) ** 2) * (4.0 if q < 3 else 1.0) for q in range(6)]
    want = [raw[O.COMPONENTS.index(O._PERMUTE["x"][c])] / sum(raw) for c in O.COMPONENTS]
    np.testing.assert_allclose(W, want, rtol=1e-12)
    assert sum(W) == pytest.approx(1.0)
    with pytest.raises(NotImplementedError):
        m.find_mode_index(0, 0)
