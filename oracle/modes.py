"""CPU restatement of the reference's full-vector mode solver (test oracle).

Test infrastructure only: the GPU mode solver (emopt_b200/modes.py,
emopt_b200/csrc/modes.cu) is checked against this.  It restates
``ModeFullVector`` (emopt/modes.py:1099-2298):

* ``build_system``: the matrices A and B of ``A x = n B x`` row by row as
  ``ModeFullVector.build`` assembles them (emopt/modes.py:1278-1588), the
  boundary rows included, with the assignments in the reference's order;
* ``solve``: the eigenpairs closest to the target ``n0`` -- the reference runs
  SLEPc with a shift-and-invert transform about ``n0`` and MUMPS LU
  (emopt/modes.py:1188-1216, 1590-1627); here SuperLU factors ``A - n0 B``
  and ARPACK finds the largest eigenvalues theta of ``(A - n0 B)^-1 B``, so
  ``n = n0 + 1/theta``, closest first;
* ``get_field``, ``get_field_interp`` and ``get_source``
  (emopt/modes.py:1629-2298).

Eigenvectors are normalised to unit 2-norm with the entry of largest modulus
real and positive (the reference's phase is whatever SLEPc's start vector
gives; any phase is an eigenvector).

Parity unpinned against the reference itself: petsc4py and slepc4py are not
in this image, so ``ModeFullVector`` cannot run here.  The assembly is pinned
by a known answer instead: for a uniform medium in the box every nonzero
eigenvalue satisfies the discrete dispersion relation of the compressed Yee
grid, n^2 = eps mu - (2R/dx sin(p pi/2N))^2 - (2R/dy sin(q pi/2M))^2, with
the half-shifted wavenumbers sin((p + 1/2) pi/2N) for the second parity
along an axis with the 'E' symmetry letter (tests/test_modes.py); the
shift-invert solve is pinned by a dense eigen-solve of the same pencil.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def plane_orientation(shape):
    """(ndir, M, N) of a plane domain of shape (Nz, Ny, Nx)
    (emopt/modes.py:1165-1187)."""
    Nz, Ny, Nx = shape
    if Nx == 1:
        return "x", Nz, Ny
    if Ny == 1:
        return "y", Nz, Nx
    if Nz == 1:
        return "z", Ny, Nx
    raise AttributeError("3D domains are not supported for 2D mode calculations!")


def material_planes(eps_fn, mu_fn, ndir, M, N, k0, j0, i0):
    """The six (M, N) coefficient planes eps_x, eps_y, eps_z, mu_x, mu_y,
    mu_z at the positions of ``ModeFullVector.build``'s lambdas for a
    Material3D (emopt/modes.py:1327-1352); ``eps_fn(k, j, i)`` and
    ``mu_fn(k, j, i)`` take fractional grid indices (numpy broadcast)."""
    y, x = np.meshgrid(np.arange(M, dtype=float), np.arange(N, dtype=float), indexing="ij")
    if ndir == "x":
        at = {"ex": (k0 + 0 * x, j0 + x + 0.5, i0 + y - 0.5), "ey": (k0 + 0 * x, j0 + x, i0 + y),
              "ez": (k0 + 0 * x, j0 + x, i0 + y - 0.5), "mx": (k0 + 0 * x, j0 + x, i0 + y),
              "my": (k0 + 0 * x, j0 + x + 0.5, i0 + y - 0.5), "mz": (k0 + 0 * x, j0 + x + 0.5, i0 + y)}
    elif ndir == "y":
        at = {"ex": (k0 + y, j0 + 0 * x, i0 + x), "ey": (k0 + y + 0.5, j0 + 0 * x, i0 + x - 0.5),
              "ez": (k0 + y, j0 + 0 * x, i0 + x - 0.5), "mx": (k0 + y + 0.5, j0 + 0 * x, i0 + x - 0.5),
              "my": (k0 + y, j0 + 0 * x, i0 + x), "mz": (k0 + y + 0.5, j0 + 0 * x, i0 + x)}
    else:
        c = (k0 + x, j0 + y, i0 + 0 * x)
        at = {q: c for q in ("ex", "ey", "ez", "mx", "my", "mz")}
    out = []
    for q in ("ex", "ey", "ez"):
        out.append(np.asarray(eps_fn(*at[q]), dtype=np.complex128) * np.ones((M, N)))
    for q in ("mx", "my", "mz"):
        out.append(np.asarray(mu_fn(*at[q]), dtype=np.complex128) * np.ones((M, N)))
    return out


def build_system(planes, M, N, dx, dy, wavelength, bc=("0", "0"), backwards=False):
    """A and B (scipy CSR, 6MN square) of emopt/modes.py:1278-1588.  ``dx``,
    ``dy``: the plane's grid spacings along its first and second axes;
    ``planes``: the six coefficient planes of :func:`material_planes`."""
    R = wavelength / (2 * np.pi)
    odx, ody = R / dx, R / dy
    d = -1.0 if backwards else 1.0
    ex, ey, ez, mx, my, mz = planes
    MN = M * N
    Ar, Ac, Av, Br, Bc, Bv = [], [], [], [], [], []
    for I in range(6 * MN):
        blk, rem = divmod(I, MN)
        y, x = divmod(rem, N)
        row = {I: 0.0}                       # the explicit diagonal entry
        brow = {}
        if blk == 0:
            Hz1, Hz0, Ex, Hy = 5 * MN + y * N + x, 5 * MN + (y - 1) * N + x, y * N + x, 4 * MN + y * N + x
            if y > 0:
                row[Hz0] = -ody
            row[Hz1] = ody
            row[Ex] = 1j * ex[y, x]
            brow[Hy] = 1j * d
            if y == 0:
                if bc[1] == "0":
                    row[Ex] = 0
                elif bc[1] == "E":
                    row[Hz1] = 2 * ody
                elif bc[1] == "H":
                    row[Hz1] = 0
                    row[Ex] = 0
        elif blk == 1:
            Hz1, Hz0, Ey, Hx = 5 * MN + y * N + x, 5 * MN + y * N + x - 1, MN + y * N + x, 3 * MN + y * N + x
            if x > 0:
                row[Hz0] = odx
            row[Hz1] = -odx
            row[Ey] = 1j * ey[y, x]
            brow[Hx] = -1j * d
            if x == 0:
                if bc[0] == "0":
                    row[Ey] = 0
                elif bc[0] == "E":
                    row[Hz1] = -2 * odx
                elif bc[0] == "H":
                    row[Hz1] = 0
        elif blk == 2:
            Ey0, Ey1 = MN + y * N + x, MN + y * N + x + 1
            Ex0, Ex1 = y * N + x, (y + 1) * N + x
            Hz = 5 * MN + y * N + x
            row[Ey0] = -odx
            if x < N - 1:
                row[Ey1] = odx
            row[Ex0] = ody
            if y < M - 1:
                row[Ex1] = -ody
            row[Hz] = -1j * mz[y, x]
            if x == 0 and bc[0] == "0":
                row[Ey0] = 0
            if y == 0 and bc[1] in ("0", "H"):
                row[Ex0] = 0
        elif blk == 3:
            Ez0, Ez1 = 2 * MN + y * N + x, 2 * MN + (y + 1) * N + x
            Hx, Ey = 3 * MN + y * N + x, MN + y * N + x
            row[Ez0] = -ody
            if y < M - 1:
                row[Ez1] = ody
            row[Hx] = -1j * mx[y, x]
            brow[Ey] = 1j * d
            if x == 0 and bc[0] == "0":
                row[Hx] = 0
            if y == 0 and bc[1] in ("0", "H"):
                row[Ez0] = 0
        elif blk == 4:
            Ez0, Ez1 = 2 * MN + y * N + x, 2 * MN + y * N + x + 1
            Hy, Ex = 4 * MN + y * N + x, y * N + x
            row[Ez0] = odx
            if x < N - 1:
                row[Ez1] = -odx
            row[Hy] = -1j * my[y, x]
            brow[Ex] = -1j * d
            if x == 0 and bc[0] == "0":
                row[Ez0] = 0
            if y == 0 and bc[1] in ("0", "H"):
                row[Hy] = 0
        else:
            Hy0, Hy1 = 4 * MN + y * N + x - 1, 4 * MN + y * N + x
            Hx0, Hx1 = 3 * MN + (y - 1) * N + x, 3 * MN + y * N + x
            Ez = 2 * MN + y * N + x
            if x > 0:
                row[Hy0] = -odx
            row[Hy1] = odx
            if y > 0:
                row[Hx0] = ody
            row[Hx1] = -ody
            row[Ez] = 1j * ez[y, x]
            if x == 0:
                if bc[0] == "0":
                    row[Hx1] = 0
                    if y > 0:
                        row[Hx0] = 0
                elif bc[0] == "E":
                    row[Hy1] = 2 * odx
                elif bc[0] == "H":
                    row[Hy1] = 0
            if y == 0:
                if bc[1] == "0":
                    row[Hy1] = 0
                    if x > 0:
                        row[Hy0] = 0
                elif bc[1] == "E":
                    row[Hx1] = -2 * ody
                elif bc[1] == "H":
                    row[Hx1] = 0
                    row[Hy1] = 0
                    if x > 0:
                        row[Hy0] = 0
        for c, v in row.items():
            Ar.append(I); Ac.append(c); Av.append(v)
        for c, v in brow.items():
            Br.append(I); Bc.append(c); Bv.append(v)
    n = 6 * MN
    A = sp.csr_matrix((np.asarray(Av, dtype=np.complex128), (Ar, Ac)), shape=(n, n))
    B = sp.csr_matrix((np.asarray(Bv, dtype=np.complex128), (Br, Bc)), shape=(n, n))
    return A, B


def _normalise(v):
    v = v / np.linalg.norm(v)
    q = int(np.argmax(np.abs(v)))
    return v * (abs(v[q]) / v[q])


def solve(A, B, n0, neigs, v0=None):
    """The ``neigs`` eigenpairs of ``A x = n B x`` closest to ``n0``, closest
    first: (neff[neigs], vectors[neigs, 6MN])."""
    lu = spla.splu((A - n0 * B).tocsc())
    n = A.shape[0]
    op = spla.LinearOperator((n, n), matvec=lambda v: lu.solve(B @ v), dtype=np.complex128)
    if v0 is None:
        v0 = np.random.default_rng(0).standard_normal(n) + 0j
    theta, V = spla.eigs(op, k=neigs, which="LM", v0=v0, tol=0)
    order = np.argsort(-np.abs(theta))
    neff = n0 + 1.0 / theta[order]
    return neff, np.stack([_normalise(V[:, q]) for q in order])


def solve_dense(A, B, n0, neigs):
    """The same eigenpairs from a dense QZ solve of the pencil (small grids)."""
    w, V = sla.eig(A.toarray(), B.toarray())
    ok = np.isfinite(w)
    w, V = w[ok], V[:, ok]
    order = np.argsort(np.abs(w - n0))[:neigs]
    return w[order], np.stack([_normalise(V[:, q]) for q in order])


_PERMUTE = {"x": {"Ex": "Ez", "Ey": "Ex", "Ez": "Ey", "Hx": "Hz", "Hy": "Hx", "Hz": "Hy"},
            "y": {"Ex": "Ey", "Ey": "Ez", "Ez": "Ex", "Hx": "Hy", "Hy": "Hz", "Hz": "Hx"},
            "z": {c: c for c in COMPONENTS}}


def get_field(vec, component, M, N, ndir, permute=True):
    """(M, N) plane of one component (emopt/modes.py:1629-1787)."""
    if permute:
        component = _PERMUTE[ndir][component]
    q = COMPONENTS.index(component)
    return vec[q * M * N:(q + 1) * M * N].reshape(M, N)


def _ghost_x(f, bc0):
    if bc0 == "E":
        f[:, 0] = -1 * f[:, 1]
    elif bc0 == "H":
        f[:, 0] = f[:, 1]


def _ghost_y(f, bc1):
    if bc1 == "E":
        f[0, :] = -1 * f[1, :]
    elif bc1 == "H":
        f[0, :] = f[1, :]


def get_field_interp(vec, component, M, N, ndir, bc):
    """(M, N) plane of one component averaged onto the plane's Ez-equivalent
    points (emopt/modes.py:1789-2052).  Two cases of the reference fail
    (the y-normal Ex reads an undefined name, the y-normal Hy returns the
    padded array); they are restated here as the evident intent: the raw
    field."""
    f = np.pad(get_field(vec, component, M, N, ndir), 1, "constant", constant_values=0)
    c = _PERMUTE[ndir][component]
    if ndir == "x":
        if c in ("Ex", "Hy"):
            g = np.copy(f)
            _ghost_x(f, bc[0])
            g[:, 1:] += f[:, 0:-1]
            g[0:-1, 1:] += f[1:, 0:-1]
            g[0:-1, :] += f[1:, :]
            return g[1:-1, 1:-1] / 4.0
        if c in ("Ey", "Hx"):
            return f[1:-1, 1:-1]
        if c == "Ez":
            g = np.copy(f)
            g[0:-1, :] += g[1:, :]
            return g[1:-1, 1:-1] / 2.0
        g = np.copy(f)                                    # Hz
        _ghost_x(f, bc[0])
        g[:, 1:] += f[:, 0:-1]
        return g[1:-1, 1:-1] / 2.0
    if ndir == "y":
        if c in ("Ex", "Hy"):
            return f[1:-1, 1:-1]
        if c in ("Ey", "Hx"):
            g = np.copy(f)
            _ghost_y(f, bc[1])
            g[:, 0:-1] += g[:, 1:]
            g[1:, :] += g[0:-1, :]
            g[1:, 0:-1] += g[0:-1, 1:]
            return g[1:-1, 1:-1] / 4.0
        if c == "Ez":
            g = np.copy(f)
            g[:, 0:-1] += g[:, 1:]
            return g[1:-1, 1:-1] / 2.0
        g = np.copy(f)                                    # Hz
        _ghost_y(f, bc[1])
        g[1:, :] += f[0:-1, :]
        return g[1:-1, 1:-1] / 2.0
    if c in ("Ex", "Hy"):
        g = np.copy(f)
        _ghost_x(f, bc[0])
        g[:, 1:] += f[:, 0:-1]
        return g[1:-1, 1:-1] / 2.0
    if c in ("Ey", "Hx"):
        g = np.copy(f)
        _ghost_y(f, bc[1])
        g[1:, :] += f[0:-1, :]
        return g[1:-1, 1:-1] / 2.0
    if c == "Ez":
        return f[1:-1, 1:-1]
    g = np.copy(f)                                        # Hz
    _ghost_y(f, bc[1])
    _ghost_x(f, bc[0])
    g[:, 1:] += f[:, 0:-1]
    g[1:, :] += f[0:-1, :]
    g[1:, 1:] += f[0:-1, 0:-1]
    return g[1:-1, 1:-1] / 4.0


def get_source(vec, neff, M, N, ndir, bc, wavelength, dx, dy, dz, eps_plane, mu_plane_05, mu_plane_50,
               backwards=False):
    """(Jx, Jy, Jz, Mx, My, Mz) planes of the mode (emopt/modes.py:2144-2296),
    in the caller's component order.  ``eps_plane``: eps at the plane's cell
    positions; ``mu_plane_05`` / ``mu_plane_50``: mu shifted by half a cell
    along the plane's second / first axis (the reference's get_mu(0, 0.5) and
    get_mu(0.5, 0))."""
    R = wavelength / (2 * np.pi)
    d = -1.0 if backwards else 1.0
    if ndir == "x":
        mydx, mydy, mydz = dy, dz, dx
    elif ndir == "y":
        mydx, mydy, mydz = dz, dx, dy
    else:
        mydx, mydy, mydz = dx, dy, dz
    dxn, dyn, dzn = mydx / R, mydy / R, mydz / R
    ekz = np.exp(1j * d * neff * dzn / 2)
    F = {c: get_field(vec, c, M, N, ndir, permute=False) for c in COMPONENTS}
    S = 0.5 * mydx * mydy * np.sum(F["Ex"] * np.conj(F["Hy"]) - F["Ey"] * np.conj(F["Hx"]))
    F = {c: v / np.sqrt(S) for c, v in F.items()}
    Jx, Jy, Jz, Mx, My, Mz = (np.zeros((M, N), dtype=np.complex128) for _ in range(6))
    Ex = np.pad(F["Ex"], 1)
    My += Ex[1:-1, 1:-1] * ekz / dzn
    Ey = np.pad(F["Ey"], 1)
    Mx += -Ey[1:-1, 1:-1] * ekz / dzn
    Ez = np.pad(F["Ez"], 1)
    Jz += 1j * eps_plane * Ez[1:-1, 1:-1]
    Mx += (Ez[2:, 1:-1] - Ez[1:-1, 1:-1]) / dyn
    My += -1 * (Ez[1:-1, 2:] - Ez[1:-1, 1:-1]) / dxn
    Hx = np.pad(F["Hx"], 1)
    if bc[1] == "E":
        Hx[0, :] = -1 * Hx[1, :]
    elif bc[1] == "H":
        Hx[0, :] = Hx[1, :]
    Jy += Hx[1:-1, 1:-1] / dzn
    Jz += -1 * (Hx[1:-1, 1:-1] - Hx[0:-2, 1:-1]) / dyn
    Mx += -1j * mu_plane_05 * Hx[1:-1, 1:-1]
    Hy = np.pad(F["Hy"], 1)
    if bc[0] == "E":
        Hy[:, 0] = -1 * Hy[:, 1]
    elif bc[0] == "H":
        Hy[:, 0] = Hy[:, 1]
    Jx += -Hy[1:-1, 1:-1] / dzn
    Jz += (Hy[1:-1, 1:-1] - Hy[1:-1, 0:-2]) / dxn
    My += -1j * mu_plane_50 * Hy[1:-1, 1:-1]
    if ndir == "x":
        return Jz, Jx, Jy, Mz, Mx, My
    if ndir == "y":
        return Jy, Jz, Jx, My, Mz, Mx
    return Jx, Jy, Jz, Mx, My, Mz


def discrete_box_spectrum(eps, mu, M, N, dx, dy, wavelength, bc=("0", "0")):
    """n^2 allowed for a uniform medium in the box of the compressed Yee grid:
    eps mu - kx^2 - ky^2 with kx = 2R/dx sin(p pi/2N), ky = 2R/dy sin(q pi/2M)
    (p = 0..N-1, q = 0..M-1); where an axis has the 'E' symmetry letter, the
    modes of the other parity take the half-shifted wavenumbers
    sin((p + 1/2) pi/2N) along it, so the spectrum is the union of both
    families.  Flattened."""
    R = wavelength / (2 * np.pi)

    def k(n, d, half):
        return 2 * R / d * np.sin((np.arange(n) + (0.5 if half else 0.0)) * np.pi / (2 * n))

    fam = [(k(N, dx, False), k(M, dy, False)), (k(N, dx, bc[0] == "E"), k(M, dy, bc[1] == "E"))]
    return np.concatenate([(eps * mu - kx[None, :] ** 2 - ky[:, None] ** 2).ravel() for kx, ky in fam])
