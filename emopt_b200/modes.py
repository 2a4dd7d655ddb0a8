"""Full-vector waveguide modes on the GPU: ``ModeFullVector`` of the reference
(emopt/modes.py:1099-2298) with the same constructor, properties and
methods, so that a mode source or a mode-match field comes from the device.

The reference assembles the 6 M N x 6 M N system A x = n B x of the plane's
six field components (emopt/modes.py:1278-1588) and solves it with SLEPc,
shift-and-invert about the target ``n0``, factoring ``A - n0 B`` with MUMPS.
Here the same rows are assembled on the GPU into a block-tridiagonal matrix
(the plane cut into lines; ``emopt_b200/csrc/modes.cu``), the Schur
complements of its block LU are inverted on the device, and a Krylov-Schur
iteration (Stewart, SIAM J. Matrix Anal. Appl. 23 (2001) 601-614) on
``(A - n0 B)^-1 B`` finds the eigenvalues theta of largest modulus, i.e. the
effective indices ``n = n0 + 1/theta`` closest to ``n0``, closest first (the
order SLEPc returns with a target).  Every application of the operator is a
forward and a backward sweep of dense matrix-vector products over the
inverted blocks, HBM-bound.

Eigenvectors are normalised to unit 2-norm with their entry of largest
modulus real and positive (SLEPc's phase follows its random start vector;
any phase is a valid mode).
"""
from __future__ import annotations

import ctypes

import numpy as np
import scipy.linalg as sla

from . import fdtd_ctypes as _ct
from .fdtd_ctypes import libFDTD
from .grid import Material3D
from .misc import warning_message

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_PERMUTE = {"x": {"Ex": "Ez", "Ey": "Ex", "Ez": "Ey", "Hx": "Hz", "Hy": "Hx", "Hz": "Hy"},
            "y": {"Ex": "Ey", "Ey": "Ez", "Ez": "Ex", "Hx": "Hy", "Hy": "Hz", "Hz": "Hx"},
            "z": {c: c for c in COMPONENTS}}
_BCS = ("0", "M", "E", "H", "P", "EM", "HM")


def _check(rc, what):
    if rc != _ct.FDTD_OK:
        raise _ct.FDTDError("%s: %s" % (what, libFDTD.FDTD_mode_last_error().decode()))


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class ModeFullVector:
    """Modes of a 2D slice of a 3D structure (emopt/modes.py:1099-1276).

    Parameters as the reference: ``wavelength``, ``eps`` and ``mu``
    (Material3D), ``domain`` (a plane: one of its three sizes is 1), ``n0``
    (the effective index the modes are sought near), ``neigs``,
    ``backwards``, ``verbose``.  Additions: ``device`` (CUDA device index)
    and ``sweep`` ('y' or 'x': the lines of the block-tridiagonal solve; by
    default the shorter of the plane's two directions).
    """

    def __init__(self, wavelength, eps, mu, domain, n0=1.0, neigs=1, backwards=False, verbose=True,
                 device=None, sweep=None):
        import torch
        self._neff = np.zeros(neigs, dtype=np.complex128)
        self.n0 = n0
        self.neigs = neigs
        self.wavelength = wavelength
        self.eps, self.mu, self.domain = eps, mu, domain
        self._fshape = domain.shape
        if domain.Nx == 1:
            self.ndir, self._M, self._N, self.dx, self.dy = "x", domain.Nz, domain.Ny, domain.dy, domain.dz
        elif domain.Ny == 1:
            self.ndir, self._M, self._N, self.dx, self.dy = "y", domain.Nz, domain.Nx, domain.dx, domain.dz
        elif domain.Nz == 1:
            self.ndir, self._M, self._N, self.dx, self.dy = "z", domain.Ny, domain.Nx, domain.dx, domain.dy
        else:
            raise AttributeError("3D domains are not supported for 2D mode calculations!")
        self.verbose = verbose
        self._dir = -1.0 if backwards else 1.0
        self.R = self.wavelength / (2 * np.pi)
        self._bc = ["0", "0"]
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._dev = torch.device("cuda", self.device)
        if sweep is None:
            sweep = "y" if self._N <= self._M else "x"
        if sweep not in ("x", "y"):
            raise ValueError("sweep must be 'x' or 'y'")
        self._lines = _ct.ModeLines(self._M, self._N, 1 if sweep == "y" else 0)
        self._planes = None
        self._x = None
        self.stats = {}

    # ------------------------------------------------------------ attributes
    @property
    def neff(self):
        return self._neff

    @neff.setter
    def neff(self, value):
        warning_message("neff cannot be set by the user.", module="emopt_b200.modes")

    @property
    def bc(self):
        return self._bc

    @bc.setter
    def bc(self, bc):
        for b in bc[:2]:
            if b not in _BCS:
                raise ValueError("Boundary condition type '%s' not found. Use 0, M, E, H, P, EM, HM." % b)
        self._bc = list(bc)

    def _bc_code(self):
        """The two boundary letters the kernels test ('0', 'E', 'H'; the other
        types change no row of the reference's system)."""
        return "".join(b if b in ("0", "E", "H") else "-" for b in self._bc[:2]).encode()

    # --------------------------------------------------------------- build
    def _values(self, mat, k1, k2, j1, j2, i1, i2, sx=0.0, sy=0.0, sz=0.0):
        import torch
        try:
            v = mat.get_values(k1, k2, j1, j2, i1, i2, sx, sy, sz, device=self._dev)
        except TypeError:
            v = mat.get_values(k1, k2, j1, j2, i1, i2, sx, sy, sz)
        return torch.as_tensor(v, dtype=torch.complex128, device=self._dev)

    def _material_planes(self):
        """eps_x, eps_y, eps_z, mu_x, mu_y, mu_z as ModeFullVector.build samples
        them for a Material3D (emopt/modes.py:1327-1352), [M][N] each."""
        if not isinstance(self.eps, Material3D) or not isinstance(self.mu, Material3D):
            raise TypeError("the GPU mode solver takes Material3D slices")
        d, M, N = self.domain, self._M, self._N
        k0, j0, i0 = d.k1, d.j1, d.i1
        out = []
        if self.ndir == "x":
            offs = [(self.eps, 0.5, -0.5), (self.eps, 0.0, 0.0), (self.eps, 0.0, -0.5),
                    (self.mu, 0.0, 0.0), (self.mu, 0.5, -0.5), (self.mu, 0.5, 0.0)]
            for mat, sy, sz in offs:
                out.append(self._values(mat, k0, k0 + 1, j0, j0 + N, i0, i0 + M, 0.0, sy, sz)[:, :, 0])
        elif self.ndir == "y":
            # the reference's lambdas put the plane's x along z and its y along x
            offs = [(self.eps, 0.0, 0.0), (self.eps, 0.5, -0.5), (self.eps, 0.0, -0.5),
                    (self.mu, 0.5, -0.5), (self.mu, 0.0, 0.0), (self.mu, 0.5, 0.0)]
            for mat, sx, sz in offs:
                out.append(self._values(mat, k0, k0 + M, j0, j0 + 1, i0, i0 + N, sx, 0.0, sz)[:, 0, :].T)
        else:
            for mat in (self.eps,) * 3 + (self.mu,) * 3:
                out.append(self._values(mat, k0, k0 + N, j0, j0 + M, i0, i0 + 1)[0])
        return [p.contiguous() for p in out]

    def build(self):
        """Sample the materials on the plane (the reference assembles A and B
        here; the GPU blocks depend on the target and are assembled in
        :meth:`solve`)."""
        self._planes = self._material_planes()

    # --------------------------------------------------------------- solve
    def _factor(self, sigma):
        """Assemble A - sigma B by lines and factor it by block cyclic
        reduction: at every level the odd lines of the remaining ones are
        eliminated (their blocks inverted in one batched call), which leaves
        dense corrections on the rows of the even lines that couple to them.
        Every row of a line couples to at most one unknown of the line before
        (rows P to columns Qp) and one of the line after (rows N to columns
        Qn), so all couplings stay 2L x 2L blocks Lc (P x Qp) and Uc (N x Qn)."""
        import torch
        g, dev = self._lines, self._dev
        L = self._N if g.sweep_y else self._M
        NL = self._M if g.sweep_y else self._N
        nb = 6 * L
        self._L, self._NL, self._nb = L, NL, nb
        c128 = torch.complex128
        D, pcol, pval, ncol, nval = self._assemble(sigma)
        # the coupling rows and columns, the same on every line that has the neighbour
        pc, nc = pcol.cpu().numpy(), ncol.cpu().numpy()
        P = np.flatnonzero(pc[1] >= 0) if NL > 1 else np.zeros(0, dtype=np.int64)
        Nr = np.flatnonzero(nc[0] >= 0) if NL > 1 else np.zeros(0, dtype=np.int64)
        Qp, Qn = (pc[1][P], nc[0][Nr]) if NL > 1 else (P, Nr)
        if NL > 1:
            ok = bool((pc[0] < 0).all() and (nc[-1] < 0).all())
            ok &= bool(((pc[1:] >= 0) == (pc[1] >= 0)).all() and (pc[1:, P] == Qp).all())
            ok &= bool(((nc[:-1] >= 0) == (nc[0] >= 0)).all() and (nc[:-1, Nr] == Qn).all())
            ok &= len(np.unique(Qp)) == len(Qp) and len(np.unique(Qn)) == len(Qn)
            if not ok:
                raise RuntimeError("line couplings differ from line to line")
        lt = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64), device=dev)
        P_t, N_t, Qp_t, Qn_t = lt(P), lt(Nr), lt(Qp), lt(Qn)
        nP, nN = len(P), len(Nr)
        Lc = torch.zeros((NL, nP, nP), dtype=c128, device=dev)
        Uc = torch.zeros((NL, nN, nN), dtype=c128, device=dev)
        if NL > 1:
            ar, an = torch.arange(nP, device=dev), torch.arange(nN, device=dev)
            Lc[1:, ar, ar] = pval[1:][:, P_t]
            Uc[:-1, an, an] = nval[:-1][:, N_t]

        def inv_into(lines):
            W, info = torch.linalg.inv_ex(D[lines])
            if bool((info != 0).any()):
                raise RuntimeError("A - n0 B is singular on a line: move n0 off the eigenvalue")
            D[lines] = W

        levels = []
        act = list(range(NL))
        while len(act) > 1:
            odd, even = act[1::2], act[0::2]
            e1, o1 = even[1:], odd[:len(even) - 1]          # even[j] with the odd line before it
            e2, o2 = even[:len(odd)], odd                    # even[j] with the odd line after it
            has_next = [j for j in range(len(odd)) if j + 1 < len(even)]
            i32 = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int32), device=dev)
            odd_n, nxt = [odd[j] for j in has_next], [even[j + 1] for j in has_next]
            lev = {"odd": lt(odd), "odd32": i32(odd), "e1": lt(e1), "o1": lt(o1), "e2": lt(e2), "o2": lt(o2),
                   "e1_32": i32(e1), "o1_32": i32(o1), "e2_32": i32(e2), "o2_32": i32(o2),
                   "Lc_e1": Lc[lt(e1)].clone(), "Uc_e2": Uc[lt(e2)].clone(),
                   "prev32": i32(even[:len(odd)]), "Lc_odd": Lc[lt(odd)].clone(),
                   "odd_n32": i32(odd_n), "next32": i32(nxt), "Uc_odd_n": Uc[lt(odd_n)].clone()}
            inv_into(lev["odd"])
            newLc = newUc = None
            # the corrections land on distinct (line, row, column) entries, so
            # a gather, a subtraction and a scatter apply them (no sort)
            if e1:
                Wq = D[lev["o1"]][:, Qp_t]
                idx = (lev["e1"][:, None, None], P_t[None, :, None], Qn_t[None, None, :])
                D[idx] = D[idx] - Lc[lev["e1"]] @ Wq[:, :, N_t] @ Uc[lev["o1"]]
                newLc = -(Lc[lev["e1"]] @ Wq[:, :, P_t] @ Lc[lev["o1"]])
            if e2:
                Wq = D[lev["o2"]][:, Qn_t]
                idx = (lev["e2"][:, None, None], N_t[None, :, None], Qp_t[None, None, :])
                D[idx] = D[idx] - Uc[lev["e2"]] @ Wq[:, :, P_t] @ Lc[lev["o2"]]
                newUc = -(Uc[lev["e2"]] @ Wq[:, :, N_t] @ Uc[lev["o2"]])
            Lc[even[0]] = 0
            if newLc is not None:
                Lc[lev["e1"]] = newLc
            if newUc is not None:
                Uc[lev["e2"]] = newUc
            if len(even) > len(odd):
                Uc[even[-1]] = 0
            levels.append(lev)
            act = even
        self._top = torch.as_tensor(act, dtype=torch.int32, device=dev)
        inv_into(lt(act))
        self._W, self._levels = D, levels
        self._P, self._Nr, self._Qp, self._Qn = P_t, N_t, Qp_t, Qn_t
        self._P32, self._N32, self._Qp32, self._Qn32 = (t.to(torch.int32) for t in (P_t, N_t, Qp_t, Qn_t))
        self._QpQn32 = torch.cat([Qp_t, Qn_t]).unique().to(torch.int32)
        self._b = torch.empty((NL, nb), dtype=c128, device=dev)
        self._y = torch.empty((NL, nb), dtype=c128, device=dev)
        self._xs = torch.empty((NL, nb), dtype=c128, device=dev)
        self._corr = torch.empty((NL, nb), dtype=c128, device=dev)
        self.stats_levels = len(levels)

    def _assemble(self, sigma):
        """Blocks D_l of A - sigma B and the couplings to the neighbouring
        lines, on the device (FDTD_mode_assemble)."""
        import torch
        g, dev, NL, nb = self._lines, self._dev, self._NL, self._nb
        c128 = torch.complex128
        D = torch.empty((NL, nb, nb), dtype=c128, device=dev)
        pcol = torch.empty((NL, nb), dtype=torch.int32, device=dev)
        ncol = torch.empty((NL, nb), dtype=torch.int32, device=dev)
        pval = torch.empty((NL, nb), dtype=c128, device=dev)
        nval = torch.empty((NL, nb), dtype=c128, device=dev)
        planes = (ctypes.c_void_p * 6)(*[p.data_ptr() for p in self._planes])
        stream = torch.cuda.current_stream(dev).cuda_stream
        odx, ody = self.R / self.dx, self.R / self.dy
        _check(libFDTD.FDTD_mode_assemble(ctypes.byref(g), self.device, stream, odx, ody, self._dir,
                                          float(np.real(sigma)), float(np.imag(sigma)), planes,
                                          self._bc_code(), _ptr(D), _ptr(pcol), _ptr(pval), _ptr(ncol),
                                          _ptr(nval)), "FDTD_mode_assemble")
        return D, pcol, pval, ncol, nval

    def _bmul(self, v, out):
        import torch
        stream = torch.cuda.current_stream(self._dev).cuda_stream
        _check(libFDTD.FDTD_mode_bmul(ctypes.byref(self._lines), self.device, stream, self._dir, _ptr(v),
                                      _ptr(out)), "FDTD_mode_bmul")

    def _gemv(self, lines32, rows32, rhs, corr, out):
        import torch
        stream = torch.cuda.current_stream(self._dev).cuda_stream
        nrows = int(rows32.numel()) if rows32 is not None else self._nb
        _check(libFDTD.FDTD_mode_lines_gemv(self._nb, self.device, stream, _ptr(self._W), _ptr(lines32),
                                            int(lines32.numel()), _ptr(rows32) if rows32 is not None else None,
                                            nrows, _ptr(rhs), _ptr(corr) if corr is not None else None,
                                            _ptr(out)), "FDTD_mode_lines_gemv")

    def _couple(self, lines32, nbrs32, C, rows32, cols32, src, dst, sign):
        import torch
        stream = torch.cuda.current_stream(self._dev).cuda_stream
        _check(libFDTD.FDTD_mode_couple(self._nb, self.device, stream, int(lines32.numel()), int(rows32.numel()),
                                        int(cols32.numel()), _ptr(C), _ptr(lines32), _ptr(nbrs32), _ptr(rows32),
                                        _ptr(cols32), _ptr(src), _ptr(dst), float(sign)), "FDTD_mode_couple")

    def _apply_direct(self, v, out):
        """out = (A - n0 B)^-1 B v: reduction over the levels, the top line,
        back-substitution over the levels."""
        b, y, x, corr = self._b, self._y, self._xs, self._corr
        self._bmul(v, b)
        y.zero_()
        x.zero_()
        corr.zero_()
        for lev in self._levels:
            self._gemv(lev["odd32"], self._QpQn32, b, None, y)
            if lev["e1_32"].numel():
                self._couple(lev["e1_32"], lev["o1_32"], lev["Lc_e1"], self._P32, self._Qp32, y, b, -1.0)
            if lev["e2_32"].numel():
                self._couple(lev["e2_32"], lev["o2_32"], lev["Uc_e2"], self._N32, self._Qn32, y, b, -1.0)
        self._gemv(self._top, None, b, None, x)
        for lev in reversed(self._levels):
            self._couple(lev["odd32"], lev["prev32"], lev["Lc_odd"], self._P32, self._Qp32, x, corr, 1.0)
            if lev["odd_n32"].numel():
                self._couple(lev["odd_n32"], lev["next32"], lev["Uc_odd_n"], self._N32, self._Qn32, x, corr, 1.0)
            self._gemv(lev["odd32"], None, b, corr, x)
        out.copy_(x.view(-1))
        return out

    def _capture(self):
        """One application of (A - n0 B)^-1 B as a CUDA graph on fixed
        buffers, replayed by :meth:`_apply`."""
        import torch
        n = self._NL * self._nb
        self._vin = torch.zeros(n, dtype=torch.complex128, device=self._dev)
        self._xout = torch.empty(n, dtype=torch.complex128, device=self._dev)
        self._graph = None
        if self._dev.type != "cuda":      # host emulation of the device calls (tests)
            return
        self._apply_direct(self._vin, self._xout)          # outside the capture first
        torch.cuda.synchronize(self._dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._apply_direct(self._vin, self._xout)
        self._graph = g

    def _apply(self, v, out):
        if self._graph is None:
            return self._apply_direct(v, out)
        self._vin.copy_(v)
        self._graph.replay()
        out.copy_(self._xout)
        return out

    def _sync(self):
        import torch
        if self._dev.type == "cuda":
            torch.cuda.synchronize(self._dev)

    def _to_solver_order(self, X):
        """[k][NL*nb] line order -> [k][6][M][N]."""
        k = X.shape[0]
        Y = X.view(k, self._NL, 6, self._L)
        if self._lines.sweep_y:                       # [k][y][c][x]
            return Y.permute(0, 2, 1, 3).contiguous()
        return Y.permute(0, 2, 3, 1).contiguous()     # [k][x][c][y] -> [k][c][y][x]

    def solve(self, tol=1e-12, maxit=100, ncv=None, seed=0):
        """Solve for the ``neigs`` modes closest to ``n0``."""
        import time

        import torch
        if self._planes is None:
            self.build()
        t0 = time.perf_counter()
        sigma = complex(self.n0)
        self._factor(sigma)
        self._capture()
        self._sync()
        t1 = time.perf_counter()
        k = self.neigs
        m = ncv or max(3 * k, k + 20)
        n = self._NL * self._nb
        m = min(m, n - 1)
        rng = np.random.default_rng(seed)
        v0 = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n), device=self._dev)
        theta, X, nconv, napply = _krylov_schur(self._apply, n, k, m, tol, maxit, v0, self._dev)
        self._sync()
        t2 = time.perf_counter()
        if nconv < k:
            warning_message("%d eigenmodes were requested, however only %d eigenmodes were found."
                            % (k, nconv), module="emopt_b200.modes")
        F = self._to_solver_order(X)
        # unit 2-norm, the entry of largest modulus real and positive
        flat = F.view(F.shape[0], -1)
        flat /= torch.linalg.vector_norm(flat, dim=1, keepdim=True)
        big = flat.gather(1, flat.abs().argmax(dim=1, keepdim=True))
        flat *= (big.abs() / big)
        self._x = F
        self._neff = np.zeros(k, dtype=np.complex128)
        self._neff[:len(theta)] = sigma + 1.0 / np.asarray(theta)
        self.stats = {"factor_s": t1 - t0, "iterate_s": t2 - t1, "applications": napply,
                      "lines": self._NL, "block": self._nb, "levels": self.stats_levels}

    # ----------------------------------------------------------- the fields
    def _raw(self, i, component):
        q = COMPONENTS.index(component)
        return self._x[i, q]

    def get_field(self, i, component, permute=True, squeeze=False):
        """Raw field component of mode i (emopt/modes.py:1651-1787)."""
        if permute:
            component = _PERMUTE[self.ndir][component]
        f = self._raw(i, component).cpu().numpy()
        return f if squeeze else np.reshape(f, self._fshape)

    def get_field_interp(self, i, component, squeeze=False):
        """Field component of mode i averaged onto the plane's Ez-equivalent
        points (emopt/modes.py:1789-2052; the y-normal Ex and Hy, which fail
        in the reference, give the raw field)."""
        f = np.pad(self.get_field(i, component, squeeze=True), 1, "constant", constant_values=0)
        c = _PERMUTE[self.ndir][component]
        b0, b1 = self._bc[0], self._bc[1]

        def gx(a):                      # x ghost column by the first boundary
            if b0 == "E":
                a[:, 0] = -1 * a[:, 1]
            elif b0 == "H":
                a[:, 0] = a[:, 1]

        def gy(a):
            if b1 == "E":
                a[0, :] = -1 * a[1, :]
            elif b1 == "H":
                a[0, :] = a[1, :]

        g = np.copy(f)
        if self.ndir == "x":
            if c in ("Ex", "Hy"):
                gx(f); g[:, 1:] += f[:, :-1]; g[:-1, 1:] += f[1:, :-1]; g[:-1, :] += f[1:, :]; out = g / 4.0
            elif c in ("Ey", "Hx"):
                out = f
            elif c == "Ez":
                g[:-1, :] += g[1:, :]; out = g / 2.0
            else:
                gx(f); g[:, 1:] += f[:, :-1]; out = g / 2.0
        elif self.ndir == "y":
            if c in ("Ex", "Hy"):
                out = f
            elif c in ("Ey", "Hx"):
                gy(f); g[:, :-1] += g[:, 1:]; g[1:, :] += g[:-1, :]; g[1:, :-1] += g[:-1, 1:]; out = g / 4.0
            elif c == "Ez":
                g[:, :-1] += g[:, 1:]; out = g / 2.0
            else:
                gy(f); g[1:, :] += f[:-1, :]; out = g / 2.0
        else:
            if c in ("Ex", "Hy"):
                gx(f); g[:, 1:] += f[:, :-1]; out = g / 2.0
            elif c in ("Ey", "Hx"):
                gy(f); g[1:, :] += f[:-1, :]; out = g / 2.0
            elif c == "Ez":
                out = f
            else:
                gy(f); gx(f); g[:, 1:] += f[:, :-1]; g[1:, :] += f[:-1, :]; g[1:, 1:] += f[:-1, :-1]; out = g / 4.0
        out = out[1:-1, 1:-1]
        return out if squeeze else np.reshape(out, self._fshape)

    def component_energy(self, i):
        """Fractions of the mode's energy in Ex..Hz (emopt/modes.py:2054-2097)."""
        eps = np.asarray(self.eps.get_values_in(self.domain, squeeze=True)).real
        mu = np.asarray(self.mu.get_values_in(self.domain, squeeze=True)).real
        W = [np.sum((eps if c[0] == "E" else mu) * np.abs(self.get_field(i, c, squeeze=True)) ** 2)
             for c in COMPONENTS]
        tot = sum(W)
        return [w / tot for w in W]

    def get_mode_number(self, i):
        raise NotImplementedError("mode numbering is not implemented (it is a stub in the reference)")

    def find_mode_index(self, P, Q):
        for i in range(self.neigs):
            p, q = self.get_mode_number(i)
            if p == P and q == Q:
                return i
        warning_message("Desired mode number was not found.", "emopt_b200.modes")
        return 0

    def get_source(self, i, dx, dy, dz):
        """(Jx, Jy, Jz, Mx, My, Mz) that launch mode i (emopt/modes.py:2144-2296),
        each shaped like the domain, in the caller's axes."""
        import torch
        if not isinstance(self.eps, Material3D):
            raise Exception("Source calculation only possible for slices of Material3D's..")
        d = self.domain
        if self.ndir == "x":
            mydx, mydy, mydz = dy, dz, dx
            mu05 = self._values(self.mu, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2, 0.0, 0.0, 0.5)[:, :, 0]
            mu50 = self._values(self.mu, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2, 0.0, 0.5, 0.0)[:, :, 0]
        elif self.ndir == "y":
            mydx, mydy, mydz = dz, dx, dy
            mu05 = self._values(self.mu, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2, 0.0, 0.0, 0.5)[:, 0, :]
            mu50 = self._values(self.mu, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2, 0.5, 0.0, 0.0)[:, 0, :]
        else:
            mydx, mydy, mydz = dx, dy, dz
            mu05 = self._values(self.mu, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2, 0.0, 0.5, 0.0)[0]
            mu50 = self._values(self.mu, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2, 0.5, 0.0, 0.0)[0]
        eps = self._values(self.eps, d.k1, d.k2, d.j1, d.j2, d.i1, d.i2).reshape(self._M, self._N).contiguous()
        mu05, mu50 = mu05.contiguous(), mu50.contiguous()
        neff = complex(self._neff[i])
        dxn, dyn, dzn = mydx / self.R, mydy / self.R, mydz / self.R
        ekz = np.exp(1j * self._dir * neff * dzn / 2)
        F = self._x[i]
        S = complex(0.5 * mydx * mydy * torch.sum(F[0] * F[4].conj() - F[1] * F[3].conj()).item())
        s = 1.0 / np.sqrt(S)
        out = torch.empty((6, self._M, self._N), dtype=torch.complex128, device=self._dev)
        stream = torch.cuda.current_stream(self._dev).cuda_stream
        bc = self._bc_code()
        _check(libFDTD.FDTD_mode_source(self.device, stream, self._M, self._N, _ptr(F), s.real, s.imag,
                                        ekz.real, ekz.imag, dxn, dyn, dzn, _ptr(eps), _ptr(mu05), _ptr(mu50),
                                        bc, _ptr(out)), "FDTD_mode_source")
        Jx, Jy, Jz, Mx, My, Mz = (np.reshape(a, self._fshape) for a in out.cpu().numpy())
        if self.ndir == "x":
            return Jz, Jx, Jy, Mz, Mx, My
        if self.ndir == "y":
            return Jy, Jz, Jx, My, Mz, Mx
        return Jx, Jy, Jz, Mx, My, Mz


def _krylov_schur(apply, n, k, m, tol, maxit, v0, dev, check_every=4):
    """Krylov-Schur iteration for the k eigenvalues of largest modulus of the
    operator ``apply`` (n x n, device vectors), m-dimensional subspace; the
    Ritz values are tested every ``check_every`` new vectors, so a solve stops
    as soon as the wanted pairs have converged.  Returns (theta[k'],
    vectors[k'][n], k' converged, applications)."""
    import torch
    V = torch.empty((m + 1, n), dtype=torch.complex128, device=dev)
    H = np.zeros((m + 1, m), dtype=np.complex128)
    V[0] = v0 / torch.linalg.vector_norm(v0)
    w = torch.empty(n, dtype=torch.complex128, device=dev)
    p, napply, mc = 0, 0, 0

    def ritz(size):
        theta, S = np.linalg.eig(H[:size, :size])
        order = np.argsort(-np.abs(theta))
        res = np.abs(H[size, size - 1] * S[size - 1, :])
        return theta, S, order, res

    for _ in range(maxit):
        done = False
        for j in range(p, m):
            apply(V[j], w)
            napply += 1
            Vj = V[:j + 1]
            h = Vj.conj() @ w                      # classical Gram-Schmidt, twice
            w -= h @ Vj
            h2 = Vj.conj() @ w
            w -= h2 @ Vj
            h += h2
            beta = float(torch.linalg.vector_norm(w))
            H[:j + 1, j] = h.cpu().numpy()
            H[j + 1, j] = beta
            mc = j + 1
            if beta == 0.0:                        # an invariant subspace: the Ritz pairs are exact
                done = True
                break
            V[j + 1] = w / beta
            if mc == m or (mc >= k + 2 and (mc - p) % check_every == 0):
                theta, S, order, res = ritz(mc)
                if all(res[q] <= tol * abs(theta[q]) for q in order[:k]):
                    done = True
                    break
        if done:
            break
        # restart: keep the Schur vectors of the wanted part and some more
        theta, S, order, res = ritz(m)
        keep = min(m - 1, max(k + (m - k) // 2, k + 1))
        thr = np.abs(theta[order[keep - 1]])
        T, Z, sdim = sla.schur(H[:m, :m], output="complex", sort=lambda z: abs(z) >= thr * (1 - 1e-12))
        p = int(min(max(sdim, k), m - 1))
        Zt = torch.as_tensor(np.ascontiguousarray(Z[:, :p].T), device=dev)
        V[:p] = Zt @ V[:m]
        V[p] = V[m]
        Hn = np.zeros_like(H)
        Hn[:p, :p] = T[:p, :p]
        Hn[p, :p] = H[m, m - 1] * Z[m - 1, :p]
        H = Hn
    theta, S, order, res = ritz(mc)
    good = [q for q in order[:k] if res[q] <= max(tol, 1e-8) * abs(theta[q])]
    Sk = torch.as_tensor(np.ascontiguousarray(S[:, good].T), device=dev)
    X = Sk @ V[:mc]
    return theta[good], X, len(good), napply
