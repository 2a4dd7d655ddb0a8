"""Figure-of-merit helpers of ``emopt.fomutils`` with the reference's numpy
interface, for scripts that compute their adjoint sources by hand.

* ``ModeMatch`` (emopt/fomutils.py:925-1197): overlap of interpolated fields
  with a mode on a plane -- ``compute``, the forward and backward mode match,
  and the derivatives of the unnormalised forward match with respect to each
  interpolated field component.
* ``interpolated_dFdx_3D`` (emopt/fomutils.py:1282-1426): the transpose of the
  interpolation onto the Ez grid (``FDTD.get_field_interp``), which turns
  derivatives with respect to interpolated fields into derivatives with
  respect to the staggered Yee fields (the adjoint current sources), on the
  domain grown by one cell towards -x, -y and +z.

The differentiation form of this package (``emopt_b200.adjoint``) computes the
same quantities on the GPU with autograd; these are the host forms with the
reference's call signatures.  The formulas are the reference's: they define
the figure of merit and its gradient.
"""
from __future__ import annotations

import numpy as np

_C = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


class ModeMatch:
    """Mode match of fields with the mode (Exm..Hzm) on a plane with normal
    ``normal`` and cell sides ``ds1``, ``ds2`` (emopt/fomutils.py:925-1092)."""

    def __init__(self, normal, ds1, ds2=1.0, Exm=None, Eym=None, Ezm=None, Hxm=None, Hym=None, Hzm=None):
        given = [Exm, Eym, Ezm, Hxm, Hym, Hzm]
        self.fshape = next((f.shape[:] for f in given if f is not None), None)
        if self.fshape is None:
            raise ValueError("No fields were passed to ModeMatch.  Mode matching is impossible "
                             "without fields!")
        z = lambda f: f if f is not None else np.zeros(self.fshape, dtype=np.complex128)
        self.Exm, self.Eym, self.Ezm, self.Hxm, self.Hym, self.Hzm = (z(f) for f in given)
        self.normal = np.array(normal)
        self.ds1, self.ds2 = ds1, ds2
        self.xhat, self.yhat, self.zhat = np.array([1, 0, 0]), np.array([0, 1, 0]), np.array([0, 0, 1])
        self.x_dot_s = self.xhat.dot(self.normal)
        self.y_dot_s = self.yhat.dot(self.normal)
        self.z_dot_s = self.zhat.dot(self.normal)
        self.Pm = ds1 * ds2 * np.sum(self._flux(self.Exm, self.Eym, self.Ezm, self.Hxm, self.Hym, self.Hzm))
        self.efficiency = 0.0
        self.Ex, self.Ey, self.Ez, self.Hx, self.Hy, self.Hz = (z(None) for _ in range(6))

    def _flux(self, Ex, Ey, Ez, Hx, Hy, Hz):
        """(E x H*) . normal, pointwise."""
        cj = np.conj
        return (self.x_dot_s * (Ey * cj(Hz) - Ez * cj(Hy)) + self.y_dot_s * (-Ex * cj(Hz) + Ez * cj(Hx))
                + self.z_dot_s * (Ex * cj(Hy) - Ey * cj(Hx)))

    def compute(self, Ex=None, Ey=None, Ez=None, Hx=None, Hy=None, Hz=None):
        """Overlap coefficients am (forward) and bm (backward) of the given
        interpolated fields (None: zero) and the two mode matches."""
        z = lambda f: f if f is not None else np.zeros(self.fshape, dtype=np.complex128)
        self.Ex, self.Ey, self.Ez, self.Hx, self.Hy, self.Hz = (z(f) for f in (Ex, Ey, Ez, Hx, Hy, Hz))
        cj = np.conj
        ds = self.ds1 * self.ds2
        xs, ys, zs = self.x_dot_s, self.y_dot_s, self.z_dot_s
        self.am1 = 0.5 * ds * np.sum((self.Ey * cj(self.Hzm) - self.Ez * cj(self.Hym)) * xs -
                                     (self.Ex * cj(self.Hzm) - self.Ez * cj(self.Hxm)) * ys +
                                     (self.Ex * cj(self.Hym) - self.Ey * cj(self.Hxm)) * zs) / self.Pm
        self.am2 = 0.5 * ds * np.sum((cj(self.Eym) * self.Hz - cj(self.Ezm) * self.Hy) * xs -
                                     (cj(self.Exm) * self.Hz - cj(self.Ezm) * self.Hx) * ys +
                                     (cj(self.Exm) * self.Hy - cj(self.Eym) * self.Hx) * zs) / cj(self.Pm)
        self.am = self.am1 + self.am2
        self.bm = self.am1 - self.am2
        self.mode_match_fwd = 0.5 * self.am * cj(self.am) * np.real(self.Pm)
        self.mode_match_back = 0.5 * self.bm * cj(self.bm) * np.real(self.Pm)

    def get_mode_match_forward(self, P_in):
        return self.mode_match_fwd.real / P_in

    def get_mode_match_back(self, P_in):
        return self.mode_match_back.real / P_in

    def _k(self, denom):
        return 0.25 * self.ds1 * self.ds2 * np.real(self.Pm) * np.conj(self.am) / denom

    def get_dFdEx(self):
        return self._k(self.Pm) * (-np.conj(self.Hzm) * self.y_dot_s + np.conj(self.Hym) * self.z_dot_s)

    def get_dFdEy(self):
        return self._k(self.Pm) * (np.conj(self.Hzm) * self.x_dot_s - np.conj(self.Hxm) * self.z_dot_s)

    def get_dFdEz(self):
        return self._k(self.Pm) * (-np.conj(self.Hym) * self.x_dot_s + np.conj(self.Hxm) * self.y_dot_s)

    def get_dFdHx(self):
        return self._k(np.conj(self.Pm)) * (np.conj(self.Ezm) * self.y_dot_s - np.conj(self.Eym) * self.z_dot_s)

    def get_dFdHy(self):
        return self._k(np.conj(self.Pm)) * (-np.conj(self.Ezm) * self.x_dot_s + np.conj(self.Exm) * self.z_dot_s)

    def get_dFdHz(self):
        return self._k(np.conj(self.Pm)) * (np.conj(self.Eym) * self.x_dot_s - np.conj(self.Exm) * self.y_dot_s)


def _on_device(arrays) -> bool:
    """Are the given derivative arrays CUDA tensors?"""
    for a in arrays:
        if a is not None and type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False):
            return True
    return False


# Where get_field_interp reads each component (offsets (dz, dy, dx) of the
# samples averaged onto a cell of the Ez grid) and with which weight.
_TAPS = {
    "Ex": ([(0, 0, 0), (0, 0, -1), (1, 0, 0), (1, 0, -1)], 0.25),
    "Ey": ([(0, 0, 0), (0, -1, 0), (1, 0, 0), (1, -1, 0)], 0.25),
    "Ez": ([(0, 0, 0)], 1.0),
    "Hx": ([(0, 0, 0), (0, -1, 0)], 0.5),
    "Hy": ([(0, 0, 0), (0, 0, -1)], 0.5),
    "Hz": ([(dz, dy, dx) for dz in (0, 1) for dy in (0, -1) for dx in (0, -1)], 0.125),
}


def interpolated_dFdx_3D(sim, domain, dFdExi, dFdEyi, dFdEzi, dFdHxi, dFdHyi, dFdHzi):
    """Derivatives with respect to the staggered fields from derivatives with
    respect to the interpolated ones (emopt/fomutils.py:1282-1426).  Returns
    (grown domain, dFdEx, dFdEy, dFdEz, dFdHx, dFdHy, dFdHz); the arrays are
    shaped like the grown domain.  On a domain touching a symmetric min face
    ('E' or 'H' in ``sim.bc``) the mirrored samples of the interpolation add
    (or, for 'E', subtract) their share to the first plane, as the reference
    does -- including its use of the y face for Ex under an 'E' letter.
    Given complex CUDA tensors (None for a zero component) it returns CUDA
    tensors computed on the device."""
    dF = dict(zip(_C, (dFdExi, dFdEyi, dFdEzi, dFdHxi, dFdHyi, dFdHzi)))
    bc = sim.bc
    if _on_device(dF.values()):
        # CUDA tensors: the same mapping by the device kernel (FDTD_dfdx_interp)
        from .fieldops import dfdx_interp
        grown, out = dfdx_interp(domain, dF, bc)
        return (grown, *(out[c] for c in _C))
    Nz, Ny, Nx = domain.shape
    out = []
    for c in _C:
        a = np.zeros((Nz + 2, Ny + 2, Nx + 2), dtype=np.complex128)
        taps, w = _TAPS[c]
        v = np.asarray(dF[c]) * w
        for dz, dy, dx in taps:
            a[1 + dz:1 + dz + Nz, 1 + dy:1 + dy + Ny, 1 + dx:1 + dx + Nx] += v
        # mirrored samples at a symmetric min face
        if c == "Ex" and domain.k1 == 0 and bc[0] in "EH":
            for dz in (0, 1):
                if bc[0] == "H":
                    a[1 + dz:1 + dz + Nz, 1:1 + Ny, 1] += v[:, :, 0]
                else:
                    a[1 + dz:1 + dz + Nz, 1, 1:1 + Nx] -= v[:, 0, :]
        if c in ("Ey", "Hx", "Hz") and domain.j1 == 0 and bc[1] in "EH":
            sgn = 1.0 if bc[1] == "H" else -1.0
            for dz, dy, dx in taps:
                if dy == 0:
                    a[1 + dz:1 + dz + Nz, 1, 1 + dx:1 + dx + Nx] += sgn * v[:, 0, :]
        if c == "Ez":
            a[1:-1, 1:-1, 1:-1] = dF[c]
        out.append(a[1:, 0:-1, 0:-1])
    grown = domain.copy()
    grown.grow(1, 0, 1, 0, 0, 1)
    return (grown, *out)


# Derivative of the plane flux s (E x H*) . e_axis with respect to each
# interpolated component, before the factor 0.25 dA and the outward sign:
# (component, sign, conjugated partner).
_DFLUX = {
    0: [("Ey", 1.0, "Hz"), ("Ez", -1.0, "Hy"), ("Hy", -1.0, "Ez"), ("Hz", 1.0, "Ey")],
    1: [("Ex", -1.0, "Hz"), ("Ez", 1.0, "Hx"), ("Hx", 1.0, "Ez"), ("Hz", -1.0, "Ex")],
    2: [("Ex", 1.0, "Hy"), ("Ey", -1.0, "Hx"), ("Hx", -1.0, "Ey"), ("Hy", 1.0, "Ex")],
}


def power_norm_dFdx_3D(sim, f, domain, dfdEx, dfdEy, dfdEz, dfdHx, dfdHy, dfdHz):
    """Adjoint sources of F = f / Psrc (emopt/fomutils.py:1654-1920): the
    derivative of f (with respect to interpolated fields on ``domain``)
    divided by the source power, plus -f / Psrc^2 times the derivative of the
    source power through each of the six planes one cell inside the CPML
    (planes on symmetric min faces left out), every block mapped to the
    staggered fields by :func:`interpolated_dFdx_3D`.  Returns
    [sources, domains].  As in the reference, a face without CPML puts its
    plane at the domain edge (X, not X - dx as the source power itself)."""
    Psrc = sim.source_power
    srcs, doms = [], []
    g = interpolated_dFdx_3D(sim, domain, *(np.asarray(a) / Psrc for a in
                                            (dfdEx, dfdEy, dfdEz, dfdHx, dfdHy, dfdHz)))
    srcs.append(g[1:])
    doms.append(g[0])
    w = sim.w_pml
    d = (sim.dx, sim.dy, sim.dz)
    L = (sim.X, sim.Y, sim.Z)
    lo = [w[2 * a] + d[a] if w[2 * a] > 0 else 0.0 for a in range(3)]
    hi = [L[a] - w[2 * a + 1] - d[a] if w[2 * a + 1] > 0 else L[a] for a in range(3)]
    from .misc import DomainCoordinates
    for axis in range(3):
        for side, pos in ((-1.0, lo[axis]), (1.0, hi[axis])):
            if side < 0 and sim.bc[axis] in ("E", "H"):
                continue
            b = [[lo[0], hi[0]], [lo[1], hi[1]], [lo[2], hi[2]]]
            b[axis] = [pos, pos]
            plane = DomainCoordinates(b[0][0], b[0][1], b[1][0], b[1][1], b[2][0], b[2][1], *d)
            dA = np.prod([d[q] for q in range(3) if q != axis])
            need = {p for _, _, p in _DFLUX[axis]}
            F = {c: sim.get_field_interp(c, domain=plane) for c in sorted(need)}
            dP = {c: np.zeros(plane.shape, dtype=np.complex128) for c in _C}
            for c, sgn, partner in _DFLUX[axis]:
                dP[c] = -1 * f * (side * sgn * 0.25 * dA * np.conj(F[partner])) / Psrc ** 2
            g = interpolated_dFdx_3D(sim, plane, *(dP[c] for c in _C))
            srcs.append(g[1:])
            doms.append(g[0])
    return [srcs, doms]
