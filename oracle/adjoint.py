"""Restatement of the reference's adjoint gradient path (test infrastructure).

Used only by tests as the checker of the differentiation form; nothing in
the product imports it.  It follows the reference step by step, in numpy, on
fields from the CPU oracle:

* ``interp`` -- ``FDTD.get_field_interp`` (emopt/fdtd.py:1401-1553): a field
  component averaged onto the Ez grid from the block grown by one cell.
* ``mode_match`` -- ``ModeMatch.compute`` and ``get_dFdE*`` / ``get_dFdH*``
  (emopt/fomutils.py:925-1197): forward mode match 0.5 |a_m|^2 Re(P_m) and
  its derivatives with respect to the interpolated fields.
* ``interpolated_dFdx`` -- ``interpolated_dFdx_3D`` (emopt/fomutils.py:
  1282-1426): maps those derivatives back onto the staggered fields (the
  transpose of the interpolation) on a domain grown by (1, 0, 1, 0, 0, 1).
* ``calc_gradient`` -- ``AdjointMethod.calc_gradient`` with ``calc_ydAx``
  (emopt/adjoint_method.py:448-547, emopt/fdtd.py:1694-1717): for each
  parameter a forward difference of the permittivity, ydAx = sum of
  y * 1j * d(eps) * x over the E components, gradient -2 Re(ydAx / step).

``reference_gradient`` strings these together around two oracle solves
(forward, then adjoint with the dF/dx arrays as J/M sources, as
``AdjointMethod.gradient`` does, emopt/adjoint_method.py:549-606).
"""
from __future__ import annotations

import numpy as np

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


class Box:
    """Index box [i1, i2) x [j1, j2) x [k1, k2) (DomainCoordinates indices)."""

    def __init__(self, k1, k2, j1, j2, i1, i2):
        self.k1, self.k2, self.j1, self.j2, self.i1, self.i2 = k1, k2, j1, j2, i1, i2

    @property
    def shape(self):
        return (self.i2 - self.i1, self.j2 - self.j1, self.k2 - self.k1)

    def take(self, a):
        return a[self.i1:self.i2, self.j1:self.j2, self.k1:self.k2]


def grown(box: Box, shape, d) -> Box:
    """The interpolation block (emopt/fdtd.py:1437-1456): one cell more on each
    side where the grid allows, rebuilt from coordinates like DomainCoordinates."""
    Nz, Ny, Nx = shape
    k1, k2, j1, j2, i1, i2 = box.k1, box.k2, box.j1, box.j2, box.i1, box.i2
    if k1 > 0: k1 -= 1
    if k2 < Nx - 1: k2 += 1
    if j1 > 0: j1 -= 1
    if j2 < Ny - 1: j2 += 1
    if i1 > 0: i1 -= 1
    if i2 < Nz - 1: i2 += 1
    dx, dy, dz = d
    # DomainCoordinates(xmin, xmax, ...): k1 = int(xmin/dx), k2 = int(xmax/dx) + 1
    return Box(int(k1 * dx / dx), int(k2 * dx / dx) + 1, int(j1 * dy / dy), int(j2 * dy / dy) + 1,
               int(i1 * dz / dz), int(i2 * dz / dz) + 1)


def interp(full: np.ndarray, component: str, box: Box, bc: str, d) -> np.ndarray:
    """One component of the full (Nz, Ny, Nx) field interpolated on ``box``."""
    if component == "Ez":
        return box.take(full).copy()
    g = grown(box, full.shape, d)
    f = np.pad(g.take(full), 1, "constant", constant_values=0)
    crop = lambda a: a[1 + box.i1 - g.i1:-1 - (g.i2 - box.i2),
                       1 + box.j1 - g.j1:-1 - (g.j2 - box.j2),
                       1 + box.k1 - g.k1:-1 - (g.k2 - box.k2)]

    def symx(a):
        if g.k1 == 0 and bc[0] == "E": a[:, :, 0] = -a[:, :, 1]
        elif g.k1 == 0 and bc[0] == "H": a[:, :, 0] = a[:, :, 1]

    def symy(a):
        if g.j1 == 0 and bc[1] == "E": a[:, 0, :] = -a[:, 1, :]
        elif g.j1 == 0 and bc[1] == "H": a[:, 0, :] = a[:, 1, :]

    if component == "Ex":
        symx(f)
        o = f.copy()
        o[1:-1, :, 1:-1] += f[1:-1, :, 0:-2] + f[2:, :, 1:-1] + f[2:, :, 0:-2]
        return crop(o / 4.0)
    if component == "Ey":
        symy(f)
        o = f.copy()
        o[1:-1, 1:-1, :] += f[1:-1, 0:-2, :] + f[2:, 1:-1, :] + f[2:, 0:-2, :]
        return crop(o / 4.0)
    if component == "Hx":
        symy(f)
        o = f.copy()
        o[:, 1:, :] += f[:, 0:-1, :]
        return crop(o / 2.0)
    if component == "Hy":
        symx(f)
        o = f.copy()
        o[:, :, 1:] += f[:, :, 0:-1]
        return crop(o / 2.0)
    if component == "Hz":
        symx(f)
        symy(f)
        o = f.copy()
        o[0:-1, 1:, 1:] += (f[0:-1, 1:, 0:-1] + f[0:-1, 0:-1, 1:] + f[0:-1, 0:-1, 0:-1] +
                            f[1:, 1:, 1:] + f[1:, 1:, 0:-1] + f[1:, 0:-1, 1:] + f[1:, 0:-1, 0:-1])
        return crop(o / 8.0)
    raise ValueError(component)


def mode_match(fields: dict, mode: dict, normal, ds1, ds2):
    """Forward mode match and dF/d(interpolated field) for each component."""
    shape = next(v.shape for v in mode.values() if v is not None)
    z = np.zeros(shape, dtype=np.complex128)
    m = {c: (np.asarray(mode[c]) if mode.get(c) is not None else z) for c in COMPONENTS}
    f = {c: (np.asarray(fields[c]).reshape(shape) if fields.get(c) is not None else z)
         for c in COMPONENTS}
    xs, ys, zs = normal
    ds = ds1 * ds2
    cj = np.conj
    Pm = ds * np.sum(xs * (m["Ey"] * cj(m["Hz"]) - m["Ez"] * cj(m["Hy"])) +
                     ys * (-m["Ex"] * cj(m["Hz"]) + m["Ez"] * cj(m["Hx"])) +
                     zs * (m["Ex"] * cj(m["Hy"]) - m["Ey"] * cj(m["Hx"])))
    am1 = 0.5 * ds * np.sum((f["Ey"] * cj(m["Hz"]) - f["Ez"] * cj(m["Hy"])) * xs -
                            (f["Ex"] * cj(m["Hz"]) - f["Ez"] * cj(m["Hx"])) * ys +
                            (f["Ex"] * cj(m["Hy"]) - f["Ey"] * cj(m["Hx"])) * zs) / Pm
    am2 = 0.5 * ds * np.sum((cj(m["Ey"]) * f["Hz"] - cj(m["Ez"]) * f["Hy"]) * xs -
                            (cj(m["Ex"]) * f["Hz"] - cj(m["Ez"]) * f["Hx"]) * ys +
                            (cj(m["Ex"]) * f["Hy"] - cj(m["Ey"]) * f["Hx"]) * zs) / cj(Pm)
    am = am1 + am2
    F = (0.5 * am * cj(am) * np.real(Pm)).real
    k = 0.25 * ds * np.real(Pm) * cj(am)
    dF = {
        "Ex": k * (-cj(m["Hz"]) * ys + cj(m["Hy"]) * zs) / Pm,
        "Ey": k * (cj(m["Hz"]) * xs - cj(m["Hx"]) * zs) / Pm,
        "Ez": k * (-cj(m["Hy"]) * xs + cj(m["Hx"]) * ys) / Pm,
        "Hx": k * (cj(m["Ez"]) * ys - cj(m["Ey"]) * zs) / cj(Pm),
        "Hy": k * (-cj(m["Ez"]) * xs + cj(m["Ex"]) * zs) / cj(Pm),
        "Hz": k * (cj(m["Ey"]) * xs - cj(m["Ex"]) * ys) / cj(Pm),
    }
    return F, dF


def interpolated_dFdx(box: Box, dF: dict, bc: str):
    """Derivatives with respect to the staggered fields; returns (grown box, dict)."""
    Nz, Ny, Nx = box.shape
    shape = (Nz + 2, Ny + 2, Nx + 2)
    z = lambda: np.zeros(shape, dtype=np.complex128)
    out = {}
    a = z(); v = dF["Ex"] / 4.0
    a[1:-1, 1:-1, 1:-1] += v; a[1:-1, 1:-1, 0:-2] += v; a[2:, 1:-1, 1:-1] += v; a[2:, 1:-1, 0:-2] += v
    if box.k1 == 0 and bc[0] == "H":
        a[1:-1, 1:-1, 1] += v[:, :, 0]; a[2:, 1:-1, 1] += v[:, :, 0]
    elif box.k1 == 0 and bc[0] == "E":
        a[1:-1, 1, 1:-1] -= v[:, 0, :]; a[2:, 1, 1:-1] -= v[:, 0, :]
    out["Ex"] = a[1:, 0:-1, 0:-1]
    a = z(); v = dF["Ey"] / 4.0
    a[1:-1, 1:-1, 1:-1] += v; a[1:-1, 0:-2, 1:-1] += v; a[2:, 1:-1, 1:-1] += v; a[2:, 0:-2, 1:-1] += v
    if box.j1 == 0 and bc[1] == "H":
        a[1:-1, 1, 1:-1] += v[:, 0, :]; a[2:, 1, 1:-1] += v[:, 0, :]
    elif box.j1 == 0 and bc[1] == "E":
        a[1:-1, 1, 1:-1] -= v[:, 0, :]; a[2:, 1, 1:-1] -= v[:, 0, :]
    out["Ey"] = a[1:, 0:-1, 0:-1]
    a = z(); a[1:-1, 1:-1, 1:-1] = dF["Ez"]
    out["Ez"] = a[1:, 0:-1, 0:-1]
    a = z(); v = dF["Hx"] / 2.0
    a[1:-1, 1:-1, 1:-1] += v; a[1:-1, 0:-2, 1:-1] += v
    if box.j1 == 0 and bc[1] == "H":
        a[1:-1, 1, 1:-1] += v[:, 0, :]
    elif box.j1 == 0 and bc[1] == "E":
        a[1:-1, 1, 1:-1] -= v[:, 0, :]
    out["Hx"] = a[1:, 0:-1, 0:-1]
    a = z(); v = dF["Hy"] / 2.0
    a[1:-1, 1:-1, 1:-1] += v; a[1:-1, 1:-1, 0:-2] += v
    out["Hy"] = a[1:, 0:-1, 0:-1]
    a = z(); v = dF["Hz"] / 8.0
    for s in ((slice(1, -1), slice(1, -1), slice(1, -1)), (slice(1, -1), slice(0, -2), slice(1, -1)),
              (slice(1, -1), slice(1, -1), slice(0, -2)), (slice(1, -1), slice(0, -2), slice(0, -2)),
              (slice(2, None), slice(1, -1), slice(1, -1)), (slice(2, None), slice(0, -2), slice(1, -1)),
              (slice(2, None), slice(1, -1), slice(0, -2)), (slice(2, None), slice(0, -2), slice(0, -2))):
        a[s] += v
    if box.j1 == 0 and bc[1] == "H":
        for s in ((slice(1, -1), 1, slice(1, -1)), (slice(1, -1), 1, slice(0, -2)),
                  (slice(2, None), 1, slice(1, -1)), (slice(2, None), 1, slice(0, -2))):
            a[s] += v[:, 0, :]
    elif box.j1 == 0 and bc[1] == "E":
        for s in ((slice(1, -1), 1, slice(1, -1)), (slice(1, -1), 1, slice(0, -2)),
                  (slice(2, None), 1, slice(1, -1)), (slice(2, None), 1, slice(0, -2))):
            a[s] -= v[:, 0, :]
    out["Hz"] = a[1:, 0:-1, 0:-1]
    # DomainCoordinates.grow(1, 0, 1, 0, 0, 1): k1-1, j1-1, i2+1
    g = Box(box.k1 - 1, box.k2, box.j1 - 1, box.j2, box.i1, box.i2 + 1)
    return g, out


def calc_gradient(x: list, y: list, eps0: list, eps_steps: list, step: float) -> np.ndarray:
    """-2 Re(y^T dA x / step) for each perturbed permittivity set in ``eps_steps``."""
    grad = np.zeros(len(eps_steps))
    for q, eps in enumerate(eps_steps):
        ydAx = 0.0 + 0.0j
        for c in range(3):
            ydAx += np.sum(y[c] * 1j * (eps[c] - eps0[c]) * x[c])
        grad[q] = -2.0 * np.real(ydAx / step)
    return grad


def clip_to_grid(g: Box, arrays: dict, shape):
    """Crop a source box (and its arrays) to the grid (FDTD.__get_local_domain_overlap)."""
    Nz, Ny, Nx = shape
    lo = (max(g.i1, 0), max(g.j1, 0), max(g.k1, 0))
    hi = (min(g.i2, Nz), min(g.j2, Ny), min(g.k2, Nx))
    sl = tuple(slice(l - o, h - o) for l, h, o in zip(lo, hi, (g.i1, g.j1, g.k1)))
    return lo, [np.ascontiguousarray(arrays[c][sl]) for c in COMPONENTS]


def reference_gradient(make_oracle, problem, params: np.ndarray, indices, step: float,
                       n_main: int, nthreads: int, eps_fn, mode, plane: Box, normal=(1, 0, 0)):
    """Forward solve, FOM, adjoint solve and calc_gradient on the CPU oracle.

    ``make_oracle(eps3)`` returns a configured OracleFDTD for permittivity
    arrays ``eps3`` (with the problem's forward sources); ``eps_fn(params)``
    gives the three permittivity arrays of a design.  Returns (F, gradient at
    ``indices``, forward fields, adjoint fields)."""
    eps0 = [np.asarray(e) for e in eps_fn(params)]
    shape = eps0[0].shape
    d = (problem.dx, problem.dy, problem.dz)
    fwd_sim = make_oracle(eps0)
    x = fwd_sim.run_fixed_slabs(n_main, nthreads)["fields"]
    bc = problem.bc
    f = {c: interp(x[COMPONENTS.index(c)], c, plane, bc, d) for c in COMPONENTS}
    ds = {0: (d[1], d[2]), 1: (d[0], d[2]), 2: (d[0], d[1])}[int(np.argmax(np.abs(normal)))]
    F, dF = mode_match(f, mode, normal, ds[0], ds[1])
    g, dFdx = interpolated_dFdx(plane, dF, bc)
    lo, arrays = clip_to_grid(g, dFdx, shape)
    adj_sim = make_oracle(eps0)
    adj_sim.sources = []
    adj_sim.add_source(arrays, *lo)
    y = adj_sim.run_fixed_slabs(n_main, nthreads)["fields"]
    eps_steps = []
    for q in indices:
        p1 = np.array(params, dtype=np.float64, copy=True)
        p1.flat[q] += step
        eps_steps.append([np.asarray(e) for e in eps_fn(p1)])
    return F, calc_gradient(x, y, eps0, eps_steps, step), x, y
