"""Differentiation form: the CW solve as a ``torch.autograd.Function``.

Forward: write the design permittivity into the device-resident material
arrays, run the CW solve on the GPU (``FDTD_solve_cw``, phasors written
straight into CUDA tensors) and return the raw Yee fields on a monitor box.
The figure of merit is ordinary torch code on those fields (the reference's
field interpolation ``emopt/fdtd.py:1401-1553`` and mode match
``emopt/fomutils.py:925-1197`` restated as torch operations), so its
derivative with respect to the raw fields -- the transpose that
``interpolated_dFdx_3D`` (``emopt/fomutils.py:1282-1426``) writes out by hand
-- comes from autograd.

Backward: the adjoint sources are the holomorphic derivative dF/dx of the
figure of merit with respect to the monitor fields (J = dF/dE, M = dF/dH, as
``AdjointMethod.gradient`` passes ``calc_dFdx`` to ``set_adjoint_sources``,
``emopt/adjoint_method.py:549-606``); torch delivers 2 dF/d(conj x) for a real
loss, so dF/dx = conj(grad) / 2.  One adjoint CW solve (same materials, no
coefficient upload) gives y, and the fused kernel ``FDTD_grad_eps`` returns
g_c = -2 Re(1j y_c x_c) per unit permittivity change, summed along z for a
planar design with Kahan-compensated float64 sums.  That is the permittivity
part of ``-2 Re(y^T dA/dp x)`` of ``AdjointMethod.calc_gradient``
(``emopt/adjoint_method.py:505-544``); autograd applies the rest of the chain
rule (design map, projection, blur).  No checkpointing is needed: the CW
adjoint uses only the two steady-state fields.

The solver may run in float32 (fields, coefficients, CPML state); phasors,
the figure of merit and the gradient sums stay float64.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch
import torch.nn.functional as F

from . import fdtd_ctypes as _ct
from . import fieldops
from .misc import DomainCoordinates

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

# array setters that take raw (device) pointers
_raw = _ct.raw


def _ptr(t: torch.Tensor) -> int:
    assert t.is_contiguous()
    return t.data_ptr()


# --------------------------------------------------------------- design map
def gaussian_blur(rho: torch.Tensor, sigma: float, truncate: float = 4.0) -> torch.Tensor:
    """Separable Gaussian blur with edge replication: the same weights and
    support as ``scipy.ndimage.gaussian_filter(rho, sigma, mode='nearest')``."""
    r = int(truncate * sigma + 0.5)
    x = torch.arange(-r, r + 1, dtype=rho.dtype, device=rho.device)
    w = torch.exp(-0.5 * (x / sigma) ** 2)
    w = w / w.sum()
    out = rho[None, None]
    out = F.conv2d(F.pad(out, (0, 0, r, r), mode="replicate"), w.view(1, 1, -1, 1))
    out = F.conv2d(F.pad(out, (r, r, 0, 0), mode="replicate"), w.view(1, 1, 1, -1))
    return out[0, 0]


def tanh_project(r: torch.Tensor, beta: float, eta: float) -> torch.Tensor:
    """Threshold projection (tanh(b e) + tanh(b (r - e))) / (tanh(b e) + tanh(b (1 - e)))."""
    a = np.tanh(beta * eta)
    return (a + torch.tanh(beta * (r - eta))) / (a + np.tanh(beta * (1.0 - eta)))


@dataclass
class PlanarDesign:
    """Permittivity of an extruded design region driven by a 2-D density.

    Component c (Ex, Ey, Ez) of column (j, k) takes eps_lo + (eps_hi - eps_lo)
    * rho[ix, iy] when its Yee position lies in the design rectangle, with
    (ix, iy) the density pixel that contains it, on the planes [i0_c, i1_c) of
    the layer; columns of the box outside the rectangle keep their background
    value.  This is the voxel sampling of the problem builders.
    """
    k0: int
    k1: int
    j0: int
    j1: int
    iz: tuple          # ((i0, i1) for Ex, Ey, Ez)
    pix: torch.Tensor  # (3, nj, nk) long: flat pixel index ix * nyd + iy, or -1
    background: torch.Tensor  # (3, nj, nk) float64
    eps_lo: float
    eps_hi: float

    @property
    def box(self):
        b = [self.k0, self.k1, self.j0, self.j1]
        for i0, i1 in self.iz:
            b += [i0, i1]
        return b

    def eps_columns(self, rho: torch.Tensor) -> torch.Tensor:
        flat = rho.reshape(-1)
        inside = self.pix >= 0
        e = self.eps_lo + (self.eps_hi - self.eps_lo) * flat[self.pix.clamp(min=0)]
        return torch.where(inside, e, self.background)


def planar_design(shape, d, rect, layer, nd, eps_lo, eps_hi, base_eps, device) -> PlanarDesign:
    """Build the map for design rectangle ``rect = (xd0, xd1, yd0, yd1)`` (um),
    layer ``|z - zc| <= h`` given as ``layer = (zc, h)``, density grid ``nd``
    and the background permittivity arrays ``base_eps`` (3 x (Nz, Ny, Nx))."""
    from .problems import YEE_OFFSETS
    Nz, Ny, Nx = shape
    xd0, xd1, yd0, yd1 = rect
    zc, hz = layer
    nxd, nyd = nd
    k0 = max(int(np.floor(xd0 / d - 0.5)) - 1, 0)
    k1 = min(int(np.ceil(xd1 / d)) + 2, Nx)
    j0 = max(int(np.floor(yd0 / d - 0.5)) - 1, 0)
    j1 = min(int(np.ceil(yd1 / d)) + 2, Ny)
    pix, bg, iz = [], [], []
    for c in range(3):
        sx, sy, sz = YEE_OFFSETS[c]
        z = (np.arange(Nz) + sz) * d
        planes = np.nonzero(np.abs(z - zc) <= hz)[0]
        i0, i1 = int(planes[0]), int(planes[-1]) + 1
        iz.append((i0, i1))
        x = (np.arange(k0, k1) + sx) * d
        y = (np.arange(j0, j1) + sy) * d
        Y, X = np.meshgrid(y, x, indexing="ij")
        inside = (X >= xd0) & (X <= xd1) & (Y >= yd0) & (Y <= yd1)
        ix = np.clip(((X - xd0) / (xd1 - xd0) * nxd).astype(int), 0, nxd - 1)
        iy = np.clip(((Y - yd0) / (yd1 - yd0) * nyd).astype(int), 0, nyd - 1)
        pix.append(np.where(inside, ix * nyd + iy, -1))
        bg.append(np.real(base_eps[c][i0, j0:j1, k0:k1]))
    return PlanarDesign(k0, k1, j0, j1, tuple(iz),
                        torch.as_tensor(np.stack(pix), dtype=torch.long, device=device),
                        torch.as_tensor(np.stack(bg), dtype=torch.float64, device=device),
                        eps_lo, eps_hi)


# ------------------------------------------------ interpolation (device)
# The raw blocks of the monitors are interpolated onto the Ez grid and their
# source-power planes summed by the kernels of fields_kernels.cu (fieldops);
# autograd runs through their transposes.
grow_domain = fieldops.grow_domain


class ModeMatch:
    """Torch form of ``emopt.fomutils.ModeMatch`` (emopt/fomutils.py:925-1092):
    the forward mode match 0.5 |a_m|^2 Re(P_m) of interpolated fields with
    reference mode fields on a plane with normal ``normal``."""

    def __init__(self, normal, ds1, ds2, mode: dict, device):
        self.n = [float(v) for v in normal]
        self.ds = ds1 * ds2
        shape = next(v.shape for v in mode.values() if v is not None)
        z = np.zeros(shape, dtype=np.complex128)
        m = {c: np.asarray(mode.get(c, z) if mode.get(c) is not None else z, dtype=np.complex128)
             for c in COMPONENTS}
        self.m = {c: torch.as_tensor(v, device=device) for c, v in m.items()}
        xs, ys, zs = self.n
        Pxm = m["Ey"] * np.conj(m["Hz"]) - m["Ez"] * np.conj(m["Hy"])
        Pym = -m["Ex"] * np.conj(m["Hz"]) + m["Ez"] * np.conj(m["Hx"])
        Pzm = m["Ex"] * np.conj(m["Hy"]) - m["Ey"] * np.conj(m["Hx"])
        self.Pm = complex(self.ds * np.sum(xs * Pxm + ys * Pym + zs * Pzm))

    def __call__(self, f: dict) -> torch.Tensor:
        m, (xs, ys, zs), ds = self.m, self.n, self.ds
        g = lambda c: f.get(c) if f.get(c) is not None else torch.zeros_like(m[c])
        Ex, Ey, Ez, Hx, Hy, Hz = (g(c) for c in COMPONENTS)
        cj = torch.conj
        am1 = 0.5 * ds * torch.sum((Ey * cj(m["Hz"]) - Ez * cj(m["Hy"])) * xs -
                                   (Ex * cj(m["Hz"]) - Ez * cj(m["Hx"])) * ys +
                                   (Ex * cj(m["Hy"]) - Ey * cj(m["Hx"])) * zs) / self.Pm
        am2 = 0.5 * ds * torch.sum((cj(m["Ey"]) * Hz - cj(m["Ez"]) * Hy) * xs -
                                   (cj(m["Ex"]) * Hz - cj(m["Ez"]) * Hx) * ys +
                                   (cj(m["Ex"]) * Hy - cj(m["Ey"]) * Hx) * zs) / np.conj(self.Pm)
        am = am1 + am2
        return 0.5 * (am * torch.conj(am)).real * self.Pm.real


# ------------------------------------------------------------ adjoint solve
class AdjointSolver:
    """Device-resident forward and adjoint CW solves for one configured
    :class:`emopt_b200.fdtd.FDTD` (grid, CPML, forward sources), with the
    design written into device material arrays and the phasors kept on the
    device.  ``monitor`` is the raw-field box the figure of merit reads."""

    def __init__(self, sim, design: PlanarDesign, monitor, base_mats, device: int = 0,
                 discrete_time: bool = False):
        self.sim = sim
        # The reference's A = diag(1j eps, ...) takes the CW frequency as 1 (in
        # units of omega).  The leapfrog's steady state obeys the same system
        # with 2 sin(dt/2)/dt in its place, so the exact derivative of the
        # discrete solution carries that factor (1 - dt^2/24 + ...).
        self.dt_factor = float(np.sin(sim.dt / 2) / (sim.dt / 2)) if discrete_time else 1.0
        self.design = design
        # one raw-field box or a list of them (e.g. a mode-match plane and the
        # six planes of the source power)
        self.monitors = list(monitor) if isinstance(monitor, (list, tuple)) else [monitor]
        self.monitor = self.monitors[0]
        self.dev = torch.device("cuda", device)
        self.device = device
        shape = (sim.Nz, sim.Ny, sim.Nx)
        self.shape = shape
        self.mats = [torch.as_tensor(np.asarray(a, dtype=np.complex128).reshape(shape),
                                     device=self.dev).contiguous() for a in base_mats]
        self.fwd = [torch.zeros(shape, dtype=torch.complex128, device=self.dev) for _ in range(6)]
        self.adj = [torch.zeros(shape, dtype=torch.complex128, device=self.dev) for _ in range(6)]
        self._t1 = torch.zeros(shape, dtype=torch.complex128, device=self.dev)
        self.last = {}

    # raw block of the six components in monitor box m
    def monitor_fields(self, which, m=None) -> torch.Tensor:
        m = self.monitor if m is None else m
        return torch.stack([a[m.i1:m.i2, m.j1:m.j2, m.k1:m.k2] for a in which])

    def _set_eps(self, eps_cols: torch.Tensor):
        d = self.design
        for c in range(3):
            i0, i1 = d.iz[c]
            blk = eps_cols[c].to(torch.complex128)
            self.mats[c][i0:i1, d.j0:d.j1, d.k0:d.k1] = blk.unsqueeze(0).expand(i1 - i0, -1, -1)

    def _solve(self, out, sources, materials_changed: bool):
        sim, h = self.sim, self.sim._libfdtd
        torch.cuda.synchronize(self.dev)
        if materials_changed:
            # registering arrays drops the handle's cached coefficients, so only
            # when they changed; the adjoint solve reuses the forward ones
            _raw.FDTD_set_mat_arrays(h, *[_ptr(a) for a in self.mats])
        for a in out:
            a.zero_()
        torch.cuda.synchronize(self.dev)
        _raw.FDTD_set_t0_arrays(h, *[_ptr(a) for a in out])
        _raw.FDTD_set_t1_arrays(h, *([_ptr(self._t1)] * 6))
        lib = _ct.libFDTD
        lib.FDTD_clear_sources(h)
        for s in sources:
            lib.FDTD_add_source(h, s.Jx, s.Jy, s.Jz, s.Mx, s.My, s.Mz,
                                s.i0, s.j0, s.k0, s.I, s.J, s.K, False)
        conv = np.ascontiguousarray(sim._conv_pts, dtype=np.int64)
        opt = _ct.SolveOptions()
        opt.Tn = int(np.int64(sim._Ncycle * 3 / 4))
        opt.Nmax = float(sim.Nmax)
        opt.rtol = float(sim._rtol)
        opt.conv_pts = conv.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
        opt.nconv = len(conv)
        opt.fixed_steps = int(sim.fixed_steps) if sim.fixed_steps else 0
        opt.materials_unchanged = 0 if materials_changed else 1
        opt.copy_t1 = 0
        res = _ct.SolveResult()
        st = lib.FDTD_solve_cw(h, ctypes.byref(opt), ctypes.byref(res))
        if st not in (_ct.FDTD_OK, _ct.FDTD_NMAX, _ct.FDTD_NONFINITE):
            raise _ct.FDTDError("FDTD_solve_cw failed: %s" % (_ct.last_error(h)[1],))
        sim._materials_dirty = True   # the handle now points at device materials
        return {"steps": res.steps, "n_main": res.n_main, "device_ms": res.device_ms,
                "total_ms": res.total_ms, "status": st}

    def forward(self, eps_cols: torch.Tensor):
        self._set_eps(eps_cols.detach())
        self.last["forward"] = self._solve(self.fwd, self.sim._sources, True)
        blocks = [self.monitor_fields(self.fwd, m) for m in self.monitors]
        return blocks[0] if len(blocks) == 1 else tuple(blocks)

    def backward(self, *grads) -> torch.Tensor:
        """Adjoint solve with the currents dF/dx of every monitor box (boxes
        that overlap add up, as the reference's adjoint source lists do,
        emopt/adjoint_method.py:1458-1486), then the overlap kernel."""
        from .fdtd import SourceArray
        h = self.sim._libfdtd
        _ct.libFDTD.FDTD_clear_sources(h)
        srcs = []
        # the currents as complex boxes (before the library's amplitude/phase
        # conversion), for solving the same adjoint problem elsewhere
        self.last_adjoint_currents = []
        for m, g in zip(self.monitors, grads):
            if g is None:
                continue
            dFdx = (torch.conj(g) / 2).detach().cpu().numpy()
            arrays = [np.ascontiguousarray(dFdx[c]).ravel() for c in range(6)]
            I, J, K = m.i2 - m.i1, m.j2 - m.j1, m.k2 - m.k1
            self.last_adjoint_currents.append(([a.reshape(I, J, K).copy() for a in arrays], m.i1, m.j1, m.k1))
            s = SourceArray(*arrays, m.i1, m.j1, m.k1, I, J, K)
            # amplitude / phase conversion of the adjoint currents (src/fdtd.cpp:1517-1576)
            _ct.libFDTD.FDTD_add_source(h, s.Jx, s.Jy, s.Jz, s.Mx, s.My, s.Mz,
                                        s.i0, s.j0, s.k0, s.I, s.J, s.K, True)
            _ct.check(h, "FDTD_add_source")
            srcs.append(s)
        self.last["adjoint"] = self._solve(self.adj, srcs, False)
        return self.grad_eps()

    def grad_eps(self) -> torch.Tensor:
        d = self.design
        nj, nk = d.j1 - d.j0, d.k1 - d.k0
        out = torch.empty((3, nj, nk), dtype=torch.float64, device=self.dev)
        fp = (ctypes.c_void_p * 3)(*[_ptr(a) for a in self.fwd[:3]])
        ap = (ctypes.c_void_p * 3)(*[_ptr(a) for a in self.adj[:3]])
        box = (ctypes.c_int * 10)(*d.box)
        msg = ctypes.create_string_buffer(256)
        Nz, Ny, Nx = self.shape
        stream = torch.cuda.current_stream(self.dev).cuda_stream
        st = _ct.libFDTD.FDTD_grad_eps(self.device, stream, fp, ap, Nx, Ny, Nz, box, 1,
                                       out.data_ptr(), msg, len(msg))
        if st != _ct.FDTD_OK:
            raise _ct.FDTDError(msg.value.decode())
        return out if self.dt_factor == 1.0 else out * self.dt_factor


class CWSolve(torch.autograd.Function):
    """eps columns (3, nj, nk) -> raw fields (6, mz, my, mx), complex128, of
    each monitor box (a tuple when the solver has several)."""

    @staticmethod
    def forward(ctx, eps_cols, solver: AdjointSolver):
        ctx.solver = solver
        return solver.forward(eps_cols)

    @staticmethod
    def backward(ctx, *grads):
        return ctx.solver.backward(*grads), None


def source_power_planes(sim):
    """The six planes one cell inside the CPML through which the source power
    is measured (emopt/fdtd.py:1555-1667), as (domain, normal axis, sign) with
    the planes on symmetric min faces ('E' / 'H') left out."""
    dx, dy, dz = sim.dx, sim.dy, sim.dz
    w = sim._w_pml
    X, Y, Z = sim.X, sim.Y, sim.Z
    xmin = w[0] + dx if w[0] > 0 else 0.0
    xmax = X - w[1] - dx if w[1] > 0 else X - dx
    ymin = w[2] + dy if w[2] > 0 else 0.0
    ymax = Y - w[3] - dy if w[3] > 0 else Y - dy
    zmin = w[4] + dz if w[4] > 0 else 0.0
    zmax = Z - w[5] - dz if w[5] > 0 else Z - dz
    D = lambda a, b, c, d, e, f: DomainCoordinates(a, b, c, d, e, f, dx, dy, dz)
    bc = sim.bc
    planes = []
    if bc[0] not in "EH":
        planes.append((D(xmin, xmin, ymin, ymax, zmin, zmax), 0, -1.0))
    planes.append((D(xmax, xmax, ymin, ymax, zmin, zmax), 0, 1.0))
    if bc[1] not in "EH":
        planes.append((D(xmin, xmax, ymin, ymin, zmin, zmax), 1, -1.0))
    planes.append((D(xmin, xmax, ymax, ymax, zmin, zmax), 1, 1.0))
    if bc[2] not in "EH":
        planes.append((D(xmin, xmax, ymin, ymax, zmin, zmin), 2, -1.0))
    planes.append((D(xmin, xmax, ymin, ymax, zmax, zmax), 2, 1.0))
    return planes


class ModeMatchObjective(torch.nn.Module):
    """Design density -> projected density -> eps -> CW solve -> mode match.

    ``forward(rho)`` returns the figure of merit (float64 scalar tensor);
    ``backward`` runs the adjoint solve.  ``plane`` is the domain of the
    monitor plane, ``mode`` the reference mode fields on it (dict of arrays
    on the interpolated grid), ``normal`` its normal."""

    def __init__(self, solver: AdjointSolver, plane: DomainCoordinates, mode: dict, normal,
                 sigma: float = 2.0, beta: float = 8.0, eta: float = 0.5, components=None):
        super().__init__()
        self.solver = solver
        self.plane = plane
        sim = solver.sim
        self.d = (sim.dx, sim.dy, sim.dz)
        self.interp_domain = solver.monitor
        ds = {0: (sim.dy, sim.dz), 1: (sim.dx, sim.dz), 2: (sim.dx, sim.dy)}[int(np.argmax(np.abs(normal)))]
        self.mm = ModeMatch(normal, ds[0], ds[1], mode, solver.dev)
        self.sigma, self.beta, self.eta = sigma, beta, eta
        self.components = components or [c for c in COMPONENTS if mode.get(c) is not None]
        self.bc = sim.bc

    def density(self, rho):
        return tanh_project(gaussian_blur(rho, self.sigma), self.beta, self.eta)

    def forward(self, rho: torch.Tensor) -> torch.Tensor:
        eps = self.solver.design.eps_columns(self.density(rho))
        raw = CWSolve.apply(eps, self.solver)
        f = {}
        for c in self.components:
            q = COMPONENTS.index(c)
            f[c] = fieldops.interp(raw[q], c, self.plane, self.interp_domain, self.bc).reshape(
                self.mm.m[c].shape)
        return self.mm(f)


class PowerNormModeMatchObjective(ModeMatchObjective):
    """The mode match divided by the source power, F = f / Psrc -- the
    reference's power-normalized figure of merit (emopt/adjoint_method.py:
    1418-1486 with fomutils.power_norm_dFdx_3D): the solver's monitors are the
    mode-match box followed by the six grown source-power planes of
    :func:`source_power_planes`, and autograd gives the adjoint currents on all
    seven boxes."""

    def __init__(self, solver: AdjointSolver, plane: DomainCoordinates, mode: dict, normal, **kw):
        super().__init__(solver, plane, mode, normal, **kw)
        sim = solver.sim
        self.planes = source_power_planes(sim)
        self.grown = solver.monitors[1:]
        if len(self.grown) != len(self.planes):
            raise ValueError("the solver needs the mode-match box and the source-power planes as monitors")

    def forward(self, rho: torch.Tensor) -> torch.Tensor:
        eps = self.solver.design.eps_columns(self.density(rho))
        raws = CWSolve.apply(eps, self.solver)
        f = {}
        for c in self.components:
            q = COMPONENTS.index(c)
            f[c] = fieldops.interp(raws[0][q], c, self.plane, self.interp_domain, self.bc).reshape(
                self.mm.m[c].shape)
        self.last_power = fieldops.source_power(raws[1:], self.planes, self.grown, self.solver.sim)
        return self.mm(f) / self.last_power


def mmi_objective(p, precision: str = "fp64", kernel: str = "auto", device: int = 0,
                  discrete_time: bool = False, power_norm: bool = False):
    """The mode-match objective of :func:`emopt_b200.problems.mmi_gradient`:
    returns (objective module, design parameters as a float64 CUDA tensor).
    ``discrete_time``: include the leapfrog's frequency factor in the gradient
    (exact for the time-stepped solution; the reference omits it).
    ``power_norm``: divide by the source power (the reference's PNF3D form)."""
    from .problems import EPS_SI, EPS_SIO2, make_solver
    sim = make_solver(p, precision=precision, kernel=kernel, device=device)
    dev = torch.device("cuda", device)
    design = planar_design(p.shape, p.dx, p.design_rect, p.design_layer, p.design_nd,
                           EPS_SIO2, EPS_SI, p.mats[:3], dev)
    k, j1, j2, i1, i2 = p.fom_plane
    d = (p.dx, p.dy, p.dz)
    plane = DomainCoordinates.from_indices(k, k + 1, j1, j2, i1, i2, *d)
    monitor = grow_domain(plane, p.shape, d)
    if power_norm:
        monitors = [monitor] + [grow_domain(dom, p.shape, d) for dom, _, _ in source_power_planes(sim)]
        solver = AdjointSolver(sim, design, monitors, p.mats, device, discrete_time)
        obj = PowerNormModeMatchObjective(solver, plane, p.fom_mode, (1, 0, 0))
    else:
        solver = AdjointSolver(sim, design, monitor, p.mats, device, discrete_time)
        obj = ModeMatchObjective(solver, plane, p.fom_mode, (1, 0, 0))
    params = torch.as_tensor(p.design_params, dtype=torch.float64, device=dev)
    return obj, params
