"""Seeded synthetic CW-FDTD workloads (the benchmark and parity configurations).

Each builder returns a :class:`Problem`: grid, wavelength, CPML widths (cells),
boundary string, solve mode, the six Yee-staggered material arrays
``(eps_x, eps_y, eps_z, mu_x, mu_y, mu_z)`` of shape ``(Nz, Ny, Nx)`` and the
current sources.  Materials are voxel-sampled at the staggered positions used
by ``FDTD.build`` (``emopt/fdtd.py:842-880``: eps_x at (x+dx/2, y, z-dz/2),
eps_y at (x, y+dy/2, z-dz/2), eps_z at (x, y, z)); mu = 1.  The same arrays
feed this package's solver and the CPU oracle, so parity is defined on them.

* :func:`waveguide` -- Si strip waveguide (0.5 x 0.22 um, eps 12.25) in SiO2
  (2.085), 4.0 x 3.0 x 2.56 um at 0.04 um (101 x 76 x 65 cells by the
  reference's ``ceil(L/d)+1`` rule), 15-cell CPML, Jy sheet at x = 0.6 um with a
  Gaussian profile (w0 = 0.4 um), 5-cycle ramp, 4000 fixed steps.
* :func:`mmi_block` -- 2x2 MMI-like block, 8.0 x 4.0 x 2.5 um at 0.025 um
  (321 x 161 x 101 cells), 20-cell CPML, 0.22 um Si layer with 0.5 um access
  waveguides and a 3 x 2 um design region whose eps comes from a seeded
  uniform[0,1] density (120 x 80), Gaussian blur (sigma = 2 cells), tanh
  projection (beta = 8, eta = 0.5), mapped linearly between 2.085 and 12.25;
  Jy Gaussian sheet in the lower input guide; run to rtol = 1e-6.
* :func:`random_box` -- small random lossy/lossless blocks for parity sweeps.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

EPS_SI = 12.25
EPS_SIO2 = 2.085
YEE_OFFSETS = ((0.5, 0.0, -0.5), (0.0, 0.5, -0.5), (0.0, 0.0, 0.0),
               (0.0, 0.5, 0.0), (0.5, 0.0, 0.0), (0.5, 0.5, -0.5))


def n_cells(L: float, d: float) -> int:
    """Grid points along an axis (``emopt/fdtd.py:252-254``)."""
    return int(np.ceil(L / d) + 1)


@dataclass
class Problem:
    name: str
    X: float
    Y: float
    Z: float
    dx: float
    dy: float
    dz: float
    wavelength: float
    w_pml: tuple = (15, 15, 15, 15, 15, 15)
    bc: str = "000"
    rtol: float = 1e-6
    fixed_steps: int | None = None
    src_ramp_time: float | None = None
    complex_eps: bool = False
    mats: tuple = ()
    sources: list = field(default_factory=list)   # [(arrays6, i0, j0, k0)]
    nconv: int | None = None
    Nmax: float | None = None

    @property
    def shape(self):
        return (n_cells(self.Z, self.dz), n_cells(self.Y, self.dy), n_cells(self.X, self.dx))

    @property
    def ncells(self):
        Nz, Ny, Nx = self.shape
        return Nz * Ny * Nx


def sample_yee(eps_fn, shape, dx, dy, dz, mu_fn=None):
    """Sample eps_fn(x, y, z) (and mu_fn) at the six staggered Yee positions."""
    Nz, Ny, Nx = shape
    out = []
    for c, (sx, sy, sz) in enumerate(YEE_OFFSETS):
        z = (np.arange(Nz) + sz) * dz
        y = (np.arange(Ny) + sy) * dy
        x = (np.arange(Nx) + sx) * dx
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        fn = eps_fn if c < 3 else mu_fn
        if fn is None:
            out.append(np.ones(shape, dtype=np.complex128))
        else:
            out.append(np.ascontiguousarray(fn(X, Y, Z), dtype=np.complex128))
    return tuple(out)


def gaussian_sheet(shape, k, dy, dz, yc, zc, w0, component=1, phase_y=0.0):
    """Current sheet on the plane x index k: exp(-((y-yc)^2+(z-zc)^2)/w0^2) in one
    J component (0,1,2 = Jx,Jy,Jz), optional linear phase exp(i phase_y y)."""
    Nz, Ny, _ = shape
    z = np.arange(Nz) * dz
    y = np.arange(Ny) * dy
    Z, Y = np.meshgrid(z, y, indexing="ij")
    prof = np.exp(-((Y - yc) ** 2 + (Z - zc) ** 2) / w0 ** 2) * np.exp(1j * phase_y * Y)
    arrays = [np.zeros((Nz, Ny, 1), dtype=np.complex128) for _ in range(6)]
    arrays[component][:, :, 0] = prof
    return (arrays, 0, 0, k)


def waveguide(fixed_steps: int | None = 4000) -> Problem:
    X, Y, Z, d = 4.0, 3.0, 2.56, 0.04
    p = Problem("waveguide_101x76x65", X, Y, Z, d, d, d, 1.55, w_pml=(15,) * 6,
                fixed_steps=fixed_steps, src_ramp_time=5 * 2 * np.pi)
    shape = p.shape
    Ny, Nz = shape[1], shape[0]
    yc, zc = (Ny - 1) * d / 2, (Nz - 1) * d / 2

    def eps(x, y, z):
        core = (np.abs(y - yc) <= 0.25) & (np.abs(z - zc) <= 0.11)
        return np.where(core, EPS_SI, EPS_SIO2)

    p.mats = sample_yee(eps, shape, d, d, d)
    p.sources = [gaussian_sheet(shape, int(0.6 / d), d, d, yc, zc, 0.4)]
    return p


def projected_density(rho: np.ndarray, sigma: float = 2.0, beta: float = 8.0,
                      eta: float = 0.5) -> np.ndarray:
    """Gaussian blur then tanh projection of a density in [0, 1]."""
    from scipy.ndimage import gaussian_filter
    r = gaussian_filter(rho, sigma=sigma, mode="nearest")
    num = np.tanh(beta * eta) + np.tanh(beta * (r - eta))
    den = np.tanh(beta * eta) + np.tanh(beta * (1 - eta))
    return num / den


def mmi_geometry(rho_design: np.ndarray, shape, d):
    """eps(x, y, z) of the 2x2 MMI-like block for a projected design density
    sampled on a regular grid over the 3 x 2 um design region."""
    Nz, Ny, Nx = shape
    xc, yc, zc = (Nx - 1) * d / 2, (Ny - 1) * d / 2, (Nz - 1) * d / 2
    xd0, xd1, yd0, yd1 = xc - 1.5, xc + 1.5, yc - 1.0, yc + 1.0
    nxd, nyd = rho_design.shape

    def eps(x, y, z):
        in_slab = np.abs(z - zc) <= 0.11
        guides = ((np.abs(y - (yc - 0.5)) <= 0.25) | (np.abs(y - (yc + 0.5)) <= 0.25)) & \
                 ((x < xd0) | (x > xd1))
        in_design = (x >= xd0) & (x <= xd1) & (y >= yd0) & (y <= yd1)
        ix = np.clip(((x - xd0) / (xd1 - xd0) * nxd).astype(int), 0, nxd - 1)
        iy = np.clip(((y - yd0) / (yd1 - yd0) * nyd).astype(int), 0, nyd - 1)
        e_design = EPS_SIO2 + (EPS_SI - EPS_SIO2) * rho_design[ix, iy]
        e = np.where(guides, EPS_SI, EPS_SIO2)
        e = np.where(in_design, e_design, e)
        return np.where(in_slab, e, EPS_SIO2)

    return eps


def mmi_block(seed: int = 0, nd=(120, 80), rtol: float = 1e-6,
              fixed_steps: int | None = None) -> Problem:
    X, Y, Z, d = 8.0, 4.0, 2.5, 0.025
    p = Problem("mmi_321x161x101", X, Y, Z, d, d, d, 1.55, w_pml=(20,) * 6, rtol=rtol,
                fixed_steps=fixed_steps)
    shape = p.shape
    rng = np.random.default_rng(seed)
    rho = projected_density(rng.uniform(0.0, 1.0, nd))
    p.mats = sample_yee(mmi_geometry(rho, shape, d), shape, d, d, d)
    Nz, Ny, Nx = shape
    yc, zc = (Ny - 1) * d / 2, (Nz - 1) * d / 2
    p.sources = [gaussian_sheet(shape, int(1.0 / d), d, d, yc - 0.5, zc, 0.35)]
    p.design_density = rho
    return p


def mmi_gradient(seed: int = 1, nd=(80, 80), d: float = 0.025, w_pml: int = 20,
                 rtol: float = 1e-6, fixed_steps: int | None = None) -> Problem:
    """Differentiation workload: the MMI block with a seeded uniform[0,1]
    design density on an ``nd`` grid (blur sigma = 2 cells, tanh projection
    beta = 8, eta = 0.5), the Jy Gaussian sheet in the lower input guide and a
    mode-match figure of merit on the output plane x = 7.0 um against a fixed
    Gaussian (w0 = 0.35 um) centred on the upper output guide: Ey = G,
    Hz = n_clad G with n_clad = sqrt(2.085) (not power-normalised).

    Extra attributes: ``design_params`` (the density), ``design_rect`` (um),
    ``design_layer`` (zc, half height), ``fom_plane`` (indices k, j1, j2, i1,
    i2 of the x-normal plane, the part outside the CPML) and ``fom_mode``
    (dict of mode fields on it).
    The default is the full 321 x 161 x 101 grid; ``d = 0.05, w_pml = 10``
    gives a 161 x 81 x 51 version of the same geometry for tests."""
    X, Y, Z = 8.0, 4.0, 2.5
    p = Problem(f"mmi_grad_d{d}", X, Y, Z, d, d, d, 1.55, w_pml=(w_pml,) * 6, rtol=rtol,
                fixed_steps=fixed_steps)
    shape = p.shape
    Nz, Ny, Nx = shape
    rng = np.random.default_rng(seed)
    p.design_params = rng.uniform(0.0, 1.0, nd)
    rho = projected_density(p.design_params)
    p.mats = sample_yee(mmi_geometry(rho, shape, d), shape, d, d, d)
    xc, yc, zc = (Nx - 1) * d / 2, (Ny - 1) * d / 2, (Nz - 1) * d / 2
    p.sources = [gaussian_sheet(shape, int(round(1.0 / d)), d, d, yc - 0.5, zc, 0.35)]
    p.design_rect = (xc - 1.5, xc + 1.5, yc - 1.0, yc + 1.0)
    p.design_layer = (zc, 0.11)
    p.design_nd = tuple(nd)
    k = int(round(7.0 / d))
    p.fom_plane = (k, w_pml, Ny - w_pml, w_pml, Nz - w_pml)   # outside the CPML
    z = np.arange(w_pml, Nz - w_pml) * d
    y = np.arange(w_pml, Ny - w_pml) * d
    Zg, Yg = np.meshgrid(z, y, indexing="ij")
    G = np.exp(-((Yg - (yc + 0.5)) ** 2 + (Zg - zc) ** 2) / 0.35 ** 2).astype(np.complex128)
    p.fom_mode = {"Ey": G[:, :, None], "Hz": np.sqrt(EPS_SIO2) * G[:, :, None]}
    return p


def design_eps(p: Problem, params: np.ndarray):
    """The three eps arrays of :func:`mmi_gradient`'s geometry for a design density."""
    Nz, Ny, Nx = p.shape
    mats = sample_yee(mmi_geometry(projected_density(params), p.shape, p.dx), p.shape,
                      p.dx, p.dy, p.dz)
    return mats[:3]


def random_box(seed: int, shape=(9, 11, 14), d=0.04, w_pml=(3, 4, 3, 2, 3, 4), bc="000",
               complex_eps=False, fixed_steps: int | None = 120, mu_random=False,
               n_sources=1, rtol=1e-6, edge_source=False) -> Problem:
    """Small random medium with random complex current boxes (parity sweeps).

    ``edge_source``: one more current box over the last 4 x cells of a few rows
    and planes (drawn after the others), so that sources reach the x-max face.
    """
    Nz, Ny, Nx = shape
    # lengths half a cell short of (N-1) d so that ceil(L/d)+1 gives back N exactly
    X, Y, Z = (Nx - 1.5) * d, (Ny - 1.5) * d, (Nz - 1.5) * d
    p = Problem(f"box_{Nx}x{Ny}x{Nz}_s{seed}", X, Y, Z, d, d, d, 1.55, w_pml=tuple(w_pml), bc=bc,
                fixed_steps=fixed_steps, complex_eps=complex_eps, rtol=rtol,
                src_ramp_time=5 * 2 * np.pi)
    assert p.shape == tuple(shape), (p.shape, shape)
    rng = np.random.default_rng(seed)
    mats = []
    for c in range(6):
        if c < 3:
            v = 2.0 + 3.0 * rng.random(shape)
            if complex_eps:
                v = v + 0.3j * rng.random(shape)
        else:
            v = (1.0 + 0.5 * rng.random(shape)) if mu_random else np.ones(shape)
        mats.append(np.ascontiguousarray(v, dtype=np.complex128))
    p.mats = tuple(mats)
    for _ in range(n_sources):
        I, J, K = (int(rng.integers(1, max(2, Nz // 2))), int(rng.integers(1, max(2, Ny // 2))),
                   int(rng.integers(1, max(2, Nx // 2))))
        i0, j0, k0 = (int(rng.integers(0, Nz - I + 1)), int(rng.integers(0, Ny - J + 1)),
                      int(rng.integers(0, Nx - K + 1)))
        arrays = [rng.standard_normal((I, J, K)) + 1j * rng.standard_normal((I, J, K))
                  for _ in range(6)]
        p.sources.append((arrays, i0, j0, k0))
    if edge_source:
        I, J, K = max(1, Nz // 2), max(1, Ny // 2), min(4, Nx)
        arrays = [rng.standard_normal((I, J, K)) + 1j * rng.standard_normal((I, J, K))
                  for _ in range(6)]
        p.sources.append((arrays, int(rng.integers(0, Nz - I + 1)), int(rng.integers(0, Ny - J + 1)),
                          Nx - K))
    return p


def make_solver(p: Problem, precision: str = "fp64", kernel: str = "auto", device=None):
    """Configure an ``emopt_b200.fdtd.FDTD`` for problem ``p`` (sources added, not solved)."""
    from .fdtd import FDTD
    from .misc import DomainCoordinates
    sim = FDTD(p.X, p.Y, p.Z, p.dx, p.dy, p.dz, p.wavelength, rtol=p.rtol, nconv=p.nconv,
               complex_eps=p.complex_eps, precision=precision, kernel=kernel, device=device)
    assert (sim.Nz, sim.Ny, sim.Nx) == p.shape
    sim.set_pml_cells(p.w_pml)
    if p.bc != "000":
        sim.bc = p.bc
    if p.src_ramp_time is not None:
        sim._src_T = p.src_ramp_time
        from .fdtd_ctypes import libFDTD
        libFDTD.FDTD_set_source_properties(sim._libfdtd, sim._src_T, sim._src_min)
    if p.Nmax is not None:
        sim.Nmax = p.Nmax
    sim.fixed_steps = p.fixed_steps
    sim.set_material_arrays(p.mats[:3], p.mats[3:])
    for arrays, i0, j0, k0 in p.sources:
        I, J, K = arrays[0].shape
        dom = DomainCoordinates.from_indices(k0, k0 + K, j0, j0 + J, i0, i0 + I, p.dx, p.dy, p.dz)
        sim.set_sources(tuple(arrays), dom)
    return sim
