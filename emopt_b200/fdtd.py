"""Drop-in ``FDTD`` solver class backed by the B200 CUDA library.

``emopt_b200.fdtd.FDTD`` keeps the public interface of ``emopt.fdtd.FDTD``
(``emopt/fdtd.py:93-1730``): the same constructor, properties and methods,
with the same parameter derivation (grid-size rule, time step, CPML defaults,
source ramp, step budget, convergence probes) and the same array semantics of
the library it drives.  Differences, all consequences of running on one GPU
instead of MPI ranks:

* one process owns the whole grid, so arrays are plain numpy arrays in the
  natural ``[Nz, Ny, Nx]`` order (the reference's one-rank layout) and the
  PETSc/MPI plumbing (``GhostComm``, scatters, barriers) disappears;
* ``solve_forward``/``solve_adjoint`` call ``FDTD_solve_cw``, which runs the
  whole time loop of ``FDTD.__solve`` (``emopt/fdtd.py:994-1194``) on the
  device and returns the complex steady-state fields;
* extra keyword arguments: ``precision`` (``'fp64'`` = reference arithmetic,
  ``'fp32'`` = float32 storage), ``kernel`` (one of ``FDTD.KERNELS``,
  default ``'auto'``) and
  ``device`` (CUDA device index).

Materials are any objects with ``get_values(k1, k2, j1, j2, i1, i2, sx, sy, sz,
arr)`` (the ``emopt.grid.Material3D`` protocol, ``emopt/grid.py:762``); see
``emopt_b200.grid`` for simple implementations.
"""
from __future__ import annotations

import ctypes
from math import pi

import numpy as np

from . import fdtd_ctypes as _ct
from .fdtd_ctypes import libFDTD
from .misc import DomainCoordinates, FieldComponent, warning_message


def derive_parameters(X, Y, Z, dx, dy, dz, wavelength, min_rindex=1.0, nconv=10, Sc=0.95):
    """Grid and timing parameters of a solve (``emopt/fdtd.py:248-413``, one rank).

    Returns a dict with Nx, Ny, Nz, the physical extents X, Y, Z (snapped to the
    grid), R, dt, Nlambda, Ncycle, src_T, src_min, Nmax, Tn and conv_pts.
    """
    Nx = int(np.ceil(X / dx) + 1)
    Ny = int(np.ceil(Y / dy) + 1)
    Nz = int(np.ceil(Z / dz) + 1)
    R = wavelength / (2 * pi)
    dt = Sc * np.min([dx, dy, dz]) / R / np.sqrt(3) * min_rindex
    Nlambda = wavelength / np.min([dx, dy, dz]) / min_rindex
    Ncycle = Nlambda * np.sqrt(3)
    n = Nx * Ny * Nz
    return {
        "Nx": Nx, "Ny": Ny, "Nz": Nz,
        "X": dx * (Nx - 1), "Y": dy * (Ny - 1), "Z": dz * (Nz - 1),
        "R": R, "dt": dt, "Nlambda": Nlambda, "Ncycle": Ncycle,
        "src_T": Ncycle * 20.0 * dt, "src_min": 1e-4, "Nmax": Nlambda * 500,
        "Tn": int(np.int64(Ncycle * 3 / 4)),
        "conv_pts": np.arange(0, n, int(n / int(nconv))),
    }


class SourceArray:
    """Cropped source block handed to the library (``emopt/fdtd.py:49-91``)."""

    def __init__(self, Jx, Jy, Jz, Mx, My, Mz, i0, j0, k0, I, J, K):
        self.Jx, self.Jy, self.Jz = Jx, Jy, Jz
        self.Mx, self.My, self.Mz = Mx, My, Mz
        self.i0, self.j0, self.k0 = i0, j0, k0
        self.I, self.J, self.K = I, J, K


class MaxwellSolver:
    """Minimal form of ``emopt.simulation.MaxwellSolver`` (``emopt/simulation.py:20-175``)."""

    def __init__(self, ndims):
        self._field_domains = []
        self._saved_fields = []
        self._source_power = 0.0
        self._ndims = ndims

    @property
    def field_domains(self):
        return self._field_domains

    @field_domains.setter
    def field_domains(self, domains):
        self._field_domains = domains

    @property
    def saved_fields(self):
        return self._saved_fields

    @property
    def source_power(self):
        return self._source_power

    @property
    def ndims(self):
        return self._ndims


class FDTD(MaxwellSolver):
    """3D continuous-wave FDTD solver (drop-in for ``emopt.fdtd.FDTD``)."""

    # time-stepping kernels of FDTD_solve_cw (include/emopt_fdtd.h, FDTD_set_kernel)
    KERNELS = {"auto": 0, "scalar": 1, "fused": 3, "vector": 5, "split": 6}

    def __init__(self, X, Y, Z, dx, dy, dz, wavelength, rtol=1e-6, nconv=None,
                 min_rindex=1.0, complex_eps=False, dist_method="auto",
                 precision="fp64", kernel="auto", device=None):
        super().__init__(3)
        if nconv is None:
            nconv = 10
        elif nconv < 2:
            warning_message("Number of convergence test points (nconv) is likely too low.",
                            "emopt_b200.fdtd")
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if kernel not in self.KERNELS:
            raise ValueError("kernel must be one of %s" % (sorted(self.KERNELS),))
        self._dx, self._dy, self._dz = dx, dy, dz
        prm = derive_parameters(X, Y, Z, dx, dy, dz, wavelength, min_rindex, nconv)
        Nx, Ny, Nz = prm["Nx"], prm["Ny"], prm["Nz"]
        self._Nx, self._Ny, self._Nz = Nx, Ny, Nz
        self._X, self._Y, self._Z = prm["X"], prm["Y"], prm["Z"]
        self._wavelength = wavelength
        self._R = prm["R"]
        self._Sc = 0.95
        self._min_rindex = min_rindex
        self._dt = prm["dt"]
        self._precision = precision
        self._kernel = kernel

        I, J, K = Nz, Ny, Nx
        npad = (K + 2) * (J + 2) * (I + 2)
        self._Ex = np.zeros(npad); self._Ey = np.zeros(npad); self._Ez = np.zeros(npad)
        self._Hx = np.zeros(npad); self._Hy = np.zeros(npad); self._Hz = np.zeros(npad)
        n = I * J * K
        z = lambda: np.zeros(n, dtype=np.complex128)
        self._eps_x, self._eps_y, self._eps_z = z(), z(), z()
        self._mu_x, self._mu_y, self._mu_z = z(), z(), z()
        for a in (self._eps_x, self._eps_y, self._eps_z, self._mu_x, self._mu_y, self._mu_z):
            a[:] = 1.0
        self._Ex_fwd_t0, self._Ey_fwd_t0, self._Ez_fwd_t0 = z(), z(), z()
        self._Hx_fwd_t0, self._Hy_fwd_t0, self._Hz_fwd_t0 = z(), z(), z()
        self._Ex_fwd_t1, self._Ey_fwd_t1, self._Ez_fwd_t1 = z(), z(), z()
        self._Hx_fwd_t1, self._Hy_fwd_t1, self._Hz_fwd_t1 = z(), z(), z()
        self._Ex_adj_t0, self._Ey_adj_t0, self._Ez_adj_t0 = z(), z(), z()
        self._Hx_adj_t0, self._Hy_adj_t0, self._Hz_adj_t0 = z(), z(), z()
        self._Ex_adj_t1, self._Ey_adj_t1, self._Ez_adj_t1 = z(), z(), z()
        self._Hx_adj_t1, self._Hy_adj_t1, self._Hz_adj_t1 = z(), z(), z()

        h = libFDTD.FDTD_new()
        self._libfdtd = h
        self._pinned = []
        code, msg = _ct.last_error(h)
        if code == _ct.FDTD_ERR_NODEVICE:
            libFDTD.FDTD_delete(h)
            self._libfdtd = None
            raise _ct.FDTDError("emopt_b200 needs a CUDA device: " + msg)
        # the materials go to the GPU and the forward phasors come back on every
        # solve: page-lock those host arrays once so the copies run at full DMA
        # speed (pageable copies are staged through a driver buffer, 2-3x slower)
        self._pin([self._eps_x, self._eps_y, self._eps_z, self._mu_x, self._mu_y, self._mu_z,
                   self._Ex_fwd_t0, self._Ey_fwd_t0, self._Ez_fwd_t0,
                   self._Hx_fwd_t0, self._Hy_fwd_t0, self._Hz_fwd_t0])
        self._device = None if device is None else int(device)
        # materials that can be evaluated on the GPU are built there and stay
        # there (build/update); False keeps the host evaluation
        self.device_materials = True
        self._dev_mats = None
        self._host_mats_stale = False
        if device is not None and libFDTD.FDTD_set_device(h, int(device)) != _ct.FDTD_OK:
            raise _ct.FDTDError(_ct.last_error(h)[1])
        libFDTD.FDTD_set_wavelength(h, wavelength)
        libFDTD.FDTD_set_physical_dims(h, X, Y, Z, dx, dy, dz)
        libFDTD.FDTD_set_grid_dims(h, Nx, Ny, Nz)
        libFDTD.FDTD_set_local_grid(h, 0, 0, 0, K, J, I)
        libFDTD.FDTD_set_dt(h, self._dt)
        libFDTD.FDTD_set_field_arrays(h, self._Ex, self._Ey, self._Ez,
                                      self._Hx, self._Hy, self._Hz)
        libFDTD.FDTD_set_mat_arrays(h, self._eps_x, self._eps_y, self._eps_z,
                                    self._mu_x, self._mu_y, self._mu_z)
        libFDTD.FDTD_set_complex_eps(h, complex_eps)
        libFDTD.FDTD_set_precision(h, 32 if precision == "fp32" else 64)
        libFDTD.FDTD_set_kernel(h, self.KERNELS[kernel])

        # CPML defaults (emopt/fdtd.py:368-390)
        w_pml = 15
        self._w_pml = [w_pml * dx, w_pml * dx, w_pml * dy, w_pml * dy, w_pml * dz, w_pml * dz]
        self._w_pml_xmin = self._w_pml_xmax = w_pml
        self._w_pml_ymin = self._w_pml_ymax = w_pml
        self._w_pml_zmin = self._w_pml_zmax = w_pml
        self._pml_sigma, self._pml_alpha, self._pml_kappa, self._pml_pow = 3.0, 0.0, 1.0, 3.0
        libFDTD.FDTD_set_pml_widths(h, w_pml, w_pml, w_pml, w_pml, w_pml, w_pml)
        libFDTD.FDTD_set_pml_properties(h, self._pml_sigma, self._pml_alpha,
                                        self._pml_kappa, self._pml_pow)
        libFDTD.FDTD_build_pml(h)
        _ct.check(h, "FDTD_build_pml")

        # source timing and step budget (emopt/fdtd.py:393-402)
        self._Nlambda = prm["Nlambda"]
        self._Ncycle = prm["Ncycle"]
        self._src_T = prm["src_T"]
        self._src_min = prm["src_min"]
        self.Nmax = prm["Nmax"]
        libFDTD.FDTD_set_source_properties(h, self._src_T, self._src_min)
        self._rtol = rtol
        self.verbose = 2

        # convergence probes: indices into the padded local E arrays (:411-413)
        self._conv_pts = prm["conv_pts"]
        self._nconv = len(self._conv_pts)

        self._sources = []
        self._adj_sources = []
        self._bc = ["0", "0", "0"]
        libFDTD.FDTD_set_bc(h, "".join(self._bc).encode("ascii"))
        self._eps = None
        self._mu = None
        self._materials_dirty = True
        self.forward_count = 0
        self.adjoint_count = 0
        self.last_solve = None
        self.fixed_steps = None
        # True: a solve whose convergence probe sees NaN/Inf stops there (status
        # NONFINITE) instead of running on to Nmax as the reference does
        self.stop_nonfinite = False

    # at most this many bytes of one solver's host arrays are page-locked
    PIN_LIMIT = 4 << 30

    def _pin(self, arrays):
        if sum(a.nbytes for a in arrays) > self.PIN_LIMIT:
            return
        for a in arrays:
            if libFDTD.FDTD_host_register(a.ctypes.data, a.nbytes) != _ct.FDTD_OK:
                break
            self._pinned.append((a.ctypes.data, a))

    def __del__(self):
        h = getattr(self, "_libfdtd", None)
        if h:
            libFDTD.FDTD_delete(h)
            self._libfdtd = None
        for ptr, _ in getattr(self, "_pinned", []):
            libFDTD.FDTD_host_unregister(ptr)
        self._pinned = []

    # ------------------------------------------------------------ properties
    @property
    def wavelength(self):
        return self._wavelength

    @wavelength.setter
    def wavelength(self, wlen):
        if wlen <= 0:
            raise ValueError("Wavelength must be >= 0.")
        self._wavelength = wlen
        self._R = wlen / 2 / pi
        libFDTD.FDTD_set_wavelength(self._libfdtd, wlen)
        ds = np.min([self._dx, self._dy, self._dz])
        self._dt = self._Sc * ds / self._R / np.sqrt(3) * self._min_rindex
        libFDTD.FDTD_set_dt(self._libfdtd, self._dt)

    X = property(lambda s: s._X)
    Y = property(lambda s: s._Y)
    Z = property(lambda s: s._Z)
    dx = property(lambda s: s._dx)
    dy = property(lambda s: s._dy)
    dz = property(lambda s: s._dz)
    Nx = property(lambda s: s._Nx)
    Ny = property(lambda s: s._Ny)
    Nz = property(lambda s: s._Nz)
    eps = property(lambda s: s._eps)
    mu = property(lambda s: s._mu)
    dt = property(lambda s: s._dt)
    Nlambda = property(lambda s: s._Nlambda)
    Ncycle = property(lambda s: s._Ncycle)
    precision = property(lambda s: s._precision)

    @property
    def courant_num(self):
        return self._Sc

    @courant_num.setter
    def courant_num(self, Sc):
        if Sc > 1.0:
            warning_message("A courant number greater than 1 will lead to instability.",
                            "emopt_b200.fdtd")
        self._Sc = Sc
        ds = np.min([self._dx, self._dy, self._dz])
        self._dt = self._Sc * ds / self._R / np.sqrt(3) * self._min_rindex
        libFDTD.FDTD_set_dt(self._libfdtd, self._dt)

    @property
    def rtol(self):
        return self._rtol

    @rtol.setter
    def rtol(self, rtol):
        if rtol <= 0:
            raise ValueError("Relative tolerance must be greater than zero.")
        self._rtol = rtol

    @property
    def src_min_value(self):
        return self._src_min

    @src_min_value.setter
    def src_min_value(self, new_min):
        if new_min <= 0:
            raise ValueError("Minimum source value must be greater than zero.")
        self._src_min = new_min
        libFDTD.FDTD_set_source_properties(self._libfdtd, self._src_T, self._src_min)

    @property
    def src_ramp_time(self):
        return self._src_T

    @src_ramp_time.setter
    def src_ramp_time(self, new_T):
        if new_T <= 0:
            raise ValueError("Source ramp time must be greater than zero.")
        if new_T <= self._Nlambda * 5:
            warning_message("Source ramp time is likely too short. Simulations may not converge.",
                            "emopt_b200.fdtd")
        self._src_T = new_T
        libFDTD.FDTD_set_source_properties(self._libfdtd, self._src_T, self._src_min)

    @property
    def bc(self):
        return "".join(self._bc)

    @bc.setter
    def bc(self, newbc):
        if len(newbc) != 3:
            raise ValueError("Incorrect number of boundary conditions specified!")
        for b in newbc:
            if b not in "0EHP":
                raise ValueError("Unrecognized boundary condition: %s" % (b))
            if b == "P":
                raise NotImplementedError("Periodic boundary conditions not yet implemented")
        self._bc = list(newbc)
        libFDTD.FDTD_set_bc(self._libfdtd, "".join(self._bc).encode("ascii"))

    @property
    def w_pml(self):
        return self._w_pml

    @w_pml.setter
    def w_pml(self, w_pml):
        if len(w_pml) != 6:
            raise ValueError("Incorrect number of pml widths specified. You must specify 6 "
                             "widths (xmin, xmax, ymin, ymax, zmin, zmax).")
        dx, dy, dz = self._dx, self._dy, self._dz
        self._w_pml_xmin = int(w_pml[0] / dx)
        self._w_pml_xmax = int(w_pml[1] / dx)
        self._w_pml_ymin = int(w_pml[2] / dy)
        self._w_pml_ymax = int(w_pml[3] / dy)
        self._w_pml_zmin = int(w_pml[4] / dz)
        self._w_pml_zmax = int(w_pml[5] / dz)
        self._w_pml = [self._w_pml_xmin * dx, self._w_pml_xmax * dx, self._w_pml_ymin * dy,
                       self._w_pml_ymax * dy, self._w_pml_zmin * dz, self._w_pml_zmax * dz]
        libFDTD.FDTD_set_pml_widths(self._libfdtd, self._w_pml_xmin, self._w_pml_xmax,
                                    self._w_pml_ymin, self._w_pml_ymax,
                                    self._w_pml_zmin, self._w_pml_zmax)
        libFDTD.FDTD_build_pml(self._libfdtd)
        _ct.check(self._libfdtd, "FDTD_build_pml")
        self._materials_dirty = True

    def set_pml_cells(self, widths):
        """Set the six CPML widths directly in cells (xmin, xmax, ymin, ymax, zmin, zmax)."""
        d = [self._dx, self._dx, self._dy, self._dy, self._dz, self._dz]
        self.w_pml = [(int(w) + 0.5) * di for w, di in zip(widths, d)]

    w_pml_xmin = property(lambda s: s._w_pml_xmin)
    w_pml_xmax = property(lambda s: s._w_pml_xmax)
    w_pml_ymin = property(lambda s: s._w_pml_ymin)
    w_pml_ymax = property(lambda s: s._w_pml_ymax)
    w_pml_zmin = property(lambda s: s._w_pml_zmin)
    w_pml_zmax = property(lambda s: s._w_pml_zmax)
    X_real = property(lambda s: s._X - s._w_pml[0] - s._w_pml[1])
    Y_real = property(lambda s: s._Y - s._w_pml[2] - s._w_pml[3])
    Z_real = property(lambda s: s._Z - s._w_pml[4] - s._w_pml[5])

    # ------------------------------------------------------------- materials
    def set_materials(self, eps, mu):
        self._eps = eps
        self._mu = mu

    def set_material_arrays(self, eps_xyz, mu_xyz):
        """Set the six Yee-staggered material arrays directly, each ``(Nz, Ny, Nx)``.

        Equivalent to what ``build`` samples from material objects
        (``emopt/fdtd.py:842-880``); used when the arrays come from elsewhere.
        """
        if self._dev_mats is not None:
            self._register_host_materials()
        targets = (self._eps_x, self._eps_y, self._eps_z, self._mu_x, self._mu_y, self._mu_z)
        for dst, src in zip(targets, list(eps_xyz) + list(mu_xyz)):
            dst[:] = np.asarray(src, dtype=np.complex128).ravel()
        self._materials_dirty = True

    # Yee sampling offsets (sx, sy, sz) of eps_x, eps_y, eps_z, mu_x, mu_y, mu_z
    # (emopt/fdtd.py:842-880)
    _YEE = ((0.5, 0.0, -0.5), (0.0, 0.5, -0.5), (0.0, 0.0, 0.0),
            (0.0, 0.5, 0.0), (0.5, 0.0, 0.0), (0.5, 0.5, -0.5))

    def _device_capable(self):
        """Can both materials be evaluated on the GPU (layered primitives,
        constants)?"""
        from .grid import ConstantMaterial3D, StructuredMaterial3D
        ok = (StructuredMaterial3D, ConstantMaterial3D)
        return (getattr(self, "device_materials", False) and isinstance(self._eps, ok)
                and isinstance(self._mu, ok))

    def _torch_device(self):
        import torch
        return torch.device("cuda", self._device if self._device is not None else torch.cuda.current_device())

    def _register_host_materials(self):
        libFDTD.FDTD_set_mat_arrays(self._libfdtd, self._eps_x, self._eps_y, self._eps_z,
                                    self._mu_x, self._mu_y, self._mu_z)
        self._dev_mats = None
        self._host_mats_stale = False

    def _sync_host_materials(self):
        """Bring the host material arrays up to date with the device-built ones."""
        if getattr(self, "_dev_mats", None) is not None and self._host_mats_stale:
            targets = (self._eps_x, self._eps_y, self._eps_z, self._mu_x, self._mu_y, self._mu_z)
            for dst, src in zip(targets, self._dev_mats):
                dst[:] = src.reshape(-1).cpu().numpy()
            self._host_mats_stale = False

    def _build_device(self):
        """Evaluate the six Yee-staggered arrays on the GPU, keep them there and
        hand their device addresses to the library: the solve reads them in
        place, nothing crosses PCIe (the host arrays follow on demand)."""
        K, J, I = self._Nx, self._Ny, self._Nz
        dev = self._torch_device()
        mats = []
        for q, (sx, sy, sz) in enumerate(self._YEE):
            m = self._eps if q < 3 else self._mu
            mats.append(m.get_values(0, K, 0, J, 0, I, sx=sx, sy=sy, sz=sz, device=dev).contiguous())
        self._dev_mats = mats
        _ct.raw.FDTD_set_mat_arrays(self._libfdtd, *[a.data_ptr() for a in mats])
        self._host_mats_stale = True
        self._materials_dirty = True

    def build(self):
        """Sample eps/mu at the Yee positions (``emopt/fdtd.py:842-880``); on
        the GPU, kept there, when both materials can be evaluated there."""
        if FDTD._device_capable(self):
            self._build_device()
            return
        if getattr(self, "_dev_mats", None) is not None:
            self._register_host_materials()
        K, J, I = self._Nx, self._Ny, self._Nz
        eps, mu = self._eps, self._mu
        eps.get_values(0, K, 0, J, 0, I, sx=0.5, sy=0.0, sz=-0.5, arr=self._eps_x)
        eps.get_values(0, K, 0, J, 0, I, sx=0.0, sy=0.5, sz=-0.5, arr=self._eps_y)
        eps.get_values(0, K, 0, J, 0, I, sx=0.0, sy=0.0, sz=0.0, arr=self._eps_z)
        mu.get_values(0, K, 0, J, 0, I, sx=0.0, sy=0.5, sz=0.0, arr=self._mu_x)
        mu.get_values(0, K, 0, J, 0, I, sx=0.5, sy=0.0, sz=0.0, arr=self._mu_y)
        mu.get_values(0, K, 0, J, 0, I, sx=0.5, sy=0.5, sz=-0.5, arr=self._mu_z)
        self._materials_dirty = True

    def update(self, bbox=None):
        """Re-sample eps/mu, everywhere or inside ``bbox`` (``emopt/fdtd.py:882-992``)."""
        if bbox is None:
            self.build()
            return
        d = DomainCoordinates(bbox[0], bbox[1], bbox[2], bbox[3], bbox[4], bbox[5],
                              self._dx, self._dy, self._dz)
        i1, i2 = max(d.i1, 0), min(d.i2, self._Nz)
        j1, j2 = max(d.j1, 0), min(d.j2, self._Ny)
        k1, k2 = max(d.k1, 0), min(d.k2, self._Nx)
        if i1 >= i2 or j1 >= j2 or k1 >= k2:
            return
        if getattr(self, "_dev_mats", None) is not None and FDTD._device_capable(self):
            # re-sample the box on the GPU into the resident arrays
            dev = self._torch_device()
            for q, (sx, sy, sz) in enumerate(self._YEE):
                m = self._eps if q < 3 else self._mu
                self._dev_mats[q][i1:i2, j1:j2, k1:k2] = m.get_values(k1, k2, j1, j2, i1, i2, sx=sx, sy=sy,
                                                                       sz=sz, device=dev)
            self._host_mats_stale = True
            self._materials_dirty = True
            return
        FDTD._sync_host_materials(self)
        temp = np.zeros((i2 - i1, j2 - j1, k2 - k1), dtype=np.complex128)
        shape = (self._Nz, self._Ny, self._Nx)
        spec = ((self._eps, self._eps_x, (0.5, 0.0, -0.5)), (self._eps, self._eps_y, (0.0, 0.5, -0.5)),
                (self._eps, self._eps_z, (0.0, 0.0, 0.0)), (self._mu, self._mu_x, (0.0, 0.5, 0.0)),
                (self._mu, self._mu_y, (0.5, 0.0, 0.0)), (self._mu, self._mu_z, (0.5, 0.5, -0.5)))
        for mat, arr, (sx, sy, sz) in spec:
            mat.get_values(k1, k2, j1, j2, i1, i2, sx=sx, sy=sy, sz=sz, arr=temp)
            arr.reshape(shape)[i1:i2, j1:j2, k1:k2] = temp
        self._materials_dirty = True

    # --------------------------------------------------------------- sources
    def _domain_overlap(self, domain):
        # whole grid is local: overlap of the domain with [0, N) on each axis
        # (emopt/fdtd.py:658-708 with k0 = j0 = i0 = 0)
        I, J, K = self._Nz, self._Ny, self._Nx
        if 0 >= domain.i2 or I <= domain.i1 or 0 >= domain.j2 or J <= domain.j1 \
                or 0 >= domain.k2 or K <= domain.k1:
            return None, None, None, None
        imax, jmax, kmax = min(I, domain.i2), min(J, domain.j2), min(K, domain.k2)
        imin, jmin, kmin = max(0, domain.i1), max(0, domain.j1), max(0, domain.k1)
        return ((imin, jmin, kmin), (imin, jmin, kmin),
                (imin - domain.i1, jmin - domain.j1, kmin - domain.k1),
                (imax - imin, jmax - jmin, kmax - kmin))

    def _set_sources(self, src, domain, adjoint=False):
        Jx, Jy, Jz, Mx, My, Mz = src
        g, l, d, sizes = self._domain_overlap(domain)
        if g is None:
            return
        sl = (slice(d[0], d[0] + sizes[0]), slice(d[1], d[1] + sizes[1]),
              slice(d[2], d[2] + sizes[2]))
        cp = [np.copy(np.asarray(a, dtype=np.complex128)[sl]).ravel() for a in (Jx, Jy, Jz, Mx, My, Mz)]
        s = SourceArray(*cp, l[0], l[1], l[2], sizes[0], sizes[1], sizes[2])
        (self._adj_sources if adjoint else self._sources).append(s)
        libFDTD.FDTD_add_source(self._libfdtd, s.Jx, s.Jy, s.Jz, s.Mx, s.My, s.Mz,
                                s.i0, s.j0, s.k0, s.I, s.J, s.K, True)
        _ct.check(self._libfdtd, "FDTD_add_source")

    def set_sources(self, src, domain, mindex=0):
        """Add a source (six arrays, or an object with ``get_source``) in ``domain``."""
        if hasattr(src, "get_source"):
            src = src.get_source(mindex, self._dx, self._dy, self._dz)
        self._set_sources(src, domain, adjoint=False)

    def set_adjoint_sources(self, src):
        self.clear_adjoint_sources()
        for dFdx, domain in zip(src[0], src[1]):
            self.add_adjoint_sources(dFdx, domain)

    def add_adjoint_sources(self, src, domain):
        self._set_sources(src, domain, adjoint=True)

    def clear_sources(self):
        self._sources = []

    def clear_adjoint_sources(self):
        self._adj_sources = []

    # ----------------------------------------------------------------- solve
    def _solve(self, t0, t1, sources):
        # FDTD_solve_cw writes every element of the t0 arrays (the extracted
        # phasors); the t1 arrays are scratch of the reference's loop that the
        # device-resident solve does not use (opt.copy_t1 = 0), so neither set
        # is cleared here (clearing 12 full-grid arrays cost ~0.1-0.2 s a solve)
        h = self._libfdtd
        libFDTD.FDTD_set_t0_arrays(h, *t0)
        libFDTD.FDTD_set_t1_arrays(h, *t1)
        libFDTD.FDTD_clear_sources(h)
        for s in sources:
            libFDTD.FDTD_add_source(h, s.Jx, s.Jy, s.Jz, s.Mx, s.My, s.Mz,
                                    s.i0, s.j0, s.k0, s.I, s.J, s.K, False)
        conv = np.ascontiguousarray(self._conv_pts, dtype=np.int64)
        opt = _ct.SolveOptions()
        opt.Tn = int(np.int64(self._Ncycle * 3 / 4))
        opt.Nmax = float(self.Nmax)
        opt.rtol = float(self._rtol)
        opt.conv_pts = conv.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
        opt.nconv = len(conv)
        opt.fixed_steps = int(self.fixed_steps) if self.fixed_steps else 0
        opt.materials_unchanged = 0 if self._materials_dirty else 1
        opt.copy_t1 = 0
        opt.stop_nonfinite = 1 if self.stop_nonfinite else 0
        res = _ct.SolveResult()
        status = libFDTD.FDTD_solve_cw(h, ctypes.byref(opt), ctypes.byref(res))
        if status not in (_ct.FDTD_OK, _ct.FDTD_NMAX, _ct.FDTD_NONFINITE):
            raise _ct.FDTDError("FDTD_solve_cw failed: %s" % (_ct.last_error(h)[1],))
        self._materials_dirty = False
        if status != _ct.FDTD_OK:
            warning_message("Maximum number of time steps exceeded.", "emopt_b200.fdtd")
        self.last_solve = {"n_main": res.n_main, "steps": res.steps, "A_change": res.A_change,
                           "phi_change": res.phi_change, "nprobes": res.nprobes,
                           "device_ms": res.device_ms, "total_ms": res.total_ms,
                           "launches": res.launches, "zchunk": res.zchunk, "status": status}
        return self.last_solve

    def solve_forward(self):
        """Forward CW solve (``emopt/fdtd.py:1196-1250``)."""
        t0 = [self._Ex_fwd_t0, self._Ey_fwd_t0, self._Ez_fwd_t0,
              self._Hx_fwd_t0, self._Hy_fwd_t0, self._Hz_fwd_t0]
        t1 = [self._Ex_fwd_t1, self._Ey_fwd_t1, self._Ez_fwd_t1,
              self._Hx_fwd_t1, self._Hy_fwd_t1, self._Hz_fwd_t1]
        self._solve(t0, t1, self._sources)
        self.update_saved_fields()
        self._source_power = self._forward_source_power()
        self.forward_count += 1

    def _forward_source_power(self):
        """The source power of the forward fields for ``source_power``: the
        Poynting sums of ``get_source_power`` (the same planes, components
        and interpolation) on the GPU (fieldops.source_power, fixed-order fp64
        sums) from the six grown plane blocks of the phasors, which agrees
        with the host form to ~1e-13 relative and takes a few ms instead of
        tens; the host form when a plane holds no cells."""
        from . import adjoint as A
        from . import fieldops as FO
        import torch
        planes = A.source_power_planes(self)
        shape = (self._Nz, self._Ny, self._Nx)
        d = (self._dx, self._dy, self._dz)
        grown = [FO.grow_domain(dom, shape, d) for dom, _, _ in planes]
        if any(g.i2 <= g.i1 or g.j2 <= g.j1 or g.k2 <= g.k1 for g in grown) or \
                any(dom.i2 <= dom.i1 or dom.j2 <= dom.j1 or dom.k2 <= dom.k1 for dom, _, _ in planes):
            return self.get_source_power()
        dev = self._torch_device()
        raws = []
        for g in grown:
            blk = np.stack([self._raw(c, False)[g.i1:g.i2, g.j1:g.j2, g.k1:g.k2]
                            for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])
            raws.append(torch.as_tensor(blk).to(dev))
        with torch.no_grad():
            return float(FO.source_power(raws, planes, grown, self))

    def solve_adjoint(self):
        """Adjoint CW solve with the adjoint sources (``emopt/fdtd.py:1252-1300``)."""
        t0 = [self._Ex_adj_t0, self._Ey_adj_t0, self._Ez_adj_t0,
              self._Hx_adj_t0, self._Hy_adj_t0, self._Hz_adj_t0]
        t1 = [self._Ex_adj_t1, self._Ey_adj_t1, self._Ez_adj_t1,
              self._Hx_adj_t1, self._Hy_adj_t1, self._Hz_adj_t1]
        self._solve(t0, t1, self._adj_sources)
        self.adjoint_count += 1

    def update_saved_fields(self):
        self._saved_fields = []
        for domain in self._field_domains:
            self._saved_fields.append(tuple(self.get_field_interp(c, domain) for c in
                                            ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")))

    # -------------------------------------------------------- field access
    def _raw(self, component, adjoint):
        name = "_%s_%s_t0" % (component, "adj" if adjoint else "fwd")
        return getattr(self, name).reshape(self._Nz, self._Ny, self._Nx)

    def _get_field(self, component, domain=None, adjoint=False):
        if domain is None:
            domain = DomainCoordinates(0, self._X, 0, self._Y, 0, self._Z,
                                       self._dx, self._dy, self._dz)
        return np.array(self._raw(component, adjoint)[domain.i, domain.j, domain.k])

    def get_field(self, component, domain=None):
        return self._get_field(component, domain, adjoint=False)

    def get_adjoint_field(self, component, domain=None):
        return self._get_field(component, domain, adjoint=True)

    def get_field_interp(self, component, domain=None, squeeze=False):
        """Interpolate a component onto the Ez grid (``emopt/fdtd.py:1401-1553``)."""
        if component == FieldComponent.Ez:
            f = self.get_field(component, domain)
            return np.squeeze(f) if squeeze else f
        if domain is None:
            domain_interp = DomainCoordinates(0, self._X, 0, self._Y, 0, self._Z,
                                              self._dx, self._dy, self._dz)
            domain = domain_interp
        else:
            k1, k2, j1, j2, i1, i2 = domain.k1, domain.k2, domain.j1, domain.j2, domain.i1, domain.i2
            if k1 > 0: k1 -= 1
            if k2 < self._Nx - 1: k2 += 1
            if j1 > 0: j1 -= 1
            if j2 < self._Ny - 1: j2 += 1
            if i1 > 0: i1 -= 1
            if i2 < self._Nz - 1: i2 += 1
            domain_interp = DomainCoordinates(k1 * self._dx, k2 * self._dx, j1 * self._dy,
                                              j2 * self._dy, i1 * self._dz, i2 * self._dz,
                                              self._dx, self._dy, self._dz)
        k1, k2 = domain_interp.k1, domain_interp.k2
        j1, j2 = domain_interp.j1, domain_interp.j2
        i1, i2 = domain_interp.i1, domain_interp.i2
        fraw = np.pad(self.get_field(component, domain_interp), 1, "constant", constant_values=0)
        crop = lambda f: f[1 + domain.i1 - i1:-1 - (i2 - domain.i2),
                           1 + domain.j1 - j1:-1 - (j2 - domain.j2),
                           1 + domain.k1 - k1:-1 - (k2 - domain.k2)]
        bc = self._bc

        def sym_x():
            if k1 == 0 and bc[0] == "E": fraw[:, :, 0] = -1 * fraw[:, :, 1]
            elif k1 == 0 and bc[0] == "H": fraw[:, :, 0] = fraw[:, :, 1]

        def sym_y():
            if j1 == 0 and bc[1] == "E": fraw[:, 0, :] = -1 * fraw[:, 1, :]
            elif j1 == 0 and bc[1] == "H": fraw[:, 0, :] = fraw[:, 1, :]

        if component == FieldComponent.Ex:
            sym_x()
            f = np.copy(fraw)
            f[1:-1, :, 1:-1] += fraw[1:-1, :, 0:-2]
            f[1:-1, :, 1:-1] += fraw[2:, :, 1:-1]
            f[1:-1, :, 1:-1] += fraw[2:, :, 0:-2]
            field = crop(f / 4.0)
        elif component == FieldComponent.Ey:
            sym_y()
            f = np.copy(fraw)
            f[1:-1, 1:-1, :] += fraw[1:-1, 0:-2, :]
            f[1:-1, 1:-1, :] += fraw[2:, 1:-1, :]
            f[1:-1, 1:-1, :] += fraw[2:, 0:-2, :]
            field = crop(f / 4.0)
        elif component == FieldComponent.Hx:
            sym_y()
            f = np.copy(fraw)
            f[:, 1:, :] += fraw[:, 0:-1, :]
            field = crop(f / 2.0)
        elif component == FieldComponent.Hy:
            sym_x()
            f = np.copy(fraw)
            f[:, :, 1:] += fraw[:, :, 0:-1]
            field = crop(f / 2.0)
        elif component == FieldComponent.Hz:
            sym_x()
            sym_y()
            f = np.copy(fraw)
            f[0:-1, 1:, 1:] += fraw[0:-1, 1:, 0:-1]
            f[0:-1, 1:, 1:] += fraw[0:-1, 0:-1, 1:]
            f[0:-1, 1:, 1:] += fraw[0:-1, 0:-1, 0:-1]
            f[0:-1, 1:, 1:] += fraw[1:, 1:, 1:]
            f[0:-1, 1:, 1:] += fraw[1:, 1:, 0:-1]
            f[0:-1, 1:, 1:] += fraw[1:, 0:-1, 1:]
            f[0:-1, 1:, 1:] += fraw[1:, 0:-1, 0:-1]
            field = crop(f / 8.0)
        else:
            raise ValueError("unknown field component %r" % (component,))
        return np.squeeze(field) if squeeze else field

    def get_source_power(self):
        """Poynting flux through a box one cell inside the CPML (``emopt/fdtd.py:1555-1667``)."""
        dx, dy, dz = self._dx, self._dy, self._dz
        w = self._w_pml
        xmin = w[0] + dx if w[0] > 0 else 0.0
        xmax = self._X - w[1] - dx if w[1] > 0 else self._X - dx
        ymin = w[2] + dy if w[2] > 0 else 0.0
        ymax = self._Y - w[3] - dy if w[3] > 0 else self._Y - dy
        zmin = w[4] + dz if w[4] > 0 else 0.0
        zmax = self._Z - w[5] - dz if w[5] > 0 else self._Z - dz
        D = lambda a, b, c, d, e, f: DomainCoordinates(a, b, c, d, e, f, dx, dy, dz)
        g = self.get_field_interp
        P = 0.0
        bc = self._bc
        x1, x2 = D(xmin, xmin, ymin, ymax, zmin, zmax), D(xmax, xmax, ymin, ymax, zmin, zmax)
        y1, y2 = D(xmin, xmax, ymin, ymin, zmin, zmax), D(xmin, xmax, ymax, ymax, zmin, zmax)
        z1, z2 = D(xmin, xmax, ymin, ymax, zmin, zmin), D(xmin, xmax, ymin, ymax, zmax, zmax)
        if bc[0] != "E" and bc[0] != "H":
            P += -0.5 * dy * dz * np.sum(np.real(g("Ey", x1) * np.conj(g("Hz", x1)) -
                                                 g("Ez", x1) * np.conj(g("Hy", x1))))
        P += 0.5 * dy * dz * np.sum(np.real(g("Ey", x2) * np.conj(g("Hz", x2)) -
                                            g("Ez", x2) * np.conj(g("Hy", x2))))
        if bc[1] != "E" and bc[1] != "H":
            P += 0.5 * dx * dz * np.sum(np.real(g("Ex", y1) * np.conj(g("Hz", y1)) -
                                                g("Ez", y1) * np.conj(g("Hx", y1))))
        P += -0.5 * dx * dz * np.sum(np.real(g("Ex", y2) * np.conj(g("Hz", y2)) -
                                             g("Ez", y2) * np.conj(g("Hx", y2))))
        if bc[2] != "E" and bc[2] != "H":
            P += -0.5 * dx * dy * np.sum(np.real(g("Ex", z1) * np.conj(g("Hy", z1)) -
                                                 g("Ey", z1) * np.conj(g("Hx", z1))))
        P += 0.5 * dx * dy * np.sum(np.real(g("Ex", z2) * np.conj(g("Hy", z2)) -
                                            g("Ey", z2) * np.conj(g("Hx", z2))))
        return P

    def get_A_diag(self):
        """Copies of the six material arrays (``emopt/fdtd.py:1669-1692``)."""
        FDTD._sync_host_materials(self)
        return tuple(np.copy(a) for a in (self._eps_x, self._eps_y, self._eps_z,
                                          self._mu_x, self._mu_y, self._mu_z))

    def calc_ydAx_topology(self, domain, update_mu=False, sig_eps=None, sig_mu=None, del_eps=1.0,
                           del_mu=1.0, planar=False, lam=0.0):
        """Topology gradient of ``emopt.experimental.fdtd.FDTD``
        (``emopt/experimental/fdtd.py:37-158``):
        ``sig_eps * (lam / n + 2 del_eps Im(E . E_adj))`` over the domain (summed
        over z when ``planar``), followed for ``update_mu`` by
        ``sig_mu * (lam / n - 2 del_mu Im(H . H_adj))``; unstaggered t0 arrays,
        as the reference.  The products run on the GPU (``FDTD_grad_eps``,
        Kahan-compensated z sums); ``sig_eps`` / ``sig_mu`` None means 1."""
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
        box = [domain.k.start, domain.k.stop, domain.j.start, domain.j.stop] + \
            [domain.i.start, domain.i.stop] * 3

        def overlap(comps):
            f = [torch.as_tensor(self._raw(c, False)).to(dev) for c in comps]
            a = [torch.as_tensor(self._raw(c, True)).to(dev) for c in comps]
            nj, nk = box[3] - box[2], box[1] - box[0]
            ni = box[5] - box[4]
            out = torch.empty((3, nj, nk) if planar else (3, ni, nj, nk), dtype=torch.float64, device=dev)
            ptr = lambda t: ctypes.c_void_p(t.data_ptr())
            fp = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in f])
            ap = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in a])
            msg = ctypes.create_string_buffer(256)
            st = libFDTD.FDTD_grad_eps(dev.index, torch.cuda.current_stream(dev).cuda_stream, fp, ap,
                                       self._Nx, self._Ny, self._Nz, (ctypes.c_int * 10)(*box),
                                       1 if planar else 0, ptr(out), msg, len(msg))
            if st != _ct.FDTD_OK:
                raise _ct.FDTDError(msg.value.decode())
            # 2 Im(adj * fwd) per component, summed over the three components
            return out.sum(dim=0).cpu().numpy()

        g = overlap(("Ex", "Ey", "Ez"))
        se = 1.0 if sig_eps is None else sig_eps
        size = np.size(se) if sig_eps is not None else g.size
        grad_eps = se * (lam / size + del_eps * g)
        if not update_mu:
            return np.ravel(grad_eps)
        gh = overlap(("Hx", "Hy", "Hz"))
        sm = 1.0 if sig_mu is None else sig_mu
        size = np.size(sm) if sig_mu is not None else gh.size
        grad_mu = sm * (lam / size - del_mu * gh)
        return np.concatenate([np.ravel(grad_eps), np.ravel(grad_mu)])

    def calc_ydAx_autograd(self, domain, update_mu, eps_autograd, mu_autograd):
        """Pseudo figure of merit for reverse-mode autodiff of the material
        arrays (``emopt/experimental/fdtd.py:160-223``):
        ``2 sum Im(eps . E . E_adj)`` over the domain, minus
        ``2 sum Im(mu . H . H_adj)`` when ``update_mu``.  ``eps_autograd`` /
        ``mu_autograd``: three torch tensors each (the staggered x, y, z
        arrays on the domain), on any device; the fields follow them there, so
        the gradient with respect to them is the adjoint overlap."""
        import torch

        def pair(c, like):
            f = torch.as_tensor(self.get_field(c, domain)).to(like.device)
            a = torch.as_tensor(self.get_adjoint_field(c, domain)).to(like.device)
            return f, a

        loss = 0
        for c, e in zip(("Ex", "Ey", "Ez"), eps_autograd):
            f, a = pair(c, e)
            loss = loss + e * f * a
        if update_mu:
            for c, m in zip(("Hx", "Hy", "Hz"), mu_autograd):
                f, a = pair(c, m)
                loss = loss - m * f * a
        return 2 * loss.imag.sum()

    def calc_ydAx(self, Adiag0):
        """y^T dA x with dA = i (eps - eps0) for E and -i (mu - mu0) for H
        (``emopt/fdtd.py:1694-1717``)."""
        FDTD._sync_host_materials(self)
        eps_x0, eps_y0, eps_z0, mu_x0, mu_y0, mu_z0 = Adiag0
        ydAx = np.zeros(eps_x0.shape, dtype=np.complex128)
        ydAx = ydAx + self._Ex_adj_t0 * 1j * (self._eps_x - eps_x0) * self._Ex_fwd_t0
        ydAx = ydAx + self._Ey_adj_t0 * 1j * (self._eps_y - eps_y0) * self._Ey_fwd_t0
        ydAx = ydAx + self._Ez_adj_t0 * 1j * (self._eps_z - eps_z0) * self._Ez_fwd_t0
        ydAx = ydAx + self._Hx_adj_t0 * -1j * (self._mu_x - mu_x0) * self._Hx_fwd_t0
        ydAx = ydAx + self._Hy_adj_t0 * -1j * (self._mu_y - mu_y0) * self._Hy_fwd_t0
        ydAx = ydAx + self._Hz_adj_t0 * -1j * (self._mu_z - mu_z0) * self._Hz_fwd_t0
        return np.sum(ydAx)
