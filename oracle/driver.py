"""Single-process restatement of EMopt's FDTD driver loop (test infrastructure only).

This module is the oracle's Python half.  Only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg import it, as a checker or as the timed CPU
baseline; the ``emopt_b200`` product never does.

``emopt.fdtd`` itself cannot be imported without PETSc/MPI, so this file restates
what the reference Python layer does for a solve and drives an FDTD C library
through the reference ABI (``emopt/fdtd_ctypes.py:26-149``):

* ``OracleFDTD.__init__`` follows ``emopt/fdtd.py:236-437`` for one rank
  (``N_PROC = 1``): grid-size rule, dt, PML defaults, source timing, Nmax and
  the convergence-probe indices.
* ``OracleFDTD.solve`` follows ``FDTD.__solve`` (``emopt/fdtd.py:994-1194``),
  including the probe window, the norm test and the t0/t1/3T extraction.
* ``GhostComm`` on one rank writes periodic copies of the opposite face into
  the face ghosts after every half step (``emopt/fdtd.py:1733-1873``); this is
  reproduced by ``_periodic_faces`` so that convergence probes which land on a
  ghost see the same value as in the reference.
* ``OracleFDTD.run_fixed_slabs`` splits the grid into z-slabs, one library
  instance per slab on its own thread, exchanging ghost planes in shared memory
  -- the reference's MPI decomposition (``dist_method='z'``) without MPI.  It
  is used for the multi-core CPU baseline and for full-size fixed-step parity.

The library is either the reference ``FDTD.so`` compiled from its own sources
(``oracle/_ref/FDTD.so``) or this project's C restatement
(``oracle/_build/libfdtd_oracle.so``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from concurrent.futures import ThreadPoolExecutor
from ctypes import c_bool, c_char_p, c_double, c_int, c_void_p
from math import pi

import numpy as np
from numpy.ctypeslib import ndpointer

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "FDTD.so")
ORACLE_SO = os.path.join(HERE, "_build", "libfdtd_oracle.so")
REF_SRC = "/root/reference/src"

_c_complex_p = ndpointer(np.complex128, ndim=1, flags="C")
_c_double_p = ndpointer(np.double, ndim=1, flags="C")


def build(ref: bool = True) -> None:
    """Compile the C restatement (and the reference core when its sources exist)."""
    targets = ["oracle"]
    if ref and os.path.isdir(REF_SRC):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def available(which: str) -> bool:
    return os.path.exists(REF_SO if which == "ref" else ORACLE_SO)


_LIBS: dict = {}


def load(which: str = "ref"):
    """Load one of the two checker libraries ("ref", "oracle") -- or any library
    with the reference ABI given by path -- and declare the reference argtypes."""
    if which in ("ref", "oracle"):
        path = REF_SO if which == "ref" else ORACLE_SO
    else:
        path = which
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path) and which in ("ref", "oracle"):
        build(ref=(which == "ref"))
    lib = ctypes.CDLL(path)
    sig = {
        "FDTD_new": ([], c_void_p),
        "FDTD_set_wavelength": ([c_void_p, c_double], None),
        "FDTD_set_physical_dims": ([c_void_p] + [c_double] * 6, None),
        "FDTD_set_grid_dims": ([c_void_p, c_int, c_int, c_int], None),
        "FDTD_set_local_grid": ([c_void_p] + [c_int] * 6, None),
        "FDTD_set_dt": ([c_void_p, c_double], None),
        "FDTD_set_complex_eps": ([c_void_p, c_bool], None),
        "FDTD_set_field_arrays": ([c_void_p] + [_c_double_p] * 6, None),
        "FDTD_set_mat_arrays": ([c_void_p] + [_c_complex_p] * 6, None),
        "FDTD_update_H": ([c_void_p, c_int, c_double], None),
        "FDTD_update_E": ([c_void_p, c_int, c_double], None),
        "FDTD_set_pml_widths": ([c_void_p] + [c_int] * 6, None),
        "FDTD_set_pml_properties": ([c_void_p] + [c_double] * 4, None),
        "FDTD_build_pml": ([c_void_p], None),
        "FDTD_reset_pml": ([c_void_p], None),
        "FDTD_set_t0_arrays": ([c_void_p] + [_c_complex_p] * 6, None),
        "FDTD_set_t1_arrays": ([c_void_p] + [_c_complex_p] * 6, None),
        "FDTD_calc_phase_2T": ([c_double] * 4, c_double),
        "FDTD_calc_phase_3T": ([c_double] * 6, c_double),
        "FDTD_calc_amplitude_2T": ([c_double] * 5, c_double),
        "FDTD_calc_amplitude_3T": ([c_double] * 7, c_double),
        "FDTD_capture_t0_fields": ([c_void_p], None),
        "FDTD_capture_t1_fields": ([c_void_p], None),
        "FDTD_calc_complex_fields_2T": ([c_void_p, c_double, c_double], None),
        "FDTD_calc_complex_fields_3T": ([c_void_p, c_double, c_double, c_double], None),
        "FDTD_add_source": ([c_void_p] + [_c_complex_p] * 6 + [c_int] * 6 + [c_bool], None),
        "FDTD_clear_sources": ([c_void_p], None),
        "FDTD_set_source_properties": ([c_void_p, c_double, c_double], None),
        "FDTD_src_func_t": ([c_void_p, c_int, c_double, c_double], c_double),
        "FDTD_set_bc": ([c_void_p, c_char_p], None),
        "FDTD_copy_to_ghost_comm": ([_c_double_p, _c_complex_p, c_int, c_int, c_int], None),
        "FDTD_copy_from_ghost_comm": ([_c_double_p, _c_complex_p, c_int, c_int, c_int], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIBS[path] = lib
    return lib


def _periodic_faces(a: np.ndarray, I: int, J: int, K: int) -> None:
    """One-rank GhostComm: copy each face's opposite interior plane into the ghost."""
    v = a.reshape(I + 2, J + 2, K + 2)
    v[1:-1, 1:-1, 0] = v[1:-1, 1:-1, K]
    v[1:-1, 1:-1, K + 1] = v[1:-1, 1:-1, 1]
    v[1:-1, 0, 1:-1] = v[1:-1, J, 1:-1]
    v[1:-1, J + 1, 1:-1] = v[1:-1, 1, 1:-1]
    v[0, 1:-1, 1:-1] = v[I, 1:-1, 1:-1]
    v[I + 1, 1:-1, 1:-1] = v[1, 1:-1, 1:-1]


def _to_source(arr: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(arr, dtype=np.complex128).ravel().copy()


class OracleFDTD:
    """One-rank restatement of ``emopt.fdtd.FDTD`` sufficient for a CW solve.

    Materials are given directly as six complex arrays of shape ``(Nz, Ny, Nx)``
    (the Yee-staggered eps_x, eps_y, eps_z, mu_x, mu_y, mu_z that
    ``FDTD.build`` would have sampled, ``emopt/fdtd.py:842-880``).
    """

    def __init__(self, X, Y, Z, dx, dy, dz, wavelength, rtol=1e-6, nconv=None,
                 min_rindex=1.0, complex_eps=False, lib="ref"):
        self.lib = load(lib)
        self.lib_name = lib
        if nconv is None:
            nconv = 10
        self.dx, self.dy, self.dz = dx, dy, dz
        Nx = int(np.ceil(X / dx) + 1)
        Ny = int(np.ceil(Y / dy) + 1)
        Nz = int(np.ceil(Z / dz) + 1)
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.X, self.Y, self.Z = dx * (Nx - 1), dy * (Ny - 1), dz * (Nz - 1)
        self.wavelength = wavelength
        self.R = wavelength / (2 * pi)
        self.Sc = 0.95
        self.min_rindex = min_rindex
        self.dt = self.Sc * np.min([dx, dy, dz]) / self.R / np.sqrt(3) * min_rindex
        self.complex_eps = complex_eps
        self.w_pml_cells = [15] * 6
        self.pml = (3.0, 0.0, 1.0, 3.0)
        Nlambda = wavelength / np.min([dx, dy, dz]) / min_rindex
        self.Nlambda = Nlambda
        self.Ncycle = Nlambda * np.sqrt(3)
        self.src_T = self.Ncycle * 20.0 * self.dt
        self.src_min = 1e-4
        self.Nmax = Nlambda * 500
        self.rtol = rtol
        I, J, K = Nz, Ny, Nx
        n_pts = int(nconv / 1)
        self.conv_pts = np.arange(0, I * J * K, int(I * J * K / n_pts))
        self.bc = "000"
        shape = (Nz, Ny, Nx)
        one = np.ones(shape, dtype=np.complex128)
        self.eps = [one.copy() for _ in range(3)]
        self.mu = [one.copy() for _ in range(3)]
        self.sources = []          # (arrays(6), i0, j0, k0, I, J, K) in global indices

    # ----------------------------------------------------------- configuration
    def set_materials(self, eps, mu):
        self.eps = [np.ascontiguousarray(e, dtype=np.complex128) for e in eps]
        self.mu = [np.ascontiguousarray(m, dtype=np.complex128) for m in mu]

    def set_w_pml_cells(self, w):
        self.w_pml_cells = [int(v) for v in w]

    def add_source(self, arrays, i0, j0, k0):
        """``arrays`` = (Jx, Jy, Jz, Mx, My, Mz), each of shape (I, J, K)."""
        I, J, K = np.asarray(arrays[0]).shape
        self.sources.append(([np.asarray(a, dtype=np.complex128) for a in arrays],
                             i0, j0, k0, I, J, K))

    def _configure(self, h, k0, j0, i0, K, J, I, E, H, mats, t0, t1):
        lib = self.lib
        lib.FDTD_set_wavelength(h, self.wavelength)
        lib.FDTD_set_physical_dims(h, self.X, self.Y, self.Z, self.dx, self.dy, self.dz)
        lib.FDTD_set_grid_dims(h, self.Nx, self.Ny, self.Nz)
        lib.FDTD_set_local_grid(h, k0, j0, i0, K, J, I)
        lib.FDTD_set_dt(h, self.dt)
        lib.FDTD_set_field_arrays(h, *E, *H)
        lib.FDTD_set_mat_arrays(h, *mats)
        lib.FDTD_set_complex_eps(h, self.complex_eps)
        lib.FDTD_set_pml_widths(h, *self.w_pml_cells)
        lib.FDTD_set_pml_properties(h, *self.pml)
        lib.FDTD_build_pml(h)
        lib.FDTD_set_source_properties(h, self.src_T, self.src_min)
        lib.FDTD_set_bc(h, self.bc.encode("ascii"))
        lib.FDTD_set_t0_arrays(h, *t0)
        lib.FDTD_set_t1_arrays(h, *t1)

    def _add_sources(self, h, i0, I, keep):
        """Crop every source to the z-range [i0, i0+I) and hand it to the library
        with calc_phase=True (``emopt/fdtd.py:710-747``)."""
        for arrays, si0, sj0, sk0, sI, sJ, sK in self.sources:
            lo, hi = max(si0, i0), min(si0 + sI, i0 + I)
            if lo >= hi:
                continue
            cropped = [_to_source(a[lo - si0:hi - si0]) for a in arrays]
            keep.append(cropped)
            self.lib.FDTD_add_source(h, *cropped, lo - i0, sj0, sk0, hi - lo, sJ, sK, True)

    # ------------------------------------------------------------------ solve
    def solve(self, fixed_steps: int | None = None, record=False):
        """Run ``__solve`` on one instance; returns a dict with the complex fields."""
        lib = self.lib
        I, J, K = self.Nz, self.Ny, self.Nx
        npad = (I + 2) * (J + 2) * (K + 2)
        E = [np.zeros(npad) for _ in range(3)]
        H = [np.zeros(npad) for _ in range(3)]
        mats = [a.ravel() for a in self.eps + self.mu]
        t0 = [np.zeros(I * J * K, dtype=np.complex128) for _ in range(6)]
        t1 = [np.zeros(I * J * K, dtype=np.complex128) for _ in range(6)]
        h = lib.FDTD_new()
        self._configure(h, 0, 0, 0, K, J, I, E, H, mats, t0, t1)
        keep = []
        self._add_sources(h, 0, I, keep)
        Nmax = float(fixed_steps - 1) if fixed_steps is not None else self.Nmax
        rtol = 1e-300 if fixed_steps is not None else self.rtol

        dt = self.dt
        lib.FDTD_reset_pml(h)
        for a in E + H:
            a.fill(0)
        Tn = np.int64(self.Ncycle * 3 / 4)
        nconv = len(self.conv_pts)
        win = np.zeros((3, 3, nconv))        # [component][sample][point]
        phi0 = np.zeros(nconv); phi1 = np.zeros(nconv)
        A0 = np.zeros(nconv); A1 = np.zeros(nconv)
        t_0 = t_1 = t_2 = 0
        A_change = 1
        phi_change = 1
        amp_rtol, phi_rtol = rtol, np.sqrt(rtol)
        history = []
        p = 0
        n = 0

        def step(nn, tH, tE):
            lib.FDTD_update_H(h, nn, tH)
            for a in H:
                _periodic_faces(a, I, J, K)
            lib.FDTD_update_E(h, nn, tE)
            for a in E:
                _periodic_faces(a, I, J, K)

        while (A_change > amp_rtol or phi_change > phi_rtol or np.isnan(A_change)
               or np.isinf(A_change) or np.isnan(phi_change) or np.isinf(phi_change)):
            if n > Nmax:
                break
            step(n, n * dt, (n + 0.5) * dt)
            if p == Tn - 1:
                t_0, t_1, t_2 = t_1, t_2, n * dt
                phi0[:] = phi1
                A0[:] = A1
                for q in range(nconv):
                    ci = self.conv_pts[q]
                    phs, amps = [], []
                    for c in range(3):
                        win[c, 0, q] = win[c, 1, q]
                        win[c, 1, q] = win[c, 2, q]
                        win[c, 2, q] = E[c][ci]
                        f0, f1, f2 = win[c, :, q]
                        ph = lib.FDTD_calc_phase_3T(t_0, t_1, t_2, f0, f1, f2)
                        am = lib.FDTD_calc_amplitude_3T(t_0, t_1, t_2, f0, f1, f2, ph)
                        if am < 0:
                            am *= -1
                            ph += pi
                        phs.append(ph)
                        amps.append(am)
                    phi1[q] = phs[0] + phs[1] + phs[2]
                    A1[q] = amps[0] + amps[1] + amps[2]
                with np.errstate(divide="ignore", invalid="ignore"):
                    A_change = np.linalg.norm(A1 - A0) / np.linalg.norm(A0)
                    phi_change = np.linalg.norm(phi1 - phi0) / np.linalg.norm(phi0)
                if record:
                    history.append((n, float(A_change), float(phi_change)))
                p = 0
            else:
                p += 1
            n += 1

        lib.FDTD_capture_t0_fields(h)
        n0 = n
        for m in range(Tn):
            step(m + n0, (m + n0) * dt, (m + n0 + 0.5) * dt)
        lib.FDTD_capture_t1_fields(h)
        for m in range(Tn):
            step(m + n0 + Tn, (m + n0 + Tn) * dt, (m + n0 + Tn + 0.5) * dt)
        lib.FDTD_calc_complex_fields_3T(h, n0 * dt, (n0 + Tn) * dt, (n0 + 2 * Tn) * dt)
        shape = (I, J, K)
        return {
            "fields": [a.reshape(shape) for a in t0],
            "n_main": n0,
            "steps": int(n0 + 2 * Tn),
            "Tn": int(Tn),
            "A_change": float(A_change),
            "phi_change": float(phi_change),
            "history": history,
            "E": [a.reshape(I + 2, J + 2, K + 2) for a in E],
            "H": [a.reshape(I + 2, J + 2, K + 2) for a in H],
        }

    # ------------------------------------------------- z-slab multi-instance
    def _slab_machine(self, ranges):
        """One library instance per slab [(i0, I), ...] and a step function
        that advances all of them with the ghost exchange of GhostComm for a
        z-only decomposition (x/y faces wrap onto the slab itself, z faces come
        from the adjacent slab with wrap-around, emopt/fdtd.py:1733-1873)."""
        lib = self.lib
        Ny, Nx = self.Ny, self.Nx
        P = len(ranges)
        slabs = []
        keep = []
        for i0, I in ranges:
            J, K = Ny, Nx
            npad = (I + 2) * (J + 2) * (K + 2)
            E = [np.zeros(npad) for _ in range(3)]
            H = [np.zeros(npad) for _ in range(3)]
            mats = [np.ascontiguousarray(a[i0:i0 + I]).ravel() for a in self.eps + self.mu]
            t0 = [np.zeros(I * J * K, dtype=np.complex128) for _ in range(6)]
            t1 = [np.zeros(I * J * K, dtype=np.complex128) for _ in range(6)]
            h = lib.FDTD_new()
            self._configure(h, 0, 0, i0, K, J, I, E, H, mats, t0, t1)
            self._add_sources(h, i0, I, keep)
            lib.FDTD_reset_pml(h)
            slabs.append(dict(h=h, i0=i0, I=I, E=E, H=H, mats=mats, t0=t0, t1=t1))
        dt = self.dt
        pool = ThreadPoolExecutor(max_workers=P)

        def exchange(fields_key):
            views = []
            for sl in slabs:
                I = sl["I"]
                vs = [a.reshape(I + 2, Ny + 2, Nx + 2) for a in sl[fields_key]]
                for v in vs:
                    v[1:-1, 1:-1, 0] = v[1:-1, 1:-1, Nx]
                    v[1:-1, 1:-1, Nx + 1] = v[1:-1, 1:-1, 1]
                    v[1:-1, 0, 1:-1] = v[1:-1, Ny, 1:-1]
                    v[1:-1, Ny + 1, 1:-1] = v[1:-1, 1, 1:-1]
                views.append(vs)
            for s in range(P):
                lo = views[(s - 1) % P]
                hi = views[(s + 1) % P]
                I_lo = slabs[(s - 1) % P]["I"]
                for c in range(3):
                    views[s][c][0, 1:-1, 1:-1] = lo[c][I_lo, 1:-1, 1:-1]
                    views[s][c][-1, 1:-1, 1:-1] = hi[c][1, 1:-1, 1:-1]

        def half(fn, n, t):
            list(pool.map(lambda sl: fn(sl["h"], n, t), slabs))

        def step(n):
            half(lib.FDTD_update_H, n, n * dt)
            exchange("H")
            half(lib.FDTD_update_E, n, (n + 0.5) * dt)
            exchange("E")

        return slabs, keep, step, pool

    def solve_slabs(self, ranges, fixed_steps: int | None = None, nconv: int = 10, record=False):
        """The reference's multi-rank solve over the z slabs ``ranges``.

        Every rank picks int(nconv / nranks) probe points of its own padded
        local E arrays (emopt/fdtd.py:411-413) and reads them after the ghost
        exchange; the amplitudes and phases of all ranks are concatenated in
        rank order before the change norms are taken (:1119-1145)."""
        lib = self.lib
        Ny, Nx = self.Ny, self.Nx
        slabs, keep, step, pool = self._slab_machine([(int(a), int(b)) for a, b in ranges])
        P = len(slabs)
        n_pts = int(nconv / P)
        pts = [np.arange(0, sl["I"] * Ny * Nx, int(sl["I"] * Ny * Nx / n_pts)) for sl in slabs]
        npt = sum(len(q) for q in pts)
        Nmax = float(fixed_steps - 1) if fixed_steps is not None else self.Nmax
        rtol = 1e-300 if fixed_steps is not None else self.rtol
        dt = self.dt
        Tn = int(np.int64(self.Ncycle * 3 / 4))
        win = np.zeros((3, 3, npt))
        phi0 = np.zeros(npt); phi1 = np.zeros(npt)
        A0 = np.zeros(npt); A1 = np.zeros(npt)
        t_0 = t_1 = t_2 = 0
        A_change = phi_change = 1
        history = []
        p = n = 0
        while (A_change > rtol or phi_change > np.sqrt(rtol) or np.isnan(A_change)
               or np.isinf(A_change) or np.isnan(phi_change) or np.isinf(phi_change)):
            if n > Nmax:
                break
            step(n)
            if p == Tn - 1:
                t_0, t_1, t_2 = t_1, t_2, n * dt
                phi0[:] = phi1
                A0[:] = A1
                q = 0
                for sl, sp in zip(slabs, pts):
                    for ci in sp:
                        phs = amps = 0.0
                        for c in range(3):
                            win[c, 0, q] = win[c, 1, q]
                            win[c, 1, q] = win[c, 2, q]
                            win[c, 2, q] = sl["E"][c][ci]
                            f0, f1, f2 = win[c, :, q]
                            ph = lib.FDTD_calc_phase_3T(t_0, t_1, t_2, f0, f1, f2)
                            am = lib.FDTD_calc_amplitude_3T(t_0, t_1, t_2, f0, f1, f2, ph)
                            if am < 0:
                                am *= -1
                                ph += pi
                            phs += ph
                            amps += am
                        phi1[q] = phs
                        A1[q] = amps
                        q += 1
                with np.errstate(divide="ignore", invalid="ignore"):
                    A_change = np.linalg.norm(A1 - A0) / np.linalg.norm(A0)
                    phi_change = np.linalg.norm(phi1 - phi0) / np.linalg.norm(phi0)
                if record:
                    history.append((n, float(A_change), float(phi_change)))
                p = 0
            else:
                p += 1
            n += 1
        n0 = n
        list(pool.map(lambda sl: lib.FDTD_capture_t0_fields(sl["h"]), slabs))
        for m in range(Tn):
            step(n0 + m)
        list(pool.map(lambda sl: lib.FDTD_capture_t1_fields(sl["h"]), slabs))
        for m in range(Tn):
            step(n0 + Tn + m)
        list(pool.map(lambda sl: lib.FDTD_calc_complex_fields_3T(
            sl["h"], n0 * dt, (n0 + Tn) * dt, (n0 + 2 * Tn) * dt), slabs))
        pool.shutdown()
        fields = [np.concatenate([sl["t0"][c].reshape(sl["I"], Ny, Nx) for sl in slabs])
                  for c in range(6)]
        return {"fields": fields, "steps": int(n0 + 2 * Tn), "n_main": n0, "Tn": Tn,
                "A_change": float(A_change), "phi_change": float(phi_change), "history": history}

    def solve_threads(self, nthreads: int, record=False):
        """The one-rank ``__solve`` of ``solve`` (same probe points, same loop,
        emopt/fdtd.py:994-1194) with the time steps run on ``nthreads`` z slabs
        in parallel threads: the slab exchange reproduces the one-rank ghost
        layers (periodic faces, zero edges), so the fields, the probe values
        and therefore the step count equal those of ``solve`` bit for bit,
        while a full-size grid takes minutes instead of hours."""
        lib = self.lib
        Nz, Ny, Nx = self.Nz, self.Ny, self.Nx
        P = max(1, min(nthreads, Nz))
        bounds = np.linspace(0, Nz, P + 1).round().astype(int)
        ranges = [(int(bounds[s]), int(bounds[s + 1] - bounds[s])) for s in range(P)]
        slabs, keep, step, pool = self._slab_machine(ranges)
        # probe point (padded global index) -> (slab, padded local index); a
        # z ghost plane holds the periodic copy of the opposite interior plane
        K2, J2 = Nx + 2, Ny + 2
        where = []
        for ci in self.conv_pts:
            ip, rem = divmod(int(ci), J2 * K2)
            ghosts = (ip in (0, Nz + 1)) + (rem // K2 in (0, Ny + 1)) + (rem % K2 in (0, Nx + 1))
            if ip == 0:
                ip = Nz if ghosts == 1 else -1
            elif ip == Nz + 1:
                ip = 1 if ghosts == 1 else -1
            if ip < 0 or ghosts > 1:
                where.append(None)      # an edge or corner ghost: zero forever
                continue
            for sidx, (i0, I) in enumerate(ranges):
                if i0 < ip <= i0 + I:
                    where.append((sidx, (ip - i0) * J2 * K2 + rem))
                    break
        dt = self.dt
        Tn = int(np.int64(self.Ncycle * 3 / 4))
        nconv = len(self.conv_pts)
        win = np.zeros((3, 3, nconv))
        phi0 = np.zeros(nconv); phi1 = np.zeros(nconv)
        A0 = np.zeros(nconv); A1 = np.zeros(nconv)
        t_0 = t_1 = t_2 = 0
        A_change = phi_change = 1
        amp_rtol, phi_rtol = self.rtol, np.sqrt(self.rtol)
        history = []
        p = n = 0
        while (A_change > amp_rtol or phi_change > phi_rtol or np.isnan(A_change)
               or np.isinf(A_change) or np.isnan(phi_change) or np.isinf(phi_change)):
            if n > self.Nmax:
                break
            step(n)
            if p == Tn - 1:
                t_0, t_1, t_2 = t_1, t_2, n * dt
                phi0[:] = phi1
                A0[:] = A1
                for q in range(nconv):
                    w = where[q]
                    phs, amps = [], []
                    for c in range(3):
                        win[c, 0, q] = win[c, 1, q]
                        win[c, 1, q] = win[c, 2, q]
                        win[c, 2, q] = 0.0 if w is None else slabs[w[0]]["E"][c][w[1]]
                        f0, f1, f2 = win[c, :, q]
                        ph = lib.FDTD_calc_phase_3T(t_0, t_1, t_2, f0, f1, f2)
                        am = lib.FDTD_calc_amplitude_3T(t_0, t_1, t_2, f0, f1, f2, ph)
                        if am < 0:
                            am *= -1
                            ph += pi
                        phs.append(ph)
                        amps.append(am)
                    phi1[q] = phs[0] + phs[1] + phs[2]
                    A1[q] = amps[0] + amps[1] + amps[2]
                with np.errstate(divide="ignore", invalid="ignore"):
                    A_change = np.linalg.norm(A1 - A0) / np.linalg.norm(A0)
                    phi_change = np.linalg.norm(phi1 - phi0) / np.linalg.norm(phi0)
                if record:
                    history.append((n, float(A_change), float(phi_change)))
                p = 0
            else:
                p += 1
            n += 1
        n0 = n
        list(pool.map(lambda sl: lib.FDTD_capture_t0_fields(sl["h"]), slabs))
        for m in range(Tn):
            step(n0 + m)
        list(pool.map(lambda sl: lib.FDTD_capture_t1_fields(sl["h"]), slabs))
        for m in range(Tn):
            step(n0 + Tn + m)
        list(pool.map(lambda sl: lib.FDTD_calc_complex_fields_3T(
            sl["h"], n0 * dt, (n0 + Tn) * dt, (n0 + 2 * Tn) * dt), slabs))
        pool.shutdown()
        fields = [np.concatenate([sl["t0"][c].reshape(sl["I"], Ny, Nx) for sl in slabs])
                  for c in range(6)]
        return {"fields": fields, "steps": int(n0 + 2 * Tn), "n_main": n0, "Tn": Tn,
                "nprobes": len(history) if record else None,
                "A_change": float(A_change), "phi_change": float(phi_change), "history": history}

    def run_fixed_slabs(self, n_main: int, nthreads: int, extract=True, time_only_steps=None,
                        ranges=None):
        """Fixed-step solve over ``nthreads`` z-slabs on as many threads.

        Each slab is one library instance configured with ``set_local_grid``
        (the reference's MPI chunking, ``emopt/fdtd.py:273-297``); ghost planes
        are exchanged with the GhostComm rule for a z-only decomposition
        (x/y faces wrap onto the slab itself, z faces come from the adjacent
        slab with wrap-around).  ctypes releases the GIL during each call, so the
        slabs advance in parallel.

        ``time_only_steps``: run that many steps and return the wall time only
        (CPU-baseline timing); otherwise run ``n_main`` + 2 Tn steps and
        extract like ``solve`` (without convergence probes).  ``ranges``: the
        slabs as [(i0, I), ...] instead of an even split; the result then also
        holds each slab's padded E arrays after the last exchange ("E_pad").
        """
        import time as _time
        lib = self.lib
        Nz, Ny, Nx = self.Nz, self.Ny, self.Nx
        if ranges is None:
            P = max(1, min(nthreads, Nz))
            bounds = np.linspace(0, Nz, P + 1).round().astype(int)
            ranges_ = [(int(bounds[s]), int(bounds[s + 1] - bounds[s])) for s in range(P)]
        else:
            ranges_ = [(int(a), int(b)) for a, b in ranges]
        slabs, keep, step, pool = self._slab_machine(ranges_)
        dt = self.dt
        P = len(slabs)

        if time_only_steps is not None:
            t_start = _time.perf_counter()
            for n in range(time_only_steps):
                step(n)
            elapsed = _time.perf_counter() - t_start
            pool.shutdown()
            return elapsed

        Tn = int(np.int64(self.Ncycle * 3 / 4))
        for n in range(n_main):
            step(n)
        n0 = n_main
        list(pool.map(lambda sl: lib.FDTD_capture_t0_fields(sl["h"]), slabs))
        for m in range(Tn):
            step(n0 + m)
        list(pool.map(lambda sl: lib.FDTD_capture_t1_fields(sl["h"]), slabs))
        for m in range(Tn):
            step(n0 + Tn + m)
        if extract:
            list(pool.map(lambda sl: lib.FDTD_calc_complex_fields_3T(
                sl["h"], n0 * dt, (n0 + Tn) * dt, (n0 + 2 * Tn) * dt), slabs))
        pool.shutdown()
        fields = [np.concatenate([sl["t0"][c].reshape(sl["I"], Ny, Nx) for sl in slabs])
                  for c in range(6)]
        out = {"fields": fields, "steps": n_main + 2 * Tn, "n_main": n_main, "Tn": Tn}
        if ranges is not None:
            out["E_pad"] = [[a.reshape(sl["I"] + 2, Ny + 2, Nx + 2) for a in sl["E"]] for sl in slabs]
        return out
