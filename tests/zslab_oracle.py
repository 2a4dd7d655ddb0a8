"""A z slab of the CPU oracle with the interface of ``emopt_b200.zslab.CudaSlab``.

Test infrastructure: drives ``emopt_b200.zslab.run`` (the multi-GPU loop and
its transports) on the CPU, one reference-core instance per slab configured
with ``set_local_grid`` (the reference's MPI chunking).  Halo planes are torch
views of the instance's padded field arrays, so a transport writes straight
into the ghost planes that the reference's update_H / update_E read.
"""
from __future__ import annotations

from math import pi

import numpy as np
import torch

from helpers import oracle_for


class OracleSlab:
    def __init__(self, p, i0, I, lib="oracle"):
        o = oracle_for(p, lib)
        self.o, self.lib = o, o.lib
        Nz, Ny, Nx = o.Nz, o.Ny, o.Nx
        self.Nx, self.Ny, self.Nz, self.i0, self.I = Nx, Ny, Nz, i0, I
        self.dt = o.dt
        npad = (I + 2) * (Ny + 2) * (Nx + 2)
        self.E = [np.zeros(npad) for _ in range(3)]
        self.H = [np.zeros(npad) for _ in range(3)]
        self._mats = [np.ascontiguousarray(a[i0:i0 + I]).ravel() for a in o.eps + o.mu]
        self.t0 = [np.zeros(I * Ny * Nx, dtype=np.complex128) for _ in range(6)]
        self._t1 = [np.zeros(I * Ny * Nx, dtype=np.complex128) for _ in range(6)]
        self.h = self.lib.FDTD_new()
        o._configure(self.h, 0, 0, i0, Nx, Ny, I, self.E, self.H, self._mats, self.t0, self._t1)
        self._keep = []
        o._add_sources(self.h, i0, I, self._keep)
        self.lib.FDTD_reset_pml(self.h)
        plane = (Ny + 2) * (Nx + 2)

        def view(a, ip):
            return torch.from_numpy(a[ip * plane:(ip + 1) * plane])

        E, H = self.E, self.H
        self.halo = {"E_send": [view(E[0], 1), view(E[1], 1)],
                     "E_recv": [view(E[0], I + 1), view(E[1], I + 1)],
                     "H_send": [view(H[0], I), view(H[1], I)],
                     "H_recv": [view(H[0], 0), view(H[1], 0)]}
        self.has_lo, self.has_hi = i0 > 0, i0 + I < Nz

    def begin(self, Tn, fixed_steps, Nmax, cells):
        Ny, Nx, i0, I = self.Ny, self.Nx, self.i0, self.I
        self.np_ = len(cells)
        self.own = []
        for q, cell in enumerate(cells):
            if cell < 0:
                continue
            iz, rem = divmod(int(cell), Ny * Nx)
            j, k = divmod(rem, Nx)
            if i0 <= iz < i0 + I:
                self.own.append((q, ((iz - i0 + 1) * (Ny + 2) + j + 1) * (Nx + 2) + k + 1))
        self.samples = torch.zeros(3 * self.np_, dtype=torch.float64)
        self.win = np.zeros((3, 3, self.np_))
        self.A = np.zeros((2, self.np_))
        self.phi = np.zeros((2, self.np_))
        self.t = [0.0, 0.0, 0.0]

    def half_step_part(self, n, half, part):
        """The reference core updates a whole chunk at once: the half step runs
        in the call that comes after the halo it needs has arrived -- part 2
        when the slab has a neighbour on that side (above for H, below for E),
        else part 1 -- so the overlapped loop gives the same fields."""
        edge = self.has_hi if half == 0 else self.has_lo
        if part == 0 or (part == 2) == edge:
            self.half_step(n, half)

    def half_step(self, n, half):
        if half == 0:
            self.lib.FDTD_update_H(self.h, n, n * self.dt)
        else:
            self.lib.FDTD_update_E(self.h, n, (n + 0.5) * self.dt)

    def sample(self):
        s = self.samples.numpy()
        s[:] = 0
        for q, off in self.own:
            for c in range(3):
                s[c * self.np_ + q] = self.E[c][off]
        return self.samples

    def probe(self, n_last):
        """The probe of emopt/fdtd.py:1072-1138 on the summed samples."""
        lib, npt = self.lib, self.np_
        self.t = [self.t[1], self.t[2], n_last * self.dt]
        t0, t1, t2 = self.t
        self.phi[0] = self.phi[1]
        self.A[0] = self.A[1]
        s = self.samples.numpy()
        for q in range(npt):
            phs = amps = 0.0
            for c in range(3):
                w = self.win[c, :, q]
                w[0], w[1], w[2] = w[1], w[2], s[c * npt + q]
                ph = lib.FDTD_calc_phase_3T(t0, t1, t2, *w)
                am = lib.FDTD_calc_amplitude_3T(t0, t1, t2, *w, ph)
                if am < 0:
                    am *= -1
                    ph += pi
                phs += ph
                amps += am
            self.phi[1, q] = phs
            self.A[1, q] = amps
        with np.errstate(divide="ignore", invalid="ignore"):
            return (float(np.linalg.norm(self.A[1] - self.A[0]) / np.linalg.norm(self.A[0])),
                    float(np.linalg.norm(self.phi[1] - self.phi[0]) / np.linalg.norm(self.phi[0])))

    def capture(self, which):
        (self.lib.FDTD_capture_t1_fields if which else self.lib.FDTD_capture_t0_fields)(self.h)

    def finish(self, n0, Tn):
        dt = self.dt
        self.lib.FDTD_calc_complex_fields_3T(self.h, n0 * dt, (n0 + Tn) * dt, (n0 + 2 * Tn) * dt)
        return [a.reshape(self.I, self.Ny, self.Nx) for a in self.t0]

    def close(self):
        pass
