"""Serving form: continuous batching of CW-FDTD solves on one GPU.

A request is a CW solve of its own grid, spacing, wavelength, structure and
source.  :class:`ServeEngine` wraps the library's ``FDTD_serve_*`` calls: it
admits requests against a device-memory budget, keeps their fields resident
and advances all admitted requests together -- each ``advance`` replays one
CUDA graph of batched stepping kernels that also run every request's probe,
convergence test and captures on the device -- and retires finished requests
(3-sample extraction into device tensors).  :func:`run_stream` drives the
engine with a timed arrival stream and reports latency percentiles beside the
aggregate throughput.

Requests are configured through the reference ABI (``FDTD_new``,
``FDTD_set_*``, ``FDTD_add_source``) with the parameter rules of
``emopt/fdtd.py:236-437``; their permittivity is assembled on the GPU from
the request's box list (voxel sampling at the Yee positions of
``emopt/fdtd.py:842-880``) and handed to the library as device arrays.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import fdtd_ctypes as _ct
from .adjoint import _raw
from .fdtd import derive_parameters
from .problems import EPS_SI, EPS_SIO2, YEE_OFFSETS

lib = _ct.libFDTD


@dataclass
class RequestSpec:
    """A block-structure CW solve: grid (Nz, Ny, Nx) cells at spacing d,
    wavelength, boxes (x0, x1, y0, y1, z0, z1, eps) in um over an SiO2
    background, a Jy Gaussian sheet source, CPML width in cells."""
    rid: int
    shape: tuple            # (Nz, Ny, Nx)
    d: float
    wavelength: float
    boxes: list
    w_pml: int = 15
    rtol: float = 1e-6
    src_k: int = 0
    src_yz: tuple = (0.0, 0.0)
    src_w0: float = 0.4
    arrival: float = 0.0
    fixed_steps: int = 0
    src_phase_y: float = 0.0    # linear source phase exp(i src_phase_y y), 1/um
    precision: int = 32          # storage precision of the solve (32 or 64)

    @property
    def ncells(self):
        Nz, Ny, Nx = self.shape
        return Nz * Ny * Nx


def random_request(rng, rid, shape=None, d=None, wavelength=None, w_pml=15) -> RequestSpec:
    """One request of the serving stream: grid uniform from 64^3 up to
    384 x 256 x 128 cells, d in {0.02, 0.025, 0.04} um, wavelength uniform in
    1.50-1.60 um, 3-12 Si/SiO2 boxes with sides uniform 0.2-2.0 um."""
    if shape is None:
        shape = (int(rng.integers(64, 129)), int(rng.integers(64, 257)), int(rng.integers(64, 385)))
    if d is None:
        d = float(rng.choice([0.02, 0.025, 0.04]))
    if wavelength is None:
        wavelength = float(rng.uniform(1.50, 1.60))
    Nz, Ny, Nx = shape
    L = [(n - 1) * d for n in (Nx, Ny, Nz)]
    boxes = []
    for _ in range(int(rng.integers(3, 13))):
        s = rng.uniform(0.2, 2.0, 3)
        c = [rng.uniform(0, L[a]) for a in range(3)]
        eps = EPS_SI if rng.random() < 0.5 else EPS_SIO2
        boxes.append((c[0] - s[0] / 2, c[0] + s[0] / 2, c[1] - s[1] / 2, c[1] + s[1] / 2,
                      c[2] - s[2] / 2, c[2] + s[2] / 2, eps))
    return RequestSpec(rid, tuple(shape), d, wavelength, boxes, w_pml=w_pml,
                       src_k=w_pml + 5, src_yz=(L[1] / 2, L[2] / 2), src_w0=0.4)


def grating_spec(seed: int = 4, d: float = 0.02, precision: int = 32) -> RequestSpec:
    """The large single solve: a grating-coupler-like slab, 24 x 12 x 6 um at
    d = 0.02 um (1201 x 601 x 301 cells, 217 M), 25-cell CPML: Si substrate
    (eps 12.25) below z = 1.5 um, a 2 um SiO2 box, a 0.22 um Si layer with 40
    seeded etch trenches (width uniform 0.1-0.4 um, depth 0.11 um, across y)
    under SiO2, wavelength 1.55 um; Jy Gaussian sheet (w0 = 2 um) on an
    x-normal plane, tilted by 10 degrees through the linear phase
    exp(i k0 n_clad sin(10 deg) y)."""
    rng = np.random.default_rng(seed)
    Nx, Ny, Nz = (int(round(24.0 / d)) + 1, int(round(12.0 / d)) + 1, int(round(6.0 / d)) + 1)
    X, Y, Z = (Nx - 1) * d, (Ny - 1) * d, (Nz - 1) * d
    big = 1e3
    z_sub, z_box, t_si = 1.5, 2.0, 0.22
    z0, z1 = z_sub + z_box, z_sub + z_box + t_si
    boxes = [(-big, big, -big, big, -big, z_sub, EPS_SI),
             (-big, big, -big, big, z0, z1, EPS_SI)]
    centres = np.sort(rng.uniform(6.0, 18.0, 40))
    for xc in centres:
        w = rng.uniform(0.1, 0.4)
        boxes.append((xc - w / 2, xc + w / 2, -big, big, z1 - 0.11, z1 + 1e-9, EPS_SIO2))
    k0 = 2 * np.pi / 1.55
    w_pml = 25
    return RequestSpec(0, (Nz, Ny, Nx), d, 1.55, boxes, w_pml=w_pml, src_k=w_pml + 5,
                       src_yz=(Y / 2, (z0 + z1) / 2), src_w0=2.0,
                       src_phase_y=k0 * np.sqrt(EPS_SIO2) * np.sin(np.deg2rad(10.0)),
                       precision=precision)


def poisson_stream(n, rate, seed=3, **kw):
    """``n`` requests with exponential inter-arrival times (mean 1/rate s)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for q in range(n):
        r = random_request(rng, q, **kw)
        r.arrival = float(t[q])
        reqs.append(r)
    return reqs


def eps_arrays(spec: RequestSpec, device) -> list:
    """The three Yee-staggered permittivity arrays of a request (complex128 on
    the GPU): SiO2 background, then the boxes in order, each voxel-sampled."""
    Nz, Ny, Nx = spec.shape
    d = spec.d
    out = []
    for c in range(3):
        sx, sy, sz = YEE_OFFSETS[c]
        x = (torch.arange(Nx, device=device, dtype=torch.float64) + sx) * d
        y = (torch.arange(Ny, device=device, dtype=torch.float64) + sy) * d
        z = (torch.arange(Nz, device=device, dtype=torch.float64) + sz) * d
        e = torch.full(spec.shape, EPS_SIO2, dtype=torch.float64, device=device)
        for (x0, x1, y0, y1, z0, z1, val) in spec.boxes:
            mx = (x >= x0) & (x <= x1)
            my = (y >= y0) & (y <= y1)
            mz = (z >= z0) & (z <= z1)
            m = mz[:, None, None] & my[None, :, None] & mx[None, None, :]
            e = torch.where(m, torch.tensor(val, dtype=torch.float64, device=device), e)
        out.append(e.to(torch.complex128).contiguous())
    return out


class Request:
    """A configured library handle for one spec (storage precision from the spec)."""

    def __init__(self, spec: RequestSpec, device: int, mu_ones: torch.Tensor):
        self.spec = spec
        self.device = device
        Nz, Ny, Nx = spec.shape
        d = spec.d
        X, Y, Z = (Nx - 1.5) * d, (Ny - 1.5) * d, (Nz - 1.5) * d
        prm = derive_parameters(X, Y, Z, d, d, d, spec.wavelength)
        assert (prm["Nz"], prm["Ny"], prm["Nx"]) == spec.shape, (prm, spec.shape)
        self.prm = prm
        h = lib.FDTD_new()
        self.h = h
        lib.FDTD_set_device(h, device)
        lib.FDTD_set_wavelength(h, spec.wavelength)
        lib.FDTD_set_physical_dims(h, prm["X"], prm["Y"], prm["Z"], d, d, d)
        lib.FDTD_set_grid_dims(h, Nx, Ny, Nz)
        lib.FDTD_set_local_grid(h, 0, 0, 0, Nx, Ny, Nz)
        lib.FDTD_set_dt(h, prm["dt"])
        lib.FDTD_set_complex_eps(h, False)
        w = spec.w_pml
        lib.FDTD_set_pml_widths(h, w, w, w, w, w, w)
        lib.FDTD_set_pml_properties(h, 3.0, 0.0, 1.0, 3.0)
        lib.FDTD_build_pml(h)
        lib.FDTD_set_source_properties(h, prm["src_T"], prm["src_min"])
        lib.FDTD_set_precision(h, spec.precision)
        self.eps = eps_arrays(spec, torch.device("cuda", device))
        torch.cuda.synchronize(device)   # the library reads them on its own stream
        _raw.FDTD_set_mat_arrays(h, *[e.data_ptr() for e in self.eps],
                                 mu_ones.data_ptr(), mu_ones.data_ptr(), mu_ones.data_ptr())
        # Jy Gaussian sheet on the plane x = src_k
        z = np.arange(Nz) * d
        y = np.arange(Ny) * d
        Zg, Yg = np.meshgrid(z, y, indexing="ij")
        yc, zc = spec.src_yz
        prof = np.exp(-((Yg - yc) ** 2 + (Zg - zc) ** 2) / spec.src_w0 ** 2) * \
            np.exp(1j * spec.src_phase_y * Yg)
        self.src = [np.zeros(Nz * Ny, dtype=np.complex128) for _ in range(6)]
        self.src[1][:] = prof.ravel()
        lib.FDTD_add_source(h, *self.src, 0, 0, spec.src_k, Nz, Ny, 1, True)
        self.conv = np.ascontiguousarray(prm["conv_pts"], dtype=np.int64)
        o = _ct.SolveOptions()
        o.Tn = prm["Tn"]
        o.Nmax = float(prm["Nmax"])
        o.rtol = spec.rtol
        o.conv_pts = self.conv.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
        o.nconv = len(self.conv)
        o.fixed_steps = int(spec.fixed_steps)
        o.materials_unchanged = 0
        o.copy_t1 = 0
        self.opt = o
        self.out = None

    def set_outputs(self):
        """Allocate the six complex128 output arrays on the device."""
        dev = torch.device("cuda", self.device)
        self.out = [torch.empty(self.spec.shape, dtype=torch.complex128, device=dev) for _ in range(6)]
        _raw.FDTD_set_t0_arrays(self.h, *[a.data_ptr() for a in self.out])

    def release_inputs(self):
        self.eps = None     # consumed into the update coefficients at admission

    def close(self):
        if self.h:
            lib.FDTD_delete(self.h)
            self.h = None


class ServeEngine:
    """Python front of ``FDTD_serve_*``."""

    def __init__(self, device: int = 0, budget_bytes: float = 150e9, max_requests: int = 128,
                 steps_per_replay: int = 32):
        self.device = device
        self.s = lib.FDTD_serve_new(device, float(budget_bytes), max_requests, steps_per_replay)
        st, msg = self.last_error()
        if st != _ct.FDTD_OK:
            raise _ct.FDTDError("FDTD_serve_new: %s" % msg)
        self.steps_per_replay = steps_per_replay
        self.max_requests = max_requests
        self.active = {}

    def last_error(self):
        buf = ctypes.create_string_buffer(512)
        st = lib.FDTD_serve_last_error(self.s, buf, 512)
        return st, buf.value.decode()

    def admit(self, req: Request) -> bool:
        slot = lib.FDTD_serve_admit(self.s, req.h, ctypes.byref(req.opt))
        if slot == -1:
            return False
        if slot < 0:
            raise _ct.FDTDError("FDTD_serve_admit: %s" % self.last_error()[1])
        self.active[req.h] = req
        req.release_inputs()
        return True

    def advance(self) -> int:
        n = lib.FDTD_serve_advance(self.s)
        if n < 0:
            raise _ct.FDTDError("FDTD_serve_advance: %s" % self.last_error()[1])
        return n

    def collect(self, ready: int) -> list:
        """Retire finished requests; returns [(request, result dict)]."""
        if ready <= 0:
            return []
        hs = (ctypes.c_void_p * ready)()
        n = lib.FDTD_serve_finished(self.s, hs, ready)
        for k in range(n):
            self.active[hs[k]].set_outputs()
        done = (ctypes.c_void_p * ready)()
        res = (_ct.SolveResult * ready)()
        n = lib.FDTD_serve_collect(self.s, done, res, ready)
        if n < 0:
            raise _ct.FDTDError("FDTD_serve_collect: %s" % self.last_error()[1])
        out = []
        for k in range(n):
            req = self.active.pop(done[k])
            r = res[k]
            out.append((req, {"n_main": r.n_main, "steps": r.steps, "A_change": r.A_change,
                              "phi_change": r.phi_change, "nprobes": r.nprobes, "status": r.status,
                              "launches": r.launches}))
        return out

    def info(self):
        used = ctypes.c_double()
        act = ctypes.c_int()
        lib.FDTD_serve_info(self.s, ctypes.byref(used), ctypes.byref(act))
        return used.value, act.value

    def close(self):
        if self.s:
            lib.FDTD_serve_delete(self.s)
            self.s = None


def run_stream(specs, engine: ServeEngine, realtime: bool = True, keep_fields: bool = False,
               on_done=None):
    """Serve ``specs`` through ``engine`` in arrival order; returns a dict with
    per-request latency (completion - arrival) and service time (completion -
    admission: the time a request spends in the engine, queueing excluded),
    the makespan and the aggregate cell updates.  With ``realtime`` the
    arrivals follow the wall clock; otherwise every request is available at
    time 0."""
    dev = torch.device("cuda", engine.device)
    max_cells = max(s.ncells for s in specs)
    mu_ones = torch.ones(max_cells, dtype=torch.complex128, device=dev)
    pending = list(sorted(specs, key=lambda s: s.arrival))
    waiting = []          # arrived, not yet admitted (FIFO)
    head = None           # the built head of the queue, kept across retries
    lat, svc, adm, results = {}, {}, {}, {}
    cell_updates = 0.0
    t0 = time.perf_counter()
    clock = lambda: time.perf_counter() - t0
    while pending or waiting or engine.active:
        now = clock()
        while pending and (not realtime or pending[0].arrival <= now):
            waiting.append(pending.pop(0))
        while waiting:
            if head is None:
                head = Request(waiting[0], engine.device, mu_ones)
            if not engine.admit(head):
                break
            adm[head.spec.rid] = clock()
            waiting.pop(0)
            head = None
        if engine.active:
            ready = engine.advance()
            for req, r in engine.collect(ready):
                t = clock()
                arr = req.spec.arrival if realtime else 0.0
                lat[req.spec.rid] = t - arr
                svc[req.spec.rid] = t - adm[req.spec.rid]
                cell_updates += float(req.spec.ncells) * r["steps"]
                r["latency"] = t - arr
                r["service"] = svc[req.spec.rid]
                if keep_fields:
                    r["fields"] = [a.cpu().numpy() for a in req.out]
                results[req.spec.rid] = r
                if on_done:
                    on_done(req, r)
                req.out = None
                req.close()
        elif pending:
            time.sleep(max(0.0, min(0.005, pending[0].arrival - clock())))
    makespan = clock()
    L = np.array([lat[k] for k in sorted(lat)])
    S = np.array([svc[k] for k in sorted(svc)])
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    return {"latency": L, "service": S, "results": results, "makespan": makespan,
            "cell_updates": cell_updates, "p50": pct(L, 50), "p99": pct(L, 99),
            "service_p50": pct(S, 50), "service_p99": pct(S, 99)}
