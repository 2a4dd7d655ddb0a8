"""One CW solve split into z slabs over several GPUs (one process per GPU).

The reference runs a large grid over MPI ranks: PETSc cuts the grid into
blocks (``emopt/fdtd.py:263-297``, ``dist_method='x'`` gives one block of
whole planes per rank), and ``GhostComm`` refreshes the one-cell ghost layer
of every block after each half step (``emopt/fdtd.py:1733-1873``,
``src/fdtd.cpp:1789-1929``).  Here each rank holds a slab of planes on its GPU
(``FDTD_slab_*`` in ``include/emopt_fdtd.h``) and exchanges only what the next
half step reads across a slab face (``src/fdtd.cpp:180`` and ``:508``):

* before the H update, Ex and Ey of the first plane of the slab above;
* before the E update, Hx and Hy of the last plane of the slab below.

Two planes of ``Ny * px`` words per direction per half step, sent with NCCL
point-to-point operations on the stream the kernels run on.  The convergence
test is the reference's multi-rank one (``emopt/fdtd.py:411-413`` and
``:1119-1145``): every rank picks ``int(nconv / nranks)`` points of its own
padded local arrays, the values at all points are summed over the ranks (each
value is held by exactly one rank, so the sum is exact), and every rank runs
the same probe on the full list, so every rank takes the same decisions.  The
fields equal those of the single-GPU solve cell for cell.

``LocalLink`` runs several slabs in one process (one GPU or several) with
device copies instead of NCCL; ``TorchLink`` is the multi-process transport
over ``torch.distributed``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import fdtd_ctypes as _ct
from .fdtd import derive_parameters
from .fdtd_ctypes import libFDTD

# the same library without argument types, for device pointers where the
# typed binding expects host arrays
_raw = ctypes.CDLL(_ct.so_path)


def ownership(N: int, n: int) -> list[tuple[int, int]]:
    """(start, count) of the planes of each of ``n`` slabs: the first ``N % n``
    slabs take one plane more (the split of a PETSc DMDA)."""
    if n <= 0 or n > N:
        raise ValueError("cannot split %d planes into %d slabs" % (N, n))
    out, start = [], 0
    for r in range(n):
        c = N // n + (1 if r < N % n else 0)
        out.append((start, c))
        start += c
    return out


def probe_cells(Nx: int, Ny: int, Nz: int, ranges, nconv: int) -> np.ndarray:
    """Global cells read by the convergence probes of a multi-rank run.

    Rank r takes ``arange(0, I*J*K, int(I*J*K / n_pts))`` with
    ``n_pts = int(nconv / nranks)``, indexed into its padded local E arrays
    (``emopt/fdtd.py:411-413``).  A point on a face ghost reads the value the
    ghost exchange leaves there: the adjacent block across a z face, the
    periodic copy within the block across an x or y face, both with
    wrap-around at the grid ends (``emopt/fdtd.py:1795-1842``); edge and corner
    ghosts stay zero (-1 here).  Returns (i*Ny + j)*Nx + k per point, in rank
    order.
    """
    n_pts = int(nconv / len(ranges))
    if n_pts <= 0:
        raise ValueError("nconv = %d gives no probe point per rank for %d ranks" % (nconv, len(ranges)))
    K2, J2 = Nx + 2, Ny + 2
    cells = []
    for i0, I in ranges:
        n = I * Ny * Nx
        for p in np.arange(0, n, int(n / n_pts)):
            ip, rem = divmod(int(p), J2 * K2)
            jp, kp = divmod(rem, K2)
            ghosts = (ip in (0, I + 1)) + (jp in (0, Ny + 1)) + (kp in (0, Nx + 1))
            if ghosts > 1:
                cells.append(-1)
                continue
            k = Nx - 1 if kp == 0 else (0 if kp == Nx + 1 else kp - 1)
            j = Ny - 1 if jp == 0 else (0 if jp == Ny + 1 else jp - 1)
            i = (i0 + ip - 1) % Nz
            cells.append((i * Ny + j) * Nx + k)
    return np.asarray(cells, dtype=np.int64)


def _device_tensor(ptr: int, n: int, dtype, device: int):
    """A torch tensor over ``n`` elements of device memory owned by the library."""
    import torch

    typestr = {np.float32: "<f4", np.float64: "<f8"}[dtype]

    class _Mem:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                    "version": 3, "strides": None}

    return torch.as_tensor(_Mem(), device=torch.device("cuda", device))


class CudaSlab:
    """Planes ``[i0, i0 + I)`` of a CW solve as one resident slab on a GPU.

    ``p`` describes the whole solve like ``emopt_b200.problems.Problem``:
    X, Y, Z, dx, dy, dz, wavelength, w_pml (cells), bc, complex_eps,
    src_ramp_time, mats (six global [Nz, Ny, Nx] complex arrays: eps x/y/z,
    mu x/y/z) and sources [(six arrays [I, J, K], i0, j0, k0)] in global cells.
    """

    def __init__(self, p, i0: int, I: int, precision: str = "fp32", device: int = 0,
                 stream: int | None = None, t0_device: bool = False):
        prm = derive_parameters(p.X, p.Y, p.Z, p.dx, p.dy, p.dz, p.wavelength, 1.0,
                                p.nconv or 10)
        Nx, Ny, Nz = prm["Nx"], prm["Ny"], prm["Nz"]
        if not (0 <= i0 and I > 0 and i0 + I <= Nz):
            raise ValueError("slab [%d, %d) outside %d planes" % (i0, i0 + I, Nz))
        self.Nx, self.Ny, self.Nz, self.i0, self.I = Nx, Ny, Nz, i0, I
        self.dt = prm["dt"]
        self.device = device
        self.stream = stream
        self.dtype = np.float32 if precision == "fp32" else np.float64
        h = libFDTD.FDTD_new()
        self.h = h
        if libFDTD.FDTD_set_device(h, int(device)) != _ct.FDTD_OK:
            raise _ct.FDTDError(_ct.last_error(h)[1])
        libFDTD.FDTD_set_wavelength(h, p.wavelength)
        libFDTD.FDTD_set_physical_dims(h, prm["X"], prm["Y"], p.dz * (I - 1), p.dx, p.dy, p.dz)
        libFDTD.FDTD_set_grid_dims(h, Nx, Ny, I)
        libFDTD.FDTD_set_local_grid(h, 0, 0, 0, Nx, Ny, I)
        libFDTD.FDTD_set_dt(h, self.dt)
        self._mats = [np.ascontiguousarray(np.asarray(a)[i0:i0 + I], dtype=np.complex128).ravel()
                      for a in p.mats]
        libFDTD.FDTD_set_mat_arrays(h, *self._mats)
        libFDTD.FDTD_set_complex_eps(h, bool(p.complex_eps))
        libFDTD.FDTD_set_precision(h, 32 if precision == "fp32" else 64)
        libFDTD.FDTD_set_kernel(h, 5)
        libFDTD.FDTD_set_pml_widths(h, *[int(w) for w in p.w_pml])
        libFDTD.FDTD_set_pml_properties(h, 3.0, 0.0, 1.0, 3.0)
        libFDTD.FDTD_build_pml(h)
        src_T = p.src_ramp_time if p.src_ramp_time is not None else prm["src_T"]
        libFDTD.FDTD_set_source_properties(h, src_T, prm["src_min"])
        libFDTD.FDTD_set_bc(h, p.bc.encode("ascii"))
        n = Nx * Ny * I
        self._t1 = [np.zeros(n, dtype=np.complex128) for _ in range(6)]
        self.t0_device = t0_device
        if t0_device:
            # phasors stay on the GPU (torch tensors the extraction writes into)
            import torch
            self.t0 = [torch.zeros((I, Ny, Nx), dtype=torch.complex128,
                                   device=torch.device("cuda", device)) for _ in range(6)]
            _raw.FDTD_set_t0_arrays(h, *[ctypes.c_void_p(t.data_ptr()) for t in self.t0])
        else:
            self.t0 = [np.zeros(n, dtype=np.complex128) for _ in range(6)]
            libFDTD.FDTD_set_t0_arrays(h, *self.t0)
        libFDTD.FDTD_set_t1_arrays(h, *self._t1)
        # sources cropped to the slab, in slab coordinates, converted to
        # amplitude/phase by the library (emopt/fdtd.py:710-747)
        self._src = []
        for arrays, si0, sj0, sk0 in p.sources:
            sI, sJ, sK = np.asarray(arrays[0]).shape
            lo, hi = max(si0, i0), min(si0 + sI, i0 + I)
            if lo >= hi:
                continue
            cut = [np.ascontiguousarray(np.asarray(a, dtype=np.complex128)[lo - si0:hi - si0]).ravel().copy()
                   for a in arrays]
            self._src.append(cut)
            libFDTD.FDTD_add_source(h, *cut, lo - i0, sj0, sk0, hi - lo, sJ, sK, True)
        _ct.check(h, "slab set-up")
        if libFDTD.FDTD_slab_set(h, i0, Nz, int(i0 > 0), int(i0 + I < Nz)) != _ct.FDTD_OK:
            raise _ct.FDTDError(_ct.last_error(h)[1])
        if stream is not None and libFDTD.FDTD_set_stream(h, ctypes.c_void_p(stream)) != _ct.FDTD_OK:
            raise _ct.FDTDError(_ct.last_error(h)[1])
        self.has_lo, self.has_hi = i0 > 0, i0 + I < Nz
        self.halo = None
        self.samples = None

    def _ok(self, rc, what):
        if rc != _ct.FDTD_OK:
            raise _ct.FDTDError("%s: %s" % (what, _ct.last_error(self.h)[1]))

    def begin(self, Tn: int, fixed_steps: int, Nmax: float, cells: np.ndarray):
        opt = _ct.SolveOptions()
        opt.Tn = int(Tn)
        opt.Nmax = float(Nmax)
        opt.fixed_steps = int(fixed_steps or 0)
        opt.materials_unchanged = 0
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        self._ok(libFDTD.FDTD_slab_begin(self.h, ctypes.byref(opt), cells, len(cells)), "FDTD_slab_begin")
        ptrs = (ctypes.c_void_p * 8)()
        pe = ctypes.c_longlong()
        self._ok(libFDTD.FDTD_slab_halo(self.h, ptrs, ctypes.byref(pe)), "FDTD_slab_halo")
        t = [_device_tensor(ptrs[q], pe.value, self.dtype, self.device) for q in range(8)]
        self.halo = {"E_send": t[0:2], "E_recv": t[2:4], "H_send": t[4:6], "H_recv": t[6:8]}
        sp = ctypes.c_void_p()
        self._ok(libFDTD.FDTD_slab_sample(self.h, ctypes.byref(sp)), "FDTD_slab_sample")
        self.samples = _device_tensor(sp.value, 3 * max(len(cells), 1), np.float64, self.device)

    def set_halo_source(self, above=None, below=None):
        """Read the neighbour planes from other planes of this device:
        ``above`` = (Ex, Ey) of the plane above the slab, ``below`` = (Hx, Hy)
        of the plane below (tensors); None keeps the slab's own halo planes
        (FDTD_slab_set_halo_source)."""
        ptrs = (ctypes.c_void_p * 4)(*([t.data_ptr() for t in above] if above else [None, None]),
                                     *([t.data_ptr() for t in below] if below else [None, None]))
        self._ok(libFDTD.FDTD_slab_set_halo_source(self.h, ptrs), "FDTD_slab_set_halo_source")

    def half_step(self, n: int, half: int):
        self._ok(libFDTD.FDTD_slab_step(self.h, n, half), "FDTD_slab_step")

    def set_step(self, base: int):
        """Device step base of the half steps (FDTD_slab_set_step)."""
        self._ok(libFDTD.FDTD_slab_set_step(self.h, int(base)), "FDTD_slab_set_step")

    def use_stream(self, stream):
        """Launch on ``stream`` (a CUDA stream handle) until told otherwise;
        the slab's own stream is ``self.stream``."""
        self._ok(libFDTD.FDTD_set_stream(self.h, ctypes.c_void_p(stream)), "FDTD_set_stream")

    def half_step_part(self, n: int, half: int, part: int):
        """Part 1: the planes that read no halo plane; part 2: the plane next to
        the neighbour's halo (FDTD_slab_step_part)."""
        self._ok(libFDTD.FDTD_slab_step_part(self.h, n, half, part), "FDTD_slab_step_part")

    def sample(self):
        sp = ctypes.c_void_p()
        self._ok(libFDTD.FDTD_slab_sample(self.h, ctypes.byref(sp)), "FDTD_slab_sample")
        return self.samples

    def probe(self, n_last: int):
        A, P = ctypes.c_double(), ctypes.c_double()
        self._ok(libFDTD.FDTD_slab_probe(self.h, n_last, ctypes.byref(A), ctypes.byref(P)),
                 "FDTD_slab_probe")
        return A.value, P.value

    def capture(self, which: int):
        self._ok(libFDTD.FDTD_slab_capture(self.h, which), "FDTD_slab_capture")

    def finish(self, n0: int, Tn: int):
        self._ok(libFDTD.FDTD_slab_finish(self.h, n0, Tn), "FDTD_slab_finish")
        if self.t0_device:
            return list(self.t0)
        return [a.reshape(self.I, self.Ny, self.Nx) for a in self.t0]

    def close(self):
        if self.h is not None:
            libFDTD.FDTD_delete(self.h)
            self.h = None


class LocalLink:
    """Slabs of one process: halo planes and probe sums move by device copies.

    Direct (``direct=True``, every slab on one device and one stream): no
    copies at all -- each slab's half steps read the neighbour planes in the
    neighbouring slabs' own arrays (``attach``, FDTD_slab_set_halo_source);
    stream order puts every H half step of a step before every E half step.
    Plain (``overlap=False``): the copies run in stream order on the slabs'
    stream, between the half steps.  Overlapped: each copy runs on a side
    stream of the receiving device, after everything queued so far on the
    sending slab's stream, and the receiving slab's stream waits for it only
    before the plane that reads the halo; the half steps run in two parts
    around it like the NCCL transport's.  With ``graphs`` (one device and one
    stream, plain schedule) the steps between two probes are captured once as
    a CUDA graph and replayed from the slabs' device step base."""

    def __init__(self, slabs, overlap=False, direct=False, graphs=False):
        one_stream = (not (direct or graphs)) or len({(s.device, s.stream) for s in slabs}) == 1
        if direct and overlap:
            raise ValueError("direct halo reads need no exchange to overlap")
        if direct and not one_stream:
            raise ValueError("direct halo reads need all slabs on one device and one stream")
        if graphs and (overlap or not one_stream):
            raise ValueError("graph replays need the plain schedule on one device and one stream")
        self.slabs = slabs
        self.direct = bool(direct)
        self.overlap = bool(overlap)
        # graphs: run() replays one captured time step of every slab (kernels
        # and copies) instead of launching from the host step by step
        self.graphs = bool(graphs)
        self._graphs = {}
        self._sides = {}
        self._streams = {}
        self._pending = {"E": [], "H": []}
        if self.overlap and any(s.stream is None for s in slabs):
            raise ValueError("overlapped device copies need the slabs' streams")

    def _stream(self, slab):
        """The torch stream object of the stream the slab's library calls
        run on.  Handle 0 is the device's legacy default stream:
        ``torch.cuda.ExternalStream(0)`` does not stand for it, so it is taken
        from ``torch.cuda.default_stream``."""
        st = self._streams.get(id(slab))
        if st is None:
            import torch
            dev = torch.device("cuda", slab.device)
            st = (torch.cuda.default_stream(dev) if not slab.stream
                  else torch.cuda.ExternalStream(slab.stream, device=dev))
            if st.cuda_stream != (slab.stream or 0):
                raise RuntimeError("no torch stream object for the slab's stream")
            self._streams[id(slab)] = st
        return st

    def attach(self):
        """After every slab's begin (which places its arrays): drop the
        captured step; in direct mode point every slab at its neighbours'
        boundary planes."""
        self._graphs = {}
        if not self.direct:
            return
        for q, s in enumerate(self.slabs):
            above = self.slabs[q + 1].halo["E_send"] if q + 1 < len(self.slabs) else None
            below = self.slabs[q - 1].halo["H_send"] if q > 0 else None
            s.set_halo_source(above, below)

    def _steps_graph(self, count):
        """``count`` time steps of every slab captured as one CUDA graph (per
        step: the E exchange, every H half step, the H exchange, every E half
        step), the half steps captured with n = 0 .. count - 1 relative to the
        slabs' device step base."""
        g = self._graphs.get(count)
        if g is None:
            import torch
            s0 = self.slabs[0]
            main = self._stream(s0)
            cap = torch.cuda.Stream(device=torch.device("cuda", s0.device))
            cap.wait_stream(main)
            g = torch.cuda.CUDAGraph()
            for s in self.slabs:
                s.use_stream(cap.cuda_stream)
            try:
                with torch.cuda.graph(g, stream=cap):
                    for m in range(count):
                        self.exchange_E()
                        for s in self.slabs:
                            s.half_step(m, 0)
                        self.exchange_H()
                        for s in self.slabs:
                            s.half_step(m, 1)
            finally:
                for s in self.slabs:
                    s.use_stream(s.stream)
            main.wait_stream(cap)
            self._graphs[count] = g
        return g

    def steps(self, n, count):
        """Steps n .. n + count - 1 of every slab as one graph replay (one
        graph per distinct count: the probe period, the tail run)."""
        if count <= 0:
            return
        import torch
        g = self._steps_graph(count)
        for s in self.slabs:
            s.set_step(n)
        with torch.cuda.stream(self._stream(self.slabs[0])):
            g.replay()
        for s in self.slabs:
            s.set_step(0)

    def _start(self, which, pairs):
        """pairs: (receiving slab, destination, sending slab, source)."""
        if self.direct:
            return
        if not self.overlap:
            for _, dst, _, src in pairs:
                dst.copy_(src)
            return
        import torch
        done = []
        for rs, dst, ss, src in pairs:
            side = self._sides.get(rs.device)
            if side is None:
                side = self._sides[rs.device] = torch.cuda.Stream(device=torch.device("cuda", rs.device))
            # the source plane is written, and the previous reader of the
            # destination has run, by everything queued so far
            side.wait_stream(self._stream(ss))
            side.wait_stream(self._stream(rs))
            with torch.cuda.stream(side):
                dst.copy_(src, non_blocking=True)
            done.append((rs, side.record_event()))
        self._pending[which] = done

    def _wait(self, which):
        for rs, ev in self._pending[which]:
            self._stream(rs).wait_event(ev)
        self._pending[which] = []

    def start_E(self):
        self._start("E", [(lo, lo.halo["E_recv"][c], hi, hi.halo["E_send"][c])
                          for lo, hi in zip(self.slabs[:-1], self.slabs[1:]) for c in range(2)])

    def start_H(self):
        self._start("H", [(hi, hi.halo["H_recv"][c], lo, lo.halo["H_send"][c])
                          for lo, hi in zip(self.slabs[:-1], self.slabs[1:]) for c in range(2)])

    def wait_E(self):
        self._wait("E")

    def wait_H(self):
        self._wait("H")

    def exchange_E(self):
        self.start_E()
        self.wait_E()

    def exchange_H(self):
        self.start_H()
        self.wait_H()

    def sum_samples(self, tensors):
        total = tensors[0].clone()
        for t in tensors[1:]:
            total += t.to(total.device)
        for t in tensors:
            t.copy_(total)


class TorchLink:
    """One slab per process; neighbours are ranks - 1 and + 1 of the default
    ``torch.distributed`` group (NCCL on GPUs, gloo on CPU tensors)."""

    # transfers between processes run beside the kernels: overlap them with
    # the planes that do not need the halo
    overlap = True

    def __init__(self, slab):
        import torch.distributed as dist
        self.dist = dist
        self.slabs = [slab]
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()

        self._pending = {"E": [], "H": []}

    def _swap(self, send, send_to, recv, recv_from):
        """Start the point-to-point operations; returns their works."""
        dist = self.dist
        ops = []
        if recv_from is not None:
            ops += [dist.P2POp(dist.irecv, t, recv_from) for t in recv]
        if send_to is not None:
            ops += [dist.P2POp(dist.isend, t, send_to) for t in send]
        return dist.batch_isend_irecv(ops) if ops else []

    def start_E(self):
        s = self.slabs[0]
        self._pending["E"] = self._swap(s.halo["E_send"], self.rank - 1 if s.has_lo else None,
                                        s.halo["E_recv"], self.rank + 1 if s.has_hi else None)

    def start_H(self):
        s = self.slabs[0]
        self._pending["H"] = self._swap(s.halo["H_send"], self.rank + 1 if s.has_hi else None,
                                        s.halo["H_recv"], self.rank - 1 if s.has_lo else None)

    def _wait(self, which):
        # on CUDA tensors the wait orders the current stream after the
        # transfer (the host does not block); on CPU tensors it blocks
        for w in self._pending[which]:
            w.wait()
        self._pending[which] = []

    def wait_E(self):
        self._wait("E")

    def wait_H(self):
        self._wait("H")

    def exchange_E(self):
        self.start_E()
        self.wait_E()

    def exchange_H(self):
        self.start_H()
        self.wait_H()

    def sum_samples(self, tensors):
        for t in tensors:
            self.dist.all_reduce(t)


@dataclass
class SlabResult:
    n_main: int
    steps: int
    A_change: float
    phi_change: float
    nprobes: int
    converged: bool


def run(slabs, link, Tn: int, rtol: float, Nmax: float, fixed_steps: int | None = None,
        history: list | None = None) -> SlabResult:
    """The loop of ``FDTD_solve_cw`` (``emopt/fdtd.py:1016-1194``) over the
    slabs of this process, with the halo exchange before each half step and
    the probe on the values of all slabs every Tn steps."""
    fixed = bool(fixed_steps)
    last = fixed_steps - 1 if fixed else int(np.floor(Nmax))

    def steps_plain(n, count):
        for m in range(n, n + count):
            link.exchange_E()
            for s in slabs:
                s.half_step(m, 0)
            link.exchange_H()
            for s in slabs:
                s.half_step(m, 1)

    def steps_overlapped(n, count):
        # Each exchange overlaps the planes that do not need it: the H update
        # of every plane but the top one runs while the E halo from above is in
        # flight, then the top plane; the H halo goes up while the E update of
        # every plane but the bottom one runs, then the bottom plane; the E
        # halo leaves at the end of the step (the fields it carries do not
        # change before the next step's H update reads them).
        if count <= 0:
            return
        link.start_E()
        for m in range(n, n + count):
            for s in slabs:
                s.half_step_part(m, 0, 1)
            link.wait_E()
            for s in slabs:
                s.half_step_part(m, 0, 2)
            link.start_H()
            for s in slabs:
                s.half_step_part(m, 1, 1)
            link.wait_H()
            for s in slabs:
                s.half_step_part(m, 1, 2)
            if m + 1 < n + count:
                link.start_E()

    steps = steps_overlapped if getattr(link, "overlap", False) else steps_plain
    if getattr(link, "graphs", False):
        steps = link.steps

    def probe(n_last):
        link.sum_samples([s.sample() for s in slabs])
        vals = [s.probe(n_last) for s in slabs]
        return vals[0]

    n, Ach, Pch, nprobes = 0, 1.0, 1.0, 0
    amp_tol, phi_tol = rtol, np.sqrt(rtol)

    def not_converged():
        if fixed:
            return True
        return (Ach > amp_tol or Pch > phi_tol or not np.isfinite(Ach) or not np.isfinite(Pch))

    while not_converged():
        if n > (last if fixed else Nmax):
            break
        if n + Tn - 1 > last:
            steps(n, last - n + 1)
            n = last + 1
            continue
        steps(n, Tn)
        Ach, Pch = probe(n + Tn - 1)
        nprobes += 1
        if history is not None:
            history.append((n + Tn - 1, Ach, Pch))
        n += Tn
    n0 = n
    for s in slabs:
        s.capture(0)
    steps(n0, Tn)
    for s in slabs:
        s.capture(1)
    steps(n0 + Tn, Tn)
    converged = fixed or not not_converged()
    return SlabResult(n_main=n0, steps=n0 + 2 * Tn, A_change=Ach, phi_change=Pch,
                      nprobes=nprobes, converged=converged)


class SlabSet:
    """The slabs of problem ``p`` that this process holds, set up and linked.

    In one process (``rank`` None) every slab of ``ranges`` [(i0, I), ...] is
    built here, on ``devices[s]`` (one device or none: that device, or GPU 0,
    for all), and linked by device copies.  Under ``torch.distributed`` (``rank`` given) this process
    builds slab ``rank`` only, on ``devices[0]``, and exchanges through
    ``TorchLink``.  ``begin()`` resets the fields for a new solve, ``run()``
    steps it, ``finish()`` extracts {slab index: six complex [I, Ny, Nx] arrays}.
    """

    def __init__(self, p, ranges, precision="fp32", devices=None, link=None, rank=None,
                 stream=None, t0_device=False, overlap=False, direct=None, graphs=None):
        prm = derive_parameters(p.X, p.Y, p.Z, p.dx, p.dy, p.dz, p.wavelength, 1.0, p.nconv or 10)
        Nx, Ny, Nz = prm["Nx"], prm["Ny"], prm["Nz"]
        self.p = p
        self.Tn = prm["Tn"]
        self.Nmax = p.Nmax if p.Nmax is not None else prm["Nmax"]
        self.cells = probe_cells(Nx, Ny, Nz, ranges, p.nconv or 10)
        self.mine = list(range(len(ranges))) if rank is None else [rank]
        devices = list(devices or [0])
        if rank is None and len(devices) == 1:
            devices = devices * len(ranges)
        devs = [devices[s] if rank is None else devices[0] for s in self.mine]
        if stream is None:
            # the kernels, the copies or NCCL transfers and the probe sums share
            # each device's current torch stream, which orders them
            import torch
            streams = [torch.cuda.current_stream(d).cuda_stream for d in devs]
        else:
            streams = [stream] * len(self.mine)
        self.slabs = []
        try:
            for s, d, st in zip(self.mine, devs, streams):
                self.slabs.append(CudaSlab(p, *ranges[s], precision=precision, device=d, stream=st,
                                           t0_device=t0_device))
        except Exception:
            self.close()
            raise
        self.link = link
        self.rank = rank
        self.overlap = overlap
        # slabs of one process on one device read each other's planes
        # directly unless told otherwise (or asked to overlap copies)
        if direct is None:
            direct = (rank is None and not overlap and len(self.slabs) > 1 and
                      len({(s.device, s.stream) for s in self.slabs}) == 1)
        self.direct = bool(direct)
        # ... and replay one captured step (CUDA graph) on one device and stream
        if graphs is None:
            graphs = (rank is None and not overlap and
                      len({(s.device, s.stream) for s in self.slabs}) == 1)
        self.graphs = bool(graphs)
        self.res = None

    def begin(self):
        for s in self.slabs:
            s.begin(self.Tn, self.p.fixed_steps, self.Nmax, self.cells)
        if self.link is None:
            self.link = (LocalLink(self.slabs, overlap=self.overlap, direct=self.direct,
                                   graphs=self.graphs)
                         if self.rank is None else TorchLink(self.slabs[0]))
        if hasattr(self.link, "attach"):
            self.link.attach()

    def run(self, history=None) -> SlabResult:
        self.res = run(self.slabs, self.link, self.Tn, self.p.rtol, self.Nmax, self.p.fixed_steps,
                       history)
        return self.res

    def finish(self):
        return {s_idx: sl.finish(self.res.n_main, self.Tn) for s_idx, sl in zip(self.mine, self.slabs)}

    def close(self):
        for s in self.slabs:
            s.close()


def grad_eps_planar(fwd, adj, box, ranges, link, device=0):
    """Permittivity gradient of a planar design over the slabs: each slab runs
    the fused overlap ``FDTD_grad_eps`` (Kahan z-sums) on its own planes of the
    design layer, and the per-column partial sums are added over the slabs --
    in one process directly, over ranks with an all-reduce (``link``).

    ``fwd`` / ``adj``: {slab index: six device phasor tensors [I, Ny, Nx]} of
    the slabs this process holds (``SlabSet(..., t0_device=True).finish()``);
    ``box``: k0, k1, j0, j1 and the z range [i0_c, i1_c) of each E component
    in global planes.  Returns the (3, j1 - j0, k1 - k0) float64 tensor that
    ``adjoint.AdjointSolver.grad_eps`` gives on one GPU."""
    import torch
    k0, k1, j0, j1 = box[:4]
    dev = torch.device("cuda", device)
    total = torch.zeros((3, j1 - j0, k1 - k0), dtype=torch.float64, device=dev)
    for s, F in fwd.items():
        i0s, I = ranges[s]
        A = adj[s]
        Iz, Ny, Nx = F[0].shape
        local = [k0, k1, j0, j1]
        for c in range(3):
            a, b = box[4 + 2 * c], box[5 + 2 * c]
            lo, hi = max(a, i0s), min(b, i0s + I)
            local += [lo - i0s, hi - i0s] if lo < hi else [0, 0]
        out = torch.empty((3, j1 - j0, k1 - k0), dtype=torch.float64, device=F[0].device)
        fp = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in F[:3]])
        ap = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in A[:3]])
        msg = ctypes.create_string_buffer(256)
        st = libFDTD.FDTD_grad_eps(F[0].device.index, torch.cuda.current_stream(F[0].device).cuda_stream,
                                   fp, ap, Nx, Ny, Iz, (ctypes.c_int * 10)(*local), 1,
                                   ctypes.c_void_p(out.data_ptr()), msg, len(msg))
        if st != _ct.FDTD_OK:
            raise _ct.FDTDError(msg.value.decode())
        total += out.to(dev)
    if isinstance(link, TorchLink):
        link.dist.all_reduce(total)
    return total


def solve(p, ranges, precision="fp32", devices=None, link=None, rank=None, stream=None,
          overlap=False, direct=None, graphs=None):
    """Solve problem ``p`` split into the slabs ``ranges`` (see ``SlabSet``).
    Returns (result, {slab index: six complex [I, Ny, Nx] arrays})."""
    ss = SlabSet(p, ranges, precision, devices, link, rank, stream, overlap=overlap, direct=direct,
                 graphs=graphs)
    try:
        ss.begin()
        res = ss.run()
        return res, ss.finish()
    finally:
        ss.close()
