"""CPU tests of the z-slab decomposition (emopt_b200/zslab.py).

* the slab split and the probe-point rule against the reference's multi-rank
  ghost semantics (the oracle's z-slab run keeps GhostComm's padded arrays);
* the multi-GPU loop (``zslab.run``) with its transports, driven on the CPU
  by one oracle instance per slab: in one process (``LocalLink``) and as two
  gloo ranks (``TorchLink``), against the oracle's own multi-rank solve.
"""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from emopt_b200 import problems as P
from emopt_b200 import zslab
from helpers import ROOT, oracle_for, oracle_lib

CASES = {
    # 3 slabs of 3 planes; z CPML of 3 / 4 planes covers slabs 0 and 2 whole
    "pec3": (dict(seed=31, shape=(9, 7, 12), bc="000", edge_source=True), 3),
    # symmetric min faces, a source box across both slab faces
    "sym2": (dict(seed=32, shape=(8, 6, 10), bc="EH0", n_sources=2), 2),
    # lossy, z-min symmetry plane ('E'), uneven split 4 + 3 + 3
    "lossy3": (dict(seed=33, shape=(10, 6, 9), complex_eps=True, bc="0HE"), 3),
}


def _problem(name, **over):
    kw, nslab = CASES[name]
    kw = dict(kw, **over)
    return P.random_box(**kw), nslab


def test_ownership_is_the_dmda_split():
    assert zslab.ownership(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert zslab.ownership(9, 3) == [(0, 3), (3, 3), (6, 3)]
    assert zslab.ownership(5, 5) == [(q, 1) for q in range(5)]
    for N, n in [(101, 8), (301, 8), (17, 4)]:
        r = zslab.ownership(N, n)
        assert sum(c for _, c in r) == N and all(r[q + 1][0] == r[q][0] + r[q][1] for q in range(n - 1))
    with pytest.raises(ValueError):
        zslab.ownership(3, 4)
    with pytest.raises(ValueError):
        zslab.probe_cells(10, 10, 10, zslab.ownership(10, 3), 2)


@pytest.mark.parametrize("name", list(CASES))
def test_probe_cells_read_what_the_reference_ghosts_hold(name):
    """Every rank's probe points in its padded local E arrays (ghosts filled as
    GhostComm leaves them) hold the value of the global cell probe_cells names."""
    p, nslab = _problem(name, fixed_steps=12)
    Nz, Ny, Nx = p.shape
    ranges = zslab.ownership(Nz, nslab)
    nconv = 40                       # 40 / nslab points per rank: x/y ghosts among them
    cells = zslab.probe_cells(Nx, Ny, Nz, ranges, nconv)
    o = oracle_for(p, oracle_lib())
    slab_run = o.run_fixed_slabs(12, len(ranges), ranges=ranges, extract=False)
    whole = oracle_for(p, oracle_lib()).solve(fixed_steps=12)
    Eg = [a[1:-1, 1:-1, 1:-1].ravel() for a in whole["E"]]
    q = 0
    ghosts = 0
    for (i0, I), Epad in zip(ranges, slab_run["E_pad"]):
        n = I * Ny * Nx
        for pt in np.arange(0, n, int(n / int(nconv / nslab))):
            for c in range(3):
                want = Eg[c][cells[q]] if cells[q] >= 0 else 0.0
                assert Epad[c].ravel()[pt] == want, (q, c)
            ip, rem = divmod(int(pt), (Ny + 2) * (Nx + 2))
            jp, kp = divmod(rem, Nx + 2)
            ghosts += ip in (0, I + 1) or jp in (0, Ny + 1) or kp in (0, Nx + 1)
            q += 1
    assert q == len(cells) and ghosts > 0


def _oracle_slabs(p, ranges, cells, fixed):
    from zslab_oracle import OracleSlab
    prm_Tn = int(np.int64(oracle_for(p, oracle_lib()).Ncycle * 3 / 4))
    slabs = [OracleSlab(p, i0, I, oracle_lib()) for i0, I in ranges]
    Nmax = p.Nmax if p.Nmax is not None else oracle_for(p, oracle_lib()).Nmax
    for s in slabs:
        s.begin(prm_Tn, fixed, Nmax, cells)
    return slabs, prm_Tn, Nmax


@pytest.mark.parametrize("name", list(CASES))
def test_loop_in_one_process_matches_reference_multirank(name):
    """zslab.run over LocalLink reproduces the oracle's multi-rank solve: step
    count, convergence history and fields, bit for bit."""
    p, nslab = _problem(name, fixed_steps=None, rtol=1e-4)
    p.Nmax = 3000
    Nz, Ny, Nx = p.shape
    ranges = zslab.ownership(Nz, nslab)
    cells = zslab.probe_cells(Nx, Ny, Nz, ranges, 10)
    ref = oracle_for(p, oracle_lib()).solve_slabs(ranges, nconv=10, record=True)
    slabs, Tn, Nmax = _oracle_slabs(p, ranges, cells, None)
    hist = []
    res = zslab.run(slabs, zslab.LocalLink(slabs), Tn, p.rtol, Nmax, None, history=hist)
    assert res.n_main == ref["n_main"] and res.steps == ref["steps"]
    assert [h[0] for h in hist] == [h[0] for h in ref["history"]]
    assert [h[1:] for h in hist] == [h[1:] for h in ref["history"]]
    F = [np.concatenate(parts) for parts in zip(*[s.finish(res.n_main, Tn) for s in slabs])]
    for c in range(6):
        assert np.array_equal(F[c], ref["fields"][c]), c


def _gloo_worker(rank, world, port, name, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p, _ = _problem(name, fixed_steps=None, rtol=1e-4)
        p.Nmax = 3000
        Nz, Ny, Nx = p.shape
        ranges = zslab.ownership(Nz, world)
        cells = zslab.probe_cells(Nx, Ny, Nz, ranges, 10)
        slabs, Tn, Nmax = _oracle_slabs(p, [ranges[rank]], cells, None)
        res = zslab.run(slabs, zslab.TorchLink(slabs[0]), Tn, p.rtol, Nmax, None)
        F = slabs[0].finish(res.n_main, Tn)
        out.put((rank, res.n_main, res.steps, res.A_change, [np.array(a) for a in F]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_match_reference_multirank():
    """Two processes, one slab each, halos and probe sums over gloo."""
    name = "sym2"
    p, _ = _problem(name, fixed_steps=None, rtol=1e-4)
    p.Nmax = 3000
    ranges = zslab.ownership(p.shape[0], 2)
    ref = oracle_for(p, oracle_lib()).solve_slabs(ranges, nconv=10)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, name, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted((q.get(timeout=280) for _ in procs), key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=30)
        assert pr.exitcode == 0
    for rank, n_main, steps, A, F in res:
        assert n_main == ref["n_main"] and steps == ref["steps"]
        assert A == ref["A_change"]
    for c in range(6):
        assert np.array_equal(np.concatenate([r[4][c] for r in res]), ref["fields"][c]), c


def test_halo_source_checks_on_the_host():
    """FDTD_slab_set_halo_source accepts neighbour planes only on the faces that
    have a neighbour, and only on a slab handle (host-side checks; no device
    work)."""
    import ctypes
    from emopt_b200 import fdtd_ctypes as ct
    lib = ct.libFDTD
    h = lib.FDTD_new()
    try:
        lib.FDTD_set_grid_dims(h, 10, 8, 4)
        lib.FDTD_set_local_grid(h, 0, 0, 0, 10, 8, 4)
        buf = ctypes.create_string_buffer(64)
        some = ctypes.cast(buf, ctypes.c_void_p).value
        none4 = (ctypes.c_void_p * 4)()
        above = (ctypes.c_void_p * 4)(some, some, None, None)
        below = (ctypes.c_void_p * 4)(None, None, some, some)
        assert lib.FDTD_slab_set_halo_source(h, none4) == ct.FDTD_ERR_ARG        # not a slab
        assert lib.FDTD_slab_set(h, 0, 12, 0, 1) == ct.FDTD_OK                    # bottom slab
        assert lib.FDTD_slab_set_halo_source(h, below) == ct.FDTD_ERR_ARG         # nothing below
        assert lib.FDTD_slab_set_halo_source(h, above) == ct.FDTD_OK
        assert lib.FDTD_slab_set_halo_source(h, none4) == ct.FDTD_OK              # back to its own halo
        assert lib.FDTD_slab_set(h, 8, 12, 1, 0) == ct.FDTD_OK                    # top slab
        assert lib.FDTD_slab_set_halo_source(h, above) == ct.FDTD_ERR_ARG         # nothing above
        assert lib.FDTD_slab_set_halo_source(h, below) == ct.FDTD_OK
    finally:
        lib.FDTD_delete(h)
