"""GPU tests of the z-slab solve (FDTD_slab_* through emopt_b200/zslab.py).

All slabs run on one GPU in one process (``LocalLink``: halo planes move by
device copies on the stream the kernels use), which exercises every kernel
and exchange path of the multi-GPU solve; the NCCL transport differs only in
how the same planes travel (``TorchLink``, covered over gloo on the CPU).

* fixed step counts: the fields equal the single-GPU solve of the whole grid
  bit for bit (fp64 and fp32), for 2 and 3 slabs, with CPML slabs and source
  boxes across slab faces and symmetric / lossy cases;
* converging runs: step count and fields of the reference's multi-rank solve
  (the oracle over the same slabs), fp64 to 1e-11 relative.
"""
import numpy as np
import pytest

from emopt_b200 import problems as P
from emopt_b200 import zslab
from helpers import oracle_for, oracle_lib, rel_l2

pytestmark = pytest.mark.gpu

CASES = {
    "pec3": (dict(seed=31, shape=(9, 7, 12), bc="000", edge_source=True), 3),
    "sym2": (dict(seed=32, shape=(8, 6, 10), bc="EH0", n_sources=2), 2),
    "lossy3": (dict(seed=33, shape=(10, 6, 9), complex_eps=True, bc="0HE"), 3),
    "mu_wide": (dict(seed=34, shape=(16, 9, 70), mu_random=True, bc="000",
                     w_pml=(5, 5, 4, 4, 6, 5), edge_source=True), 4),
}


def _single(p, precision):
    sim = P.make_solver(p, precision=precision, kernel="vector")
    info = sim._solve([sim._Ex_fwd_t0, sim._Ey_fwd_t0, sim._Ez_fwd_t0, sim._Hx_fwd_t0,
                       sim._Hy_fwd_t0, sim._Hz_fwd_t0],
                      [sim._Ex_fwd_t1, sim._Ey_fwd_t1, sim._Ez_fwd_t1, sim._Hx_fwd_t1,
                       sim._Hy_fwd_t1, sim._Hz_fwd_t1], sim._sources)
    return np.stack([sim._raw(c, False) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")]), info


def _slabs(p, nslab, precision, mode="direct"):
    """mode: "direct" (the slabs read each other's boundary planes in place,
    one captured time step replayed as a CUDA graph), "direct-loop" (the same
    launched from the host step by step), "copy" (halo planes exchanged by
    device copies between the half steps, graph replays) or "overlap" (copies
    on a side stream, the half steps in two parts around them)."""
    ranges = zslab.ownership(p.shape[0], nslab)
    direct = mode.startswith("direct")
    ss = zslab.SlabSet(p, ranges, precision=precision, overlap=mode == "overlap",
                       direct=None if direct else False,
                       graphs=False if mode == "direct-loop" else None)
    try:
        ss.begin()
        assert ss.link.direct == direct and ss.link.overlap == (mode == "overlap")
        assert ss.link.graphs == (mode in ("direct", "copy"))
        res = ss.run()
        parts = ss.finish()
    finally:
        ss.close()
    F = np.stack([np.concatenate([parts[s][c] for s in range(len(ranges))]) for c in range(6)])
    return F, res


@pytest.mark.parametrize("mode", ["direct", "direct-loop", "copy"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(CASES))
def test_fixed_steps_equal_single_gpu_solve(name, precision, mode):
    kw, nslab = CASES[name]
    p = P.random_box(**dict(kw, fixed_steps=150))
    F1, info = _single(p, precision)
    F, res = _slabs(p, nslab, precision, mode)
    assert res.steps == info["steps"] and res.n_main == info["n_main"]
    assert np.array_equal(F, F1)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(CASES))
def test_overlapped_schedule_equals_single_gpu_solve(name, precision):
    """The split half steps of the overlapped loop give the same fields, bit
    for bit, as the whole-grid solve."""
    kw, nslab = CASES[name]
    p = P.random_box(**dict(kw, fixed_steps=150))
    F1, info = _single(p, precision)
    F, res = _slabs(p, nslab, precision, "overlap")
    assert res.steps == info["steps"] and res.n_main == info["n_main"]
    assert np.array_equal(F, F1)


@pytest.mark.parametrize("name", ["pec3", "sym2", "lossy3"])
def test_converging_run_matches_reference_multirank(name):
    kw, nslab = CASES[name]
    p = P.random_box(**dict(kw, fixed_steps=None, rtol=1e-4))
    p.Nmax = 3000
    ranges = zslab.ownership(p.shape[0], nslab)
    ref = oracle_for(p, oracle_lib()).solve_slabs(ranges, nconv=10)
    F, res = _slabs(p, nslab, "fp64")
    assert res.n_main == ref["n_main"] and res.steps == ref["steps"]
    assert res.A_change == pytest.approx(ref["A_change"], rel=1e-6)
    assert rel_l2(F, np.stack(ref["fields"])) < 1e-11


def test_slab_api_rejects_misuse():
    from emopt_b200 import fdtd_ctypes as ct
    lib = ct.libFDTD
    h = lib.FDTD_new()
    try:
        lib.FDTD_set_grid_dims(h, 10, 8, 4)
        lib.FDTD_set_local_grid(h, 0, 0, 0, 10, 8, 4)
        # neighbours that do not match the slab's place
        assert lib.FDTD_slab_set(h, 0, 12, 1, 1) == ct.FDTD_ERR_ARG
        assert lib.FDTD_slab_set(h, 10, 12, 1, 0) == ct.FDTD_ERR_ARG
        # stepping before FDTD_slab_begin
        assert lib.FDTD_slab_step(h, 0, 0) == ct.FDTD_ERR_ARG
        assert lib.FDTD_slab_set(h, 4, 12, 1, 1) == ct.FDTD_OK
        # a slab handle is not solved by FDTD_solve_cw
        import ctypes
        opt, res = ct.SolveOptions(), ct.SolveResult()
        opt.Tn = 10
        opt.fixed_steps = 5
        assert lib.FDTD_solve_cw(h, ctypes.byref(opt), ctypes.byref(res)) == ct.FDTD_ERR_ARG
    finally:
        lib.FDTD_delete(h)


def test_distributed_gradient_equals_single_gpu():
    """Forward and adjoint solves in 3 z slabs, the overlap summed over the
    slabs (zslab.grad_eps_planar), against AdjointSolver.grad_eps on one GPU
    for the same design, adjoint currents and step count (fp64)."""
    import copy

    import torch

    from emopt_b200 import adjoint as A
    p = P.mmi_gradient(d=0.05, w_pml=10, nd=(30, 20), fixed_steps=1200)
    obj, params = A.mmi_objective(p, "fp64")
    x = params.clone().requires_grad_(True)
    obj(x).backward()
    s = obj.solver
    g1 = s.grad_eps()
    mats = tuple(t.cpu().numpy() for t in s.mats)
    ranges = zslab.ownership(p.shape[0], 3)
    pf = copy.copy(p)
    pf.mats = mats
    pa = copy.copy(pf)
    pa.sources = s.last_adjoint_currents
    parts = {}
    for name, prob in (("fwd", pf), ("adj", pa)):
        ss = zslab.SlabSet(prob, ranges, precision="fp64", t0_device=True)
        try:
            ss.begin()
            ss.run()
            parts[name] = ss.finish()
        finally:
            ss.close()
    g = zslab.grad_eps_planar(parts["fwd"], parts["adj"], s.design.box, ranges, None)
    torch.cuda.synchronize()
    err = (torch.linalg.norm(g - g1) / torch.linalg.norm(g1)).item()
    print("z-slab gradient vs one GPU: %.3e" % err)
    assert err < 1e-12
