"""Full-size parity: the fp64 solve and the gradient on the workloads
themselves, not scaled-down versions.

* Waveguide (101 x 76 x 65 cells) and MMI block (321 x 161 x 101 cells, 20-cell
  CPML), both run to rtol = 1e-6 in fp64 through FDTD_solve_cw, against the
  reference core compiled from its sources (oracle/_ref/FDTD.so; the oracle's
  C restatement where it is absent) running the one-rank __solve
  (emopt/fdtd.py:994-1194) on z-slab threads of the host: identical number of
  main steps, time steps and probes, the last amplitude and phase change norms
  within 1e-9, the complex steady-state fields within 1e-9 (relative L2).
  The device reduces the probe norms in its own order, so a step count that
  stayed equal here is evidence that no probe sits on the tolerance edge.
* Gradient of the MMI mode-match objective (321 x 161 x 101 cells, 80 x 80
  design density): against the reference's calc_gradient restated on the
  oracle's forward and adjoint fields (emopt/adjoint_method.py:448-547),
  against central finite differences of this solver's objective (h = 1e-4,
  32 seeded parameters, fp64) for the fp64 and the fp32 gradient, and fp32
  against fp64 (<= 1e-3).

The CPU runs of the oracle go to a worker thread as soon as a test asks for
them and overlap the GPU solves (ctypes releases the GIL in every call).
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
import torch

from emopt_b200 import adjoint as A
from emopt_b200 import problems as P
from helpers import oracle_for, oracle_lib, rel_l2
from oracle import adjoint as R

pytestmark = pytest.mark.gpu

NTHREADS = max(1, min(64, os.cpu_count() or 1))
_pool = ThreadPoolExecutor(max_workers=1)
_jobs = {}


def _oracle_job(name, fn):
    if name not in _jobs:
        _jobs[name] = _pool.submit(fn)
    return _jobs[name]


def _gpu_solve(p, precision):
    sim = P.make_solver(p, precision=precision, kernel="auto")
    sim.solve_forward()
    F = np.stack([sim.get_field(c) for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")])
    return F, dict(sim.last_solve)


def _check_converging(p, job):
    F, info = _gpu_solve(p, "fp64")
    ref = job.result()
    print("%s: GPU n_main %d steps %d probes %d | reference n_main %d steps %d probes %d"
          % (p.name, info["n_main"], info["steps"], info["nprobes"], ref["n_main"], ref["steps"],
             len(ref["history"])))
    assert info["n_main"] == ref["n_main"]
    assert info["steps"] == ref["steps"]
    assert info["nprobes"] == len(ref["history"])
    assert info["A_change"] == pytest.approx(ref["A_change"], rel=1e-9)
    assert info["phi_change"] == pytest.approx(ref["phi_change"], rel=1e-9)
    err = rel_l2(F, np.stack(ref["fields"]))
    print("%s: fp64 field relative L2 vs reference core %.3e" % (p.name, err))
    assert err < 1e-9


def _waveguide():
    return P.waveguide(fixed_steps=None)


def _mmi():
    return P.mmi_block(seed=0)


def test_waveguide_converging_fp64_matches_reference_core():
    p = _waveguide()
    # queue both oracle runs now: the MMI run overlaps this test's GPU solve
    job = _oracle_job("waveguide", lambda: oracle_for(_waveguide(), oracle_lib()).solve_threads(NTHREADS, record=True))
    _oracle_job("mmi", lambda: oracle_for(_mmi(), oracle_lib()).solve_threads(NTHREADS, record=True))
    _check_converging(p, job)


def test_mmi_converging_fp64_matches_reference_core():
    p = _mmi()
    job = _oracle_job("mmi", lambda: oracle_for(_mmi(), oracle_lib()).solve_threads(NTHREADS, record=True))
    _check_converging(p, job)


# ------------------------------------------------------------------ gradient
N_REF = 1500       # main steps of the reference-calc_gradient comparison (same on both sides)


def _value_and_grad(obj, params):
    x = params.clone().requires_grad_(True)
    F = obj(x)
    F.backward()
    return F.item(), x.grad.detach().cpu().numpy().ravel()


def _indices(n):
    return np.random.default_rng(2).choice(n, 32, replace=False)


def _reference_gradient_job():
    p = P.mmi_gradient(fixed_steps=N_REF)
    idx = _indices(p.design_params.size)

    def make_oracle(eps3):
        q = P.mmi_gradient()
        q.mats = tuple(list(eps3) + list(p.mats[3:]))
        return oracle_for(q, oracle_lib())

    k, j1, j2, i1, i2 = p.fom_plane
    return R.reference_gradient(make_oracle, p, p.design_params, idx, 1e-8, N_REF, NTHREADS,
                                lambda q: P.design_eps(p, q), p.fom_mode,
                                R.Box(k, k + 1, j1, j2, i1, i2))[:2]


def test_full_gradient_matches_reference_calc_gradient():
    job = _oracle_job("grad", _reference_gradient_job)
    p = P.mmi_gradient(fixed_steps=N_REF)
    obj, params = A.mmi_objective(p, "fp64")
    F, g = _value_and_grad(obj, params)
    idx = _indices(params.numel())
    Fr, gr = job.result()
    err = np.linalg.norm(g[idx] - gr) / np.linalg.norm(gr)
    print("full-size adjoint vs reference calc_gradient: F %.6e / %.6e, gradient relative L2 %.3e"
          % (F, Fr, err))
    assert F == pytest.approx(Fr, rel=1e-10)
    assert err < 1e-5


def test_full_gradient_central_differences_fp64_and_fp32():
    # fixed step count: twice what rtol = 1e-6 takes, so that every
    # perturbed solve runs the same steps and the difference quotient is not
    # disturbed by a change of the stopping step
    conv = P.mmi_gradient()
    o_conv, params = A.mmi_objective(conv, "fp64")
    with torch.no_grad():
        o_conv(params)
    n_fixed = 2 * int(o_conv.solver.last["forward"]["n_main"])
    p = P.mmi_gradient(fixed_steps=n_fixed)
    obj, params = A.mmi_objective(p, "fp64", discrete_time=True)
    o32, _ = A.mmi_objective(p, "fp32", discrete_time=True)
    F0, g = _value_and_grad(obj, params)
    F32, g32 = _value_and_grad(o32, params)
    idx = _indices(params.numel())
    h = 1e-4
    fd = np.empty(len(idx))
    for n, q in enumerate(idx):
        pp = params.clone()
        pp.view(-1)[q] += h
        pm = params.clone()
        pm.view(-1)[q] -= h
        with torch.no_grad():
            fd[n] = (obj(pp).item() - obj(pm).item()) / (2 * h)
    err64 = np.linalg.norm(fd - g[idx]) / np.linalg.norm(fd)
    err32 = np.linalg.norm(fd - g32[idx]) / np.linalg.norm(fd)
    e3264 = np.linalg.norm(g32 - g) / np.linalg.norm(g)
    print("full size, %d main steps: central FD vs adjoint fp64 %.3e, fp32 %.3e; "
          "fp32 vs fp64 gradient %.3e, objective %.3e"
          % (n_fixed, err64, err32, e3264, abs(F32 - F0) / abs(F0)))
    assert err64 < 2e-5
    assert err32 < 1e-3
    assert e3264 < 1e-3
    assert abs(F32 - F0) / abs(F0) < 1e-4
