"""GPU tests of the differentiation form (MMI design problem at half
resolution, 161 x 81 x 51 cells, 30 x 20 design density).

* against the oracle: the reference's calc_gradient restated in numpy
  (forward difference of eps, -2 Re(y^T dA x) / step) on forward and adjoint
  fields of the CPU oracle, adjoint sources from the reference's own
  ModeMatch derivatives and interpolated_dFdx_3D;
* against central finite differences (h = 1e-4) of the objective computed by
  this solver, on 32 seeded parameters;
* float32 against float64: relative gradient error <= 1e-3.
"""
import os

import numpy as np
import pytest
import torch

from emopt_b200 import adjoint as A
from emopt_b200 import problems as P
from helpers import oracle_for, oracle_lib
from oracle import adjoint as R

pytestmark = pytest.mark.gpu

SMALL = dict(d=0.05, w_pml=10, nd=(30, 20))
N_FIXED = 7000          # main steps: about twice what rtol = 1e-6 needs on this grid


def _problem(**kw):
    return P.mmi_gradient(**SMALL, **kw)


def _value_and_grad(obj, params):
    x = params.clone().requires_grad_(True)
    F = obj(x)
    F.backward()
    return F.item(), x.grad.detach().cpu().numpy().ravel()


def _indices(n):
    return np.random.default_rng(2).choice(n, 32, replace=False)


def test_gradient_matches_reference_calc_gradient():
    n_main = 1500
    p = _problem(fixed_steps=n_main)
    obj, params = A.mmi_objective(p, "fp64")
    F, g = _value_and_grad(obj, params)
    idx = _indices(params.numel())

    def make_oracle(eps3):
        q = _problem()
        q.mats = tuple(list(eps3) + list(p.mats[3:]))
        return oracle_for(q, oracle_lib())

    k, j1, j2, i1, i2 = p.fom_plane
    Fr, gr, _, _ = R.reference_gradient(make_oracle, p, p.design_params, idx, 1e-8, n_main,
                                        min(32, os.cpu_count() or 1),
                                        lambda q: P.design_eps(p, q), p.fom_mode,
                                        R.Box(k, k + 1, j1, j2, i1, i2))
    assert F == pytest.approx(Fr, rel=1e-12)
    err = np.linalg.norm(g[idx] - gr) / np.linalg.norm(gr)
    print("adjoint vs reference calc_gradient: relative L2 %.3e" % err)
    assert err < 1e-5


def test_gradient_central_differences():
    p = _problem(fixed_steps=N_FIXED)
    obj, params = A.mmi_objective(p, "fp64", discrete_time=True)
    F0, g = _value_and_grad(obj, params)
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
    err = np.linalg.norm(fd - g[idx]) / np.linalg.norm(fd)
    ref_conv = np.linalg.norm(fd - g[idx] / obj.solver.dt_factor) / np.linalg.norm(fd)
    print("central FD vs adjoint: %.3e (without the leapfrog frequency factor: %.3e)"
          % (err, ref_conv))
    assert err < 2e-5
    assert ref_conv < 1e-3


def test_gradient_fp32_against_fp64():
    p = _problem(fixed_steps=N_FIXED)
    o64, params = A.mmi_objective(p, "fp64")
    o32, _ = A.mmi_objective(p, "fp32")
    F64, g64 = _value_and_grad(o64, params)
    F32, g32 = _value_and_grad(o32, params)
    ferr = abs(F32 - F64) / abs(F64)
    gerr = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print("fp32 vs fp64: objective %.3e, gradient %.3e" % (ferr, gerr))
    assert ferr < 1e-4
    assert gerr < 1e-3


def test_grad_eps_kernel_against_torch():
    """FDTD_grad_eps (fused, Kahan z-sums) against the same overlap in torch."""
    p = _problem(fixed_steps=300)
    obj, params = A.mmi_objective(p, "fp64")
    F, _ = _value_and_grad(obj, params)
    s = obj.solver
    d = s.design
    got = s.grad_eps()
    for c in range(3):
        i0, i1 = d.iz[c]
        blk = lambda a: a[i0:i1, d.j0:d.j1, d.k0:d.k1]
        ref = (2 * torch.imag(blk(s.adj[c]) * blk(s.fwd[c]))).sum(0)
        torch.testing.assert_close(got[c], ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max()))


@pytest.mark.parametrize("planar", [True, False])
def test_calc_ydAx_topology_matches_reference_formula(planar):
    """FDTD.calc_ydAx_topology (products on the GPU) against the numpy lines of
    emopt/experimental/fdtd.py:121-158 on the same forward/adjoint fields."""
    from emopt_b200 import problems as P
    from emopt_b200.misc import DomainCoordinates
    p = P.random_box(seed=41, shape=(10, 9, 12), fixed_steps=200)
    sim = P.make_solver(p, precision="fp64")
    sim.solve_forward()
    rng = np.random.default_rng(3)
    I, J, K = 2, 3, 4
    src = [rng.standard_normal((I, J, K)) + 1j * rng.standard_normal((I, J, K)) for _ in range(6)]
    dom = DomainCoordinates.from_indices(5, 5 + K, 3, 3 + J, 4, 4 + I, p.dx, p.dy, p.dz)
    sim.add_adjoint_sources(tuple(src), dom)
    sim.solve_adjoint()
    design = DomainCoordinates.from_indices(2, 10, 1, 8, 3, 8, p.dx, p.dy, p.dz)
    E = [sim.get_field(c, design) for c in ("Ex", "Ey", "Ez")]
    Ea = [sim.get_adjoint_field(c, design) for c in ("Ex", "Ey", "Ez")]
    H = [sim.get_field(c, design) for c in ("Hx", "Hy", "Hz")]
    Ha = [sim.get_adjoint_field(c, design) for c in ("Hx", "Hy", "Hz")]
    shape = E[0].shape[1:] if planar else E[0].shape
    sig_e = rng.uniform(0.1, 1.0, shape)
    sig_m = rng.uniform(0.1, 1.0, shape)
    de, dm, lam = 10.165, 0.7, 0.01
    pe = E[0] * Ea[0] + E[1] * Ea[1] + E[2] * Ea[2]
    ph = H[0] * Ha[0] + H[1] * Ha[1] + H[2] * Ha[2]
    if planar:
        pe, ph = np.sum(pe, axis=0), np.sum(ph, axis=0)
    want = np.concatenate([np.ravel(sig_e * (lam / sig_e.size + 2 * de * np.imag(pe))),
                           np.ravel(sig_m * (lam / sig_m.size - 2 * dm * np.imag(ph)))])
    got = sim.calc_ydAx_topology(design, True, sig_e, sig_m, de, dm, planar, lam)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_source_power_matches_host_computation():
    """The torch source power on the device phasors equals FDTD.get_source_power
    (host numpy, emopt/fdtd.py:1555-1667) on the same fields."""
    p = _problem(fixed_steps=600)
    obj, params = A.mmi_objective(p, "fp64", power_norm=True)
    with torch.no_grad():
        obj(params)
    sim = obj.solver.sim
    for a, c in zip(obj.solver.fwd, ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        getattr(sim, "_%s_fwd_t0" % c)[:] = a.cpu().numpy().ravel()
    P_host = sim.get_source_power()
    assert obj.last_power.item() == pytest.approx(P_host, rel=1e-12)
    assert P_host > 0


def test_power_normalized_gradient_central_differences():
    """F = mode match / source power (the reference's PNF3D form): adjoint
    currents on the mode-match box and the six power planes, against central
    differences on 8 seeded parameters."""
    p = _problem(fixed_steps=N_FIXED)
    obj, params = A.mmi_objective(p, "fp64", discrete_time=True, power_norm=True)
    F0, g = _value_and_grad(obj, params)
    idx = _indices(params.numel())[:8]
    h = 1e-4
    fd = np.empty(len(idx))
    for n, q in enumerate(idx):
        pp = params.clone()
        pp.view(-1)[q] += h
        pm = params.clone()
        pm.view(-1)[q] -= h
        with torch.no_grad():
            fd[n] = (obj(pp).item() - obj(pm).item()) / (2 * h)
    err = np.linalg.norm(fd - g[idx]) / np.linalg.norm(fd)
    print("power-normalized: central FD vs adjoint %.3e" % err)
    assert err < 2e-5
