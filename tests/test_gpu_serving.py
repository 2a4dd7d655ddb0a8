"""GPU tests of the serving form (continuous batching, FDTD_serve_*).

Each request's result must be the same alone and in a mix: the same step
count and the same fields, bit for bit, as FDTD_solve_cw on the same request
(float32 storage; the served half steps are the single-solve kernels), whether
it is served alone or admitted while other requests of different grids and
wavelengths are running.
"""
import ctypes

import numpy as np
import pytest
import torch

from emopt_b200 import fdtd_ctypes as ct
from emopt_b200 import serving as S

pytestmark = pytest.mark.gpu


def _specs(n=6, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        shape = (int(rng.integers(26, 40)), int(rng.integers(26, 44)), int(rng.integers(28, 56)))
        out.append(S.random_request(rng, q, shape=shape, w_pml=8))
    return out


def _rel(a, b):
    a = np.stack(a)
    b = np.stack(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def mu_ones():
    return torch.ones(64 * 64 * 64, dtype=torch.complex128, device="cuda:0")


@pytest.fixture(scope="module")
def alone_solve_cw(mu_ones):
    """Every request through FDTD_solve_cw (vector kernel, float32)."""
    out = {}
    for spec in _specs():
        req = S.Request(spec, 0, mu_ones)
        ct.libFDTD.FDTD_set_kernel(req.h, 5)
        req.set_outputs()
        res = ct.SolveResult()
        st = ct.libFDTD.FDTD_solve_cw(req.h, ctypes.byref(req.opt), ctypes.byref(res))
        assert st in (ct.FDTD_OK, ct.FDTD_NMAX), ct.last_error(req.h)
        out[spec.rid] = (res.steps, res.n_main, [a.cpu().numpy() for a in req.out])
        req.close()
    return out


def _serve(specs, mu_ones, stagger, budget=8e9, steps_per_replay=16):
    """Admit specs[:stagger] first, the rest two replays later; run to the end."""
    eng = S.ServeEngine(0, budget, 16, steps_per_replay)
    reqs = {s.rid: S.Request(s, 0, mu_ones) for s in specs}
    order = [s.rid for s in specs]
    results = {}
    replay = 0
    try:
        while order or eng.active:
            if order and (replay >= 2 or len(eng.active) < stagger):
                while order and eng.admit(reqs[order[0]]):
                    order.pop(0)
                    if replay < 2 and len(eng.active) >= stagger:
                        break
            ready = eng.advance()
            replay += 1
            for req, r in eng.collect(ready):
                results[req.spec.rid] = (r["steps"], r["n_main"], [a.cpu().numpy() for a in req.out])
                req.close()
    finally:
        eng.close()
    return results


def test_each_request_same_alone_and_in_mix(alone_solve_cw, mu_ones):
    specs = _specs()
    mix = _serve(specs, mu_ones, stagger=3)
    assert set(mix) == set(alone_solve_cw)
    for rid, (steps, n_main, F) in alone_solve_cw.items():
        alone = _serve([s for s in specs if s.rid == rid], mu_ones, stagger=1)[rid]
        assert alone[0] == steps and mix[rid][0] == steps, (rid, steps, alone[0], mix[rid][0])
        assert alone[1] == n_main and mix[rid][1] == n_main
        e_alone = _rel(alone[2], F)
        e_mix = _rel(mix[rid][2], F)
        print("request %d: %d steps, served alone %.2e, in the mix %.2e vs FDTD_solve_cw"
              % (rid, steps, e_alone, e_mix))
        assert all(np.array_equal(a, b) for a, b in zip(alone[2], F))
        assert all(np.array_equal(a, b) for a, b in zip(mix[rid][2], F))


def test_budget_admission_waits_for_memory(mu_ones):
    """With room for one request, a second identical one waits until the
    first is collected, then runs to the same result."""
    spec = _specs(1, seed=11)[0]
    probe = S.ServeEngine(0, 1e12, 4, 16)
    r0 = S.Request(spec, 0, mu_ones)
    assert probe.admit(r0)
    used, active = probe.info()
    assert active == 1 and used > 0
    probe.close()
    r0.close()
    eng = S.ServeEngine(0, 1.5 * used, 4, 16)
    a, b = S.Request(spec, 0, mu_ones), S.Request(spec, 0, mu_ones)
    done = []
    try:
        assert eng.admit(a)
        assert not eng.admit(b)
        while eng.active:
            done += [(r, [x.cpu().numpy() for x in q.out]) for q, r in eng.collect(eng.advance())]
        assert eng.info() == (0.0, 0)
        assert eng.admit(b)
        while eng.active:
            done += [(r, [x.cpu().numpy() for x in q.out]) for q, r in eng.collect(eng.advance())]
    finally:
        eng.close()
        a.close()
        b.close()
    assert len(done) == 2
    assert done[0][0]["steps"] == done[1][0]["steps"]
    assert _rel(done[1][1], done[0][1]) < 1e-6


def test_nonfinite_request_retires_early(alone_solve_cw, mu_ones):
    """A request whose permittivity holds NaN and that asks to stop on a
    non-finite probe retires at its first probe with status NONFINITE; a
    request served beside it gives its solo result."""
    specs = _specs()
    bad = S.Request(specs[0], 0, mu_ones)
    for e in bad.eps:
        e.view(-1)[: e.numel() // 2] = float("nan")
    bad.opt.stop_nonfinite = 1
    good = S.Request(specs[1], 0, mu_ones)
    torch.cuda.synchronize()
    eng = S.ServeEngine(0, 8e9, 4, 16)
    res = {}
    try:
        assert eng.admit(bad) and eng.admit(good)
        while eng.active:
            for req, r in eng.collect(eng.advance()):
                res[req.spec.rid] = (r, [a.cpu().numpy() for a in req.out])
                req.close()
    finally:
        eng.close()
    r_bad, _ = res[specs[0].rid]
    Tn = bad.opt.Tn
    assert r_bad["status"] == ct.FDTD_NONFINITE
    assert r_bad["nprobes"] == 1 and r_bad["steps"] == 3 * Tn
    r_good, F = res[specs[1].rid]
    steps, n_main, F1 = alone_solve_cw[specs[1].rid]
    assert r_good["status"] == ct.FDTD_OK and r_good["steps"] == steps
    assert all(np.array_equal(a, b) for a, b in zip(F, F1))
