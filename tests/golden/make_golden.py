"""Generate the golden fixtures in tests/golden/ from the reference FDTD library.

The reference has no tests or golden vectors of its own, so the fixtures are
produced by running the reference C++ core, compiled unchanged from its own
sources (``make -C oracle ref`` -> ``oracle/_ref/FDTD.so``), through the
one-rank restatement of its Python driver loop (``oracle/driver.py``).

Fixtures (all inputs are regenerated from seeds by ``emopt_b200.problems``; an
input checksum is stored to detect generator drift):

* ``kat_fit.npz``      scalar known answers of FDTD_calc_phase/amplitude_2T/3T
                       and FDTD_src_func_t, including the branch edges
                       (zero differences, negative amplitude, f21^2 == f10^2).
* ``box_<case>.npz``   complex steady-state fields of small random blocks after
                       a fixed number of steps (boundary-condition, lossy,
                       varying-mu and multi-source cases).
* ``box_converge.npz`` a run to rtol = 1e-6: step count and probe history.
* ``waveguide.npz``    the 101 x 76 x 65 waveguide after 4000 + 2 Tn steps:
                       per-component norms and 512 sampled complex values.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from emopt_b200 import problems as P  # noqa: E402
from helpers import input_digest, oracle_for  # noqa: E402
from oracle import driver  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

BOX_CASES = {
    # name: kwargs of problems.random_box
    "pec": dict(seed=1, bc="000"),
    "sym_EH0": dict(seed=2, bc="EH0"),
    "sym_HEH": dict(seed=3, bc="HEH"),
    "sym_0EE": dict(seed=4, bc="0EE"),
    "lossy": dict(seed=5, complex_eps=True, bc="0H0"),
    "mu_two_src": dict(seed=6, mu_random=True, n_sources=2, bc="E00"),
    "wide_pml": dict(seed=7, shape=(12, 10, 16), w_pml=(5, 5, 4, 4, 5, 5), bc="000"),
    "no_pml": dict(seed=8, shape=(8, 9, 10), w_pml=(0, 0, 0, 0, 0, 0), bc="H0E"),
    # rows that end 1-17 cells past a whole number of 64-cell vector blocks,
    # with a current box over the last x cells
    "tail1": dict(seed=21, shape=(6, 7, 65), bc="000", edge_source=True),
    "tail8_sym": dict(seed=22, shape=(5, 6, 72), bc="EH0", edge_source=True),
    "tail16_lossy": dict(seed=23, shape=(5, 6, 80), complex_eps=True, bc="0H0", edge_source=True),
    "tail1_mu": dict(seed=24, shape=(4, 5, 129), mu_random=True, bc="HEH", edge_source=True),
    "tail17": dict(seed=25, shape=(5, 6, 81), bc="000", edge_source=True),
}


def kat_fit(lib):
    rng = np.random.default_rng(123)
    n = 400
    t = np.sort(rng.uniform(0, 60, (n, 3)), axis=1)
    f = rng.standard_normal((n, 3))
    # branch edges: both differences zero, one zero, |f21| == |f10|, negative A
    f[0] = [0.3, 0.3, 0.3]
    f[1] = [0.0, 0.0, 0.0]
    f[2] = [0.1, 0.1, 0.5]
    f[3] = [0.1, 0.5, 0.5]
    f[4] = [0.2, 0.5, 0.2]
    f[5] = [-0.7, 0.1, 0.9]
    ph3 = np.array([lib.FDTD_calc_phase_3T(*t[q], *f[q]) for q in range(n)])
    am3 = np.array([lib.FDTD_calc_amplitude_3T(*t[q], *f[q], ph3[q]) for q in range(n)])
    ph2 = np.array([lib.FDTD_calc_phase_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1]) for q in range(n)])
    am2 = np.array([lib.FDTD_calc_amplitude_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1], ph2[q])
                    for q in range(n)])
    h = lib.FDTD_new()
    lib.FDTD_set_source_properties(h, 37.5, 1e-4)
    ts = np.linspace(0, 80, 257)
    phs = rng.uniform(-np.pi, np.pi, ts.size)
    src = np.array([lib.FDTD_src_func_t(h, q, ts[q], phs[q]) for q in range(ts.size)])
    np.savez_compressed(os.path.join(OUT, "kat_fit.npz"), t=t, f=f, phase3=ph3, amp3=am3,
                        phase2=ph2, amp2=am2, src_T=37.5, src_min=1e-4, src_t=ts,
                        src_phase=phs, src_value=src)


def main():
    driver.build(ref=True)
    lib = driver.load("ref")
    kat_fit(lib)
    for name, kw in BOX_CASES.items():
        p = P.random_box(**kw)
        r = oracle_for(p).solve(fixed_steps=p.fixed_steps)
        np.savez_compressed(os.path.join(OUT, f"box_{name}.npz"), digest=input_digest(p),
                            steps=r["steps"], fields=np.stack(r["fields"]))
        print(name, p.shape, r["steps"])
    p = P.random_box(seed=11, shape=(10, 12, 15), fixed_steps=None, rtol=1e-6)
    p.Nmax = 40000
    r = oracle_for(p).solve(record=True)
    np.savez_compressed(os.path.join(OUT, "box_converge.npz"), digest=input_digest(p),
                        steps=r["steps"], n_main=r["n_main"], history=np.array(r["history"]),
                        fields=np.stack(r["fields"]))
    print("converge", r["steps"])
    t0 = time.time()
    p = P.waveguide()
    r = oracle_for(p).run_fixed_slabs(p.fixed_steps, os.cpu_count() or 1)
    F = np.stack(r["fields"])
    rng = np.random.default_rng(5)
    idx = np.stack([rng.integers(0, n, 512) for n in (6,) + p.shape], axis=1)
    samples = F[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]
    norms = np.sqrt(np.sum(np.abs(F) ** 2, axis=(1, 2, 3)))
    np.savez_compressed(os.path.join(OUT, "waveguide.npz"), digest=input_digest(p),
                        steps=r["steps"], idx=idx, samples=samples, norms=norms)
    print("waveguide", r["steps"], "%.1fs" % (time.time() - t0))


if __name__ == "__main__":
    main()
