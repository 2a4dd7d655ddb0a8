"""CPU tests of the oracle: the C restatement against the reference build and
against the committed golden fixtures, and the driver's z-slab decomposition."""
import numpy as np
import pytest

from emopt_b200 import problems as P
from helpers import golden, input_digest, oracle_for, rel_l2
from oracle import driver

GOLDEN_BOXES = ["pec", "sym_EH0", "sym_HEH", "sym_0EE", "lossy", "mu_two_src", "wide_pml",
                "no_pml", "tail1", "tail8_sym", "tail16_lossy", "tail1_mu", "tail17"]
BOX_KW = {
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

needs_ref = pytest.mark.skipif(not driver.available("ref"),
                               reason="reference core not compiled (sources absent)")


def test_fit_kat_restatement():
    """Scalar fit functions of the restatement equal the reference's known answers."""
    g = golden("kat_fit.npz")
    lib = driver.load("oracle")
    t, f = g["t"], g["f"]
    for q in range(len(t)):
        ph3 = lib.FDTD_calc_phase_3T(*t[q], *f[q])
        assert ph3 == g["phase3"][q]
        assert lib.FDTD_calc_amplitude_3T(*t[q], *f[q], ph3) == g["amp3"][q] or \
            (np.isnan(g["amp3"][q]) and np.isnan(lib.FDTD_calc_amplitude_3T(*t[q], *f[q], ph3)))
        ph2 = lib.FDTD_calc_phase_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1])
        assert ph2 == g["phase2"][q] or (np.isnan(ph2) and np.isnan(g["phase2"][q]))
    h = lib.FDTD_new()
    lib.FDTD_set_source_properties(h, float(g["src_T"]), float(g["src_min"]))
    vals = [lib.FDTD_src_func_t(h, q, g["src_t"][q], g["src_phase"][q]) for q in range(len(g["src_t"]))]
    assert np.array_equal(vals, g["src_value"])


@pytest.mark.parametrize("name", GOLDEN_BOXES)
def test_restatement_matches_golden(name):
    """The C restatement reproduces the reference's fields bit-for-bit."""
    g = golden(f"box_{name}.npz")
    p = P.random_box(**BOX_KW[name])
    assert input_digest(p) == str(g["digest"]), "problem generator drifted"
    r = oracle_for(p, lib="oracle").solve(fixed_steps=p.fixed_steps)
    assert r["steps"] == int(g["steps"])
    assert np.array_equal(np.stack(r["fields"]), g["fields"])


def test_restatement_converging_run_matches_golden():
    g = golden("box_converge.npz")
    p = P.random_box(seed=11, shape=(10, 12, 15), fixed_steps=None, rtol=1e-6)
    p.Nmax = 40000
    assert input_digest(p) == str(g["digest"])
    r = oracle_for(p, lib="oracle").solve(record=True)
    assert r["steps"] == int(g["steps"]) and r["n_main"] == int(g["n_main"])
    assert np.array_equal(np.array(r["history"]), g["history"])
    assert np.array_equal(np.stack(r["fields"]), g["fields"])


@needs_ref
@pytest.mark.parametrize("seed,bc,cplx,mu", [(21, "000", False, False), (22, "HHE", True, False),
                                              (23, "E0H", False, True), (24, "EEE", True, True)])
def test_restatement_bitexact_vs_reference(seed, bc, cplx, mu):
    p = P.random_box(seed, shape=(7, 9, 12), bc=bc, complex_eps=cplx, mu_random=mu,
                     n_sources=2, fixed_steps=90)
    a = oracle_for(p, "ref").solve(fixed_steps=p.fixed_steps)
    b = oracle_for(p, "oracle").solve(fixed_steps=p.fixed_steps)
    for x, y in zip(a["fields"], b["fields"]):
        assert np.array_equal(x, y)
    for x, y in zip(a["E"] + a["H"], b["E"] + b["H"]):
        assert np.array_equal(x, y)


BC_ALL = [a + b + c for a in "0EH" for b in "0EH" for c in "0EH"]


@needs_ref
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("bc", BC_ALL)
def test_restatement_bitexact_vs_reference_every_bc(bc, cplx):
    """Every boundary combination {0, E, H}^3, lossless and lossy, on a tiny
    block with a current box over the x-max face: the restatement equals the
    reference core bit for bit (fields after the fixed steps and phasors)."""
    k = BC_ALL.index(bc)
    p = P.random_box(100 + 2 * k + cplx, shape=(5, 6, 7), w_pml=(2, 1, 1, 2, 2, 1), bc=bc,
                     complex_eps=cplx, mu_random=bool(k % 2), edge_source=True, fixed_steps=50)
    a = oracle_for(p, "ref").solve(fixed_steps=p.fixed_steps)
    b = oracle_for(p, "oracle").solve(fixed_steps=p.fixed_steps)
    assert max(np.abs(f).max() for f in a["fields"]) > 0
    for x, y in zip(a["fields"] + a["E"] + a["H"], b["fields"] + b["E"] + b["H"]):
        assert np.array_equal(x, y)


def test_slab_decomposition_equals_one_rank():
    """z-slab instances with ghost exchange reproduce the one-rank result exactly
    (the CPU baseline runs this way)."""
    p = P.random_box(31, shape=(13, 8, 9), bc="E00", fixed_steps=80)
    a = oracle_for(p, "oracle").solve(fixed_steps=p.fixed_steps)
    for nt in (2, 4):
        b = oracle_for(p, "oracle").run_fixed_slabs(p.fixed_steps, nt)
        assert b["steps"] == a["steps"]
        for x, y in zip(a["fields"], b["fields"]):
            assert np.array_equal(x, y)


def test_waveguide_fingerprint_restatement():
    """Full-size 101x76x65 waveguide, 4000 + 2 Tn steps: the restatement matches
    the reference's fingerprint (sampled values and norms) exactly."""
    g = golden("waveguide.npz")
    p = P.waveguide()
    assert input_digest(p) == str(g["digest"])
    r = oracle_for(p, "oracle").run_fixed_slabs(p.fixed_steps, 8)
    F = np.stack(r["fields"])
    idx = g["idx"]
    assert r["steps"] == int(g["steps"])
    assert np.array_equal(F[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]], g["samples"])
    norms = np.sqrt(np.sum(np.abs(F) ** 2, axis=(1, 2, 3)))
    assert rel_l2(norms, g["norms"]) < 1e-14


@pytest.mark.parametrize("seed,shape,nconv,nthreads", [(11, (10, 12, 15), 10, 3), (5, (7, 6, 9), 40, 4)])
def test_threaded_converging_solve_equals_one_rank(seed, shape, nconv, nthreads):
    """solve_threads (z slabs on threads, the one-rank probe rule) reproduces
    the one-rank converging solve bit for bit: step count, probe history,
    fields.  nconv = 40 on 7 x 6 x 9 cells puts probe points on face ghosts."""
    p = P.random_box(seed=seed, shape=shape, fixed_steps=None, rtol=1e-6)
    p.nconv = nconv
    p.Nmax = 40000
    o = oracle_for(p, "oracle")
    ref = o.solve(record=True)
    thr = oracle_for(p, "oracle").solve_threads(nthreads, record=True)
    assert thr["n_main"] == ref["n_main"] and thr["steps"] == ref["steps"]
    assert thr["history"] == ref["history"]
    for a, b in zip(thr["fields"], ref["fields"]):
        np.testing.assert_array_equal(a, b)
