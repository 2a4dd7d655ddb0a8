"""The reference's own ctypes binding, byte for byte, drives this library.

emopt/fdtd_ctypes.py loads ``FDTD.so`` from its own directory and declares the
argtypes of all 32 reference symbols (emopt/fdtd_ctypes.py:14-149).  Copied
unchanged into a scratch directory beside a link ``FDTD.so`` -> this
library, it must import (every symbol it declares exists) and its calls must
give the reference's answers: the scalar fit and ramp functions against the
known answers produced by the reference core, and the ghost pack/unpack
against the reference core itself.  Needs the reference sources (present where
the oracle is built); the CUDA kernels behind the other symbols are exercised
through the same signatures by the GPU parity tests."""
import ctypes
import importlib.util
import os
import shutil

import numpy as np
import pytest

from helpers import ROOT, golden
from oracle import driver

REF_BINDING = os.path.join(os.path.dirname(driver.REF_SRC), "emopt", "fdtd_ctypes.py")


@pytest.fixture(scope="module")
def refmod(tmp_path_factory):
    if not os.path.exists(REF_BINDING):
        pytest.skip("the reference sources are not present")
    from emopt_b200 import fdtd_ctypes as ct
    d = tmp_path_factory.mktemp("refbinding")
    dst = d / "fdtd_ctypes.py"
    shutil.copyfile(REF_BINDING, dst)
    assert dst.read_bytes() == open(REF_BINDING, "rb").read()
    os.symlink(os.path.realpath(ct.so_path), d / "FDTD.so")
    spec = importlib.util.spec_from_file_location("reference_fdtd_ctypes", str(dst))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_binding_loads_this_library(refmod):
    from emopt_b200 import fdtd_ctypes as ct
    assert os.path.realpath(refmod.so_path) == os.path.realpath(ct.so_path)
    names = [n for n in ct.REFERENCE_SYMBOLS]
    assert len(names) == 32
    for n in names:
        assert getattr(refmod.libFDTD, n).argtypes is not None, n


def test_scalar_functions_through_reference_binding(refmod):
    lib = refmod.libFDTD
    g = golden("kat_fit.npz")
    t, f = g["t"], g["f"]
    ph3 = [lib.FDTD_calc_phase_3T(*t[q], *f[q]) for q in range(len(t))]
    am3 = [lib.FDTD_calc_amplitude_3T(*t[q], *f[q], g["phase3"][q]) for q in range(len(t))]
    ph2 = [lib.FDTD_calc_phase_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1]) for q in range(len(t))]
    am2 = [lib.FDTD_calc_amplitude_2T(t[q, 0], t[q, 1], f[q, 0], f[q, 1], g["phase2"][q])
           for q in range(len(t))]
    np.testing.assert_array_equal(ph3, g["phase3"])
    np.testing.assert_array_equal(am3, g["amp3"])
    np.testing.assert_array_equal(ph2, g["phase2"])
    np.testing.assert_array_equal(am2, g["amp2"])
    h = lib.FDTD_new()
    lib.FDTD_set_source_properties(h, float(g["src_T"]), float(g["src_min"]))
    vals = [lib.FDTD_src_func_t(h, int(q), float(g["src_t"][q]), float(g["src_phase"][q]))
            for q in range(len(g["src_t"]))]
    np.testing.assert_array_equal(vals, g["src_value"])


def test_ghost_helpers_through_reference_binding(refmod):
    """numpy arrays through the binding's ndpointer argtypes, against the
    reference core compiled from its sources."""
    if not driver.available("ref"):
        pytest.skip("the reference core is not built")
    ref = ctypes.CDLL(driver.REF_SO)
    for name in ("FDTD_copy_to_ghost_comm", "FDTD_copy_from_ghost_comm"):
        getattr(ref, name).argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 3
    I, J, K = 4, 6, 5
    rng = np.random.default_rng(3)
    n = 2 * (I * J + I * K + J * K)
    src = rng.standard_normal((I + 2) * (J + 2) * (K + 2))
    g1 = np.zeros(2 * n, dtype=np.complex128)
    g2 = g1.copy()
    refmod.libFDTD.FDTD_copy_to_ghost_comm(src, g1, I, J, K)
    ref.FDTD_copy_to_ghost_comm(src.ctypes.data, g2.ctypes.data, I, J, K)
    np.testing.assert_array_equal(g1, g2)
    g = rng.standard_normal(2 * n) + 1j * rng.standard_normal(2 * n)
    d1, d2 = src.copy(), src.copy()
    refmod.libFDTD.FDTD_copy_from_ghost_comm(d1, g, I, J, K)
    ref.FDTD_copy_from_ghost_comm(d2.ctypes.data, g.ctypes.data, I, J, K)
    np.testing.assert_array_equal(d1, d2)
