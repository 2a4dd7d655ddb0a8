"""Shared helpers for the test suite: build the CPU oracle for a problem and
compare complex field sets."""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import driver  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def input_digest(p) -> str:
    h = hashlib.sha256()
    for a in p.mats:
        h.update(np.ascontiguousarray(a).tobytes())
    for arrays, i0, j0, k0 in p.sources:
        for a in arrays:
            h.update(np.ascontiguousarray(a).tobytes())
        h.update(np.array([i0, j0, k0]).tobytes())
    return h.hexdigest()


def oracle_for(p, lib="ref"):
    """Configure the one-rank oracle driver exactly like ``problems.make_solver``."""
    s = driver.OracleFDTD(p.X, p.Y, p.Z, p.dx, p.dy, p.dz, p.wavelength, rtol=p.rtol,
                          nconv=p.nconv, complex_eps=p.complex_eps, lib=lib)
    assert (s.Nz, s.Ny, s.Nx) == p.shape
    s.bc = p.bc
    s.set_w_pml_cells(p.w_pml)
    if p.src_ramp_time is not None:
        s.src_T = p.src_ramp_time
    if p.Nmax is not None:
        s.Nmax = p.Nmax
    s.set_materials(p.mats[:3], p.mats[3:])
    for arrays, i0, j0, k0 in p.sources:
        s.add_source([a.copy() for a in arrays], i0, j0, k0)
    return s


def oracle_lib() -> str:
    """The reference build when present, else the C restatement."""
    return "ref" if driver.available("ref") else "oracle"


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.sqrt(np.sum(np.abs(b) ** 2))
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2)) / (den if den > 0 else 1.0))


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)
