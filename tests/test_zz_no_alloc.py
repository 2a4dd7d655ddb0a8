"""FDTD_amp_phase_noalloc, the allocation-free amplitude/phase conversion.

Its output must match what the existing entry point FDTD_add_source(...,
calc_phase=True) writes into the same source arrays, on two calls in a row
(the second one smaller, so the fixed staging array still holds the first
call's values past its end).  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

FDTD_OK, FDTD_ERR_ARG = 0, 2


def _values(rng, n):
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a[:: 97] = 0.0                      # zero: amplitude 0, phase 0
    a[1:: 89] = -rng.random(len(a[1:: 89]))   # negative real axis: phase -pi
    a[2:: 83] = 1j * rng.random(len(a[2:: 83]))
    return np.ascontiguousarray(a, dtype=np.complex128)


def _via_add_source(ct, a):
    """The six components converted in place by FDTD_add_source(calc_phase=True)."""
    comps = [np.ascontiguousarray(a * (c + 1)) for c in range(6)]
    h = ct.libFDTD.FDTD_new()
    try:
        ct.libFDTD.FDTD_set_device(h, 0)
        ct.libFDTD.FDTD_add_source(h, *comps, 0, 0, 0, 1, 1, len(a), True)
        ct.check(h, "FDTD_add_source")
    finally:
        ct.libFDTD.FDTD_delete(h)
    return comps


def _via_noalloc(ct, a):
    comps = [np.ascontiguousarray(a * (c + 1)) for c in range(6)]
    msg = ctypes.create_string_buffer(256)
    for x in comps:
        st = ct.libFDTD.FDTD_amp_phase_noalloc(0, None, x, x.size, msg, len(msg))
        assert st == FDTD_OK, msg.value.decode()
        assert msg.value == b""
    return comps


@pytest.mark.gpu
def test_noalloc_matches_add_source_two_calls():
    from emopt_b200 import fdtd_ctypes as ct
    rng = np.random.default_rng(20261203)
    for n in (200_000, 3_001):
        a = _values(rng, n)
        ref = _via_add_source(ct, a)
        out = _via_noalloc(ct, a)
        for c in range(6):
            # Same kernel on the same device: agreement is expected to the bit;
            # the tolerance below is the test's bound.
            np.testing.assert_allclose(out[c].real, ref[c].real, rtol=1e-15, atol=0)
            np.testing.assert_allclose(out[c].imag, ref[c].imag, rtol=1e-15, atol=1e-300)
            b = a * (c + 1)
            np.testing.assert_allclose(out[c].real, np.abs(b), rtol=1e-13)
            np.testing.assert_allclose(out[c].imag, -np.angle(b), rtol=1e-13, atol=1e-15)


@pytest.mark.gpu
def test_noalloc_limit_on_gpu():
    _check_limit()


def test_noalloc_rejects_bad_sizes():
    """Size checks come before any device work, so they hold without a GPU."""
    _check_limit()


def _check_limit():
    from emopt_b200 import fdtd_ctypes as ct
    a = np.arange(8, dtype=np.complex128) + 1j
    keep = a.copy()
    msg = ctypes.create_string_buffer(256)
    st = ct.libFDTD.FDTD_amp_phase_noalloc(0, None, a, ct.NOALLOC_MAX_VALUES + 1, msg, len(msg))
    assert st == FDTD_ERR_ARG
    assert b"exceed" in msg.value
    st = ct.libFDTD.FDTD_amp_phase_noalloc(0, None, a, -1, msg, len(msg))
    assert st == FDTD_ERR_ARG
    np.testing.assert_array_equal(a, keep)
