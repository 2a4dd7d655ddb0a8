"""The ghost pack/unpack helpers of the C ABI (FDTD_copy_to_ghost_comm /
FDTD_copy_from_ghost_comm, src/fdtd.cpp:1789-1929) against the reference core
compiled from its own sources (oracle/_ref/FDTD.so) and against the oracle's C
restatement: the same face order and index arithmetic, so the packed ghost
vectors and the unpacked ghost layers must be identical, bit for bit.

Both helpers are pure host functions (no handle, no device): the pack copies
the six boundary faces of a padded (I+2)(J+2)(K+2) real array into the first
2(IJ + IK + JK) entries of a complex128 vector (real parts); the unpack reads
the received faces from the entries after those -- the ghost region that
PETSc appends to the owned part of a ghosted vector (emopt/fdtd.py:1860-1873)
-- and writes them into the ghost layer."""
import ctypes

import numpy as np
import pytest

from oracle import driver

SHAPES = [(1, 1, 1), (2, 3, 4), (5, 1, 7), (6, 5, 3), (9, 8, 11)]


def _bind(path):
    lib = ctypes.CDLL(path)
    for name in ("FDTD_copy_to_ghost_comm", "FDTD_copy_from_ghost_comm"):
        fn = getattr(lib, name)
        fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        fn.restype = None
    return lib


def _libs():
    from emopt_b200 import fdtd_ctypes as ct
    ours = _bind(ct.so_path)
    refs = []
    if driver.available("ref"):
        refs.append(("reference", _bind(driver.REF_SO)))
    if driver.available("oracle"):
        refs.append(("oracle", _bind(driver.ORACLE_SO)))
    if not refs:
        pytest.skip("neither the reference core nor the oracle is built")
    return ours, refs


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("shape", SHAPES)
def test_pack_matches_reference(shape):
    I, J, K = shape
    ours, refs = _libs()
    rng = np.random.default_rng(I * 100 + J * 10 + K)
    src = rng.standard_normal((I + 2) * (J + 2) * (K + 2))
    n = 2 * (I * J + I * K + J * K)
    # the vector carries received ghosts after the owned part; the pack writes
    # only the owned part, so the tail (and every imaginary part) keeps its
    # previous contents
    init = rng.standard_normal((2 * n, 2))
    g_ours = init.copy()
    ours.FDTD_copy_to_ghost_comm(_ptr(src), _ptr(g_ours), I, J, K)
    for name, lib in refs:
        g_ref = init.copy()
        lib.FDTD_copy_to_ghost_comm(_ptr(src), _ptr(g_ref), I, J, K)
        np.testing.assert_array_equal(g_ours, g_ref, err_msg=name)
    # and the content: the faces one layer inside the ghosts, xmin first
    a = src.reshape(I + 2, J + 2, K + 2)
    faces = [a[1:-1, 1:-1, 1], a[1:-1, 1:-1, K], a[1:-1, 1, 1:-1], a[1:-1, J, 1:-1],
             a[1, 1:-1, 1:-1], a[I, 1:-1, 1:-1]]
    np.testing.assert_array_equal(g_ours[:n, 0], np.concatenate([f.ravel() for f in faces]))


@pytest.mark.parametrize("shape", SHAPES)
def test_unpack_matches_reference(shape):
    I, J, K = shape
    ours, refs = _libs()
    rng = np.random.default_rng(1000 + I * 100 + J * 10 + K)
    n = 2 * (I * J + I * K + J * K)
    ghost = rng.standard_normal((2 * n, 2))
    init = rng.standard_normal((I + 2) * (J + 2) * (K + 2))
    d_ours = init.copy()
    ours.FDTD_copy_from_ghost_comm(_ptr(d_ours), _ptr(ghost), I, J, K)
    assert not np.array_equal(d_ours, init)
    for name, lib in refs:
        d_ref = init.copy()
        lib.FDTD_copy_from_ghost_comm(_ptr(d_ref), _ptr(ghost), I, J, K)
        np.testing.assert_array_equal(d_ours, d_ref, err_msg=name)


def test_pack_unpack_round_trip_is_periodic_on_one_rank():
    """One rank exchanging with itself: packing, moving the owned part into
    the ghost region with the neighbour order a periodic 1x1x1 DMDA gives
    (xmin <-> xmax, ymin <-> ymax, zmin <-> zmax) and unpacking writes into
    each ghost face the opposite boundary face -- the periodic wrap that the
    one-rank reference run leaves in its ghosts."""
    I, J, K = 4, 3, 5
    ours, _ = _libs()
    rng = np.random.default_rng(7)
    src = rng.standard_normal((I + 2) * (J + 2) * (K + 2))
    n = 2 * (I * J + I * K + J * K)
    g = np.zeros((2 * n, 2))
    ours.FDTD_copy_to_ghost_comm(_ptr(src), _ptr(g), I, J, K)
    sizes = [I * J, I * J, I * K, I * K, J * K, J * K]
    off = np.concatenate([[0], np.cumsum(sizes)])
    owned = [g[off[q]:off[q + 1]].copy() for q in range(6)]
    recv = [owned[1], owned[0], owned[3], owned[2], owned[5], owned[4]]
    g[n:] = np.concatenate(recv)
    dst = src.copy()
    ours.FDTD_copy_from_ghost_comm(_ptr(dst), _ptr(g), I, J, K)
    a, d = src.reshape(I + 2, J + 2, K + 2), dst.reshape(I + 2, J + 2, K + 2)
    np.testing.assert_array_equal(d[1:-1, 1:-1, 0], a[1:-1, 1:-1, K])
    np.testing.assert_array_equal(d[1:-1, 1:-1, K + 1], a[1:-1, 1:-1, 1])
    np.testing.assert_array_equal(d[1:-1, 0, 1:-1], a[1:-1, J, 1:-1])
    np.testing.assert_array_equal(d[1:-1, J + 1, 1:-1], a[1:-1, 1, 1:-1])
    np.testing.assert_array_equal(d[0, 1:-1, 1:-1], a[I, 1:-1, 1:-1])
    np.testing.assert_array_equal(d[I + 1, 1:-1, 1:-1], a[1, 1:-1, 1:-1])
