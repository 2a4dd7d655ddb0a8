"""GPU tests of the layered rectangle and polygon materials
(FDTD_structured_values via emopt_b200.grid) against the CPU restatement in
oracle/structured.py.

The GPU code subtracts convex parts from convex pieces of the unclaimed
region; the oracle integrates the same areas exactly over vertical slices:
both in float64, so they agree to rounding (absolute 1e-11 on values of
order 10)."""
import numpy as np
import pytest

from emopt_b200 import grid as G
from test_structured import _oracle_prim, _random_layout

pytestmark = pytest.mark.gpu

SHIFTS = [(0.5, 0.0, -0.5), (0.0, 0.5, -0.5), (0.0, 0.0, 0.0), (0.5, 0.5, -0.5)]


@pytest.mark.parametrize("seed,polygons", [(0, False), (1, False), (2, False), (3, False),
                                           (10, True), (11, True), (12, True)])
def test_values_match_oracle(seed, polygons):
    mat, st = _random_layout(seed, n=12, polygons=polygons)
    k1, k2, j1, j2, i1, i2 = (0, 41, 0, 31, 0, 21) if not polygons else (4, 30, 3, 24, 0, 16)
    for sx, sy, sz in SHIFTS:
        got = mat.get_values(k1, k2, j1, j2, i1, i2, sx, sy, sz)
        want = np.array([[[st.value(k + sx, j + sy, i + sz, 0.1, 0.1, 0.1)
                           for k in range(k1, k2)] for j in range(j1, j2)] for i in range(i1, i2)])
        assert got.shape == want.shape
        assert np.max(np.abs(got - want)) < 1e-11, (sx, sy, sz)


def test_device_output_and_moved_primitive():
    import torch
    mat, st = _random_layout(7, n=8)
    host = mat.get_values(3, 30, 2, 25, 0, 18, 0.5, 0.0, -0.5)
    dev = mat.get_values(3, 30, 2, 25, 0, 18, 0.5, 0.0, -0.5, device=0)
    assert dev.is_cuda and np.array_equal(dev.cpu().numpy(), host)
    # primitives are held by reference: moving one changes the next evaluation
    p = mat.primitives[0]
    p.set_position(p.x0 + 0.37, p.y0 - 0.21)
    moved = mat.get_values(3, 30, 2, 25, 0, 18, 0.5, 0.0, -0.5)
    from oracle.structured import LayerStack
    st2 = LayerStack()
    for prim, z1, z2 in zip(mat.primitives, mat.zmins, mat.zmaxs):
        st2.add(_oracle_prim(prim), prim.layer, z1, z2)
    want = np.array([[[st2.value(k + 0.5, j, i - 0.5, 0.1, 0.1, 0.1) for k in range(3, 30)]
                      for j in range(2, 25)] for i in range(0, 18)])
    assert np.max(np.abs(moved - want)) < 1e-11


def test_too_many_pieces_is_an_error():
    """A staircase of rectangles over one cell corner leaves more than 32
    unclaimed pieces: reported as an error, nothing faults."""
    mat = G.StructuredMaterial3D(1.0, 1.0, 1.0, 1.0, 1.0, 1.0)
    n = 40
    for q in range(n):
        # cell [-0.5, 0.5]^2: every step holds the corner (-0.5, -0.5); x reach
        # grows and y reach shrinks, so each step cuts one more piece
        a = (q + 1) / (n + 2)
        x0, x1, y0, y1 = -1.5, a - 0.5, -1.5, 0.5 - a
        mat.add_primitive(G.Rectangle((x0 + x1) / 2, (y0 + y1) / 2, x1 - x0, y1 - y0), -1.0, 1.0)
    with pytest.raises(Exception, match="pieces"):
        mat.get_values(0, 1, 0, 1, 0, 1)
