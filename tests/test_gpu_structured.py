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


@pytest.mark.parametrize("seed,polygons,circles", [(0, False, False), (1, False, False), (2, False, False),
                                                   (3, False, False), (10, True, False), (11, True, False),
                                                   (12, True, False), (20, False, True), (21, True, True)])
def test_values_match_oracle(seed, polygons, circles):
    mat, st = _random_layout(seed, n=12, polygons=polygons, circles=circles)
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


def _layered(seed):
    """A layered structure of rectangles, polygons and circles on a small grid."""
    mat, _ = _random_layout(seed, n=10, polygons=True, circles=True)
    return mat


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fdtd_build_keeps_materials_on_device(precision):
    """FDTD.build with GPU-evaluable materials keeps the six arrays on the
    device (the solve reads them in place); they equal the host evaluation,
    the host arrays follow on demand (get_A_diag), update(bbox) re-samples the
    box on the device, and the solve equals the one on host-built arrays."""
    from emopt_b200 import problems as P
    p = P.random_box(3, shape=(20, 30, 40), d=0.1, w_pml=(4,) * 6, fixed_steps=200)
    sims = []
    for on_device in (True, False):
        sim = P.make_solver(p, precision=precision)
        sim.device_materials = on_device
        sim.set_materials(_layered(4), G.ConstantMaterial3D(1.0))
        sim.build()
        assert (sim._dev_mats is not None) == on_device
        sims.append(sim)
    dev, host = sims
    for a, b in zip(dev.get_A_diag(), host.get_A_diag()):
        np.testing.assert_array_equal(a, b)
    # move a primitive and re-sample a box on both
    idx = next(n for n, q in enumerate(dev._eps.primitives) if isinstance(q, G.Rectangle))
    x0, y0 = dev._eps.primitives[idx].x0 + 0.3, dev._eps.primitives[idx].y0 - 0.2
    for sim in sims:
        sim._eps.primitives[idx].set_position(x0, y0)
    bbox = (0.5, 2.5, 0.3, 1.9, 0.2, 1.4)
    for sim in sims:
        sim.update(bbox)
    for a, b in zip(dev.get_A_diag(), host.get_A_diag()):
        np.testing.assert_array_equal(a, b)
    for sim in sims:
        sim.solve_forward()
    for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        np.testing.assert_array_equal(dev.get_field(c), host.get_field(c))
