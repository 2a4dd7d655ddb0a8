"""CPU tests of the layered rectangle materials: the oracle restatement on
hand-computed cells, and the host-side layer tables of emopt_b200.grid
against the oracle's layer stack."""
import numpy as np
import pytest

from emopt_b200 import grid as G
from oracle.structured import LayerStack, layer_value


def test_layer_value_known_answers():
    m = 4.0 + 0.5j
    # cell [-0.5, 0.5]^2; a rectangle holding the right half (corners (x1,*) inside)
    assert layer_value([(0.0, 5.0, -5.0, 5.0, m)], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.5 * m + 0.5)
    # the whole cell inside: the material outright
    assert layer_value([(-1.0, 1.0, -1.0, 1.0, m)], 0.0, 0.0, 1.0, 1.0) == m
    # a strip through the middle with no corner inside is skipped (reference quirk)
    assert layer_value([(-0.1, 0.1, -5.0, 5.0, m)], 0.0, 0.0, 1.0, 1.0) == 1.0
    # priority: the first rectangle claims the overlap; a quarter each
    a = (0.0, 5.0, -5.0, 5.0, 2.0)            # right half
    b = (-5.0, 5.0, 0.0, 5.0, 3.0)            # top half
    assert layer_value([a, b], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.5 * 2 + 0.25 * 3 + 0.25)
    assert layer_value([b, a], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.5 * 3 + 0.25 * 2 + 0.25)
    # full coverage by two primitives leaves nothing for the background
    c = (-5.0, 0.0, -5.0, 5.0, 7.0)
    assert layer_value([a, c], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.5 * 2 + 0.5 * 7)
    # a layer without primitives is 0
    assert layer_value([], 0.0, 0.0, 1.0, 1.0) == 0.0


def test_z_averaging_known_answers():
    st = LayerStack()
    st.add((-10, 10, -10, 10, 9.0), 1, 1.0, 2.0)          # a slab 1 <= z < 2, full in x/y
    dz = 1.0
    # cell i = 1 spans [0.5, 1.5): half background below, half slab
    assert st.value(0, 0, 1, 1.0, 1.0, dz) == pytest.approx(0.5 + 0.5 * 9)
    assert st.value(0, 0, 1.5, 1.0, 1.0, dz) == pytest.approx(9.0)      # [1, 2)
    assert st.value(0, 0, 3, 1.0, 1.0, dz) == pytest.approx(1.0)        # above
    assert st.value(0, 0, -2, 1.0, 1.0, dz) == 1.0                      # below
    # a second slab above a gap: the gap layer (no primitive) counts 0
    st.add((-10, 10, -10, 10, 4.0), 1, 3.0, 4.0)
    assert st.value(0, 0, 2.5, 1.0, 1.0, dz) == pytest.approx(0.0)      # [2, 3) is the gap
    assert st.value(0, 0, 2.0, 1.0, 1.0, dz) == pytest.approx(0.5 * 9 + 0.0)


def _random_layout(seed, n=10):
    rng = np.random.default_rng(seed)
    mat = G.StructuredMaterial3D(4.0, 3.0, 2.0, 0.1, 0.1, 0.1)
    st = LayerStack()
    for q in range(n):
        r = G.Rectangle(rng.uniform(0, 4), rng.uniform(0, 3), rng.uniform(0.05, 2.5), rng.uniform(0.05, 2.0))
        r.material_value = complex(rng.uniform(1, 12), rng.uniform(0, 0.3))
        r.layer = int(rng.integers(0, 4))
        z1 = float(np.round(rng.uniform(0, 1.5), 2))
        z2 = z1 + float(np.round(rng.uniform(-0.1, 1.0), 2))
        mat.add_primitive(r, z1, z2)
        st.add((*r.bounds(), complex(r.material_value)), r.layer, z1, z2)
    return mat, st


@pytest.mark.parametrize("seed", range(6))
def test_layer_tables_match_oracle_stack(seed):
    mat, st = _random_layout(seed)
    zs, start, flat, rects, nrects = mat.tables()
    assert list(zs) == st.zs
    assert len(start) == len(st.layers) + 1
    for l, layer in enumerate(st.layers):
        got = [tuple(rects[flat[q]][:4]) + (complex(rects[flat[q]][4], rects[flat[q]][5]),)
               for q in range(start[l], start[l + 1])]
        assert got == [tuple(p) for p, _ in layer]
