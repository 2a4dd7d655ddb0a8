"""CPU tests of the layered rectangle and polygon materials: the oracle
restatement on hand-computed cells, the host-side triangulation, and the
layer tables of emopt_b200.grid against the oracle's layer stack."""
import numpy as np
import pytest

from emopt_b200 import grid as G
from oracle.structured import LayerStack, _outline, _value, layer_value


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


def _random_polygon(rng):
    """A simple, star-shaped (often concave) polygon: n angles with gaps below
    pi around the centre, radii random."""
    n = int(rng.integers(3, 9))
    ang = (np.arange(n) + rng.uniform(0, 0.8, n)) * 2 * np.pi / n
    rad = rng.uniform(0.2, 1.2, n)
    cx, cy = rng.uniform(0, 4), rng.uniform(0, 3)
    xs, ys = cx + rad * np.cos(ang), cy + rad * np.sin(ang)
    if rng.uniform() < 0.5:                     # closed the emopt way, clockwise
        xs, ys = np.append(xs[::-1], xs[-1]), np.append(ys[::-1], ys[-1])
    return G.Polygon(xs, ys)


def _oracle_prim(p):
    m = complex(p.material_value)
    if isinstance(p, G.Circle):
        return ("circle", p.get_x0(), p.get_y0(), p.get_r(), m)
    if isinstance(p, G.Rectangle):
        return (*p.bounds(), m)
    return (p.outline().tolist(), m)


def _random_layout(seed, n=10, polygons=False, circles=False):
    rng = np.random.default_rng(seed)
    mat = G.StructuredMaterial3D(4.0, 3.0, 2.0, 0.1, 0.1, 0.1)
    st = LayerStack()
    for q in range(n):
        if circles and rng.uniform() < 0.4:
            r = G.Circle(rng.uniform(0, 4), rng.uniform(0, 3), rng.uniform(0.1, 1.5))
        elif polygons and rng.uniform() < 0.6:
            r = _random_polygon(rng)
        else:
            r = G.Rectangle(rng.uniform(0, 4), rng.uniform(0, 3), rng.uniform(0.05, 2.5), rng.uniform(0.05, 2.0))
        r.material_value = complex(rng.uniform(1, 12), rng.uniform(0, 0.3))
        r.layer = int(rng.integers(0, 4))
        z1 = float(np.round(rng.uniform(0, 1.5), 2))
        z2 = z1 + float(np.round(rng.uniform(-0.1, 1.0), 2))
        mat.add_primitive(r, z1, z2)
        st.add(_oracle_prim(r), r.layer, z1, z2)
    return mat, st


def test_polygon_known_answers():
    # a triangle holding the lower-right half of the cell [-0.5, 0.5]^2 (three
    # corners on its edges are not inside, (0.5, -0.5) is): half the cell
    tri = ([(-0.5 - 1e-9, -0.5 - 1e-9), (5.0, -0.5 - 1e-9), (5.0, 5.0)], 3.0)
    assert layer_value([tri], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.5 * 3 + 0.5, rel=1e-6)
    # an L-shaped (concave) polygon covering three quarters
    L = ([(-2, -2), (2, -2), (2, 0), (0, 0), (0, 2), (-2, 2)], 5.0)
    assert layer_value([L], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.75 * 5 + 0.25)
    # a clockwise outline with a repeated closing vertex comes out
    # counter-clockwise without the repeat
    v = G.Polygon([0, 0, 2, 2, 0], [0, 2, 2, 0, 0]).outline()
    assert len(v) == 4
    assert np.sum(v[:, 0] * np.roll(v[:, 1], -1) - np.roll(v[:, 0], -1) * v[:, 1]) == pytest.approx(8.0)
    # the triangulation of a concave outline covers it exactly

    def tri_area(t):
        return 0.5 * abs((t[1][0] - t[0][0]) * (t[2][1] - t[0][1]) - (t[1][1] - t[0][1]) * (t[2][0] - t[0][0]))

    tris = G._convex_parts(G.Polygon([0, 2, 2, 1, 0], [0, 0, 2, 1, 2]).outline())
    assert len(tris) == 3 and sum(tri_area(t) for t in tris) == pytest.approx(3.0)


@pytest.mark.parametrize("seed", range(6))
def test_layer_tables_match_oracle_stack(seed):
    mat, st = _random_layout(seed, polygons=True, circles=seed % 2 == 1)
    zs, start, flat, info, vals, parts, verts, nprims, nparts, nverts = mat.tables()
    assert list(zs) == st.zs
    assert len(start) == len(st.layers) + 1
    verts = verts.reshape(-1, 2)
    info = info.reshape(-1, 4)
    vals = vals.reshape(-1, 6)
    for l, layer in enumerate(st.layers):
        got = []
        for q in range(start[l], start[l + 1]):
            pr = flat[q]
            ov, on = info[pr][0], info[pr][1]
            if on < 0:      # circle: centre and radius
                got.append(([verts[ov][0], verts[ov][1], verts[ov + 1][0]], complex(vals[pr][0], vals[pr][1])))
            else:
                got.append((verts[ov:ov + on].tolist(), complex(vals[pr][0], vals[pr][1])))
        want = [(([p[1], p[2], p[3]] if isinstance(p[0], str) else _outline(p)), _value(p))
                for p, _ in layer]
        assert [(np.asarray(a).tolist(), b) for a, b in got] == [(np.asarray(a).tolist(), b) for a, b in want]


def test_circle_known_answers():
    """The reference's circle (src/Grid.cpp:141-201): a cell wholly inside
    takes its value; a cell it only cuts gets none of it (overlap stub 0) and
    keeps the background; behind a higher-priority primitive that claimed
    part of the cell, even a wholly covering circle adds nothing."""
    m = 6.0 + 0.2j
    c = ("circle", 0.0, 0.0, 2.0, m)
    assert layer_value([c], 0.0, 0.0, 1.0, 1.0) == m
    assert layer_value([c], 2.0, 0.0, 1.0, 1.0) == 1.0           # corners (1.5, +-0.5) inside, cut only
    rect = (0.0, 5.0, -5.0, 5.0, 3.0)                             # right half of the cell
    assert layer_value([rect, c], 0.0, 0.0, 1.0, 1.0) == pytest.approx(0.5 * 3 + 0.5)
    assert layer_value([c, rect], 0.0, 0.0, 1.0, 1.0) == m
    circ = G.Circle(0.0, 0.0, 2.0)
    assert circ.contains_point(1.0, 1.0) and not circ.contains_point(2.0, 0.0)


def test_self_crossing_polygon_is_rejected():
    bowtie = G.Polygon([0, 1, 1, 0], [0, 1, 0, 1])
    with pytest.raises(ValueError, match="cross"):
        G._convex_parts(bowtie.outline())


def _check_tables(mat, info=None):
    """FDTD_structured_values on an empty cell range: the table checks run,
    no device is touched."""
    import ctypes
    from emopt_b200.fdtd_ctypes import libFDTD
    zs, start, flat, info0, vals, parts, verts, nprims, nparts, nverts = mat.tables()
    info = info0 if info is None else info
    msg = ctypes.create_string_buffer(256)
    rc = libFDTD.FDTD_structured_values(
        0, None, zs.ctypes.data, len(zs), start.ctypes.data, flat.ctypes.data, info.ctypes.data,
        vals.ctypes.data, nprims, parts.ctypes.data, nparts, verts.ctypes.data, nverts,
        1.0, 1.0, 1.0, 0, 0, 0, 4, 0, 4, 0.0, 0.0, 0.0, vals.ctypes.data, msg, 256)
    return rc, msg.value.decode()


@pytest.mark.parametrize("seed", [1, 3, 20, 21])
def test_library_accepts_circle_tables(seed):
    """Every table the host builds (circles included: outline count -1, no
    convex parts) passes the library's table checks."""
    mat, _ = _random_layout(seed, n=12, polygons=seed % 2 == 1, circles=True)
    info = mat.tables()[3].reshape(-1, 4)
    assert (info[:, 1] == -1).any()
    assert _check_tables(mat) == (0, "")


def test_library_rejects_bad_circle_entry():
    mat, _ = _random_layout(20, n=12, polygons=False, circles=True)
    info = mat.tables()[3].copy().reshape(-1, 4)
    q = int(np.nonzero(info[:, 1] == -1)[0][0])
    info[q, 3] = 1          # a circle carries no convex parts
    rc, msg = _check_tables(mat, np.ascontiguousarray(info.reshape(-1)))
    assert rc != 0 and "bad primitive table" in msg
