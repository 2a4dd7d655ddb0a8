"""CPU restatement of the reference's layered rectangle materials (test oracle).

Test infrastructure only: the GPU evaluation (emopt_b200/csrc/structured.cu,
emopt_b200/grid.py) is checked against this.  It restates
StructuredMaterial3D (src/Grid.cpp:627-826) and StructuredMaterial2D
(src/Grid.cpp:410-525) for Rectangle, Polygon and Circle primitives
(src/Grid.cpp:141-395; a circle is ("circle", x0, y0, r, value)) in
plain Python, but measures the claimed areas differently from the GPU code
(which subtracts convex parts piece by piece): each area is integrated
exactly over vertical slices of the cell, the cross-section at a slice being
interval arithmetic on the polygons' crossings (its length is linear between
the x of vertices, of edge crossings and of edges meeting the cell's top or
bottom, so one midpoint per slab is exact).

Parity unpinned: the reference's Grid.so needs Eigen and Boost.Geometry,
which are not in this image, so no reference output exists; the restatement
follows the source and is checked on hand-computed cases.
"""
from __future__ import annotations


def _is_circle(prim):
    return isinstance(prim[0], str) and prim[0] == "circle"


def _outline(prim):
    """Counter-clockwise outline of a primitive given as (xmin, xmax, ymin,
    ymax, value) or as (vertices, value)."""
    if len(prim) == 5:
        x0, x1, y0, y1, _ = prim
        return [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]
    return [tuple(map(float, p)) for p in prim[0]]


def _value(prim):
    return prim[4] if len(prim) == 5 else prim[1]


def _circle_inside(prim, x, y):
    """Circle::contains_point (src/Grid.cpp:144-149): strictly inside."""
    _, x0, y0, r, _ = prim
    dx, dy = x - x0, y - y0
    return dx * dx + dy * dy < r * r


def _inside(poly, x, y):
    """Strictly inside (a point on an edge is outside), even-odd rule."""
    inside = False
    n = len(poly)
    for q in range(n):
        (ax, ay), (bx, by) = poly[q], poly[(q + 1) % n]
        if (bx - ax) * (y - ay) - (by - ay) * (x - ax) == 0 and min(ax, bx) <= x <= max(ax, bx) \
                and min(ay, by) <= y <= max(ay, by):
            return False
        if (ay > y) != (by > y) and x < (bx - ax) * (y - ay) / (by - ay) + ax:
            inside = not inside
    return inside


def _section(poly, x):
    """y-intervals of the polygon on the vertical line x (x not a vertex x)."""
    ys = []
    n = len(poly)
    for q in range(n):
        (ax, ay), (bx, by) = poly[q], poly[(q + 1) % n]
        if (ax < x) != (bx < x):
            ys.append(ay + (by - ay) * (x - ax) / (bx - ax))
    ys.sort()
    return [(ys[q], ys[q + 1]) for q in range(0, len(ys) - 1, 2)]


def _union(ivs):
    out = []
    for a, b in sorted(ivs):
        if out and a <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], b))
        else:
            out.append((a, b))
    return out


def _minus(ivs, cut):
    out = []
    for a, b in ivs:
        pieces = [(a, b)]
        for c, d in cut:
            nxt = []
            for u, v in pieces:
                if d <= u or c >= v:
                    nxt.append((u, v))
                    continue
                if c > u:
                    nxt.append((u, c))
                if d < v:
                    nxt.append((d, v))
            pieces = nxt
        out += pieces
    return out


def _area(x0, x1, y0, y1, take, taken):
    """Exact area of (cell & take) minus the union of `taken` (polygons; take
    None means the whole cell): cross-section lengths are linear between the
    x of vertices and edge crossings, so the midpoint of each slab is exact."""
    polys = ([take] if take else []) + list(taken)
    xs = {x0, x1}
    edges = []
    for poly in polys:
        n = len(poly)
        for q in range(n):
            a, b = poly[q], poly[(q + 1) % n]
            edges.append((a, b))
            if x0 < a[0] < x1:
                xs.add(a[0])
            # where the edge meets the cell's bottom or top the clipped
            # cross-section bends too
            for yc in (y0, y1):
                if (a[1] - yc) * (b[1] - yc) < 0:
                    xc = a[0] + (b[0] - a[0]) * (yc - a[1]) / (b[1] - a[1])
                    if x0 < xc < x1:
                        xs.add(xc)
    for q in range(len(edges)):
        (ax, ay), (bx, by) = edges[q]
        for r in range(q + 1, len(edges)):
            (cx, cy), (dx_, dy_) = edges[r]
            den = (bx - ax) * (dy_ - cy) - (by - ay) * (dx_ - cx)
            if den == 0:
                continue
            t = ((cx - ax) * (dy_ - cy) - (cy - ay) * (dx_ - cx)) / den
            u = ((cx - ax) * (by - ay) - (cy - ay) * (bx - ax)) / den
            if 0 <= t <= 1 and 0 <= u <= 1:
                xi = ax + t * (bx - ax)
                if x0 < xi < x1:
                    xs.add(xi)
    xs = sorted(xs)
    total = 0.0
    for q in range(len(xs) - 1):
        xm = 0.5 * (xs[q] + xs[q + 1])
        ivs = [(y0, y1)]
        if take:
            ivs = [(max(a, y0), min(b, y1)) for a, b in _section(take, xm) if min(b, y1) > max(a, y0)]
        cut = _union([iv for poly in taken for iv in _section(poly, xm)])
        total += (xs[q + 1] - xs[q]) * sum(b - a for a, b in _minus(ivs, cut))
    return total


def layer_value(prims, xd, yd, dx, dy):
    """Cell value of one z layer (src/Grid.cpp:460-525).  ``prims``: the
    layer's primitives in priority order, each (xmin, xmax, ymin, ymax, value)
    or (vertices, value)."""
    if not prims:
        return 0.0                    # empty layer: the reference returns 0
    x0, x1, y0, y1 = xd - dx / 2.0, xd + dx / 2.0, yd - dy / 2.0, yd + dy / 2.0
    full = (x1 - x0) * (y1 - y0)
    taken = []
    val = 0.0
    free = full
    for prim in prims:
        if _is_circle(prim):
            # a circle's cell overlap is 0 (src/Grid.cpp:167-171): it gives its
            # value to a cell it holds entirely while nothing is claimed, and
            # claims nothing otherwise
            corners = [_circle_inside(prim, x, y) for x, y in ((x0, y0), (x1, y0), (x1, y1), (x0, y1))]
            if all(corners) and not taken:
                return _value(prim)
            if free == 0:
                break
            continue
        poly = _outline(prim)
        corners = [_inside(poly, x0, y0), _inside(poly, x1, y0), _inside(poly, x1, y1),
                   _inside(poly, x0, y1)]
        if all(corners) and not taken:
            return _value(prim)
        if any(corners):
            val += _area(x0, x1, y0, y1, poly, taken) / full * _value(prim)
            taken.append(poly)
            free = _area(x0, x1, y0, y1, None, taken)
        if free == 0:
            break
    if free > 0:
        val += free / full * 1.0
    return val


class LayerStack:
    """z layers of primitives (src/Grid.cpp:627-733)."""

    def __init__(self):
        self.zs = []
        self.layers = []

    @staticmethod
    def _add(layer, prim, prio):
        q = 0
        while q < len(layer) and not (prio < layer[q][1]):
            q += 1
        layer.insert(q, (prim, prio))

    def add(self, prim, prio, z1, z2):
        if z1 >= z2:
            return
        if not self.zs:
            self.zs = [z1, z2]
            self.layers = [[(prim, prio)]]
            return
        for z in (z1, z2):
            below = [q for q, zq in enumerate(self.zs) if zq <= z]
            if not below:
                self.zs.insert(0, z)
                self.layers.insert(0, [])
                continue
            q = below[-1]
            if self.zs[q] == z:
                continue
            if q == len(self.zs) - 1:
                self.zs.append(z)
                self.layers.append([])
            else:
                copy = []
                for p, pr in self.layers[q]:
                    self._add(copy, p, pr)
                self.layers.insert(q, copy)
                self.zs.insert(q + 1, z)
        for q, zq in enumerate(self.zs[:-1]):
            if z1 <= zq < z2:
                self._add(self.layers[q], prim, prio)

    def value(self, x, y, z, dx, dy, dz):
        """Cell value at fractional indices (src/Grid.cpp:737-826)."""
        if len(self.zs) < 2:
            return 1.0
        zmin, zmax = (z - 0.5) * dz, (z + 0.5) * dz
        zs = self.zs
        if zmax <= zs[0]:
            return 1.0
        v = 0.0
        if zmin < zs[0]:
            v += (zs[0] - zmin) / dz
            zmin = zs[0]

        def lv(l):
            return layer_value([p for p, _ in self.layers[l]], x * dx, y * dy, dx, dy)

        for l in range(len(zs) - 1):
            if zmin >= zs[l] and zmax <= zs[l + 1]:
                return v + (zmax - zmin) / dz * lv(l)
            if zs[l] <= zmin < zs[l + 1] < zmax:
                v += (zs[l + 1] - zmin) / dz * lv(l)
                zmin = zs[l + 1]
        return v + (zmax - zmin) / dz
