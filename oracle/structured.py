"""CPU restatement of the reference's layered rectangle materials (test oracle).

Test infrastructure only: the GPU evaluation (emopt_b200/csrc/structured.cu,
emopt_b200/grid.py) is checked against this.  It restates
StructuredMaterial3D (src/Grid.cpp:627-826) and StructuredMaterial2D
(src/Grid.cpp:410-525) for Rectangle primitives (src/Grid.cpp:203-300) in
plain Python, but measures the claimed areas differently from the GPU code:
the cell is cut along every primitive edge that crosses it, and each piece of
that grid belongs to the first primitive (in priority order, among those the
reference lets claim area) that covers it.

Parity unpinned: the reference's Grid.so needs Eigen and Boost.Geometry,
which are not in this image, so no reference output exists; the restatement
follows the source and is checked on hand-computed cases.
"""
from __future__ import annotations


def _strictly_inside(r, x, y):
    return r[0] < x < r[1] and r[2] < y < r[3]


def layer_value(rects, xd, yd, dx, dy):
    """Cell value of one z layer (src/Grid.cpp:460-525).  ``rects``: the
    layer's primitives in priority order as (xmin, xmax, ymin, ymax, value)."""
    if not rects:
        return 0.0                    # empty layer: the reference returns 0
    x0, x1, y0, y1 = xd - dx / 2.0, xd + dx / 2.0, yd - dy / 2.0, yd + dy / 2.0
    full = (x1 - x0) * (y1 - y0)
    xs = sorted({x0, x1} | {e for r in rects for e in (r[0], r[1]) if x0 < e < x1})
    ys = sorted({y0, y1} | {e for r in rects for e in (r[2], r[3]) if y0 < e < y1})
    pieces = {(a, b): (xs[a + 1] - xs[a]) * (ys[b + 1] - ys[b])
              for a in range(len(xs) - 1) for b in range(len(ys) - 1)}
    free = set(pieces)
    val = 0.0
    for r in rects:
        corners = [_strictly_inside(r, x0, y0), _strictly_inside(r, x1, y0),
                   _strictly_inside(r, x1, y1), _strictly_inside(r, x0, y1)]
        if all(corners) and len(free) == len(pieces):
            return r[4]
        if any(corners):
            took = [p for p in free
                    if r[0] < (xs[p[0]] + xs[p[0] + 1]) / 2 < r[1]
                    and r[2] < (ys[p[1]] + ys[p[1] + 1]) / 2 < r[3]]
            val += sum(pieces[p] for p in took) / full * r[4]
            free.difference_update(took)
        if not free:
            break
    if free:
        val += sum(pieces[p] for p in free) / full * 1.0
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
