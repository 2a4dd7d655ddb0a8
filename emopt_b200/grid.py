"""Layered rectangle and polygon materials for ``emopt_b200.fdtd.FDTD``, evaluated on the GPU.

The names and semantics follow ``emopt.grid`` (``emopt/grid.py``, backed by
the reference's ``Grid.so``, ``src/Grid.cpp``): ``Rectangle`` primitives with a
material value and a priority ``layer`` (lower wins), and ``Polygon``
primitives, and ``Circle`` primitives with the reference's semantics (a
cell wholly inside takes the circle's value, a cut cell gets none of it),
stacked along z by ``StructuredMaterial3D.add_primitive(prim, z1, z2)``, and
``ConstantMaterial3D``.  ``get_values`` returns the Yee-cell averages that the
reference computes -- area-weighted within a z layer, length-weighted across
layers -- with one CUDA thread per cell (``FDTD_structured_values``), into a
numpy array or, with ``device=``, into a torch tensor that stays on the GPU
(``FDTD.set_material_arrays`` takes either).

Primitives are held by reference as in the reference: moving or resizing a
rectangle after ``add_primitive`` changes the next ``get_values``; the z
ranges and the priority order are fixed when the primitive is added
(``src/Grid.cpp:410-433``, ``:627-733``).  ``Polygon`` primitives are simple
polygons (convex ones evaluated whole, others through a triangulation made
here); ``FunctionMaterial3D`` samples an analytic ``f(x, y, z)`` at the Yee
points on the host.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import fdtd_ctypes as _ct
from .fdtd_ctypes import libFDTD


class MaterialPrimitive:
    """A shape with a material value; ``layer``: lower means higher priority."""

    def __init__(self):
        self._layer = 1

    @property
    def layer(self):
        return self._layer

    @layer.setter
    def layer(self, newlayer):
        self._layer = int(newlayer)

    def get_layer(self):
        return self._layer

    def set_layer(self, layer):
        self._layer = int(layer)


class Rectangle(MaterialPrimitive):
    """Axis-aligned rectangle centred on (x0, y0) with spans (xspan, yspan)."""

    def __init__(self, x0, y0, xspan, yspan):
        super().__init__()
        self._x0, self._y0 = float(x0), float(y0)
        self._xspan, self._yspan = float(xspan), float(yspan)
        self._mat = 1.0

    x0 = property(lambda s: s._x0, lambda s, v: setattr(s, "_x0", float(v)))
    y0 = property(lambda s: s._y0, lambda s, v: setattr(s, "_y0", float(v)))
    width = property(lambda s: s._xspan, lambda s, v: setattr(s, "_xspan", float(v)))
    height = property(lambda s: s._yspan, lambda s, v: setattr(s, "_yspan", float(v)))
    material_value = property(lambda s: s._mat, lambda s, v: setattr(s, "_mat", v))

    def set_material(self, mat):
        self._mat = mat

    def set_position(self, x0, y0):
        self._x0, self._y0 = float(x0), float(y0)

    def set_width(self, width):
        self._xspan = float(width)

    def set_height(self, height):
        self._yspan = float(height)

    def bounds(self):
        """xmin, xmax, ymin, ymax (``src/Grid.cpp:203-213``)."""
        return (self._x0 - self._xspan / 2.0, self._x0 + self._xspan / 2.0,
                self._y0 - self._yspan / 2.0, self._y0 + self._yspan / 2.0)

    def contains_point(self, x, y):
        """Strictly inside (``src/Grid.cpp:222-228``)."""
        hw, hh = self._xspan / 2, self._yspan / 2
        return (x > self._x0 - hw) and (x < self._x0 + hw) and (y > self._y0 - hh) and (y < self._y0 + hh)


class Circle(MaterialPrimitive):
    """Circle centred on (x0, y0) with radius r (``emopt/grid.py:330-365``,
    ``src/Grid.cpp:141-201``).  As in the reference, a circle gives its value
    only to cells whose four corners lie strictly inside it while no
    higher-priority primitive has claimed part of the cell; its partial-cell
    overlap is 0 there (``Circle::get_cell_overlap``), so a cell it only cuts
    keeps the other primitives' and the background's share."""

    def __init__(self, x0, y0, r):
        super().__init__()
        self._x0, self._y0, self._r = float(x0), float(y0), float(r)
        self._mat = 1.0

    material_value = property(lambda s: s._mat, lambda s, v: setattr(s, "_mat", v))

    def set_material(self, mat):
        self._mat = mat

    def set_position(self, x0, y0):
        self._x0, self._y0 = float(x0), float(y0)

    def set_radius(self, r):
        self._r = float(r)

    def get_x0(self):
        return self._x0

    def get_y0(self):
        return self._y0

    def get_r(self):
        return self._r

    def contains_point(self, x, y):
        dx, dy = x - self._x0, y - self._y0
        return dx * dx + dy * dy < self._r * self._r


class Polygon(MaterialPrimitive):
    """Simple polygon given by its vertices (``emopt/grid.py`` Polygon; a
    repeated closing vertex is accepted).  Convex polygons are evaluated as
    one part, others as the triangles of an ear-clipping triangulation."""

    def __init__(self, xs=None, ys=None):
        super().__init__()
        self._xs = np.zeros(0)
        self._ys = np.zeros(0)
        self._value = 1.0
        if xs is not None and ys is not None:
            self.set_points(xs, ys)

    xs = property(lambda s: np.copy(s._xs))
    ys = property(lambda s: np.copy(s._ys))
    Np = property(lambda s: len(s._xs))
    material_value = property(lambda s: s._value, lambda s, v: setattr(s, "_value", v))

    def set_material(self, mat):
        self._value = mat

    def set_points(self, x, y):
        self._xs = np.array(x, dtype=np.float64).ravel()
        self._ys = np.array(y, dtype=np.float64).ravel()

    def add_point(self, x, y):
        self._xs = np.append(self._xs, float(x))
        self._ys = np.append(self._ys, float(y))

    def add_points(self, x, y):
        self._xs = np.concatenate([self._xs, np.asarray(x, dtype=np.float64).ravel()])
        self._ys = np.concatenate([self._ys, np.asarray(y, dtype=np.float64).ravel()])

    def set_point(self, index, x, y):
        self._xs[index] = x
        self._ys[index] = y

    def outline(self):
        """Vertices counter-clockwise, without a repeated closing vertex."""
        x, y = self._xs, self._ys
        if len(x) > 1 and x[0] == x[-1] and y[0] == y[-1]:
            x, y = x[:-1], y[:-1]
        if len(x) < 3:
            raise ValueError("a Polygon needs at least 3 vertices")
        area2 = np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)
        if area2 < 0:
            x, y = x[::-1], y[::-1]
        return np.stack([x, y], axis=1)

    def contains_point(self, x, y):
        v = self.outline()
        inside = False
        for q in range(len(v)):
            (ax, ay), (bx, by) = v[q], v[(q + 1) % len(v)]
            if (bx - ax) * (y - ay) - (by - ay) * (x - ax) == 0 and min(ax, bx) <= x <= max(ax, bx) \
                    and min(ay, by) <= y <= max(ay, by):
                return False
            if (ay > y) != (by > y) and x < (bx - ax) * (y - ay) / (by - ay) + ax:
                inside = not inside
        return inside


def _convex_parts(v):
    """Convex pieces of the counter-clockwise outline v: itself when convex,
    else the triangles of an ear-clipping triangulation."""
    n = len(v)
    cross = [(v[(q + 1) % n][0] - v[q][0]) * (v[(q + 2) % n][1] - v[(q + 1) % n][1]) -
             (v[(q + 1) % n][1] - v[q][1]) * (v[(q + 2) % n][0] - v[(q + 1) % n][0]) for q in range(n)]
    if all(c >= 0 for c in cross):
        return [v]
    idx = list(range(n))
    tris = []

    def cr(a, b, c):
        return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])

    guard = 0
    while len(idx) > 3 and guard < 10 * n * n:
        guard += 1
        m = len(idx)
        for q in range(m):
            a, b, c = v[idx[q - 1]], v[idx[q]], v[idx[(q + 1) % m]]
            if cr(a, b, c) <= 0:
                continue            # reflex or degenerate corner
            if any(cr(a, b, v[r]) >= 0 and cr(b, c, v[r]) >= 0 and cr(c, a, v[r]) >= 0
                   for r in idx if r not in (idx[q - 1], idx[q], idx[(q + 1) % m])):
                continue            # another vertex inside the ear
            tris.append(np.array([a, b, c]))
            del idx[q]
            break
        else:
            raise ValueError("polygon could not be triangulated (is it simple?)")
    tris.append(np.array([v[r] for r in idx]))

    def area(p):
        p = np.asarray(p)
        return 0.5 * abs(np.sum(p[:, 0] * np.roll(p[:, 1], -1) - np.roll(p[:, 0], -1) * p[:, 1]))

    if abs(sum(area(t) for t in tris) - area(v)) > 1e-9 * max(area(v), 1e-300):
        raise ValueError("polygon edges cross each other: only simple polygons are supported")
    return tris


def _insert_by_priority(prims, prim):
    """Before the first primitive of a larger layer (``src/Grid.cpp:410-433``)."""
    for q, other in enumerate(prims):
        if prim.layer < other.layer:
            prims.insert(q, prim)
            return
    prims.append(prim)


class Material3D:
    def get_values_in(self, domain, sx=0, sy=0, sz=0, arr=None, squeeze=False, device=None):
        vals = self.get_values(domain.k.start, domain.k.stop, domain.j.start, domain.j.stop,
                               domain.i.start, domain.i.stop, sx, sy, sz, arr, device=device)
        return vals.squeeze() if squeeze else vals


class ConstantMaterial3D(Material3D):
    """Uniform material (``emopt/grid.py`` ConstantMaterial3D)."""

    def __init__(self, value):
        self._material_value = value

    material_value = property(lambda s: s._material_value,
                              lambda s, v: setattr(s, "_material_value", v))
    value = property(lambda s: complex(s._material_value))

    def get_value(self, k, j, i):
        return complex(self._material_value)

    def get_values(self, k1, k2, j1, j2, i1, i2, sx=0, sy=0, sz=0, arr=None, reshape=True,
                   device=None):
        shape = (i2 - i1, j2 - j1, k2 - k1)
        if device is not None:
            import torch
            return torch.full(shape, complex(self._material_value), dtype=torch.complex128,
                              device=torch.device("cuda", device) if isinstance(device, int) else device)
        out = np.full(shape, self._material_value, dtype=np.complex128)
        if arr is not None:
            np.ravel(arr)[:] = out.ravel()
            out = arr
        return out if reshape else np.ravel(out)


class FunctionMaterial3D(Material3D):
    """Material given by ``f(x, y, z) -> value`` evaluated at the staggered Yee
    points (host numpy; for analytic media in tests and examples)."""

    def __init__(self, f, dx, dy, dz):
        self.f, self.dx, self.dy, self.dz = f, dx, dy, dz

    def get_values(self, k1, k2, j1, j2, i1, i2, sx=0, sy=0, sz=0, arr=None, reshape=True,
                   device=None):
        z = (np.arange(i1, i2) + sz) * self.dz
        y = (np.arange(j1, j2) + sy) * self.dy
        x = (np.arange(k1, k2) + sx) * self.dx
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        vals = np.asarray(self.f(X, Y, Z), dtype=np.complex128)
        if device is not None:
            import torch
            return torch.as_tensor(vals, device=torch.device("cuda", device) if isinstance(device, int) else device)
        if arr is None:
            return vals if reshape else vals.ravel()
        arr.reshape(-1)[:] = vals.ravel()
        return arr


class StructuredMaterial3D(Material3D):
    """Rectangles stacked in z layers (``src/Grid.cpp:610-874``)."""

    def __init__(self, X, Y, Z, dx, dy, dz):
        self._X, self._Y, self._Z = X, Y, Z
        self._dx, self._dy, self._dz = dx, dy, dz
        self._zs: list[float] = []              # layer boundaries, ascending
        self._layers: list[list] = []            # primitives of each layer, by priority
        self._primitives, self._zmins, self._zmaxs = [], [], []

    primitives = property(lambda s: s._primitives)
    zmins = property(lambda s: s._zmins)
    zmaxs = property(lambda s: s._zmaxs)

    def add_primitive(self, prim, z1, z2):
        """Add ``prim`` over z1 <= z < z2, splitting layers as needed
        (``src/Grid.cpp:627-733``)."""
        if not isinstance(prim, (Rectangle, Polygon, Circle)):
            raise TypeError("Rectangle, Polygon and Circle primitives are evaluated on the GPU")
        self._primitives.append(prim)
        self._zmins.append(z1)
        self._zmaxs.append(z2)
        if z1 >= z2:
            return          # the reference warns and ignores layers without thickness
        zs, layers = self._zs, self._layers
        if not zs:
            zs += [z1, z2]
            layers.append([prim])
            return
        for z in (z1, z2):
            ins = None                           # last boundary <= z
            for q, zq in enumerate(zs):
                if z >= zq:
                    ins = q
            if ins is None:                      # below the stack
                zs.insert(0, z)
                layers.insert(0, [])
            elif ins == len(zs) - 1 and z != zs[ins]:   # above the stack
                zs.append(z)
                layers.append([])
            elif z != zs[ins]:                   # inside layer `ins`: split it
                copy = []
                for p in layers[ins]:
                    _insert_by_priority(copy, p)
                layers.insert(ins, copy)
                zs.insert(ins + 1, z)
        for q in range(len(layers)):
            if z1 <= zs[q] < z2:
                _insert_by_priority(layers[q], prim)

    def tables(self):
        """Layer and primitive tables of FDTD_structured_values for the current
        primitive parameters: (zs, layer_start, layer_prims, prim_info,
        prim_vals, parts, verts)."""
        prims, index, start, flat = [], {}, [0], []
        for layer in self._layers:
            for p in layer:
                if id(p) not in index:
                    index[id(p)] = len(prims)
                    prims.append(p)
                flat.append(index[id(p)])
            start.append(len(flat))
        info, vals, parts, verts = [], [], [], []
        for p in prims:
            if isinstance(p, Circle):
                ov = len(verts)
                verts.extend([[p.get_x0(), p.get_y0()], [p.get_r(), 0.0]])
                info.append((ov, -1, len(parts), 0))
                m = complex(p.material_value)
                r = p.get_r()
                vals.append((m.real, m.imag, p.get_x0() - r, p.get_x0() + r, p.get_y0() - r,
                             p.get_y0() + r))
                continue
            if isinstance(p, Rectangle):
                x0, x1, y0, y1 = p.bounds()
                outline = np.array([[x0, y0], [x1, y0], [x1, y1], [x0, y1]])
                pieces = [outline]
            else:
                outline = p.outline()
                pieces = _convex_parts(outline)
            ov = len(verts)
            verts.extend(outline.tolist())
            pp = len(parts)
            for piece in pieces:
                parts.append((len(verts), len(piece)))
                verts.extend(np.asarray(piece).tolist())
            info.append((ov, len(outline), pp, len(pieces)))
            m = complex(p.material_value)
            vals.append((m.real, m.imag, outline[:, 0].min(), outline[:, 0].max(),
                         outline[:, 1].min(), outline[:, 1].max()))
        i32 = lambda a, w: np.asarray(a if len(a) else [[0] * w], dtype=np.int32).reshape(-1)
        return (np.asarray(self._zs, dtype=np.float64), np.asarray(start, dtype=np.int32),
                np.asarray(flat if flat else [0], dtype=np.int32), i32(info, 4),
                np.asarray(vals if vals else [[0.0] * 6], dtype=np.float64).reshape(-1),
                i32(parts, 2), np.asarray(verts if verts else [[0.0, 0.0]], dtype=np.float64).reshape(-1),
                len(prims), len(parts), len(verts))

    def get_values(self, k1, k2, j1, j2, i1, i2, sx=0, sy=0, sz=0, arr=None, reshape=True,
                   device=None):
        """Cell values at fractional indices (k + sx, j + sy, i + sz) for
        k1 <= k < k2, j1 <= j < j2, i1 <= i < i2, shaped [i, j, k].  With
        ``device`` (a CUDA device index or torch device) the result is a torch
        tensor on that GPU; otherwise a numpy array (``arr`` if given)."""
        zs, start, flat, info, vals, parts, verts, nprims, nparts, nverts = self.tables()
        shape = (i2 - i1, j2 - j1, k2 - k1)
        if device is not None:
            import torch
            dev = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
            out = torch.empty(shape, dtype=torch.complex128, device=dev)
            ptr, dev_index = out.data_ptr(), dev.index or 0
            stream = torch.cuda.current_stream(dev).cuda_stream
        else:
            out = np.empty(shape, dtype=np.complex128) if arr is None else arr
            if out.dtype != np.complex128 or not out.flags["C_CONTIGUOUS"] or out.size != np.prod(shape):
                raise ValueError("arr must be a C-contiguous complex128 array of %d values" % np.prod(shape))
            ptr, dev_index, stream = out.ctypes.data, 0, None
        msg = ctypes.create_string_buffer(256)
        if np.prod(shape) > 0:
            rc = libFDTD.FDTD_structured_values(
                dev_index, stream, zs.ctypes.data if len(zs) else None, len(zs), start.ctypes.data,
                flat.ctypes.data, info.ctypes.data, vals.ctypes.data, nprims, parts.ctypes.data,
                nparts, verts.ctypes.data, nverts, self._dx, self._dy, self._dz,
                k1, k2, j1, j2, i1, i2, float(sx), float(sy), float(sz), ptr, msg, 256)
            if rc != _ct.FDTD_OK:
                raise _ct.FDTDError(msg.value.decode())
        if device is None and not reshape:
            return np.ravel(out)
        return out
