"""Domain bookkeeping and field-component names used by the FDTD interface.

``DomainCoordinates`` follows ``emopt/misc.py:169-279``: a box given in real
coordinates maps to index ranges ``[int(min/d), int(max/d) + 1)`` along each
axis.  ``FieldComponent`` / ``SourceComponent`` are the string constants of
``emopt/defs.py:11-25``.  This package runs as a single process per device, so
the MPI helpers of the reference (``COMM``, ``RANK``, ``NOT_PARALLEL``) reduce
to constants.
"""
from __future__ import annotations

import warnings

import numpy as np

RANK = 0
N_PROC = 1
NOT_PARALLEL = True


class FieldComponent:
    Ex = "Ex"
    Ey = "Ey"
    Ez = "Ez"
    Hx = "Hx"
    Hy = "Hy"
    Hz = "Hz"


class SourceComponent:
    Jx = "Jx"
    Jy = "Jy"
    Jz = "Jz"
    Mx = "Mx"
    My = "My"
    Mz = "Mz"


def warning_message(message: str, module: str = "emopt_b200") -> None:
    warnings.warn(f"{module}: {message}", stacklevel=2)


class DomainCoordinates:
    """Index ranges and coordinates of a line, plane or volume of the grid."""

    def __init__(self, xmin, xmax, ymin, ymax, zmin, zmax, dx, dy, dz):
        i1, i2 = int(zmin / dz), int(zmax / dz) + 1
        j1, j2 = int(ymin / dy), int(ymax / dy) + 1
        k1, k2 = int(xmin / dx), int(xmax / dx) + 1
        self.set_region(k1, k2, j1, j2, i1, i2, dx, dy, dz)

    def set_region(self, k1, k2, j1, j2, i1, i2, dx, dy, dz):
        self.i1, self.i2, self.j1, self.j2, self.k1, self.k2 = i1, i2, j1, j2, k1, k2
        self._i, self._j, self._k = slice(i1, i2), slice(j1, j2), slice(k1, k2)
        self._z = dz * np.arange(i1, i2, dtype=np.int64).astype(np.double)
        self._y = dy * np.arange(j1, j2, dtype=np.int64).astype(np.double)
        self._x = dx * np.arange(k1, k2, dtype=np.int64).astype(np.double)
        self._Nx, self._Ny, self._Nz = k2 - k1, j2 - j1, i2 - i1
        self._dx, self._dy, self._dz = dx, dy, dz

    x = property(lambda s: s._x)
    y = property(lambda s: s._y)
    z = property(lambda s: s._z)
    i = property(lambda s: s._i)
    j = property(lambda s: s._j)
    k = property(lambda s: s._k)
    Nx = property(lambda s: s._Nx)
    Ny = property(lambda s: s._Ny)
    Nz = property(lambda s: s._Nz)
    dx = property(lambda s: s._dx)
    dy = property(lambda s: s._dy)
    dz = property(lambda s: s._dz)
    xspan = property(lambda s: s._dx * (s._Nx - 1))
    yspan = property(lambda s: s._dy * (s._Ny - 1))
    zspan = property(lambda s: s._dz * (s._Nz - 1))
    shape = property(lambda s: (s._Nz, s._Ny, s._Nx))

    @classmethod
    def from_indices(cls, k1, k2, j1, j2, i1, i2, dx, dy, dz):
        """Domain covering index ranges [k1,k2) x [j1,j2) x [i1,i2) exactly."""
        d = cls.__new__(cls)
        d.set_region(k1, k2, j1, j2, i1, i2, dx, dy, dz)
        return d

    def grow(self, x1, x2, y1, y2, z1, z2):
        """Grow by the given numbers of cells towards -x, +x, -y, +y, -z, +z
        (negative values shrink; not checked), ``emopt/misc.py`` grow."""
        self.set_region(self.k1 - x1, self.k2 + x2, self.j1 - y1, self.j2 + y2, self.i1 - z1,
                        self.i2 + z2, self._dx, self._dy, self._dz)

    def copy(self):
        """A new domain with the same index ranges and spacings."""
        return DomainCoordinates.from_indices(self.k1, self.k2, self.j1, self.j2, self.i1, self.i2,
                                              self._dx, self._dy, self._dz)

    def get_bounding_box(self):
        return [self._x[0], self._x[-1], self._y[0], self._y[-1], self._z[0], self._z[-1]]
