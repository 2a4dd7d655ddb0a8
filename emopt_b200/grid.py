"""Minimal material objects implementing the ``Material3D.get_values`` protocol.

``FDTD.build`` samples permittivity and permeability through
``get_values(k1, k2, j1, j2, i1, i2, sx, sy, sz, arr)`` (``emopt/grid.py:762``),
where ``(sx, sy, sz)`` are the Yee offsets in cells.  The reference's smoothed
``StructuredMaterial3D`` (polygon overlap in ``src/Grid.cpp``) is outside the
accelerated path; these classes cover uniform media and voxel arrays.
"""
from __future__ import annotations

import numpy as np


class ConstantMaterial3D:
    """Uniform material (``emopt/grid.py`` ConstantMaterial3D)."""

    def __init__(self, value):
        self.value = complex(value)

    def get_value(self, k, j, i):
        return self.value

    def get_values(self, k1, k2, j1, j2, i1, i2, sx=0, sy=0, sz=0, arr=None):
        shape = (i2 - i1, j2 - j1, k2 - k1)
        if arr is None:
            arr = np.zeros(shape, dtype=np.complex128)
        arr.reshape(-1)[:] = self.value
        return arr


class FunctionMaterial3D:
    """Material given by ``f(x, y, z) -> value`` evaluated at the staggered Yee points."""

    def __init__(self, f, dx, dy, dz):
        self.f, self.dx, self.dy, self.dz = f, dx, dy, dz

    def get_values(self, k1, k2, j1, j2, i1, i2, sx=0, sy=0, sz=0, arr=None):
        z = (np.arange(i1, i2) + sz) * self.dz
        y = (np.arange(j1, j2) + sy) * self.dy
        x = (np.arange(k1, k2) + sx) * self.dx
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        vals = np.asarray(self.f(X, Y, Z), dtype=np.complex128)
        if arr is None:
            return vals
        arr.reshape(-1)[:] = vals.ravel()
        return arr
