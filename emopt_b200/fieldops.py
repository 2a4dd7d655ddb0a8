"""Field access around a solve, on the GPU (``csrc/fields_kernels.cu``).

* :func:`interp` -- a field component interpolated onto the Ez grid, the
  reference's ``FDTD.get_field_interp`` (emopt/fdtd.py:1401-1553), from a
  device block of raw phasors; differentiable (:class:`InterpField`: the
  backward pass is the exact transpose, on the device).
* :func:`dfdx_interp` -- the reference's ``interpolated_dFdx_3D``
  (emopt/fomutils.py:1282-1426) on device tensors: derivatives with respect
  to interpolated fields -> the adjoint current sources on the staggered grid,
  the reference's rules at symmetric min faces included.
* :func:`source_power` -- ``FDTD.get_source_power`` (emopt/fdtd.py:1555-1667):
  the Poynting flux through the planes one cell inside the CPML, with a fixed
  order fp64 reduction on the device; differentiable (:class:`SourcePower`).

Every array is a complex128 CUDA tensor in ``[z, y, x]`` order.  The block
geometry of an interpolation (which cells are read, where the requested domain
sits in the padded block, which pad is mirrored) is computed here exactly as
the reference's numpy code slices its arrays, so results agree with
``emopt_b200.fdtd.FDTD.get_field_interp`` to the last bit.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import fdtd_ctypes as _ct
from .misc import DomainCoordinates

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_CIDX = {c: q for q, c in enumerate(COMPONENTS)}
_NBLK = 148   # partial sums per plane of the flux reduction (fields_kernels.cu)


def _check(status: int, msg) -> None:
    if status != _ct.FDTD_OK:
        raise _ct.FDTDError(msg.value.decode(errors="replace"))


def _stream(t: torch.Tensor):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


def grow_domain(domain: DomainCoordinates, shape, d) -> DomainCoordinates:
    """The domain grown by one cell where the grid allows: the block the
    interpolation reads (emopt/fdtd.py:1417-1430; rebuilt from coordinates,
    as the reference does)."""
    Nz, Ny, Nx = shape
    k1, k2, j1, j2, i1, i2 = domain.k1, domain.k2, domain.j1, domain.j2, domain.i1, domain.i2
    if k1 > 0: k1 -= 1
    if k2 < Nx - 1: k2 += 1
    if j1 > 0: j1 -= 1
    if j2 < Ny - 1: j2 += 1
    if i1 > 0: i1 -= 1
    if i2 < Nz - 1: i2 += 1
    return DomainCoordinates(k1 * d[0], k2 * d[0], j1 * d[1], j2 * d[1], i1 * d[2], i2 * d[2],
                             d[0], d[1], d[2])


def clipped_extent(lo: int, hi: int, n: int) -> int:
    """Cells a slice lo:hi selects along an axis of n cells (lo >= 0)."""
    return max(0, min(hi, n) - min(lo, n))


def geometry(component: str, domain, domain_interp, block_shape, bc: str, block_origin=(0, 0, 0),
             array_shape=None) -> tuple[np.ndarray, tuple]:
    """The 17 integers the interpolation kernels take, and the output shape.

    The block read is ``domain_interp`` clipped to the grid, ``block_shape``
    cells (z, y, x), starting at ``block_origin`` of an array of
    ``array_shape`` (default: the block itself).  For Ez the reference reads
    ``domain`` itself: pass ``domain_interp = domain``."""
    ni, nj, nk = block_shape
    Az, Ay, Ax = array_shape if array_shape is not None else block_shape
    di, dj, dk = domain.i1 - domain_interp.i1, domain.j1 - domain_interp.j1, domain.k1 - domain_interp.k1
    if component == "Ez":
        oi = min(domain.i2 - domain_interp.i1, ni) - di
        oj = min(domain.j2 - domain_interp.j1, nj) - dj
        ok = min(domain.k2 - domain_interp.k1, nk) - dk
    else:
        oi = ni - di - (domain_interp.i2 - domain.i2)
        oj = nj - dj - (domain_interp.j2 - domain.j2)
        ok = nk - dk - (domain_interp.k2 - domain.k2)
    oi, oj, ok = max(oi, 0), max(oj, 0), max(ok, 0)
    sign = {"E": -1, "H": 1}
    sx = sign.get(bc[0], 0) if domain_interp.k1 == 0 else 0
    sy = sign.get(bc[1], 0) if domain_interp.j1 == 0 else 0
    g = np.array([block_origin[0], block_origin[1], block_origin[2], ni, nj, nk, di, dj, dk,
                  oi, oj, ok, Ax, Ay, Az, sx, sy], dtype=np.int32)
    return g, (oi, oj, ok)


def _interp_raw(raw: torch.Tensor, comp: int, g: np.ndarray, shape) -> torch.Tensor:
    out = torch.empty(shape, dtype=torch.complex128, device=raw.device)
    msg = ctypes.create_string_buffer(256)
    _check(_ct.libFDTD.FDTD_interp_field(raw.device.index, _stream(raw), comp, _ptr(raw),
                                         g.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _ptr(out),
                                         msg, len(msg)), msg)
    return out


def _interp_T(gout: torch.Tensor, comp: int, g: np.ndarray, raw_shape) -> torch.Tensor:
    """Transpose of the interpolation: the cotangent of the output mapped onto
    an array of ``raw_shape`` (zero outside the block read)."""
    gout = gout.contiguous()
    ni, nj, nk = int(g[3]), int(g[4]), int(g[5])
    blk = torch.empty((ni, nj, nk), dtype=torch.complex128, device=gout.device)
    msg = ctypes.create_string_buffer(256)
    _check(_ct.libFDTD.FDTD_interp_field_T(gout.device.index, _stream(gout), comp, _ptr(gout),
                                           g.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _ptr(blk),
                                           msg, len(msg)), msg)
    if tuple(raw_shape) == (ni, nj, nk) and not (g[0] or g[1] or g[2]):
        return blk
    full = torch.zeros(tuple(raw_shape), dtype=torch.complex128, device=gout.device)
    full[g[0]:g[0] + ni, g[1]:g[1] + nj, g[2]:g[2] + nk] = blk
    return full


class InterpField(torch.autograd.Function):
    """Interpolation of one component of a raw block; the backward pass is the
    transpose kernel (FDTD_interp_field_T) onto the block."""

    @staticmethod
    def forward(ctx, raw, comp, g, shape):
        raw = raw.contiguous()
        ctx.comp, ctx.g, ctx.raw_shape = comp, g, tuple(raw.shape)
        return _interp_raw(raw, comp, g, shape)

    @staticmethod
    def backward(ctx, gout):
        return _interp_T(gout, ctx.comp, ctx.g, ctx.raw_shape), None, None, None


def interp(raw: torch.Tensor, component: str, domain, domain_interp, bc: str) -> torch.Tensor:
    """``component`` interpolated onto the Ez grid on ``domain``, from the raw
    block ``raw`` of ``domain_interp`` (the grown domain, clipped to the grid;
    for Ez any block containing ``domain``)."""
    g, shape = geometry(component, domain, domain_interp, tuple(raw.shape), bc)
    return InterpField.apply(raw, _CIDX[component], g, shape)


def interp_full(field: torch.Tensor, component: str, domain, d, bc: str, lengths=None) -> torch.Tensor:
    """``FDTD.get_field_interp`` on a whole-grid device array ``field``.
    ``domain`` None: the whole grid, rebuilt from the grid lengths ``lengths``
    = (X, Y, Z) (default (N - 1) d) as the reference does."""
    shape = tuple(field.shape)
    Nz, Ny, Nx = shape
    if domain is None:
        X, Y, Z = lengths if lengths is not None else ((Nx - 1) * d[0], (Ny - 1) * d[1], (Nz - 1) * d[2])
        domain = DomainCoordinates(0, X, 0, Y, 0, Z, *d)
        dint = domain
    else:
        dint = domain if component == "Ez" else grow_domain(domain, shape, d)
    block = (clipped_extent(dint.i1, dint.i2, Nz), clipped_extent(dint.j1, dint.j2, Ny),
             clipped_extent(dint.k1, dint.k2, Nx))
    origin = (min(dint.i1, Nz), min(dint.j1, Ny), min(dint.k1, Nx))
    g, out_shape = geometry(component, domain, dint, block, bc, origin, shape)
    return InterpField.apply(field, _CIDX[component], g, out_shape)


def dfdx_interp(domain, dF: dict, bc: str):
    """``interpolated_dFdx_3D`` on device tensors: ``dF`` maps each component
    to the derivative with respect to the interpolated field on ``domain``
    (tensors of domain.shape; a missing component counts as zero).  Returns
    (the domain grown by one cell towards -x, -y and +z, dict of the six
    adjoint source blocks on it)."""
    nz, ny, nx = domain.shape
    out = {}
    for c in COMPONENTS:
        v = dF.get(c)
        dev = next(t.device for t in dF.values() if t is not None)
        if v is None:
            v = torch.zeros((nz, ny, nx), dtype=torch.complex128, device=dev)
        v = v.to(torch.complex128).contiguous()
        qx = 0
        if c == "Ex" and domain.k1 == 0 and bc[0] in "EH":
            qx = 1 if bc[0] == "H" else 2
        qy = 0
        if c in ("Ey", "Hx", "Hz") and domain.j1 == 0 and bc[1] in "EH":
            qy = 1 if bc[1] == "H" else -1
        o = torch.empty((nz + 1, ny + 1, nx + 1), dtype=torch.complex128, device=v.device)
        msg = ctypes.create_string_buffer(256)
        _check(_ct.libFDTD.FDTD_dfdx_interp(v.device.index, _stream(v), _CIDX[c], _ptr(v), nx, ny, nz,
                                            qx, qy, _ptr(o), msg, len(msg)), msg)
        out[c] = o
    grown = domain.copy()
    grown.grow(1, 0, 1, 0, 0, 1)
    return grown, out


# ------------------------------------------------------------- source power
# (E1, H2, E2, H1) with Re(E1 H2* - E2 H1*) = Re(E x H*) . n through a plane
# normal to x, y, z (the kernel's kFluxComps)
_FLUX = {0: ("Ey", "Hz", "Ez", "Hy"), 1: ("Ez", "Hx", "Ex", "Hz"), 2: ("Ex", "Hy", "Ey", "Hx")}


def _flux_sums(raws, geoms, axes) -> torch.Tensor:
    n = len(raws)
    dev = raws[0].device
    blocks = [r[q].contiguous() for r in raws for q in range(6)]
    ptrs = (ctypes.c_void_p * (6 * n))(*[b.data_ptr() for b in blocks])
    gg = np.concatenate(geoms).astype(np.int32)
    ax = np.array(axes, dtype=np.int32)
    sums = torch.empty(6 + 6 * _NBLK, dtype=torch.float64, device=dev)
    msg = ctypes.create_string_buffer(256)
    _check(_ct.libFDTD.FDTD_plane_flux(dev.index, _stream(raws[0]), n, ptrs,
                                       gg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                       ax.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _ptr(sums),
                                       msg, len(msg)), msg)
    torch.cuda.current_stream(dev).synchronize()   # blocks and arrays outlive the launch
    return sums[:n].clone()


def _plane_geometry(dom, grown, block_shape, bc, axis) -> np.ndarray:
    """Geometry of one flux plane; its four components must give one shape."""
    gs = [geometry(c, dom, grown, block_shape, bc) for c in _FLUX[axis]]
    if len({s for _, s in gs}) != 1:
        raise ValueError("the components of a flux plane interpolate to different shapes")
    return gs[0][0]


class SourcePower(torch.autograd.Function):
    """P = sum over planes of sign 0.5 dA sum Re(E1 H2* - E2 H1*) (one fused
    kernel per call); the backward pass maps dP/d(interpolated fields) to the
    raw blocks with the transpose kernel."""

    @staticmethod
    def forward(ctx, spec, *raws):
        planes, grown, bc, dA = spec
        geoms = [_plane_geometry(dom, g, tuple(raw.shape[1:]), bc, axis)
                 for (dom, axis, sign), g, raw in zip(planes, grown, raws)]
        sums = _flux_sums(list(raws), geoms, [ax for _, ax, _ in planes])
        P = torch.zeros((), dtype=torch.float64, device=raws[0].device)
        for q, (dom, axis, sign) in enumerate(planes):
            P = P + sign * 0.5 * dA[axis] * sums[q]
        ctx.spec = spec
        ctx.save_for_backward(*raws)
        return P

    @staticmethod
    def backward(ctx, gP):
        planes, grown, bc, dA = ctx.spec
        raws = ctx.saved_tensors
        grads = []
        for raw, (dom, axis, sign), g in zip(raws, planes, grown):
            e1, h2, e2, h1 = _FLUX[axis]
            f = {c: interp(raw[_CIDX[c]], c, dom, g, bc) for c in (e1, h2, e2, h1)}
            k = gP * sign * 0.5 * dA[axis]
            # cotangents of Re(E1 conj(H2) - E2 conj(H1)) in autograd's
            # convention (2 dP/d conj(x)); the interpolation has real weights,
            # so its transpose carries them back to the raw block
            cot = {e1: k * f[h2], h2: k * f[e1], e2: -k * f[h1], h1: -k * f[e2]}
            gr = torch.zeros_like(raw)
            for c, v in cot.items():
                gc, _ = geometry(c, dom, g, tuple(raw.shape[1:]), bc)
                gr[_CIDX[c]] = _interp_T(v, _CIDX[c], gc, raw.shape[1:])
            grads.append(gr)
        return (None, *grads)


def source_power(raws, planes, grown, sim) -> torch.Tensor:
    """Differentiable source power from the raw blocks ``raws`` ([6, ...] each)
    of the grown plane domains ``grown`` (planes from
    ``emopt_b200.adjoint.source_power_planes``)."""
    dA = {0: sim.dy * sim.dz, 1: sim.dx * sim.dz, 2: sim.dx * sim.dy}
    return SourcePower.apply((planes, grown, sim.bc, dA), *raws)
