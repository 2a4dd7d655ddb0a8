"""Device field access (fields_kernels.cu via emopt_b200/fieldops.py) against
the host forms with the reference's semantics:

* interpolation onto the Ez grid == FDTD.get_field_interp (numpy restatement
  of emopt/fdtd.py:1401-1553) on interior boxes, planes on every min and max
  face, the whole grid, and the source-power planes, for every boundary
  letter of x and y ('0', 'E', 'H'): within 1e-13 of the largest value (the
  additions run in the reference's order);
* its transpose is exact: <A x, g> == <x, A^T g> to 1e-12;
* interpolated_dFdx_3D on CUDA tensors == the numpy form
  (emopt/fomutils.py:1282-1426, quirks at symmetric min faces included);
* source power == FDTD.get_source_power to 1e-12, and its gradient == autograd
  through the torch restatement of the same sums, on a grid where all six
  planes hold cells.
The phasors are seeded random complex arrays written into the solver's t0
arrays: the kernels are pure functions of them."""
import itertools

import numpy as np
import pytest
import torch

import torch_glue as G
from emopt_b200 import adjoint as A
from emopt_b200 import fieldops as FO
from emopt_b200 import fomutils
from emopt_b200 import problems as P
from emopt_b200.misc import DomainCoordinates

pytestmark = pytest.mark.gpu

COMPS = FO.COMPONENTS
BCS = ["".join(t) + "0" for t in itertools.product("0EH", repeat=2)]
SHAPE = (9, 11, 14)
# every source-power plane holds cells on this grid (on SHAPE with these
# CPML widths the planes normal to x and y are empty)
POWER_SHAPE, POWER_PML = (14, 13, 16), (3, 4, 3, 2, 2, 3)


def _sim(bc, seed=0, shape=SHAPE, w_pml=(3, 4, 3, 2, 3, 4)):
    p = P.random_box(seed, shape=shape, w_pml=w_pml, bc=bc)
    sim = P.make_solver(p, precision="fp64")
    rng = np.random.default_rng(seed + 17)
    for c in COMPS:
        a = getattr(sim, "_%s_fwd_t0" % c)
        a[:] = rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)
    return sim


def _fields(sim):
    return {c: torch.as_tensor(sim._raw(c, False).copy()).cuda() for c in COMPS}


def _domains(sim):
    dx, dy, dz = sim.dx, sim.dy, sim.dz
    X, Y, Z = sim.X, sim.Y, sim.Z
    D = lambda *a: DomainCoordinates(*a, dx, dy, dz)
    doms = {
        "box": D(3 * dx, 9 * dx, 2 * dy, 7 * dy, 2 * dz, 6 * dz),
        "xmin_plane": D(0, 0, 0, Y, 0, Z),
        "xmax_plane": D(X, X, 0, Y, 0, Z),
        "ymin_box": D(2 * dx, 8 * dx, 0, 4 * dy, 1 * dz, 5 * dz),
        "ymax_plane": D(0, X, Y, Y, 0, Z),
        "zmin_plane": D(0, X, 0, Y, 0, 0),
        "zmax_plane": D(0, X, 0, Y, Z, Z),
        "corner_box": D(0, 3 * dx, 0, 3 * dy, 0, 3 * dz),
        "max_corner_box": D(X - 3 * dx, X, Y - 2 * dy, Y, Z - 2 * dz, Z),
        "whole": None,
    }
    for q, (dom, axis, sign) in enumerate(A.source_power_planes(sim)):
        doms["power_plane_%d" % q] = dom
    return doms


@pytest.mark.parametrize("bc", BCS)
def test_interp_matches_host_form(bc):
    sim = _sim(bc, seed=BCS.index(bc))
    F = _fields(sim)
    d = (sim.dx, sim.dy, sim.dz)
    for name, dom in _domains(sim).items():
        for c in COMPS:
            ref = sim.get_field_interp(c, dom)
            got = FO.interp_full(F[c], c, dom, d, sim.bc, lengths=(sim.X, sim.Y, sim.Z)).cpu().numpy()
            assert got.shape == ref.shape, (name, c, got.shape, ref.shape)
            scale = max(np.abs(ref).max(), 1.0) if ref.size else 1.0
            np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13 * scale, err_msg="%s %s" % (name, c))


@pytest.mark.parametrize("bc", ["000", "EH0", "HE0", "EE0"])
def test_interp_transpose_is_exact(bc):
    sim = _sim(bc, seed=3)
    d = (sim.dx, sim.dy, sim.dz)
    rng = np.random.default_rng(5)
    for name, dom in _domains(sim).items():
        if dom is None:
            continue
        g = FO.grow_domain(dom, SHAPE, d)
        blk = tuple(FO.clipped_extent(a, b, n) for a, b, n in
                    ((g.i1, g.i2, SHAPE[0]), (g.j1, g.j2, SHAPE[1]), (g.k1, g.k2, SHAPE[2])))
        for c in COMPS:
            gi = dom if c == "Ez" else g
            x = torch.as_tensor(rng.standard_normal(blk) + 1j * rng.standard_normal(blk)).cuda()
            x.requires_grad_(True)
            y = FO.interp(x, c, dom, gi, bc)
            cot = torch.as_tensor(rng.standard_normal(tuple(y.shape)) +
                                  1j * rng.standard_normal(tuple(y.shape))).cuda()
            # real-linear map with real weights: sum((A x) * g) == sum(x * A^T g)
            (gx,) = torch.autograd.grad(y, x, cot)
            lhs = complex(torch.sum(y.detach() * cot))
            rhs = complex(torch.sum(x.detach() * gx))
            assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0), (name, c, lhs, rhs)


@pytest.mark.parametrize("bc", BCS)
def test_dfdx_interp_matches_host_form(bc):
    sim = _sim(bc, seed=7)
    rng = np.random.default_rng(11 + BCS.index(bc))
    for name, dom in _domains(sim).items():
        if dom is None:
            continue
        shape = dom.shape
        host = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in COMPS]
        ref = fomutils.interpolated_dFdx_3D(sim, dom, *host)
        got = fomutils.interpolated_dFdx_3D(sim, dom, *[torch.as_tensor(a).cuda() for a in host])
        g_ref, g_got = ref[0], got[0]
        assert (g_ref.i1, g_ref.i2, g_ref.j1, g_ref.j2, g_ref.k1, g_ref.k2) == \
            (g_got.i1, g_got.i2, g_got.j1, g_got.j2, g_got.k1, g_got.k2)
        for c, a, b in zip(COMPS, ref[1:], got[1:]):
            b = b.cpu().numpy()
            assert a.shape == b.shape, (name, c)
            np.testing.assert_allclose(b, a, rtol=0, atol=1e-13 * max(np.abs(a).max(), 1.0),
                                       err_msg="%s %s" % (name, c))


def _power_inputs(sim, F):
    d = (sim.dx, sim.dy, sim.dz)
    planes = A.source_power_planes(sim)
    for dom, _, _ in planes:
        assert dom.i2 > dom.i1 and dom.j2 > dom.j1 and dom.k2 > dom.k1
    assert {axis for _, axis, _ in planes} == {0, 1, 2}
    grown = [FO.grow_domain(dom, POWER_SHAPE, d) for dom, _, _ in planes]
    raws = [torch.stack([F[c][g.i1:g.i2, g.j1:g.j2, g.k1:g.k2] for c in COMPS]).contiguous()
            for g in grown]
    return planes, grown, raws


@pytest.mark.parametrize("bc", BCS)
def test_source_power_matches_host_form(bc):
    sim = _sim(bc, seed=21 + BCS.index(bc), shape=POWER_SHAPE, w_pml=POWER_PML)
    planes, grown, raws = _power_inputs(sim, _fields(sim))
    ref = sim.get_source_power()
    got = float(FO.source_power(raws, planes, grown, sim))
    assert got == pytest.approx(ref, rel=1e-12, abs=1e-14)


@pytest.mark.parametrize("bc", ["000", "EH0", "0E0"])
def test_source_power_gradient_matches_autograd(bc):
    sim = _sim(bc, seed=31, shape=POWER_SHAPE, w_pml=POWER_PML)
    planes, grown, raws = _power_inputs(sim, _fields(sim))
    r1 = [r.clone().requires_grad_(True) for r in raws]
    r2 = [r.clone().requires_grad_(True) for r in raws]
    P1 = FO.source_power(r1, planes, grown, sim)
    P2 = G.source_power(r2, planes, grown, sim)
    assert float(P1) == pytest.approx(float(P2), rel=1e-12)
    g1 = torch.autograd.grad(P1, r1)
    g2 = torch.autograd.grad(P2, r2)
    for a, b in zip(g1, g2):
        scale = float(torch.abs(b).max())
        assert float(torch.abs(a - b).max()) <= 1e-12 * max(scale, 1.0)


@pytest.mark.parametrize("bc", ["000", "HE0"])
def test_solve_forward_source_power_matches_host_form(bc):
    """FDTD.solve_forward fills source_power from the phasors' plane blocks on
    the GPU; it equals FDTD.get_source_power (host numpy) to 1e-12."""
    p = P.random_box(5, shape=POWER_SHAPE, w_pml=POWER_PML, bc=bc, fixed_steps=200, n_sources=2)
    sim = P.make_solver(p, precision="fp64")
    sim.solve_forward()
    ref = sim.get_source_power()
    assert ref != 0.0
    assert sim.source_power == pytest.approx(ref, rel=1e-12, abs=1e-14 * abs(ref))
