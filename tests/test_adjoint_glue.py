"""CPU tests of the differentiation form's host side against the oracle's
restatement of the reference glue (interpolation, mode match, its
derivatives, the transpose of the interpolation) and of the design map."""
import numpy as np
import pytest
import torch

from emopt_b200 import adjoint as A
from emopt_b200 import problems as P
from emopt_b200.misc import DomainCoordinates
import torch_glue as G
from oracle import adjoint as R

SHAPE = (9, 12, 14)
D = (0.05, 0.05, 0.05)


def _rand_fields(rng, shape=SHAPE):
    return [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(6)]


BOXES = [(4, 5, 0, 12, 0, 9), (3, 8, 2, 7, 1, 6), (0, 1, 0, 12, 0, 9), (0, 14, 0, 1, 2, 4),
         (13, 14, 3, 9, 0, 9)]


@pytest.mark.parametrize("bc", ["000", "EH0", "HE0"])
@pytest.mark.parametrize("box", BOXES)
def test_interp_matches_reference(box, bc):
    rng = np.random.default_rng(3)
    full = _rand_fields(rng)
    dom = DomainCoordinates.from_indices(*box, *D)
    g = A.grow_domain(dom, SHAPE, D)
    rb = R.Box(*box)
    for c, comp in enumerate(A.COMPONENTS):
        ref = R.interp(full[c], comp, rb, bc, D)
        raw = torch.as_tensor(full[c][g.i1:g.i2, g.j1:g.j2, g.k1:g.k2])
        got = G.interp_field(raw, comp, dom, g, bc).numpy()
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-14)


@pytest.mark.parametrize("box", [(6, 7, 0, 11, 0, 8), (5, 6, 2, 10, 1, 8)])
def test_autograd_transpose_matches_interpolated_dFdx(box):
    """dF/dx from torch autograd (conj(grad)/2) equals the reference's
    hand-written ModeMatch derivatives mapped back by interpolated_dFdx_3D."""
    rng = np.random.default_rng(5)
    full = _rand_fields(rng)
    dom = DomainCoordinates.from_indices(*box, *D)
    g = A.grow_domain(dom, SHAPE, D)
    rb = R.Box(*box)
    # a domain reaching a max face interpolates one row short (reference quirk)
    pshape = R.interp(full[1], "Ey", rb, "000", D).shape
    mode = {"Ey": rng.standard_normal(pshape) + 0.3j * rng.standard_normal(pshape),
            "Hz": rng.standard_normal(pshape) + 0.2j * rng.standard_normal(pshape),
            "Ez": 0.1 * rng.standard_normal(pshape) + 0j}
    # reference path
    f_ref = {c: R.interp(full[A.COMPONENTS.index(c)], c, rb, "000", D) for c in A.COMPONENTS}
    F_ref, dF = R.mode_match(f_ref, mode, (1, 0, 0), D[1], D[2])
    gb, dFdx = R.interpolated_dFdx(rb, dF, "000")
    # torch path
    raw = torch.as_tensor(np.stack([a[g.i1:g.i2, g.j1:g.j2, g.k1:g.k2] for a in full]),
                          dtype=torch.complex128).requires_grad_(True)
    mm = A.ModeMatch((1, 0, 0), D[1], D[2], mode, "cpu")
    f = {c: G.interp_field(raw[A.COMPONENTS.index(c)], c, dom, g, "000").reshape(pshape)
         for c in A.COMPONENTS}
    F = mm(f)
    F.backward()
    assert float(F.detach()) == pytest.approx(F_ref, rel=1e-13)
    hol = (torch.conj(raw.grad) / 2).numpy()
    # embed both in full-grid arrays and compare
    for c, comp in enumerate(A.COMPONENTS):
        a = np.zeros((SHAPE[0] + 2, SHAPE[1] + 2, SHAPE[2] + 2), dtype=np.complex128)
        b = np.zeros_like(a)
        a[g.i1 + 1:g.i2 + 1, g.j1 + 1:g.j2 + 1, g.k1 + 1:g.k2 + 1] = hol[c]
        b[gb.i1 + 1:gb.i2 + 1, gb.j1 + 1:gb.j2 + 1, gb.k1 + 1:gb.k2 + 1] += dFdx[comp]
        # the reference's grown box may reach one cell past the grid: those
        # entries are dropped by the source overlap rule
        inner = (slice(1, -1),) * 3
        np.testing.assert_allclose(a[inner], b[inner], rtol=0,
                                   atol=1e-13 * max(1.0, np.abs(b).max()), err_msg=comp)


def test_blur_and_projection_match_numpy():
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(0)
    rho = rng.uniform(0, 1, (23, 17))
    ref = P.projected_density(rho)
    got = A.tanh_project(A.gaussian_blur(torch.as_tensor(rho), 2.0), 8.0, 0.5).numpy()
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13)
    np.testing.assert_allclose(A.gaussian_blur(torch.as_tensor(rho), 2.0).numpy(),
                               gaussian_filter(rho, 2.0, mode="nearest"), rtol=0, atol=1e-14)


def test_design_map_reproduces_geometry():
    p = P.mmi_gradient(d=0.05, w_pml=10, nd=(30, 20))
    des = A.planar_design(p.shape, p.dx, p.design_rect, p.design_layer, p.design_nd,
                          P.EPS_SIO2, P.EPS_SI, p.mats[:3], "cpu")
    rng = np.random.default_rng(9)
    q = rng.uniform(0, 1, p.design_nd)
    ref = P.design_eps(p, q)
    cols = des.eps_columns(A.tanh_project(A.gaussian_blur(torch.as_tensor(q), 2.0), 8.0, 0.5))
    for c in range(3):
        e = np.real(np.array(p.mats[c]))
        i0, i1 = des.iz[c]
        e[i0:i1, des.j0:des.j1, des.k0:des.k1] = cols[c].numpy()[None]
        np.testing.assert_allclose(e, np.real(ref[c]), rtol=0, atol=1e-12, err_msg=str(c))


def test_reference_calc_gradient_formula():
    """calc_gradient's forward difference on a linear permittivity model is exact."""
    rng = np.random.default_rng(1)
    x = _rand_fields(rng)[:3]
    y = _rand_fields(rng)[:3]
    eps0 = [rng.random(SHAPE) for _ in range(3)]
    dirs = [[rng.random(SHAPE) for _ in range(3)] for _ in range(4)]
    step = 1e-3
    steps = [[e + step * d for e, d in zip(eps0, dd)] for dd in dirs]
    g = R.calc_gradient(x, y, eps0, steps, step)
    exact = [-2 * np.real(sum(np.sum(y[c] * 1j * dd[c] * x[c]) for c in range(3))) for dd in dirs]
    np.testing.assert_allclose(g, exact, rtol=1e-9)


@pytest.mark.parametrize("bc", ["000", "EH0", "0HE"])
def test_source_power_matches_reference_formula(bc):
    """The torch source power over the six planes one cell inside the CPML
    (emopt/fdtd.py:1555-1667; planes on symmetric min faces left out), on
    random fields, against the same sums over the oracle's interpolation."""
    from types import SimpleNamespace
    Nz, Ny, Nx = SHAPE
    dx, dy, dz = D
    rng = np.random.default_rng(11)
    full = _rand_fields(rng)
    sim = SimpleNamespace(dx=dx, dy=dy, dz=dz, _w_pml=(2 * dx, 3 * dx, 2 * dy, 0.0, 2 * dz, 2 * dz),
                          X=(Nx - 1) * dx, Y=(Ny - 1) * dy, Z=(Nz - 1) * dz, bc=bc)
    planes = A.source_power_planes(sim)
    assert len(planes) == 6 - sum(c in "EH" for c in bc)
    grown = [A.grow_domain(dom, SHAPE, D) for dom, _, _ in planes]
    raws = [torch.as_tensor(np.stack([f[g.i1:g.i2, g.j1:g.j2, g.k1:g.k2] for f in full])) for g in grown]
    got = float(G.source_power(raws, planes, grown, sim))
    want = 0.0
    dA = {0: dy * dz, 1: dx * dz, 2: dx * dy}
    for dom, axis, sign in planes:
        rb = R.Box(dom.k1, dom.k2, dom.j1, dom.j2, dom.i1, dom.i2)
        f = {comp: R.interp(full[c], comp, rb, bc, D) for c, comp in enumerate(A.COMPONENTS)}
        if axis == 0:
            s = f["Ey"] * np.conj(f["Hz"]) - f["Ez"] * np.conj(f["Hy"])
        elif axis == 1:
            s = -(f["Ex"] * np.conj(f["Hz"]) - f["Ez"] * np.conj(f["Hx"]))
        else:
            s = f["Ex"] * np.conj(f["Hy"]) - f["Ey"] * np.conj(f["Hx"])
        want += sign * 0.5 * dA[axis] * np.sum(s.real)
    assert got == pytest.approx(want, rel=1e-12)


@pytest.mark.parametrize("update_mu", [False, True])
def test_calc_ydAx_autograd_pseudo_loss(update_mu):
    """FDTD.calc_ydAx_autograd (emopt/experimental/fdtd.py:160-223): its value
    is 2 sum Im(eps E E_adj) (- 2 sum Im(mu H H_adj)), and autograd gives the
    adjoint overlap 2 Im(E E_adj) as the gradient of a real permittivity."""
    from types import SimpleNamespace

    from emopt_b200.fdtd import FDTD
    rng = np.random.default_rng(5)
    fwd = dict(zip(A.COMPONENTS, _rand_fields(rng)))
    adj = dict(zip(A.COMPONENTS, _rand_fields(rng)))
    dom = DomainCoordinates.from_indices(2, 9, 1, 7, 3, 6, *D)
    take = lambda a: a[dom.i1:dom.i2, dom.j1:dom.j2, dom.k1:dom.k2]
    fake = SimpleNamespace(get_field=lambda c, d: take(fwd[c]), get_adjoint_field=lambda c, d: take(adj[c]))
    shape = take(fwd["Ex"]).shape
    eps = [torch.as_tensor(rng.uniform(1, 12, shape)).requires_grad_(True) for _ in range(3)]
    mu = [torch.as_tensor(rng.uniform(1, 2, shape)).requires_grad_(True) for _ in range(3)]
    loss = FDTD.calc_ydAx_autograd(fake, dom, update_mu, eps, mu)
    want = sum(2 * np.sum(np.imag(e.detach().numpy() * take(fwd[c]) * take(adj[c])))
               for c, e in zip(("Ex", "Ey", "Ez"), eps))
    if update_mu:
        want -= sum(2 * np.sum(np.imag(m.detach().numpy() * take(fwd[c]) * take(adj[c])))
                    for c, m in zip(("Hx", "Hy", "Hz"), mu))
    assert float(loss.detach()) == pytest.approx(want, rel=1e-12)
    loss.backward()
    for c, e in zip(("Ex", "Ey", "Ez"), eps):
        np.testing.assert_allclose(e.grad.numpy(), 2 * np.imag(take(fwd[c]) * take(adj[c])), rtol=1e-12)
    if update_mu:
        np.testing.assert_allclose(mu[0].grad.numpy(), -2 * np.imag(take(fwd["Hx"]) * take(adj["Hx"])),
                                   rtol=1e-12)


@pytest.mark.parametrize("normal", [(1, 0, 0), (0, -1, 0), (0, 0, 1)])
def test_fomutils_mode_match_matches_restatement(normal):
    """emopt_b200.fomutils.ModeMatch (the reference's numpy interface) against
    the oracle's restatement: forward match and every derivative; the
    backward match is the forward match of the mode with H reversed."""
    from emopt_b200.fomutils import ModeMatch
    rng = np.random.default_rng(sum(normal) + 7)
    shape = (1, 6, 9)
    r = lambda: rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    mode = {c: r() for c in A.COMPONENTS}
    fields = {c: r() for c in A.COMPONENTS}
    mm = ModeMatch(normal, 0.05, 0.04, **{c + "m": mode[c] for c in A.COMPONENTS})
    mm.compute(**fields)
    F, dF = R.mode_match(fields, mode, normal, 0.05, 0.04)
    assert mm.get_mode_match_forward(1.0) == pytest.approx(F, rel=1e-12)
    for c in A.COMPONENTS:
        np.testing.assert_allclose(getattr(mm, "get_dFd" + c)(), dF[c], rtol=1e-12, atol=1e-15)
    back = {c: (-fields[c] if c[0] == "H" else fields[c]) for c in A.COMPONENTS}
    mm2 = ModeMatch(normal, 0.05, 0.04, **{c + "m": mode[c] for c in A.COMPONENTS})
    mm2.compute(**back)
    assert mm2.get_mode_match_back(2.0) == pytest.approx(mm.get_mode_match_forward(2.0), rel=1e-12)


@pytest.mark.parametrize("bc", ["000", "HH0", "EE0", "HE0"])
@pytest.mark.parametrize("box", [(0, 5, 0, 6, 2, 4), (3, 8, 2, 7, 1, 6), (4, 5, 0, 12, 0, 9)])
def test_fomutils_interpolated_dFdx_matches_restatement(box, bc):
    from types import SimpleNamespace

    from emopt_b200.fomutils import interpolated_dFdx_3D
    rng = np.random.default_rng(13)
    dom = DomainCoordinates.from_indices(*box, *D)
    dF = [rng.standard_normal(dom.shape) + 1j * rng.standard_normal(dom.shape) for _ in range(6)]
    g, *got = interpolated_dFdx_3D(SimpleNamespace(bc=bc), dom, *dF)
    rg, want = R.interpolated_dFdx(R.Box(*box), dict(zip(A.COMPONENTS, dF)), bc)
    assert (g.k1, g.k2, g.j1, g.j2, g.i1, g.i2) == (rg.k1, rg.k2, rg.j1, rg.j2, rg.i1, rg.i2)
    assert (dom.k1, dom.j1, dom.i2) == (box[0], box[2], box[5])          # the input is not changed
    for a, c in zip(got, A.COMPONENTS):
        assert a.shape == g.shape
        np.testing.assert_allclose(a, want[c], rtol=0, atol=1e-15)


def test_domain_grow_and_copy():
    d = DomainCoordinates.from_indices(2, 5, 3, 7, 1, 4, 0.1, 0.2, 0.3)
    e = d.copy()
    e.grow(1, 2, 0, 1, 1, 0)
    assert (d.k1, d.k2, d.j1, d.j2, d.i1, d.i2) == (2, 5, 3, 7, 1, 4)
    assert (e.k1, e.k2, e.j1, e.j2, e.i1, e.i2) == (1, 7, 3, 8, 0, 4)
    assert e.shape == (4, 5, 6) and np.allclose(e.x, 0.1 * np.arange(1, 7))


def _fake_sim(full, bc, w=2):
    """A stand-in for FDTD: fields interpolated by the oracle, the source
    power summed over the planes of the reference's get_source_power."""
    from types import SimpleNamespace
    Nz, Ny, Nx = SHAPE
    dx, dy, dz = D
    sim = SimpleNamespace(dx=dx, dy=dy, dz=dz, X=(Nx - 1) * dx, Y=(Ny - 1) * dy, Z=(Nz - 1) * dz, bc=bc,
                          w_pml=[w * dx, w * dx, w * dy, w * dy, w * dz, w * dz])
    sim._w_pml = sim.w_pml
    sim.get_field_interp = lambda c, domain=None, squeeze=False: R.interp(
        full[A.COMPONENTS.index(c)], c, R.Box(domain.k1, domain.k2, domain.j1, domain.j2, domain.i1, domain.i2),
        bc, D)
    P = 0.0
    dA = {0: dy * dz, 1: dx * dz, 2: dx * dy}
    for dom, axis, sign in A.source_power_planes(sim):
        f = {c: sim.get_field_interp(c, dom) for c in A.COMPONENTS}
        cj = np.conj
        s = {0: f["Ey"] * cj(f["Hz"]) - f["Ez"] * cj(f["Hy"]),
             1: -(f["Ex"] * cj(f["Hz"]) - f["Ez"] * cj(f["Hx"])),
             2: f["Ex"] * cj(f["Hy"]) - f["Ey"] * cj(f["Hx"])}[axis]
        P += sign * 0.5 * dA[axis] * np.sum(s.real)
    sim.source_power = P
    return sim


@pytest.mark.parametrize("bc", ["000", "0H0", "0E0", "H0E"])
def test_power_norm_dFdx_3D_matches_finite_differences(bc):
    """power_norm_dFdx_3D + interpolated_dFdx_3D (the reference's adjoint
    sources of F = f / Psrc, f a mode match) against central differences of F
    in the raw staggered fields: for a real F, dF/d(Re z) = 2 Re(dF/dz) and
    dF/d(Im z) = -2 Im(dF/dz)."""
    from emopt_b200.fomutils import ModeMatch, power_norm_dFdx_3D
    rng = np.random.default_rng(21)
    full = _rand_fields(rng)
    mon = DomainCoordinates.from_indices(9, 10, 3, 9, 3, 7, *D)
    mode = {c + "m": rng.standard_normal(mon.shape) + 1j * rng.standard_normal(mon.shape) for c in A.COMPONENTS}

    def F_of(fields):
        sim = _fake_sim(fields, bc)
        mm = ModeMatch((1, 0, 0), D[1], D[2], **mode)
        mm.compute(**{c: sim.get_field_interp(c, mon) for c in A.COMPONENTS})
        return mm, sim, mm.mode_match_fwd.real / sim.source_power

    mm, sim, F0 = F_of(full)
    f = mm.mode_match_fwd.real
    srcs, doms = power_norm_dFdx_3D(sim, f, mon, mm.get_dFdEx(), mm.get_dFdEy(), mm.get_dFdEz(),
                                    mm.get_dFdHx(), mm.get_dFdHy(), mm.get_dFdHz())
    assert len(srcs) == 1 + 6 - sum(c in "EH" for c in bc)
    D_full = [np.zeros(SHAPE, dtype=np.complex128) for _ in range(6)]
    for arrays, g in zip(srcs, doms):
        for c in range(6):
            sl = (slice(g.i1, g.i2), slice(g.j1, g.j2), slice(g.k1, g.k2))
            blk = np.asarray(arrays[c])
            assert blk.shape == g.shape
            # blocks may reach one cell past the grid (grown domain): clip
            i2, j2, k2 = min(g.i2, SHAPE[0]), min(g.j2, SHAPE[1]), min(g.k2, SHAPE[2])
            D_full[c][g.i1:i2, g.j1:j2, g.k1:k2] += blk[:i2 - g.i1, :j2 - g.j1, :k2 - g.k1]
    picks = []
    for c in range(6):
        nz = np.argwhere(np.abs(D_full[c]) > 0)
        for q in rng.choice(len(nz), size=min(6, len(nz)), replace=False):
            picks.append((c, tuple(nz[q])))
        # and anywhere (mostly where the sources are zero: F must not move)
        for _ in range(3):
            picks.append((c, tuple(int(rng.integers(0, n)) for n in SHAPE)))
    h = 1e-6
    for c, pos in picks:
        for direction in (1.0, 1j):
            up = [a.copy() for a in full]
            dn = [a.copy() for a in full]
            up[c][pos] += h * direction
            dn[c][pos] -= h * direction
            fd = (F_of(up)[2] - F_of(dn)[2]) / (2 * h)
            want = 2 * np.real(D_full[c][pos] * direction)
            assert fd == pytest.approx(want, rel=1e-5, abs=1e-9 * abs(F0)), (c, pos, direction)


def test_adjoint_method_calc_gradient_is_the_reference_formula():
    """AdjointMethod.calc_gradient over FDTD.calc_ydAx: one perturbation per
    parameter, -2 Re(y^T dA x / step), parameters and materials restored."""
    import types

    from emopt_b200.adjoint_method import AdjointMethod
    from emopt_b200.fdtd import FDTD
    rng = np.random.default_rng(4)
    n = int(np.prod(SHAPE))
    sim = types.SimpleNamespace(ndims=3, X=1.0, Y=1.0, Z=1.0, dx=0.05, updates=[])
    for c in A.COMPONENTS:
        for kind in ("fwd", "adj"):
            setattr(sim, "_%s_%s_t0" % (c, kind), rng.standard_normal(n) + 1j * rng.standard_normal(n))
    base = [rng.uniform(2, 12, n) + 0j for _ in range(3)]
    masks = [rng.uniform(0, 1, (3, n)) for _ in range(4)]
    sim._mu_x = sim._mu_y = sim._mu_z = np.ones(n, dtype=np.complex128)
    sim.update = lambda box=None: sim.updates.append(box)
    sim.calc_ydAx = types.MethodType(FDTD.calc_ydAx, sim)
    sim.get_A_diag = types.MethodType(FDTD.get_A_diag, sim)

    class AM(AdjointMethod):
        def update_system(self, params):
            for a, name in enumerate(("_eps_x", "_eps_y", "_eps_z")):
                setattr(sim, name, base[a] + sum(p * m[a] for p, m in zip(params, masks)))

        def calc_fom(self, sim, params):
            return 0.0

        def calc_dFdx(self, sim, params):
            return [[], []]

        def calc_grad_p(self, sim, params):
            return 0.0

    params = np.array([0.3, -0.2, 0.5, 0.1])
    am = AM(sim, step=1e-6)
    am.update_system(params)
    eps0 = [sim._eps_x.copy(), sim._eps_y.copy(), sim._eps_z.copy()]
    g = am.calc_gradient(sim, params)
    assert np.array_equal(params, [0.3, -0.2, 0.5, 0.1])
    assert all(np.array_equal(e, getattr(sim, nm)) for e, nm in zip(eps0, ("_eps_x", "_eps_y", "_eps_z")))
    assert len(sim.updates) == 2 * len(params) and sim.updates[0] == (0, 1.0, 0, 1.0, 0, 1.0)
    x = [getattr(sim, "_%s_fwd_t0" % c) for c in ("Ex", "Ey", "Ez")]
    y = [getattr(sim, "_%s_adj_t0" % c) for c in ("Ex", "Ey", "Ez")]
    steps = []
    for i in range(len(params)):
        p = params.copy()
        p[i] += 1e-6
        steps.append([base[a] + sum(q * m[a] for q, m in zip(p, masks)) for a in range(3)])
    want = R.calc_gradient(x, y, eps0, steps, 1e-6)
    np.testing.assert_allclose(g, want, rtol=1e-6)
    # linear in the parameters: the derivative is -2 Re(i y . mask . x)
    exact = [-2 * np.real(1j * sum(np.sum(y[a] * m[a] * x[a]) for a in range(3))) for m in masks]
    np.testing.assert_allclose(g, exact, rtol=1e-6)


def test_adjoint_method_gradient_and_check_gradient_flow():
    """gradient(): forward solve, adjoint sources, adjoint solve, then
    calc_gradient + calc_grad_p; check_gradient compares with finite
    differences of fom and reports the total relative error."""
    from types import SimpleNamespace

    from emopt_b200.adjoint_method import AdjointMethod
    calls = []
    sim = SimpleNamespace(ndims=3, X=1.0, Y=1.0, Z=1.0, dx=0.05)
    sim.update = lambda box=None: calls.append("update")
    sim.solve_forward = lambda: calls.append("forward")
    sim.solve_adjoint = lambda: calls.append("adjoint")
    sim.set_adjoint_sources = lambda src: calls.append(("sources", src))
    state = {}

    class AM(AdjointMethod):
        def update_system(self, params):
            state["p"] = np.array(params, dtype=float)

        def calc_fom(self, sim, params):
            return float(np.sum(np.sin(state["p"])) + 0.5 * state["p"][0] ** 2)

        def calc_dFdx(self, sim, params):
            return [["dF"], ["dom"]]

        def calc_gradient(self, sim, params):
            return np.cos(np.asarray(params, dtype=float))

        def calc_grad_p(self, sim, params):
            g = np.zeros(len(params))
            g[0] = params[0]
            return g

    am = AM(sim)
    p = np.array([0.2, 1.1, -0.7])
    g = am.gradient(p)
    np.testing.assert_allclose(g, np.cos(p) + np.array([0.2, 0, 0]))
    assert calls[:4] == ["update", "forward", ("sources", [["dF"], ["dom"]]), "adjoint"]
    err = am.check_gradient(p.copy(), plot=False, verbose=False, fd_step=1e-7)
    assert err < 1e-5

    class Wrong(AM):
        def calc_grad_p(self, sim, params):
            return np.zeros(len(params))

    with pytest.warns(UserWarning, match="over 1%"):
        err2, gfd, gam = Wrong(sim).check_gradient(p.copy(), indices=[0, 2], plot=False, verbose=False,
                                                  return_gradients=True, fd_step=1e-7)
    assert err2 > 0.01 and len(gfd) == 2


def test_adjoint_method_pnf3d_fom_and_sources():
    """AdjointMethodPNF3D: F = f / Psrc + penalty and the adjoint sources of
    power_norm_dFdx_3D for each fom domain."""
    from emopt_b200.adjoint_method import AdjointMethodPNF3D
    from emopt_b200.fomutils import ModeMatch, power_norm_dFdx_3D
    rng = np.random.default_rng(8)
    full = _rand_fields(rng)
    sim = _fake_sim(full, "000")
    mon = DomainCoordinates.from_indices(9, 10, 3, 9, 3, 7, *D)
    mode = {c + "m": rng.standard_normal(mon.shape) + 1j * rng.standard_normal(mon.shape) for c in A.COMPONENTS}

    class AM(AdjointMethodPNF3D):
        def update_system(self, params):
            pass

        def _mm(self, sim):
            mm = ModeMatch((1, 0, 0), D[1], D[2], **mode)
            mm.compute(**{c: sim.get_field_interp(c, mon) for c in A.COMPONENTS})
            return mm

        def calc_f(self, sim, params):
            return self._mm(sim).mode_match_fwd.real

        def calc_dfdx(self, sim, params):
            mm = self._mm(sim)
            return [[mm.get_dFdEx(), mm.get_dFdEy(), mm.get_dFdEz(), mm.get_dFdHx(), mm.get_dFdHy(),
                     mm.get_dFdHz()]]

        def get_fom_domains(self):
            return [mon]

        def calc_penalty(self, sim, params):
            return 0.25

        def calc_grad_p(self, sim, params):
            return 0.0

    am = AM(sim)
    f = am.calc_f(sim, [])
    assert am.calc_fom(sim, []) == pytest.approx(f / sim.source_power + 0.25)
    srcs, doms = am.calc_dFdx(sim, [])
    want_s, want_d = power_norm_dFdx_3D(sim, f, mon, *am.calc_dfdx(sim, [])[0])
    assert len(srcs) == len(want_s) == 7
    for a, b in zip(srcs, want_s):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_adjoint_method_mo_combines_objectives():
    """AdjointMethodMO: the combined figure of merit and gradient of several
    adjoint methods, checked against finite differences."""
    from types import SimpleNamespace

    from emopt_b200.adjoint_method import AdjointMethod, AdjointMethodMO

    def make(scale):
        sim = SimpleNamespace(ndims=3, X=1.0, Y=1.0, Z=1.0, dx=0.05)
        sim.update = lambda box=None: None
        sim.solve_forward = sim.solve_adjoint = lambda: None
        sim.set_adjoint_sources = lambda src: None
        st = {}

        class AM(AdjointMethod):
            def update_system(self, params):
                st["p"] = np.array(params, dtype=float)

            def calc_fom(self, sim, params):
                return float(scale * np.sum(st["p"] ** 2))

            def calc_dFdx(self, sim, params):
                return [[], []]

            def calc_gradient(self, sim, params):
                return 2 * scale * np.asarray(params, dtype=float)

            def calc_grad_p(self, sim, params):
                return 0.0
        return AM(sim)

    class MO(AdjointMethodMO):
        def calc_total_fom(self, foms):
            return foms[0] * foms[1]

        def calc_total_gradient(self, foms, grads):
            return foms[1] * grads[0] + foms[0] * grads[1]

    mo = MO([make(1.0), make(3.0)])
    p = np.array([0.4, -0.3])
    assert mo.fom(p) == pytest.approx(np.sum(p ** 2) * 3 * np.sum(p ** 2))
    np.testing.assert_allclose(mo.gradient(p), 2 * 6 * np.sum(p ** 2) * p)
    assert mo.check_gradient(p.copy(), plot=False, verbose=False, fd_step=1e-7) < 1e-5


@pytest.mark.parametrize("bc", ["000", "EH0", "HE0"])
@pytest.mark.parametrize("box", BOXES)
def test_fdtd_get_field_interp_matches_reference(box, bc):
    """FDTD.get_field_interp (host numpy, emopt/fdtd.py:1401-1553) on a
    stand-in holding random fields, against the oracle's restatement."""
    from types import SimpleNamespace

    from emopt_b200.fdtd import FDTD
    rng = np.random.default_rng(17)
    full = dict(zip(A.COMPONENTS, _rand_fields(rng)))
    Nz, Ny, Nx = SHAPE
    dx, dy, dz = D
    sim = SimpleNamespace(_X=(Nx - 1) * dx, _Y=(Ny - 1) * dy, _Z=(Nz - 1) * dz, _dx=dx, _dy=dy, _dz=dz,
                          _Nx=Nx, _Ny=Ny, _Nz=Nz, _bc=bc)
    sim.get_field = lambda c, d: np.array(full[c][d.i1:d.i2, d.j1:d.j2, d.k1:d.k2])
    dom = DomainCoordinates.from_indices(*box, *D)
    for c in A.COMPONENTS:
        got = FDTD.get_field_interp(sim, c, dom)
        want = R.interp(full[c], c, R.Box(*box), bc, D)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-14)


@pytest.mark.parametrize("bc", ["000", "0H0", "E0H"])
def test_fdtd_get_source_power_matches_torch_form(bc):
    """FDTD.get_source_power (host numpy, emopt/fdtd.py:1555-1667) on a
    stand-in equals the torch source power of the differentiation form."""
    import types
    from types import SimpleNamespace

    from emopt_b200.fdtd import FDTD
    rng = np.random.default_rng(19)
    full = dict(zip(A.COMPONENTS, _rand_fields(rng)))
    Nz, Ny, Nx = SHAPE
    dx, dy, dz = D
    w = (2 * dx, 3 * dx, 2 * dy, 0.0, 2 * dz, 2 * dz)
    sim = SimpleNamespace(_X=(Nx - 1) * dx, _Y=(Ny - 1) * dy, _Z=(Nz - 1) * dz, _dx=dx, _dy=dy, _dz=dz,
                          _Nx=Nx, _Ny=Ny, _Nz=Nz, _bc=bc, _w_pml=w)
    sim.get_field = lambda c, d: np.array(full[c][d.i1:d.i2, d.j1:d.j2, d.k1:d.k2])
    sim.get_field_interp = types.MethodType(FDTD.get_field_interp, sim)
    P_host = FDTD.get_source_power(sim)
    fake = SimpleNamespace(dx=dx, dy=dy, dz=dz, _w_pml=w, X=sim._X, Y=sim._Y, Z=sim._Z, bc=bc)
    planes = A.source_power_planes(fake)
    grown = [A.grow_domain(dom, SHAPE, D) for dom, _, _ in planes]
    raws = [torch.as_tensor(np.stack([full[c][g.i1:g.i2, g.j1:g.j2, g.k1:g.k2] for c in A.COMPONENTS]))
            for g in grown]
    assert P_host == pytest.approx(float(G.source_power(raws, planes, grown, fake)), rel=1e-12)


def test_source_domain_overlap_is_the_reference_rule():
    """FDTD._domain_overlap: the reference's local-domain overlap
    (emopt/fdtd.py:658-708) with the whole grid local, for domains inside,
    across and outside the grid."""
    from types import SimpleNamespace

    from emopt_b200.fdtd import FDTD
    Nz, Ny, Nx = SHAPE
    sim = SimpleNamespace(_Nz=Nz, _Ny=Ny, _Nx=Nx)

    def reference(d):
        i0 = j0 = k0 = 0
        I, J, K = Nz, Ny, Nx
        if i0 >= d.i2 or i0 + I <= d.i1 or j0 >= d.j2 or j0 + J <= d.j1 or k0 >= d.k2 or k0 + K <= d.k1:
            return None, None, None, None
        imax, jmax, kmax = min(i0 + I, d.i2), min(j0 + J, d.j2), min(k0 + K, d.k2)
        imin, jmin, kmin = max(i0, d.i1), max(j0, d.j1), max(k0, d.k1)
        return ((imin, jmin, kmin), (imin - i0, jmin - j0, kmin - k0), (imin - d.i1, jmin - d.j1, kmin - d.k1),
                (imax - imin, jmax - jmin, kmax - kmin))

    rng = np.random.default_rng(23)
    for _ in range(300):
        k1, j1, i1 = (int(rng.integers(-4, n + 2)) for n in (Nx, Ny, Nz))
        k2, j2, i2 = (a + int(rng.integers(1, 8)) for a in (k1, j1, i1))
        d = DomainCoordinates.from_indices(k1, k2, j1, j2, i1, i2, *D)
        assert FDTD._domain_overlap(sim, d) == reference(d)


def test_fdtd_build_and_box_update_sample_the_yee_positions():
    """FDTD.build samples eps at (k+1/2, j, i-1/2), (k, j+1/2, i-1/2), (k, j, i)
    and mu at (k, j+1/2, i), (k+1/2, j, i), (k+1/2, j+1/2, i-1/2)
    (emopt/fdtd.py:842-880); update(bbox) re-samples the box's cells only
    (emopt/fdtd.py:882-992)."""
    import types
    from types import SimpleNamespace

    from emopt_b200.fdtd import FDTD
    from emopt_b200.grid import FunctionMaterial3D
    Nz, Ny, Nx = SHAPE
    dx, dy, dz = D
    state = {"bump": 0.0}
    fe = lambda x, y, z: (2.0 + np.sin(3 * x) * np.cos(2 * y) + z ** 2 + state["bump"]) + 0.1j * x
    fm = lambda x, y, z: 1.0 + 0.5 * x * y + 0.25 * z + state["bump"]
    sim = SimpleNamespace(_Nx=Nx, _Ny=Ny, _Nz=Nz, _dx=dx, _dy=dy, _dz=dz,
                          _eps=FunctionMaterial3D(fe, dx, dy, dz), _mu=FunctionMaterial3D(fm, dx, dy, dz))
    for name in ("_eps_x", "_eps_y", "_eps_z", "_mu_x", "_mu_y", "_mu_z"):
        setattr(sim, name, np.zeros(Nx * Ny * Nz, dtype=np.complex128))
    sim.build = types.MethodType(FDTD.build, sim)
    FDTD.build(sim)
    i, j, k = np.meshgrid(np.arange(Nz), np.arange(Ny), np.arange(Nx), indexing="ij")
    at = lambda f, sx, sy, sz: f((k + sx) * dx, (j + sy) * dy, (i + sz) * dz)
    offsets = {"_eps_x": (fe, 0.5, 0.0, -0.5), "_eps_y": (fe, 0.0, 0.5, -0.5), "_eps_z": (fe, 0.0, 0.0, 0.0),
               "_mu_x": (fm, 0.0, 0.5, 0.0), "_mu_y": (fm, 0.5, 0.0, 0.0), "_mu_z": (fm, 0.5, 0.5, -0.5)}
    for name, (f, sx, sy, sz) in offsets.items():
        np.testing.assert_allclose(getattr(sim, name).reshape(SHAPE), at(f, sx, sy, sz), rtol=1e-14)
    before = {n: getattr(sim, n).reshape(SHAPE).copy() for n in offsets}
    state["bump"] = 1.0
    bbox = (3 * dx, 6 * dx, 2 * dy, 4 * dy, 1 * dz, 5 * dz)          # cells k 3-6, j 2-4, i 1-5
    FDTD.update(sim, bbox)
    inside = (slice(1, 6), slice(2, 5), slice(3, 7))
    for name, (f, sx, sy, sz) in offsets.items():
        now = getattr(sim, name).reshape(SHAPE)
        np.testing.assert_allclose(now[inside], at(f, sx, sy, sz)[inside], rtol=1e-14)
        mask = np.ones(SHAPE, bool)
        mask[inside] = False
        assert np.array_equal(now[mask], before[name][mask])
    assert sim._materials_dirty
