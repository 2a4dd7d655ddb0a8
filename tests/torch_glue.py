"""Torch restatement of the reference's interpolation onto the Ez grid
(emopt/fdtd.py:1401-1553) and source power (emopt/fdtd.py:1555-1667), for
the CPU tests of the adjoint glue and as the autograd reference of the device
kernels (emopt_b200/fieldops.py) in the GPU tests.  Test infrastructure: the
package computes these on the device."""
import torch
import torch.nn.functional as F

from emopt_b200.fieldops import COMPONENTS, grow_domain  # noqa: F401


def interp_field(raw: torch.Tensor, component: str, domain, domain_interp, bc: str) -> torch.Tensor:
    """Torch form of the reference interpolation onto the Ez grid: ``raw`` is the
    component on ``domain_interp``; returns it interpolated on ``domain``."""
    if component == "Ez":
        return raw[domain.i1 - domain_interp.i1:domain.i2 - domain_interp.i1,
                   domain.j1 - domain_interp.j1:domain.j2 - domain_interp.j1,
                   domain.k1 - domain_interp.k1:domain.k2 - domain_interp.k1]
    k1, k2 = domain_interp.k1, domain_interp.k2
    j1, j2 = domain_interp.j1, domain_interp.j2
    i1, i2 = domain_interp.i1, domain_interp.i2
    fraw = F.pad(raw, (1, 1, 1, 1, 1, 1))

    def sym_x(f):
        if k1 == 0 and bc[0] in "EH":
            f = f.clone()
            f[:, :, 0] = (-1 if bc[0] == "E" else 1) * f[:, :, 1]
        return f

    def sym_y(f):
        if j1 == 0 and bc[1] in "EH":
            f = f.clone()
            f[:, 0, :] = (-1 if bc[1] == "E" else 1) * f[:, 1, :]
        return f

    if component == "Ex":
        fr = sym_x(fraw)
        f = fr.clone()
        f[1:-1, :, 1:-1] = f[1:-1, :, 1:-1] + fr[1:-1, :, 0:-2] + fr[2:, :, 1:-1] + fr[2:, :, 0:-2]
        f = f / 4.0
    elif component == "Ey":
        fr = sym_y(fraw)
        f = fr.clone()
        f[1:-1, 1:-1, :] = f[1:-1, 1:-1, :] + fr[1:-1, 0:-2, :] + fr[2:, 1:-1, :] + fr[2:, 0:-2, :]
        f = f / 4.0
    elif component == "Hx":
        fr = sym_y(fraw)
        f = fr.clone()
        f[:, 1:, :] = f[:, 1:, :] + fr[:, 0:-1, :]
        f = f / 2.0
    elif component == "Hy":
        fr = sym_x(fraw)
        f = fr.clone()
        f[:, :, 1:] = f[:, :, 1:] + fr[:, :, 0:-1]
        f = f / 2.0
    elif component == "Hz":
        fr = sym_y(sym_x(fraw))
        f = fr.clone()
        f[0:-1, 1:, 1:] = (f[0:-1, 1:, 1:] + fr[0:-1, 1:, 0:-1] + fr[0:-1, 0:-1, 1:] +
                           fr[0:-1, 0:-1, 0:-1] + fr[1:, 1:, 1:] + fr[1:, 1:, 0:-1] +
                           fr[1:, 0:-1, 1:] + fr[1:, 0:-1, 0:-1])
        f = f / 8.0
    else:
        raise ValueError("unknown component %r" % (component,))
    n0 = f.shape
    return f[1 + domain.i1 - i1:n0[0] - 1 - (i2 - domain.i2),
             1 + domain.j1 - j1:n0[1] - 1 - (j2 - domain.j2),
             1 + domain.k1 - k1:n0[2] - 1 - (k2 - domain.k2)]




def source_power(raws, planes, grown, sim) -> torch.Tensor:
    """Torch form of ``FDTD.get_source_power`` (emopt/fdtd.py:1555-1667):
    0.5 * dA * sum Re(E x H*) . n over the six planes, from the raw blocks
    ``raws`` of the grown plane domains ``grown``."""
    dA = {0: sim.dy * sim.dz, 1: sim.dx * sim.dz, 2: sim.dx * sim.dy}
    P = torch.zeros((), dtype=torch.float64, device=raws[0].device)
    for raw, (dom, axis, sign), g in zip(raws, planes, grown):
        f = {c: interp_field(raw[q], c, dom, g, sim.bc) for q, c in enumerate(COMPONENTS)}
        cj = torch.conj
        if axis == 0:
            s = f["Ey"] * cj(f["Hz"]) - f["Ez"] * cj(f["Hy"])
        elif axis == 1:
            s = -(f["Ex"] * cj(f["Hz"]) - f["Ez"] * cj(f["Hx"]))
        else:
            s = f["Ex"] * cj(f["Hy"]) - f["Ey"] * cj(f["Hx"])
        P = P + sign * 0.5 * dA[axis] * torch.sum(s.real)
    return P
