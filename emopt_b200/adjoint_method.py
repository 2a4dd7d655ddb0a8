"""The reference's adjoint-method base classes (emopt/adjoint_method.py) over
this package's FDTD solver, so that optimisation scripts written as
``AdjointMethod`` subclasses run with one import changed.

* ``AdjointMethod`` (emopt/adjoint_method.py:177-721): ``fom``, ``gradient``
  (forward solve, the subclass's dF/dx as adjoint sources, adjoint solve,
  then ``calc_gradient`` + ``calc_grad_p``), ``calc_gradient`` (one
  perturbation of each design parameter: -2 Re(y^T dA x / step) from
  ``sim.calc_ydAx`` on the updated boxes) and ``check_gradient`` (one-sided
  finite differences of ``fom``, total relative error, warning above 1%).
* ``AdjointMethodPNF3D`` (emopt/adjoint_method.py:1329-1486): figures of
  merit normalised by the source power, F = f / Psrc + penalty, with the
  adjoint sources of ``fomutils.power_norm_dFdx_3D``.
* ``AdjointMethodMO`` (emopt/adjoint_method.py:723-929): several adjoint
  methods combined through ``calc_total_fom`` / ``calc_total_gradient``.

The solves and the overlap products run on the GPU (``FDTD.solve_forward`` /
``solve_adjoint`` through ``FDTD_solve_cw``); one process owns the whole grid,
so the reference's MPI gathers and broadcasts disappear.  The faster route
for many parameters is the autograd form in ``emopt_b200.adjoint``.
"""
from __future__ import annotations

import time
from abc import ABC, abstractmethod

import numpy as np

from . import fomutils
from .misc import warning_message


def info_message(message: str) -> None:
    print("[INFO] " + message, flush=True)


class AdjointMethod(ABC):
    """Adjoint-method driver of a simulation ``sim`` (emopt/adjoint_method.py:
    177-721).  Subclasses define ``update_system``, ``calc_fom``,
    ``calc_dFdx`` and ``calc_grad_p`` (and may override
    ``get_update_boxes``)."""

    def __init__(self, sim, step=1e-8):
        self.sim = sim
        self.prev_params = []
        self._step = step
        self._grad_f_time = 0.0

    @property
    def step(self):
        """Step of the finite difference of A in ``calc_gradient``."""
        return self._step

    @step.setter
    def step(self, val):
        if np.abs(val) > self.sim.dx / 1e3:
            warning_message("Step size used for adjoint method may be too large.  Consider reducing it "
                            "to ~1e-3*dx", "emopt_b200.adjoint_method")
        self._step = val

    @abstractmethod
    def update_system(self, params):
        """Map the design parameters onto the simulation's materials."""

    @abstractmethod
    def calc_fom(self, sim, params):
        """The figure of merit from the current forward fields."""

    @abstractmethod
    def calc_dFdx(self, sim, params):
        """Derivative of the figure of merit with respect to the fields:
        [sources, domains] for ``sim.set_adjoint_sources``."""

    @abstractmethod
    def calc_grad_p(self, sim, params):
        """Explicit derivative of the figure of merit with respect to the
        parameters (0 where it depends on them only through the fields)."""

    def get_update_boxes(self, sim, params):
        """The region each parameter changes: the whole grid by default."""
        if sim.ndims == 2:
            return [(0, sim.X, 0, sim.Y) for _ in range(len(params))]
        return [(0, sim.X, 0, sim.Y, 0, sim.Z) for _ in range(len(params))]

    def fom(self, params):
        self.update_system(params)
        self.prev_params = params
        self.sim.update()
        self.sim.solve_forward()
        return self.calc_fom(self.sim, params)

    def _update(self, boxes):
        if isinstance(boxes[0], (list, tuple, np.ndarray)):
            for box in boxes:
                self.sim.update(box)
        else:
            self.sim.update(boxes)

    def calc_gradient(self, sim, params):
        """d F / d p_i = -2 Re(y^T (A(p + step e_i) - A(p)) x) / step, with
        A's diagonal re-sampled only in parameter i's update boxes."""
        Ai = sim.get_A_diag()
        step = self._step
        boxes = self.get_update_boxes(sim, params)
        gradient = np.zeros(len(params))
        for i in range(len(params)):
            p0 = params[i]
            params[i] += step
            self.update_system(params)
            self._update(boxes[i])
            gradient[i] = -2 * np.real(sim.calc_ydAx(Ai) / step)
            params[i] = p0
            self.update_system(params)
            self._update(boxes[i])
        return gradient

    def gradient(self, params):
        self.update_system(params)
        self.sim.update()
        if not np.array_equal(self.prev_params, params):
            self.sim.solve_forward()
        dFdx = self.calc_dFdx(self.sim, params)
        self.sim.set_adjoint_sources(dFdx)
        self.sim.solve_adjoint()
        start = time.time()
        grad_f = self.calc_gradient(self.sim, params)
        self._grad_f_time = time.time() - start
        grad_p = self.calc_grad_p(self.sim, params)
        return grad_f + grad_p

    def check_gradient(self, params, indices=[], plot=True, verbose=True, return_gradients=False,
                       fd_step=1e-10):
        """Adjoint gradient against one-sided finite differences of ``fom``
        at ``indices`` (all parameters when empty); returns the total
        relative error (and both gradients with ``return_gradients``)."""
        if len(indices) == 0:
            indices = np.arange(0, len(params), 1)
        self.update_system(params)
        self.sim.update()
        grad_am = self.gradient(params)
        grad_fd = np.zeros(len(indices))
        fom0 = self.fom(params)
        if verbose:
            info_message("Checking gradient...")
        for q, j in enumerate(indices):
            if verbose:
                print("\tDerivative %d of %d" % (q + 1, len(indices)))
            p0 = params[j]
            params[j] += fd_step
            fom1 = self.fom(params)
            grad_fd[q] = (fom1 - fom0) / fd_step
            params[j] = p0
        errors = np.abs(grad_fd - grad_am[indices]) / np.abs(grad_fd)
        error_tot = np.linalg.norm(grad_fd - grad_am[indices]) / np.linalg.norm(grad_fd)
        if error_tot < 0.01:
            if verbose:
                info_message("The total error in the gradient is %0.4E" % error_tot)
        else:
            warning_message("The total error in the gradient is %0.4E which is over 1%%" % error_tot,
                            "emopt_b200.adjoint_method")
        if plot:
            try:
                import matplotlib.pyplot as plt
            except ImportError:
                warning_message("matplotlib is not available: no gradient plot", "emopt_b200.adjoint_method")
            else:
                f = plt.figure()
                xs = np.arange(len(indices))
                for n, (vals, title) in enumerate(((grad_fd, "Finite Differences"),
                                                   (grad_am[indices], "Adjoint Method"),
                                                   (errors, "Error in Adjoint Method"))):
                    ax = f.add_subplot(311 + n)
                    ax.bar(xs, vals)
                    ax.set_title(title)
                plt.show()
        if return_gradients:
            return error_tot, grad_fd, grad_am
        return error_tot


class AdjointMethodPNF3D(AdjointMethod):
    """Figure of merit normalised by the source power (emopt/adjoint_method.py:
    1329-1486): F = f / Psrc + penalty.  Subclasses define ``calc_f``,
    ``calc_dfdx`` (one set of six derivative arrays per domain of
    ``get_fom_domains``), ``get_fom_domains`` and optionally
    ``calc_penalty``."""

    @abstractmethod
    def calc_f(self, sim, params):
        """The unnormalised figure of merit f."""

    @abstractmethod
    def calc_dfdx(self, sim, params):
        """[[dfdEx, dfdEy, dfdEz, dfdHx, dfdHy, dfdHz], ...] per fom domain,
        with respect to the interpolated fields."""

    @abstractmethod
    def get_fom_domains(self):
        """The domains the derivatives of ``calc_dfdx`` live on."""

    def calc_penalty(self, sim, params):
        return 0.0

    def calc_fom(self, sim, params):
        return self.calc_f(sim, params) / sim.source_power + self.calc_penalty(sim, params)

    def calc_dFdx(self, sim, params):
        """The adjoint sources of every fom domain, concatenated.  The
        reference passes ``self.fom_domain`` for every domain; a subclass
        that sets it keeps that behaviour, otherwise each domain of
        ``get_fom_domains`` is used."""
        f = self.calc_f(sim, params)
        dfdxs = self.calc_dfdx(sim, params)
        sources = [[], []]
        for i, domain in enumerate(self.get_fom_domains()):
            domain = getattr(self, "fom_domain", domain)
            a_src = fomutils.power_norm_dFdx_3D(sim, f, domain, *dfdxs[i])
            sources = [sources[0] + a_src[0], sources[1] + a_src[1]]
        return sources


class AdjointMethodMO(AdjointMethod):
    """Several adjoint methods combined into one figure of merit
    (emopt/adjoint_method.py:723-929): subclasses define
    ``calc_total_fom(foms)`` and ``calc_total_gradient(foms, grads)``."""

    def __init__(self, ams, step=1e-6):
        self._ams = ams
        self._foms_current = np.zeros(len(ams))
        self._step = step
        self.prev_params = []
        self._grad_f_time = 0.0

    @property
    def adjoint_methods(self):
        return self._ams

    @adjoint_methods.setter
    def adjoint_methods(self, new_ams):
        self._ams = new_ams

    def update_system(self, params):
        for am in self._ams:
            am.update_system(params)

    def calc_fom(self, sim, params):
        return self.calc_total_fom(self._foms_current)

    def calc_dFdx(self, sim, params):
        return None

    def calc_grad_p(self, sim, params):
        return None

    @abstractmethod
    def calc_total_fom(self, foms):
        """The combined figure of merit from the individual ones."""

    @abstractmethod
    def calc_total_gradient(self, foms, grads):
        """The combined gradient from the individual figures and gradients."""

    def fom(self, params):
        foms = [am.fom(params) for am in self._ams]
        self._foms_current = foms
        return self.calc_total_fom(foms)

    def gradient(self, params):
        foms, grads = [], []
        for am in self._ams:
            grads.append(am.gradient(params))
            foms.append(am.calc_fom(am.sim, params))
        return self.calc_total_gradient(foms, grads)

    def check_gradient(self, params, indices=[], plot=True, verbose=True, return_gradients=False,
                       fd_step=1e-10):
        self.sim = self._ams[0].sim
        for am in self._ams:
            am.update_system(params)
            am.sim.update()
        return super().check_gradient(params, indices, plot, verbose, return_gradients, fd_step)
