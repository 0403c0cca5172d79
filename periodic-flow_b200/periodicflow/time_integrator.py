"""Time integrators: registry and stage rules of the reference's
time_integrator.py:7-318.

Inside ``Solver.solve`` the stages run fused on the device (one kernel per
stage, or whole steps for the linear problem); each class also exposes the
reference's ``stepping`` on device arrays for direct use.
"""
from __future__ import annotations

import numpy as np

from . import _native as N
from ._dev import Arg, real_dtype, stream_ptr

DICT_TIME_INTEGRATORS = {}


def register_integrator(name):
    """Register an integrator class under ``name`` (time_integrator.py:10-14)."""
    def decorator(cls):
        DICT_TIME_INTEGRATORS[name] = cls
        return cls
    return decorator


class TimeIntegrator:
    """Base class: dt, the shared linear operator and (1 - dt/2 L)^-1
    (time_integrator.py:17-33).  ``native_id`` names the device rule."""

    native_id = None
    n_stages = 0
    noise_factor = ()

    def __init__(self, dt: float, linear_operator: np.ndarray = None, optimization: bool = False):
        self.dt = dt
        self._lin_op = linear_operator
        self._optimization = optimization
        if linear_operator is not None:
            self._lin_op_inv = 1 / (1 - self.dt / 2 * linear_operator)
        self._on_update = None

    def update_linear_operator(self, L):
        self._lin_op[...] = L
        self._lin_op_inv = 1 / (1 - self.dt / 2 * np.asarray(L))
        if self._on_update is not None:
            self._on_update(self._lin_op)

    def stepping(self, unew, u0, stage, rhs_nonlinear, rhs_linear, forcing, noise=None):
        """One stage on device arrays, in place on ``unew`` (and ``rhs_linear``
        for the implicit corrector, time_integrator.py:116-117)."""
        if self.native_id is None:
            raise NotImplementedError(f"{type(self).__name__} has no device stage rule")
        from ._dev import precision_of
        prec = precision_of(unew)
        rd = real_dtype(prec)
        args = [Arg(a, rd, True) for a in (unew, u0, rhs_nonlinear, rhs_linear, forcing)]
        Nz = Arg(noise, rd, True) if noise is not None else None
        Lr = Arg(self._lin_op, rd, False) if self._lin_op is not None else None
        n = int(np.prod(unew.shape))
        npc = int(np.prod(unew.shape[1:]))
        rc = N.lib().pf_op_stepping(prec, self.native_id, int(stage), float(self.dt), n,
                                    args[0].ptr, args[1].ptr, args[2].ptr, args[3].ptr,
                                    args[4].ptr, Nz.ptr if Nz else None,
                                    Lr.ptr if Lr else None, npc, stream_ptr())
        N.check(rc, None, "stepping")
        args[0].write_back()
        args[3].write_back()


@register_integrator("explicit_pc")
class ExplicitPredictorCorrector(TimeIntegrator):
    """2-stage explicit predictor-corrector of Delong et al. (2013)."""
    native_id = N.PF_EXPLICIT_PC
    n_stages = 2
    noise_factor = (0.0, 1.0)


@register_integrator("implicit_pc")
class ImplicitPredictorCorrector(TimeIntegrator):
    """2-stage implicit predictor-corrector of Delong et al. (2013)."""
    native_id = N.PF_IMPLICIT_PC
    n_stages = 2
    noise_factor = (0.0, 1.0)


@register_integrator("rk2")
class RungeKuttaTVD2(TimeIntegrator):
    """TVD RK2 (Gottlieb & Shu).  The reference defines no noise_factor for it,
    so Solver.solve fails there; zeros are supplied here."""
    native_id = N.PF_RK2
    n_stages = 2
    noise_factor = (0.0, 0.0)


@register_integrator("rk3")
class RungeKuttaTVD3(TimeIntegrator):
    """Stochastic TVD RK3 of Delong et al. (2013)."""
    native_id = N.PF_RK3
    n_stages = 3
    noise_factor = ((2 * np.sqrt(2) + np.sqrt(3)) / 5,
                    (-4 * np.sqrt(2) + 3 * np.sqrt(3)) / 5,
                    (np.sqrt(2) - 2 * np.sqrt(3)) / 10)


@register_integrator("rk4")
class RungeKutta4(TimeIntegrator):
    """Low-storage RK4 of Bogey & Bailly (2004); no noise (zeros supplied)."""
    native_id = N.PF_RK4
    n_stages = 4
    noise_factor = (0.0, 0.0, 0.0, 0.0)
