"""Equipartition of the fluctuating Stokes runs with device (Philox) noise.

For thermal noise xi = mag P[i k . (W + W^T)/sqrt 2] with the reference's
normal factor 1/sqrt(prod N)/sqrt(2 - 2/d) (space_solver.py:143-145, 240-259),
E|xi_k|^2 = mag^2 d |k|^2 / prod N.  The implicit predictor-corrector
(time_integrator.py:93-119) advances a linear mode as
u1 = (1 + dt L/2)/(1 - dt L/2) u0 + sqrt(dt/2)/(1 - dt L/2) (xi(w1) + xi(w2)),
whose stationary variance is exactly E|xi|^2 / (2 nu |k|^2) for every dt:
with mag^2 = 2 nu kT, prod N E sum_a |u_k,a|^2 = d kT per mode, i.e. kT per
real transverse degree of freedom in 2D.  Snapshots every 200 steps are nearly
independent for |k| >= 3; the normalised per-mode energy X has mean 1 and
variance 1/(d-1), so the mean over M modes and S snapshots must lie within
3 sigma = 3 / sqrt((d-1) M S) of 1.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,precision", [((128, 128), "fp32"), ((32, 32, 32), "fp32"),
                                         ((64, 64), "fp64")])
def test_equipartition_implicit_pc(N, precision):
    from periodicflow import simulation as sim
    nu, kT, dt = 0.1, 1e-3, 0.01
    d = len(N)
    s = sim.Solver(list(N), dt, 1.0, is_nonlinear=False, time_integrator="implicit_pc",
                   viscosity=nu, noise_type="thermal", noise_mag=math.sqrt(2 * nu * kT),
                   dealias="2/3", precision=precision, seed=7)
    ss = s.space_solver
    kmag = np.sqrt(ss.k2) * 1.0
    sel = kmag >= 3.0
    M = int(sel.sum())
    ss.step(1000)  # burn-in: 10 time units >= 1/(nu k^2) for |k| >= 1
    S = 40
    acc = np.zeros(M)
    prodN = float(np.prod(N))
    for _ in range(S):
        ss.step(200)
        uh = ss.u_hat
        e = prodN * np.sum(np.abs(uh) ** 2, axis=0) / (d * kT)
        acc += e[sel]
    mean = acc.sum() / (M * S)
    sigma = 1.0 / math.sqrt((d - 1) * M * S)
    assert abs(mean - 1.0) < 3 * sigma, (mean, sigma)
    # energy per real transverse degree of freedom, in units of kT
    per_dof = mean * d / (2 * (d - 1))
    if d == 2:
        assert abs(per_dof - 1.0) < 3 * sigma
