"""The benchmark workloads' FP32 and FP64 results against the FP64 oracle.

* forced-turbulence headline at its full size (256^3 FP32, seed-1 field, band
  forcing, RK3 with CFL dt) one step from the same initial field;
* the shell spectrum diagnostic against oracle.spectrum;
* the 2D thermal Stokes workload (256^2, nu 0.1, explicit PC, dt 0.01) with
  the reference's NumPy draws injected into both codes, FP32 and FP64.

Tolerances (relative L2 over all modes): FP32 1e-5, FP64 1e-12.
"""
import os

import numpy as np
import pytest

import oracle as O
import oracle.pf_oracle as P
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "fp64": 1e-12}


def _spectrum_rel(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    sel = ref >= 1e-10 * ref.max()
    return float(np.max(np.abs(got[sel] - ref[sel]) / ref[sel]))


def test_headline_256_fp32_one_step_vs_oracle():
    """256^3 FP32 fused schedule, forcing + CFL + seed-1 field, vs FP64 oracle."""
    from periodicflow import simulation as sim
    n = 256
    workers = P.FFT_WORKERS
    P.FFT_WORKERS = os.cpu_count()
    try:
        g = O.Grid((n, n, n))
        uh0 = O.spectral_random_field(g, 1)
        o = O.OracleSolver((n, n, n), 1e-3, time_integrator="rk3", viscosity=2e-3,
                           forcing=(0.1, 2.5), cfl=0.5)
        o.initialize(uh0, "fourier")
        o.advance(1)
        s = sim.Solver([n] * 3, 1e-3, 1.0, time_integrator="rk3", viscosity=2e-3,
                       dealias="2/3", precision="fp32", forcing=(0.1, 2.5), cfl=0.5)
        ss = s.space_solver
        ss.initialize_velocity(uh0, "fourier")
        ss.step(1)
        assert rel_l2(ss.u_hat, o.u_hat) < TOL["fp32"]
        _, _, dt = ss.time()
        assert abs(dt - o.dt) / o.dt < 1e-5
        nb = int(np.sqrt(3 * (n // 2) ** 2)) + 2
        assert _spectrum_rel(ss.spectrum(nb), O.spectrum(g, o.u_hat, nb)) < 1e-5
    finally:
        P.FFT_WORKERS = workers


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("N", [(64, 64, 64), (32, 48, 16), (128, 128)])
def test_spectrum_vs_oracle(precision, N):
    from periodicflow import simulation as sim
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 1)
    s = sim.Solver(list(N), 0.01, 1.0, time_integrator="rk3", viscosity=2e-3, dealias="2/3",
                   precision=precision)
    s.space_solver.initialize_velocity(uh, "fourier")
    nb = int(np.sqrt(sum((n // 2) ** 2 for n in N))) + 2
    got = s.space_solver.spectrum(nb)
    ref = O.spectrum(g, uh * g.mask_k0, nb)
    tol = 1e-6 if precision == "fp32" else 1e-12
    assert _spectrum_rel(got, ref) < tol
    # the shells sum to the energy
    e, _ = s.space_solver.energy()
    assert abs(got.sum() - e) <= 1e-12 * e + (1e-6 * e if precision == "fp32" else 0)


def _stokes_pair(precision, integrator, steps):
    from periodicflow import simulation as sim
    n, nu, kT, dt = 256, 0.1, 1e-3, 0.01
    mag = float(np.sqrt(2 * nu * kT))
    g = O.Grid((n, n))
    rng = np.random.RandomState(0)
    fields = [O.numpy_noise_fields(g, "thermal", rng) for _ in range(steps)]
    o = O.OracleSolver((n, n), dt, is_nonlinear=False, time_integrator=integrator,
                       viscosity=nu, noise_type="thermal", noise_mag=mag,
                       noise=lambda step: fields[step - 1])
    o.initialize(np.zeros((2,) + g.spec_shape, complex), "fourier")
    o.advance(steps)
    s = sim.Solver([n, n], dt, 1.0, is_nonlinear=False, time_integrator=integrator,
                   viscosity=nu, noise_type="thermal", noise_mag=mag, precision=precision,
                   noise_source="injected")
    ss = s.space_solver
    for w1, w2 in fields:
        ss.inject_noise(w1, w2)
        ss.step(1)
    return ss.u_hat, o.u_hat


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_config2_thermal_stokes_256sq_explicit_pc_vs_oracle(precision):
    """Configuration 2 as specified (explicit PC, dt 0.01): unstable at 256^2,
    so ten steps; the arithmetic must still follow the oracle."""
    got, ref = _stokes_pair(precision, "explicit_pc", 10)
    assert np.all(np.isfinite(got))
    assert rel_l2(got, ref) < TOL[precision]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_config2_thermal_stokes_256sq_implicit_pc_vs_oracle(precision):
    got, ref = _stokes_pair(precision, "implicit_pc", 200)
    assert rel_l2(got, ref) < TOL[precision]
