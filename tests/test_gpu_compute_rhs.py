"""SpaceSolver.compute_rhs(a) and its arrays (space_solver.py:152-178,
273-310) against the oracle, and forward() of the physical array.

Every part is compared per array in relative L2 (FP64 1e-12, FP32 1e-5):
rhs_linear, rhs_nonlinear (projected, Nyquist mask), noise (Philox draws
of the next step or injected NumPy-order fields, thermal and correlated,
stage noise factors), forcing and p_hat.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "fp64": 1e-12}
NAMES = ("rhs_linear", "rhs_nonlinear", "noise", "forcing", "p_hat")

CASES = [
    # name, N, solver keywords (shared), oracle-only keywords
    ("3d_rk3_forcing", (32, 32, 32),
     dict(time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5)), {}),
    ("3d_thermal_philox", (16, 32, 16),
     dict(time_integrator="implicit_pc", viscosity=0.05, noise_type="thermal", noise_mag=0.02),
     dict(noise="philox", seed=7)),
    ("3d_correlated_padded", (16, 16, 32),
     dict(time_integrator="explicit_pc", viscosity=0.01, noise_type="correlated",
          noise_mag=0.1, dealias="3/2"), dict(noise="philox", seed=7)),
    ("2d_thermal_nyquist", (64, 32),
     dict(time_integrator="rk3", viscosity=1e-3, noise_type="thermal", noise_mag=0.05,
          mask_nyquist=True), dict(noise="philox", seed=7)),
    ("2d_linear_correlated", (64, 64),
     dict(is_nonlinear=False, time_integrator="implicit_pc", viscosity=0.1,
          noise_type="correlated", noise_mag=0.03), dict(noise="philox", seed=7)),
]


def _pair(name, N, kw, okw, precision, a, injected=False):
    from periodicflow import simulation as sim
    kw = dict(kw)
    dealias = kw.pop("dealias", "2/3")
    seed = okw.get("seed", 0)
    g = O.Grid(N, dealias=dealias, mask_nyquist=kw.get("mask_nyquist", False))
    o = O.OracleSolver(N, 0.01, dealias=dealias, **kw, **okw)
    s = sim.Solver(list(N), 0.01, 1.0, dealias=dealias, precision=precision, seed=seed,
                   noise_source="injected" if injected else "philox", **kw)
    uh = O.spectral_random_field(g, 3)
    o.initialize(uh, "fourier")
    s.initialize(uh, "fourier")
    if kw.get("noise_type") == "correlated":
        C = np.exp(-(np.sqrt(g.k2) / 8.0) ** 2)
        o.set_correlation_function(C)
        s.set_correlation_function(C)
    w = None
    if injected:
        w = O.numpy_noise_fields(g, kw.get("noise_type", "thermal"), np.random.RandomState(5))
        s.inject_noise(*w)
    ss = s.space_solver
    ss.compute_rhs(a)
    ref = o.compute_rhs(a, *(w or (None, None)))
    return {n: getattr(ss, n) for n in NAMES}, ref


def _compare(got, ref, precision):
    for n in NAMES:
        r = ref[n]
        if np.linalg.norm(r) == 0.0:
            assert np.max(np.abs(got[n])) == 0.0, n
        else:
            assert rel_l2(got[n], r) < TOL[precision], n


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("a", [0.0, 1.0, 0.6])
def test_compute_rhs_vs_oracle(case, precision, a):
    name, N, kw, okw = case
    got, ref = _pair(name, N, kw, okw, precision, a)
    _compare(got, ref, precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_compute_rhs_injected_noise_vs_oracle(precision):
    got, ref = _pair("2d_thermal_injected", (32, 64),
                     dict(time_integrator="explicit_pc", viscosity=0.1, noise_type="thermal",
                          noise_mag=0.05), {}, precision, 0.7, injected=True)
    _compare(got, ref, precision)


def test_compute_rhs_leaves_the_state_and_step_alone():
    from periodicflow import simulation as sim
    N = (16, 16, 16)
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 4)
    s = sim.Solver(list(N), 0.01, 1.0, time_integrator="rk3", viscosity=2e-3, dealias="2/3",
                   precision="fp64", forcing=(0.1, 2.5))
    s.initialize(uh, "fourier")
    before = s.space_solver.u_hat
    s.space_solver.compute_rhs(0.0)
    assert np.array_equal(s.space_solver.u_hat, before)
    t, step, _ = s.space_solver.time()
    assert step == 0 and t == 0.0
    # a plain step afterwards equals one without the call
    s2 = sim.Solver(list(N), 0.01, 1.0, time_integrator="rk3", viscosity=2e-3, dealias="2/3",
                    precision="fp64", forcing=(0.1, 2.5))
    s2.initialize(uh, "fourier")
    s.space_solver.step(1)
    s2.space_solver.step(1)
    assert np.array_equal(s.space_solver.u_hat, s2.space_solver.u_hat)


def test_arrays_are_zero_before_compute_rhs():
    from periodicflow import simulation as sim
    s = sim.Solver([16, 16], 0.01, 1.0, precision="fp64", dealias="2/3")
    for n in NAMES:
        assert not np.any(getattr(s, n))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_forward_without_argument_transforms_the_edited_u(precision):
    """space_solver.py:215-219: forward() transforms the solver's own u."""
    from periodicflow import simulation as sim
    N = (32, 16, 16)
    g = O.Grid(N)
    s = sim.Solver(list(N), 0.01, 1.0, precision=precision, dealias="2/3")
    ss = s.space_solver
    s.initialize(O.taylor_green(g), project=False)
    u = ss.u                      # the solver's host array
    u *= 2.0                      # edited in place
    ss.forward()
    ref = g.forward(2.0 * O.taylor_green(g))
    assert rel_l2(ss.u_hat, ref) < (1e-13 if precision == "fp64" else 2e-6)
    assert ss.u is u              # the same array object, refreshed by backward
    assert rel_l2(ss.backward(), 2.0 * O.taylor_green(g)) < (1e-13 if precision == "fp64" else 2e-6)
