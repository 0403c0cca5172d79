"""GPU parity of the fused 2D nonlinear schedule (three passes per stage).

The fused path is the default for 2D boxes with power-of-two sides 16..1024
and the 2/3 rule; ``fused=False`` runs the per-operator path.  Tolerances:
relative L2 over the state, FP64 1e-11 against the FP64 oracle, FP32 1e-5.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def solver(N, dt=0.01, **kw):
    from periodicflow import simulation as sim
    kw.setdefault("dealias", "2/3")
    return sim.Solver(list(N), dt, 1.0, **kw)


@pytest.mark.parametrize("N", [(16, 16), (64, 32), (32, 128), (256, 256), (1024, 64),
                               (128, 1024), (512, 512)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("integ", ["rk3", "rk4", "implicit_pc"])
def test_fused2d_vs_oracle(N, precision, integ):
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3)
    uh0 = O.spectral_random_field(o.grid, 11)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=2e-3, time_integrator=integ, viscosity=2e-3, precision=precision,
               fused=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < (1e-11 if precision == "fp64" else 1e-5)


@pytest.mark.parametrize("integ", ["rk2", "explicit_pc"])
def test_fused2d_other_integrators_vs_oracle(integ):
    N = (128, 128)
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3)
    uh0 = O.spectral_random_field(o.grid, 12)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=2e-3, time_integrator=integ, viscosity=2e-3, precision="fp64")
    s.initialize(uh0, "fourier")
    o.advance(3)
    s.space_solver.step(3)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


def test_fused2d_1024_fp64_vs_oracle():
    """The largest 2D side with a fused schedule, a non-square domain and
    the Nyquist mask on."""
    N = (1024, 1024)
    dom = ((0.0, 2 * np.pi), (0.0, 4 * np.pi))
    o = O.OracleSolver(N, 1e-3, time_integrator="rk3", viscosity=1e-3, domain=dom,
                       mask_nyquist=True)
    uh0 = O.spectral_random_field(o.grid, 13)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=1e-3, time_integrator="rk3", viscosity=1e-3, precision="fp64",
               domain=dom, mask_nyquist=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


@pytest.mark.parametrize("precision,noise_type", [("fp64", "thermal"), ("fp64", "correlated"),
                                                  ("fp32", "thermal")])
def test_fused2d_forcing_cfl_noise_matches_generic(precision, noise_type):
    N = (256, 128)
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision=precision,
              forcing=(0.1, 2.5), cfl=0.5, noise_mag=1e-3, noise_type=noise_type, seed=3)
    a = solver(N, fused=True, **kw)
    b = solver(N, fused=False, **kw)
    g = O.Grid(N)
    if noise_type == "correlated":
        C = np.exp(-g.k2 / 64.0)
        a.set_correlation_function(C)
        b.set_correlation_function(C)
    uh0 = O.spectral_random_field(g, 1)
    a.initialize(uh0, "fourier")
    b.initialize(uh0, "fourier")
    a.space_solver.step(3)
    b.space_solver.step(3)
    ta, sa, da = a.space_solver.time()
    tb, sb, db = b.space_solver.time()
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert sa == sb == 3 and abs(da - db) < (1e-12 if precision == "fp64" else 1e-5) * db
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < tol


def test_fused2d_energy_history_and_graph_vs_oracle():
    """E and Z per step from the fused update, and a captured graph replayed
    over a state set between replays."""
    import torch
    N = (256, 256)
    o = O.OracleSolver(N, 5e-3, time_integrator="rk4", viscosity=1e-3)
    uh0 = O.spectral_random_field(o.grid, 14)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=5e-3, time_integrator="rk4", viscosity=1e-3, precision="fp64",
               diagnostics=True)
    s.initialize(uh0, "fourier")
    ho = np.array(o.advance(4, diagnostics=True))
    s.space_solver.step(4)
    hs = s.space_solver.history()
    assert np.max(np.abs(hs - ho) / np.abs(ho)) < 1e-11
    kw = dict(dt=2e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32")
    a = solver(N, fused=True, **kw)
    b = solver(N, fused=False, **kw)
    g = O.Grid(N)
    for s_ in (a, b):
        s_.initialize(O.spectral_random_field(g, 3), "fourier")
        st = torch.cuda.Stream()
        s_.space_solver.set_stream(st.cuda_stream)
        s_.space_solver.capture(3)
        s_.space_solver.replay()
        s_.initialize(O.spectral_random_field(g, 5), "fourier")
        s_.space_solver.replay()
        st.synchronize()
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 2e-6
