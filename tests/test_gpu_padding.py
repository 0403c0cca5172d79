"""GPU parity of the 3/2 (padding) dealias rule against the oracle's
restatement (the reference's default rule, basis.py:80-81; shenfun's own
padding is not available here, so the convention is the oracle's: Nyquist
modes split in half on padding and folded on truncation)."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def solver(N, dt, **kw):
    from periodicflow import simulation as sim
    return sim.Solver(list(N), dt, 1.0, dealias="3/2", **kw)


@pytest.mark.parametrize("N", [(12, 24), (96, 48), (24, 48, 12), (192, 384), (384, 12),
                               (768, 16), (48, 96, 192)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_radix3_transforms_vs_oracle(N, precision):
    from periodicflow import simulation as sim
    rng = np.random.default_rng(3)
    g = O.Grid(N)
    s = sim.Solver(list(N), 0.01, 1.0, is_nonlinear=False, precision=precision)
    u = rng.standard_normal((len(N),) + tuple(N))
    s.space_solver.u = u
    tol = 1e-13 if precision == "fp64" else 3e-6
    assert rel_l2(s.space_solver.u_hat, g.forward(u)) < tol
    s.space_solver.u_hat = g.forward(u)
    assert rel_l2(s.space_solver.u, u) < tol


@pytest.mark.parametrize("N", [(16, 16), (32, 64), (16, 16, 16), (8, 16, 32), (32, 32, 32)])
@pytest.mark.parametrize("precision,integ", [("fp64", "rk3"), ("fp64", "implicit_pc"),
                                             ("fp32", "rk4")])
def test_padded_nonlinear_vs_oracle(N, precision, integ):
    o = O.OracleSolver(N, 5e-3, time_integrator=integ, viscosity=5e-3, dealias="3/2")
    uh0 = O.spectral_random_field(o.grid, 11, kp=2.0)
    o.initialize(uh0, "fourier")
    s = solver(N, 5e-3, time_integrator=integ, viscosity=5e-3, precision=precision)
    s.initialize(uh0, "fourier")
    o.advance(3)
    s.space_solver.step(3)
    tol = 1e-11 if precision == "fp64" else 1e-5
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < tol


def test_padded_tgv_forcing_cfl_vs_oracle():
    N = (32, 32, 32)
    o = O.OracleSolver(N, 0.01, time_integrator="rk3", viscosity=2e-3, dealias="3/2",
                       forcing=(0.1, 2.5), cfl=0.5)
    o.initialize(O.taylor_green(o.grid))
    s = solver(N, 0.01, time_integrator="rk3", viscosity=2e-3, precision="fp64",
               forcing=(0.1, 2.5), cfl=0.5)
    s.initialize(O.taylor_green(o.grid))
    o.advance(3)
    s.space_solver.step(3)
    t, step, dt = s.space_solver.time()
    assert abs(dt - o.dt) < 1e-12 * o.dt and abs(t - o.t) < 1e-12 * o.t
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


def test_padded_energy_conservation_inviscid():
    """With nu = 0 the padded nonlinear term conserves energy: E drifts only
    by the time-stepping error (RK4, small dt)."""
    N = (32, 32, 32)
    s = solver(N, 1e-3, time_integrator="rk4", viscosity=0.0, precision="fp64")
    g = O.Grid(N, dealias="3/2")
    s.initialize(O.spectral_random_field(g, 5, kp=3.0), "fourier")
    e0, _ = s.space_solver.energy()
    s.space_solver.step(20)
    e1, _ = s.space_solver.energy()
    assert abs(e1 - e0) / e0 < 1e-9


# ------------------------------------------------- fused 3/2 schedule (FP32)
@pytest.mark.parametrize("N", [(16, 16, 16), (32, 64, 32), (64, 32, 128), (128, 64, 32)])
@pytest.mark.parametrize("integ", ["rk3", "rk4", "implicit_pc"])
def test_fused_padded_vs_oracle(N, integ):
    """FP32 fused passes on the padded grid vs the FP64 oracle, 2 steps."""
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3, dealias="3/2")
    uh0 = O.spectral_random_field(o.grid, 5)
    o.initialize(uh0, "fourier")
    s = solver(N, 2e-3, time_integrator=integ, viscosity=2e-3, precision="fp32", fused=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-5


def test_fused_padded_forcing_cfl_noise_matches_generic():
    N = (64, 64, 64)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp32",
              forcing=(0.1, 2.5), cfl=0.5, noise_mag=1e-3, seed=3)
    a = solver(N, 1e-3, fused=True, **kw)
    b = solver(N, 1e-3, fused=False, **kw)
    uh0 = O.spectral_random_field(O.Grid(N), 1)
    a.initialize(uh0, "fourier")
    b.initialize(uh0, "fourier")
    a.space_solver.step(3)
    b.space_solver.step(3)
    ta, sa, da = a.space_solver.time()
    tb, sb, db = b.space_solver.time()
    assert sa == sb == 3 and abs(da - db) < 1e-5 * db
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 2e-6


def test_fused_padded_256_matches_generic():
    """The 384-point padded passes at the benchmark's grid: fused and generic
    FP32 agree after one RK3 step (the FP64 oracle is too slow at 256^3)."""
    N = (256, 256, 256)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", cfl=0.5)
    uh0 = O.spectral_random_field(O.Grid(N), 2)
    out = []
    for fused in (True, False):
        s = solver(N, 1e-3, fused=fused, **kw)
        s.initialize(uh0, "fourier")
        s.space_solver.step(1)
        out.append(s.space_solver.u_hat)
        del s
    assert rel_l2(out[0], out[1]) < 2e-6


# ------------------------------------------------- fused 3/2 schedule (FP64)
@pytest.mark.parametrize("N", [(16, 16, 16), (32, 64, 32), (64, 32, 128), (128, 64, 32)])
@pytest.mark.parametrize("integ", ["rk3", "rk4", "implicit_pc"])
def test_fused_padded_fp64_vs_oracle(N, integ):
    """FP64 fused passes on the padded grid (the reference's precision and
    default rule) vs the FP64 oracle, 2 steps."""
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3, dealias="3/2")
    uh0 = O.spectral_random_field(o.grid, 6)
    o.initialize(uh0, "fourier")
    s = solver(N, 2e-3, time_integrator=integ, viscosity=2e-3, precision="fp64", fused=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


def test_fused_padded_fp64_forcing_cfl_noise_matches_generic():
    N = (64, 64, 64)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp64",
              forcing=(0.1, 2.5), cfl=0.5, noise_mag=1e-3, seed=3)
    a = solver(N, 1e-3, fused=True, **kw)
    b = solver(N, 1e-3, fused=False, **kw)
    uh0 = O.spectral_random_field(O.Grid(N), 1)
    a.initialize(uh0, "fourier")
    b.initialize(uh0, "fourier")
    a.space_solver.step(3)
    b.space_solver.step(3)
    ta, sa, da = a.space_solver.time()
    tb, sb, db = b.space_solver.time()
    assert sa == sb == 3 and abs(da - db) < 1e-12 * db
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 1e-12


def test_fused_padded_fp64_256_matches_generic():
    """FP64 384-point padded passes at 256^3: fused and generic agree after
    one RK3 step."""
    N = (256, 256, 256)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp64", cfl=0.5)
    uh0 = O.spectral_random_field(O.Grid(N), 2)
    out = []
    for fused in (True, False):
        s = solver(N, 1e-3, fused=fused, **kw)
        s.initialize(uh0, "fourier")
        s.space_solver.step(1)
        out.append(s.space_solver.u_hat)
        del s
    assert rel_l2(out[0], out[1]) < 1e-12
