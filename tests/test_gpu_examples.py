"""The call patterns of the reference's three example scripts, run against
this backend (smaller grids and end times so the tests are quick):
examples/fluctuating_stokes_thermal_noise.py, examples/
fluctuating_stokes_correlated_noise.py and examples/tgv3d.py use the Solver
constructor keywords, the pass-through attributes (x, k, k2,
shape_local_fourier, shape_local_physical, comm, mpi_rank), initialize in
Fourier or physical space, set_linear_operator / set_correlation_function,
solve and solution_writer.reconfigure_dataset."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _random_fourier_ic(shape, n, kbt, factor_rule):
    dim = shape[0]
    factor = factor_rule(n, dim, kbt)
    u0 = np.random.randn(*shape) + 1j * np.random.randn(*shape)
    for i in range(dim):
        u0[i] /= np.std(u0[i]) * factor
    return u0


def _oracle_snapshots(o, steps, every):
    """Physical velocity of the oracle at every written step (0 included)."""
    out = {0: o.grid.backward(o.u_hat)}
    for step in range(1, steps + 1):
        o.advance(1)
        if step % every == 0:
            out[step] = o.grid.backward(o.u_hat)
    return out


def _check_snapshots(z, ref, names, width, tol):
    for step, u in ref.items():
        got = np.stack([z[f"{c}/{step:0{width}d}"] for c in names])
        err = np.linalg.norm(got - u) / max(np.linalg.norm(u), 1e-300)
        assert err < tol, (step, err)


TOL = {"fp64": 1e-11, "fp32": 1e-5}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_thermal_noise_example_pattern(tmp_path, precision):
    """examples/fluctuating_stokes_thermal_noise.py's calls (64^2, 20 steps)
    with the reference's NumPy draws; every written snapshot equals the
    oracle's velocity under the same draws."""
    import oracle as O
    from periodicflow import simulation as sim
    n, dim, nu, kbt = 64, 2, 818.72, 4.2052
    rule = lambda n, d, k: n ** (d / 2) / k ** 0.5 * np.sqrt(1 - 1 / d)
    mag = (2 * nu * kbt) ** 0.5
    np.random.seed(1234)
    sol = sim.Solver([n] * dim, 1e-3, 0.02, viscosity=nu, is_nonlinear=False,
                     time_integrator="implicit_pc", write_solution=True,
                     file_name=str(tmp_path / "thermal"), write_interval=2,
                     noise_type="thermal", noise_mag=mag, precision=precision,
                     noise_source="numpy")
    u0 = _random_fourier_ic(sol.shape_local_fourier, n, kbt, rule)
    sol.initialize(u0, "fourier")
    sol.solve()
    assert sol.step == 20 and abs(sol.t - 0.02) < 1e-12
    z = np.load(sol.solution_writer.reconfigure_dataset())
    assert {"x", "y", "t", "u/00", "v/20"} <= set(z.files)
    # the same generator sequence for the oracle: Solver reseeds NumPy's
    # global generator (simulation.py:100), then the initial field and the
    # per-step draws (space_solver.py:227-238) follow
    np.random.seed(1234)
    np.random.seed(np.random.randint(0, 2 ** 32 - 1))
    u0o = _random_fourier_ic(sol.shape_local_fourier, n, kbt, rule)
    assert np.array_equal(u0o, u0)
    o = O.OracleSolver((n, n), 1e-3, is_nonlinear=False, time_integrator="implicit_pc",
                       viscosity=nu, noise_type="thermal", noise_mag=mag, noise="numpy")
    o.initialize(u0o, "fourier")
    _check_snapshots(z, _oracle_snapshots(o, 20, 2), "uv", 2, TOL[precision])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_correlated_noise_example_pattern(tmp_path, precision):
    """examples/fluctuating_stokes_correlated_noise.py's calls (64^2, 10
    steps, L = 0.2), checked against the oracle under the same draws."""
    import oracle as O
    from periodicflow import simulation as sim
    n, dim, nu, kbt, L = 64, 2, 818.72, 4.2052, 0.2
    rule = lambda n, d, k: n ** (d / 2) / k ** 0.5 / (2 - 2 / d)
    mag = (2 * nu * kbt) ** 0.5
    np.random.seed(99)
    sol = sim.Solver([n] * dim, 0.01, 0.1, viscosity=nu, is_nonlinear=False,
                     time_integrator="implicit_pc", write_solution=True,
                     file_name=str(tmp_path / "correlated"), write_interval=5,
                     noise_type="correlated", noise_mag=mag, precision=precision,
                     noise_source="numpy")
    u0 = _random_fourier_ic(sol.shape_local_fourier, n, kbt, rule)
    sol.initialize(u0, "fourier")
    args_L = sol.comm.bcast(L if sol.mpi_rank == 0 else None, root=0)
    dx = sol.x[0][1] - sol.x[0][0]
    kx, ky = sol.k
    C = np.exp(-0.5 * ((args_L * kx) ** 2 + (args_L * ky) ** 2)) * (
        np.sqrt(2 * np.pi * args_L ** 2) / dx) ** dim
    C *= np.where(sol.k2 == 0, 0, 1)
    sol.set_linear_operator(-nu * C)
    sol.set_correlation_function(np.sqrt(C))
    sol.solve()
    assert sol.step == 10
    uh = sol.u_hat
    assert np.isfinite(uh).all() and np.all(uh[:, 0, 0] == 0)
    z = np.load(sol.solution_writer.reconfigure_dataset())
    np.random.seed(99)
    np.random.seed(np.random.randint(0, 2 ** 32 - 1))
    u0o = _random_fourier_ic(sol.shape_local_fourier, n, kbt, rule)
    o = O.OracleSolver((n, n), 0.01, is_nonlinear=False, time_integrator="implicit_pc",
                       viscosity=nu, noise_type="correlated", noise_mag=mag, noise="numpy")
    o.initialize(u0o, "fourier")
    o.set_linear_operator(-nu * C)
    o.set_correlation_function(np.sqrt(C))
    _check_snapshots(z, _oracle_snapshots(o, 10, 5), "uv", 2, TOL[precision])
    assert np.linalg.norm(uh - o.u_hat) / np.linalg.norm(o.u_hat) < TOL[precision]


def test_tgv3d_example_pattern(tmp_path):
    from periodicflow import simulation as sim
    n = 16
    sol = sim.Solver([n] * 3, 1e-3, 0.1, viscosity=1600, nonlinear=False, optimization=True,
                     time_integrator="implicit_pc", verbose=True, write_solution=True,
                     file_name=str(tmp_path / "TG"), write_interval=50, check_interval=1000)
    x = sol.x
    u0 = np.zeros(sol.shape_local_physical)
    u0[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    u0[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    sol.initialize(u0)
    sol.solve()
    path = sol.solution_writer.reconfigure_dataset()
    z = np.load(path)
    assert {"x", "y", "z", "t", "u/000", "w/100"} <= set(z.files)
    # Stokes with nu = 1600 damps the |k| = sqrt(3) mode by exp(-3 nu t)
    e = sum(float(np.mean(z[f"{c}/100"] ** 2)) for c in "uvw")
    assert e < 1e-6
    # every written snapshot against the oracle (same physical initial field)
    import oracle as O
    o = O.OracleSolver((n, n, n), 1e-3, is_nonlinear=False, time_integrator="implicit_pc",
                       viscosity=1600)
    o.initialize(u0)
    ref = _oracle_snapshots(o, 100, 50)
    for step, u in ref.items():
        got = np.stack([z[f"{c}/{step:03d}"] for c in "uvw"])
        assert np.max(np.abs(got - u)) < 1e-5 * max(np.max(np.abs(ref[0])), 1.0), step


def test_nonlinear_default_dealias_and_read_config():
    """The reference's default dealias rule is 3/2 (simulation.py:74)."""
    from periodicflow import simulation as sim
    cfg = dict(N=[16, 16, 16], dt=1e-3, end_time=0.005, time_integrator="rk3",
               viscosity=1e-2)
    sol = sim.Solver.read_config(cfg)
    x = sol.x
    u0 = np.zeros(sol.shape_local_physical)
    u0[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
    u0[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    sol.initialize(u0)
    sol.solve()
    assert sol.step == 5 and np.isfinite(sol.u).all()
