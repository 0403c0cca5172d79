"""Pin the oracle to the reference: golden vectors produced by the reference's
own Numba kernels and integrator classes (tests/golden/make_golden.py)."""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2


@pytest.mark.parametrize("d,N", [(2, (8, 8)), (3, (8, 8, 8))])
def test_pointwise_kernels(golden, d, N):
    g = O.Grid(N)
    uh = golden[f"k{d}_uh"]
    np.testing.assert_allclose(O.curl(g.k, uh), golden[f"k{d}_curl"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(O.cross(golden[f"k{d}_u"], golden[f"k{d}_w"]),
                               golden[f"k{d}_cross"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(O.apply_linear_operator(golden[f"k{d}_L"], uh),
                               golden[f"k{d}_Lu"], rtol=0, atol=1e-13)
    up, p = O.leray_projection(uh, g.k, g.k_over_k2)
    np.testing.assert_allclose(up, golden[f"k{d}_leray_u"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(p, golden[f"k{d}_leray_p"], rtol=0, atol=1e-13)
    ws = O.symmetrize(golden[f"k{d}_W"])
    np.testing.assert_allclose(ws, golden[f"k{d}_Wsym"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(O.noise_divergence(ws, g.k), golden[f"k{d}_noisediv"],
                               rtol=0, atol=1e-13)


@pytest.mark.parametrize("d,N", [(2, (8, 8)), (3, (4, 4, 4))])
@pytest.mark.parametrize("name", ["explicit_pc", "implicit_pc", "rk2", "rk3", "rk4"])
@pytest.mark.parametrize("opt", [0, 1])
def test_integrator_stages(golden, d, N, name, opt):
    L = golden[f"st{d}_L"]
    integ = O.INTEGRATORS[name](0.01, L.copy())
    for stage in range(integ.n_stages):
        key = f"st{d}_{name}_{opt}_{stage}"
        unew, u0, Nl, Lu, f, xi = (a.copy() for a in golden[key + "_in"])
        integ.stepping(unew, u0, stage, Nl, Lu, f, xi)
        np.testing.assert_allclose(unew, golden[key + "_out"], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(Lu, golden[key + "_Lu"], rtol=1e-13, atol=1e-13)


def _oracle_for(meta, golden):
    name = meta["name"]
    pre = f"p_{name}_"
    w1 = golden[pre + "w1"] if pre + "w1" in golden else None
    w2 = golden[pre + "w2"] if pre + "w2" in golden else None
    domain = [(0.0, float(x)) for x in meta["L"]]

    d = len(meta["N"])
    ncomp = d * d if meta.get("noise_type", "thermal") == "thermal" else d
    spec = tuple(meta["N"][:-1]) + (meta["N"][-1] // 2 + 1,)

    def inject(step):
        if w1 is None:
            z = np.zeros((ncomp,) + spec, dtype=np.complex128)
            return z, z
        return w1[step - 1], w2[step - 1]

    s = O.OracleSolver(meta["N"], meta["dt"], is_nonlinear=meta["nonlinear"],
                       time_integrator=meta["integ_name"], viscosity=meta["nu"],
                       noise_type=meta.get("noise_type", "thermal"),
                       noise_mag=meta.get("noise_mag", 0.0), domain=domain,
                       dealias="2/3", mask_nyquist=meta["mask_nyquist"], noise=inject)
    if meta["has_L"]:
        s.set_linear_operator(golden[pre + "L"])
    if meta["has_C"]:
        s.set_correlation_function(golden[pre + "C"])
    s.initialize(golden[pre + "uh0"], "fourier", project=False, mask_zero_mode=False)
    return s


def test_pipelines_match_reference_kernels(golden, pipeline_meta):
    assert len(pipeline_meta) >= 10
    for name, meta in pipeline_meta.items():
        s = _oracle_for(meta, golden)
        states = golden[f"p_{name}_states"]
        for i in range(meta["nsteps"]):
            s.advance(1)
            err = rel_l2(s.u_hat, states[i])
            assert err < 1e-12, (name, i, err)


@pytest.mark.parametrize("N", [(8, 8), (8, 6, 10), (16, 16, 16)])
def test_padding_rule_properties(N):
    """3/2 rule restatement: truncate(pad(u)) = u for Hermitian spectra, and
    the padded backward transform interpolates the coarse samples."""
    g = O.Grid(N, dealias="3/2")
    rng = np.random.default_rng(0)
    u = rng.standard_normal((len(N),) + tuple(N))
    uh = g.forward(u)
    np.testing.assert_allclose(g.truncate(g.pad(uh)), uh, rtol=0, atol=1e-15)
    uM = g.backward_dealiased(uh)
    idxM = tuple([slice(None)] + [slice(0, 3 * n // 2, 3) for n in N])
    idxN = tuple([slice(None)] + [slice(0, n, 2) for n in N])
    np.testing.assert_allclose(uM[idxM], u[idxN], rtol=0, atol=1e-13)


@pytest.mark.parametrize("dealias", ["2/3", "3/2"])
def test_tgv_energy_decay_rate_both_rules(dealias):
    nu = 1 / 1600
    s = O.OracleSolver((16, 16, 16), 1e-4, time_integrator="rk4", viscosity=nu, dealias=dealias)
    s.initialize(O.taylor_green(s.grid))
    e0, z0 = O.energy(s.grid, s.u_hat), O.enstrophy(s.grid, s.u_hat)
    s.advance(1)
    assert abs((O.energy(s.grid, s.u_hat) - e0) / 1e-4 + 2 * nu * z0) < 1e-6


def test_tgv_energy_decay_rate():
    """TGV at t=0: dE/dt = -2 nu Z (the nonlinear term conserves energy)."""
    nu = 1 / 1600
    s = O.OracleSolver((16, 16, 16), 1e-4, time_integrator="rk4", viscosity=nu)
    s.initialize(O.taylor_green(s.grid))
    e0, z0 = O.energy(s.grid, s.u_hat), O.enstrophy(s.grid, s.u_hat)
    assert abs(e0 - 0.125) < 1e-14 and abs(z0 - 0.375) < 1e-13
    s.advance(1)
    e1 = O.energy(s.grid, s.u_hat)
    rate = (e1 - e0) / 1e-4
    assert abs(rate - (-2 * nu * z0)) < 1e-6


def test_oracle_tgv64_history_prefix():
    """The oracle's Taylor-Green run (64^3 FP64, rk4, dt 0.005, nu 1/1600)
    against the energy/enstrophy history the reference's kernels produced
    (tests/golden/make_c1_history.py); first 40 of its 400 steps."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tgv64_fp64_rk4_400.npz"))
    ref = z["energy_enstrophy"]
    n = 64
    o = O.OracleSolver((n, n, n), 0.005, time_integrator="rk4", viscosity=1 / 1600)
    o.initialize(O.taylor_green(o.grid))
    h = np.array(o.advance(40, diagnostics=True))
    np.testing.assert_allclose(h, ref[:40], rtol=1e-12, atol=0)


@pytest.mark.parametrize("kw", [
    dict(N=(16, 16, 16), time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5)),
    dict(N=(16, 8, 16), time_integrator="implicit_pc", viscosity=0.05, noise_type="thermal",
         noise_mag=0.02, seed=3),
    dict(N=(32, 16), time_integrator="explicit_pc", viscosity=0.01, noise_type="correlated",
         noise_mag=0.1, mask_nyquist=True, seed=3),
], ids=["3d_rk3_forcing", "3d_thermal", "2d_correlated_nyquist"])
def test_oracle_compute_rhs_rebuilds_its_step(kw):
    """compute_rhs(a) per stage fed to the integrator reproduces advance(1):
    the arrays are the terms the reference's loop hands to stepping
    (simulation.py:209-213)."""
    kw = dict(kw)
    N = kw.pop("N")
    g = O.Grid(N, mask_nyquist=kw.get("mask_nyquist", False))
    uh = O.spectral_random_field(g, 2)
    a = O.OracleSolver(N, 0.01, **kw)
    b = O.OracleSolver(N, 0.01, **kw)
    if kw.get("noise_type") == "correlated":
        C = np.exp(-g.k2 / 16.0)
        a.set_correlation_function(C)
        b.set_correlation_function(C)
    a.initialize(uh, "fourier")
    b.initialize(uh, "fourier")
    a.advance(1)
    integ = b.integrator
    u0 = b.u_hat.copy()
    w = b._noise_fields_for(1) if kw.get("noise_mag") else (None, None)
    for stage in range(integ.n_stages):
        r = b.compute_rhs(integ.noise_factor[stage], *w)
        integ.stepping(b.u_hat, u0, stage, r["rhs_nonlinear"], r["rhs_linear"], r["forcing"],
                       r["noise"])
    assert rel_l2(b.u_hat, a.u_hat) < 1e-15
