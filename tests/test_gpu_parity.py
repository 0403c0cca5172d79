"""GPU parity of the CUDA path against the oracle and the golden fixtures.

Tolerances (relative L2 over all modes of the state): FP64 1e-12 per the
target (1e-11 where many FFT passes accumulate), FP32 1e-5.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-11, "fp32": 1e-5}


def solver(N, dt=0.01, **kw):
    from periodicflow import simulation as sim
    kw.setdefault("dealias", "2/3")
    return sim.Solver(list(N), dt, 1.0, **kw)


# ------------------------------------------------------------------ transforms
@pytest.mark.parametrize("N", [(8, 8), (32, 64), (256, 256), (1024, 16), (8, 8, 8),
                               (16, 8, 32), (64, 64, 64), (128, 32, 256), (4, 1024, 8)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_forward_backward_vs_oracle(N, precision):
    rng = np.random.default_rng(1)
    g = O.Grid(N)
    s = solver(N, is_nonlinear=False, precision=precision)
    u = rng.standard_normal((len(N),) + tuple(N))
    s.space_solver.u = u
    uh = s.space_solver.u_hat
    ref = g.forward(u)
    assert rel_l2(uh, ref) < (1e-13 if precision == "fp64" else 2e-6)
    # backward of a Hermitian-consistent spectrum
    s.space_solver.u_hat = ref
    back = s.space_solver.u
    assert rel_l2(back, u) < (1e-13 if precision == "fp64" else 2e-6)


def test_backward_non_hermitian_planes_match_irfftn():
    """C2R takes only the real part of the DC / Nyquist entries, like irfftn."""
    rng = np.random.default_rng(2)
    N = (16, 16, 16)
    g = O.Grid(N)
    uh = rng.standard_normal((3,) + g.spec_shape) + 1j * rng.standard_normal((3,) + g.spec_shape)
    s = solver(N, is_nonlinear=False, precision="fp64")
    s.space_solver.u_hat = uh
    assert rel_l2(s.space_solver.u, g.backward(uh)) < 1e-13


# ------------------------------------------------------------- golden pipelines
def _run_pipeline(meta, golden, precision):
    name = meta["name"]
    pre = f"p_{name}_"
    noisy = pre + "w1" in golden
    s = solver(meta["N"], dt=meta["dt"], is_nonlinear=meta["nonlinear"],
               time_integrator=meta["integ_name"], viscosity=meta["nu"],
               noise_type=meta.get("noise_type", "thermal"), noise_mag=meta.get("noise_mag", 0.0),
               domain=[(0.0, float(x)) for x in meta["L"]], mask_nyquist=meta["mask_nyquist"],
               precision=precision, noise_source="injected" if noisy else "philox")
    if meta["has_L"]:
        s.set_linear_operator(golden[pre + "L"])
    if meta["has_C"]:
        s.set_correlation_function(golden[pre + "C"])
    s.initialize(golden[pre + "uh0"], "fourier", project=False, mask_zero_mode=False)
    states = golden[pre + "states"]
    errs = []
    for i in range(meta["nsteps"]):
        if noisy:
            s.inject_noise(golden[pre + "w1"][i], golden[pre + "w2"][i])
        s.space_solver.step(1)
        errs.append(rel_l2(s.space_solver.u_hat, states[i]))
    return errs


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_golden_pipelines(golden, pipeline_meta, precision):
    bad = {}
    for name, meta in pipeline_meta.items():
        errs = _run_pipeline(meta, golden, precision)
        if max(errs) > TOL[precision]:
            bad[name] = errs
    assert not bad, bad


# ------------------------------------------------------------------ operators
@pytest.mark.parametrize("d,N", [(2, (8, 8)), (3, (8, 8, 8))])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_operator_kernels_vs_golden(golden, d, N, precision):
    from periodicflow import math as pm
    g = O.Grid(N)
    cdt = np.complex128 if precision == "fp64" else np.complex64
    rdt = np.float64 if precision == "fp64" else np.float32
    tol = 1e-13 if precision == "fp64" else 1e-6
    uh = golden[f"k{d}_uh"].astype(cdt)
    k = g.k.astype(rdt)
    c = np.zeros((3,) + g.spec_shape if d == 3 else g.spec_shape, dtype=cdt)
    pm.curl(c, k, uh)
    assert rel_l2(c, golden[f"k{d}_curl"]) < tol
    u, w = golden[f"k{d}_u"].astype(rdt), golden[f"k{d}_w"].astype(rdt)
    cr = np.zeros_like(u)
    pm.cross(cr, u, w)
    assert rel_l2(cr, golden[f"k{d}_cross"]) < tol
    Lu = np.zeros_like(uh)
    pm.apply_linear_operator(Lu, golden[f"k{d}_L"].astype(rdt), uh)
    assert rel_l2(Lu, golden[f"k{d}_Lu"]) < tol
    up = uh.copy()
    p = np.zeros(g.spec_shape, dtype=cdt)
    pm.leray_projection(up, k, g.k_over_k2.astype(rdt), p)
    assert rel_l2(up, golden[f"k{d}_leray_u"]) < tol
    assert rel_l2(p, golden[f"k{d}_leray_p"]) < tol
    W = golden[f"k{d}_W"].astype(cdt)
    ws = np.zeros_like(W)
    pm.symmetrize(ws, W)
    assert rel_l2(ws, golden[f"k{d}_Wsym"]) < tol
    div = np.zeros((d,) + g.spec_shape, dtype=cdt)
    pm.noise_divergence(div, ws, k)
    assert rel_l2(div, golden[f"k{d}_noisediv"]) < tol


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("name", ["explicit_pc", "implicit_pc", "rk2", "rk3", "rk4"])
def test_stepping_kernels_vs_golden(golden, d, name):
    from periodicflow.time_integrator import DICT_TIME_INTEGRATORS
    L = golden[f"st{d}_L"]
    integ = DICT_TIME_INTEGRATORS[name](0.01, L.copy())
    for stage in range(integ.n_stages):
        key = f"st{d}_{name}_1_{stage}"
        unew, u0, Nl, Lu, f, xi = (a.copy() for a in golden[key + "_in"])
        integ.stepping(unew, u0, stage, Nl, Lu, f, xi)
        assert rel_l2(unew, golden[key + "_out"]) < 1e-14
        assert rel_l2(Lu, golden[key + "_Lu"]) < 1e-14


# ---------------------------------------------------------------- Philox noise
@pytest.mark.parametrize("N,noise_type,integ", [
    ((16, 16), "thermal", "explicit_pc"), ((16, 16), "thermal", "implicit_pc"),
    ((16, 16), "correlated", "implicit_pc"), ((8, 8, 8), "thermal", "rk3"),
    ((8, 8, 8), "correlated", "explicit_pc")])
def test_philox_stokes_vs_oracle(N, noise_type, integ):
    """Device Philox draws (Hermitian on self-conjugate planes) == oracle's."""
    nu, mag = 0.1, 0.05
    g = O.Grid(N)
    Cf = np.exp(-g.k2 / 8.0) * g.mask_k0
    o = O.OracleSolver(N, 0.01, is_nonlinear=False, time_integrator=integ, viscosity=nu,
                       noise_type=noise_type, noise_mag=mag, noise="philox", seed=1234)
    s = solver(N, is_nonlinear=False, time_integrator=integ, viscosity=nu,
               noise_type=noise_type, noise_mag=mag, precision="fp64", seed=1234)
    if noise_type == "correlated":
        o.set_correlation_function(Cf)
        s.set_correlation_function(Cf)
    s.space_solver.step(3)
    o.advance(3)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-12


def test_philox_nonlinear_noise_generic_update_vs_oracle():
    N = (32, 32)
    o = O.OracleSolver(N, 0.01, time_integrator="rk3", viscosity=0.01, noise_mag=0.05,
                       noise="philox", seed=99)
    s = solver(N, time_integrator="rk3", viscosity=0.01, noise_mag=0.05, precision="fp64",
               seed=99)
    uh0 = O.spectral_random_field(o.grid, 3, kp=3.0)
    o.initialize(uh0, "fourier")
    s.initialize(uh0, "fourier")
    s.space_solver.step(3)
    o.advance(3)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


def test_stokes_multistep_kernel_equals_single_steps():
    N = (32, 32)
    kw = dict(is_nonlinear=False, time_integrator="explicit_pc", viscosity=0.1,
              noise_mag=0.01, precision="fp32", seed=5)
    a = solver(N, **kw)
    b = solver(N, **kw)
    a.space_solver.step(10)
    for _ in range(10):
        b.space_solver.step(1)
    np.testing.assert_array_equal(a.space_solver.u_hat, b.space_solver.u_hat)


# ---------------------------------------------------------- TGV / forcing / CFL
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tgv64_rk4_energy_enstrophy(precision):
    """Taylor-Green 64^3, nu=1/1600, rk4, dt=0.005: E, Z per step vs oracle."""
    N = (64, 64, 64)
    o = O.OracleSolver(N, 0.005, time_integrator="rk4", viscosity=1 / 1600)
    o.initialize(O.taylor_green(o.grid))
    s = solver(N, dt=0.005, time_integrator="rk4", viscosity=1 / 1600, precision=precision,
               diagnostics=True)
    s.initialize(O.taylor_green(o.grid))
    hist_o = o.advance(10, diagnostics=True)
    s.space_solver.step(10)
    hist_s = s.space_solver.history()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < tol * 10
    assert np.max(np.abs(hist_s - np.array(hist_o)) / np.abs(np.array(hist_o))) < tol


def test_forcing_and_cfl_rk3_vs_oracle():
    N = (32, 32, 32)
    o = O.OracleSolver(N, 0.01, time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5),
                       cfl=0.5)
    uh0 = O.spectral_random_field(o.grid, 1)
    o.initialize(uh0, "fourier")
    s = solver(N, time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5), cfl=0.5,
               precision="fp64")
    s.initialize(uh0, "fourier")
    o.advance(4)
    s.space_solver.step(4)
    t, step, dt = s.space_solver.time()
    assert step == 4 and abs(t - o.t) < 1e-12 * o.t and abs(dt - o.dt) < 1e-12 * o.dt
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


# ------------------------------------------------------------- fused passes
@pytest.mark.parametrize("N", [(16, 16, 16), (32, 32, 32), (64, 32, 128), (32, 128, 64),
                               (128, 128, 128)])
@pytest.mark.parametrize("integ", ["rk3", "rk4", "implicit_pc"])
def test_fused_passes_match_oracle(N, integ):
    """FP32 fused pencil path vs the FP64 oracle after 2 steps (1e-5 target)."""
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3)
    uh0 = O.spectral_random_field(o.grid, 7)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=2e-3, time_integrator=integ, viscosity=2e-3, precision="fp32", fused=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-5


def test_fused_forcing_cfl_noise_matches_generic():
    N = (64, 64, 64)
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32",
              forcing=(0.1, 2.5), cfl=0.5, noise_mag=1e-3, seed=3)
    a = solver(N, fused=True, **kw)
    b = solver(N, fused=False, **kw)
    uh0 = O.spectral_random_field(O.Grid(N), 1)
    a.initialize(uh0, "fourier")
    b.initialize(uh0, "fourier")
    a.space_solver.step(3)
    b.space_solver.step(3)
    ta, sa, da = a.space_solver.time()
    tb, sb, db = b.space_solver.time()
    assert sa == sb == 3 and abs(da - db) < 1e-5 * db
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 2e-6


def test_fused_energy_history_matches_oracle():
    N = (64, 64, 64)
    o = O.OracleSolver(N, 5e-3, time_integrator="rk4", viscosity=1 / 1600)
    o.initialize(O.taylor_green(o.grid))
    s = solver(N, dt=5e-3, time_integrator="rk4", viscosity=1 / 1600, precision="fp32",
               diagnostics=True, fused=True)
    s.initialize(O.taylor_green(o.grid))
    ho = np.array(o.advance(5, diagnostics=True))
    s.space_solver.step(5)
    hs = s.space_solver.history()
    assert np.max(np.abs(hs - ho) / np.abs(ho)) < 1e-5


def test_fused_state_replaced_between_calls_and_graph_replay():
    """A state set between calls, and each replay of a captured graph, start
    from the new u_hat: fused and generic paths agree."""
    import torch
    N = (32, 64, 32)
    kw = dict(dt=2e-3, time_integrator="rk4", viscosity=2e-3, precision="fp32")
    a = solver(N, fused=True, **kw)
    b = solver(N, fused=False, **kw)
    g = O.Grid(N)
    for s_ in (a, b):
        s_.initialize(O.spectral_random_field(g, 3), "fourier")
        s_.space_solver.step(2)
        s_.initialize(O.spectral_random_field(g, 4), "fourier")
        s_.space_solver.step(1)
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 2e-6
    for s_ in (a, b):
        st = torch.cuda.Stream()
        s_.space_solver.set_stream(st.cuda_stream)
        s_.space_solver.capture(3)
        s_.space_solver.replay()
        s_.initialize(O.spectral_random_field(g, 5), "fourier")
        s_.space_solver.replay()
        st.synchronize()
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 2e-6


@pytest.mark.parametrize("N", [(16, 16, 16), (32, 64, 32), (64, 32, 128), (128, 64, 64)])
@pytest.mark.parametrize("integ", ["rk3", "rk4", "implicit_pc"])
def test_fused_fp64_vs_oracle(N, integ):
    """FP64 fused passes (the reference's precision) vs the FP64 oracle."""
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3)
    uh0 = O.spectral_random_field(o.grid, 9)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=2e-3, time_integrator=integ, viscosity=2e-3, precision="fp64", fused=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-11


def test_fused_fp64_forcing_cfl_noise_matches_generic():
    N = (64, 64, 64)
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp64",
              forcing=(0.1, 2.5), cfl=0.5, noise_mag=1e-3, seed=3)
    a = solver(N, fused=True, **kw)
    b = solver(N, fused=False, **kw)
    uh0 = O.spectral_random_field(O.Grid(N), 1)
    a.initialize(uh0, "fourier")
    b.initialize(uh0, "fourier")
    a.space_solver.step(3)
    b.space_solver.step(3)
    ta, sa, da = a.space_solver.time()
    tb, sb, db = b.space_solver.time()
    assert sa == sb == 3 and abs(da - db) < 1e-12 * db
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 1e-12


def test_autotune_keeps_state_and_parity():
    """The autotuner leaves the state unchanged, picks among the built
    variants, and the tuned fused path still agrees with the generic one."""
    N = (256, 256, 256)
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32", cfl=0.5)
    uh0 = O.spectral_random_field(O.Grid(N), 4)
    a = solver(N, fused=True, **kw)
    a.initialize(uh0, "fourier")
    before = a.space_solver.u_hat
    picks = a.space_solver.autotune()
    assert np.array_equal(a.space_solver.u_hat, before)
    built = {1: range(0, 10), 2: range(0, 11), 3: range(0, 6), 4: range(0, 7)}
    assert all(picks["axes_256"][p] in built[p] for p in built)
    assert a.space_solver.fused_variants() == picks
    a.space_solver.step(1)
    ua = a.space_solver.u_hat
    del a
    b = solver(N, fused=False, **kw)
    b.initialize(uh0, "fourier")
    b.space_solver.step(1)
    assert rel_l2(ua, b.space_solver.u_hat) < 2e-6


@pytest.mark.parametrize("N,var", [((32, 32, 256), 4), ((32, 32, 256), 5), ((64, 32, 128), 4),
                                   ((48, 96, 256), 4), ((128, 128, 128), 4)])
def test_p3_one_exchange_form_vs_oracle(N, var, monkeypatch):
    """P3 with sixteen values per lane (one exchange per line FFT, twiddles in
    registers, shuffled output split, FP32 CFL sums): forcing + CFL vs the
    FP64 oracle after 2 steps, and against the eight-value form."""
    monkeypatch.setenv("PF_FUSED_VARIANT", f"p3:{var}")
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32",
              forcing=(0.1, 2.5), cfl=0.5)
    o = O.OracleSolver(N, 1e-3, time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5),
                       cfl=0.5)
    uh0 = O.spectral_random_field(o.grid, 5)
    o.initialize(uh0, "fourier")
    a = solver(N, fused=True, **kw)
    assert a.space_solver.fused_variants()["axes_256"][3] == var
    a.initialize(uh0, "fourier")
    o.advance(2)
    a.space_solver.step(2)
    assert rel_l2(a.space_solver.u_hat, o.u_hat) < 1e-5
    _, _, dt = a.space_solver.time()
    assert abs(dt - o.dt) < 1e-5 * o.dt
    monkeypatch.setenv("PF_FUSED_VARIANT", "p3:2")
    b = solver(N, fused=True, **kw)
    b.initialize(uh0, "fourier")
    b.space_solver.step(2)
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) < 2e-6


@pytest.mark.parametrize("N", [(16, 256, 256), (48, 256, 64), (256, 256, 256)])
def test_p2_tma_tiles_vs_oracle_and_plain_loads(N, monkeypatch):
    """P2 with its input tiles brought in by tiled bulk tensor copies (rows
    of c2 = 86 or 22 complex: multiples of 16 bytes): the same results as P2
    with plain loads to rounding, and the FP64 oracle (forcing + CFL, 2
    steps; 1 step at 256^3 against the per-operator path)."""
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32",
              forcing=(0.1, 2.5), cfl=0.5)
    uh0 = O.spectral_random_field(O.Grid(N), 8)
    steps = 1 if N[0] == 256 else 2
    out = {}
    for var in (10, 0):
        monkeypatch.setenv("PF_FUSED_VARIANT", f"p2:{var}")
        a = solver(N, fused=True, **kw)
        assert a.space_solver.fused_variants()["axes_256"][2] == var
        a.initialize(uh0, "fourier")
        a.space_solver.step(steps)
        out[var] = a.space_solver.u_hat
        del a
    assert rel_l2(out[10], out[0]) < 1e-6
    if N[0] == 256:
        b = solver(N, fused=False, **kw)
        b.initialize(uh0, "fourier")
        b.space_solver.step(steps)
        assert rel_l2(out[10], b.space_solver.u_hat) < 2e-6
    else:
        o = O.OracleSolver(N, 1e-3, time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5),
                           cfl=0.5)
        o.initialize(uh0, "fourier")
        o.advance(steps)
        assert rel_l2(out[10], o.u_hat) < 1e-5


@pytest.mark.parametrize("var", [4, 5])
def test_p3_one_exchange_form_256cubed_matches_generic(var, monkeypatch):
    N = (256, 256, 256)
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32", cfl=0.5,
              forcing=(0.1, 2.5))
    uh0 = O.spectral_random_field(O.Grid(N), 4)
    monkeypatch.setenv("PF_FUSED_VARIANT", f"p3:{var}")
    a = solver(N, fused=True, **kw)
    a.initialize(uh0, "fourier")
    a.space_solver.step(1)
    ua = a.space_solver.u_hat
    del a
    b = solver(N, fused=False, **kw)
    b.initialize(uh0, "fourier")
    b.space_solver.step(1)
    assert rel_l2(ua, b.space_solver.u_hat) < 2e-6


@pytest.mark.parametrize("N", [(48, 48, 48), (96, 48, 192), (192, 96, 48), (64, 96, 32)])
@pytest.mark.parametrize("integ", ["rk3", "implicit_pc"])
def test_fused_three_pow2_sides_vs_oracle(N, integ):
    """FP32 fused passes on sides 3 * 2^b (radix-3 stages, streamed-omega P3)
    vs the FP64 oracle."""
    o = O.OracleSolver(N, 2e-3, time_integrator=integ, viscosity=2e-3)
    uh0 = O.spectral_random_field(o.grid, 6)
    o.initialize(uh0, "fourier")
    s = solver(N, dt=2e-3, time_integrator=integ, viscosity=2e-3, precision="fp32", fused=True)
    s.initialize(uh0, "fourier")
    o.advance(2)
    s.space_solver.step(2)
    assert rel_l2(s.space_solver.u_hat, o.u_hat) < 1e-5


def test_fused_192_matches_generic():
    N = (192, 192, 192)
    kw = dict(dt=1e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32",
              forcing=(0.1, 2.5), cfl=0.5)
    uh0 = O.spectral_random_field(O.Grid(N), 3)
    out = []
    for fused in (True, False):
        s = solver(N, fused=fused, **kw)
        s.initialize(uh0, "fourier")
        s.space_solver.step(2)
        out.append(s.space_solver.u_hat)
        del s
    assert rel_l2(out[0], out[1]) < 2e-6


def test_step_graph_matches_plain_launches(monkeypatch):
    """pf_step replays a recorded one-step graph for noise-free runs; the
    states equal plain launches bit for bit, also after the linear operator
    is set between calls (the graph is recorded again)."""
    N = (32, 32, 32)
    kw = dict(dt=2e-3, time_integrator="rk3", viscosity=2e-3, precision="fp32",
              forcing=(0.1, 2.5), cfl=0.5)
    uh0 = O.spectral_random_field(O.Grid(N), 8)
    a = solver(N, **kw)
    monkeypatch.setenv("PF_STEP_GRAPH", "0")
    b = solver(N, **kw)
    monkeypatch.delenv("PF_STEP_GRAPH")
    L = -2e-3 * O.Grid(N).k2 * 1.5
    for s_ in (a, b):
        s_.initialize(uh0, "fourier")
        s_.space_solver.step(4)
        s_.set_linear_operator(L)
        s_.space_solver.step(3)
    assert np.array_equal(a.space_solver.u_hat, b.space_solver.u_hat)
    assert a.space_solver.time() == b.space_solver.time()


def test_tgv64_fp64_full_run_vs_reference_history():
    """The Taylor-Green configuration for its full 400 steps (64^3 FP64,
    rk4, dt 0.005, nu 1/1600, 2/3 rule) through the solver's public API,
    against the energy/enstrophy history and final low modes produced by the
    reference's own kernels (tests/golden/make_c1_history.py)."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "tgv64_fp64_rk4_400.npz"))
    ref = z["energy_enstrophy"]
    n = 64
    s = solver((n, n, n), dt=0.005, time_integrator="rk4", viscosity=1 / 1600,
               precision="fp64", diagnostics=True)
    g = O.Grid((n, n, n))
    s.initialize(O.taylor_green(g))
    s.space_solver.step(400)
    hs = s.space_solver.history()
    assert hs.shape == ref.shape
    assert np.max(np.abs(hs - ref) / np.abs(ref)) < 1e-10
    idx = np.r_[0:4, n - 3:n]
    low = s.space_solver.u_hat[:, idx][:, :, idx][..., 0:4]
    assert rel_l2(low, z["final_low_modes"]) < 1e-9
