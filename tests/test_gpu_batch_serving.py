"""Ensembles (one launch for many linear boxes) and the continuous-batching
server: every result equals the same solve run alone."""
import math

import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu

KT, NU = 1e-3, 0.1


def stokes(N, seed, integ="implicit_pc", noise_type="thermal", precision="fp32", C=None,
           dt=0.02):
    """Explicit schemes need nu |k|^2 dt below their stability limit (~2)."""
    from periodicflow import simulation as sim
    s = sim.Solver(list(N), dt, 1.0, is_nonlinear=False, time_integrator=integ, viscosity=NU,
                   noise_type=noise_type, noise_mag=math.sqrt(2 * NU * KT), dealias="2/3",
                   precision=precision, seed=seed)
    if C is not None:
        s.set_correlation_function(C)
    return s


@pytest.mark.parametrize("precision,integ,dt", [("fp32", "implicit_pc", 0.02),
                                               ("fp64", "implicit_pc", 0.02),
                                               ("fp32", "explicit_pc", 0.001),
                                               ("fp64", "rk3", 0.001)])
def test_ensemble_equals_individual_solves(precision, integ, dt):
    from periodicflow.ensemble import Ensemble
    sizes = [(64, 64), (128, 128), (32, 32, 32), (128, 128), (16, 16, 16)]
    a = [stokes(N, 10 + i, integ, precision=precision, dt=dt) for i, N in enumerate(sizes)]
    b = [stokes(N, 10 + i, integ, precision=precision, dt=dt) for i, N in enumerate(sizes)]
    ens = Ensemble(a)
    ens.step(40)
    ens.step(10)
    for s in b:
        s.space_solver.step(50)
    for x, y in zip(a, b):
        assert rel_l2(x.space_solver.u_hat, y.space_solver.u_hat) < 1e-6
        tx, sx, _ = x.space_solver.time()
        ty, sy, _ = y.space_solver.time()
        assert sx == sy == 50 and tx == ty


def test_ensemble_graph_replay_and_correlated_noise():
    from periodicflow.ensemble import Ensemble
    sizes = [(128, 128), (256, 256), (64, 64, 64)]
    Cs = [np.exp(-O.Grid(N).k2 / 64.0) for N in sizes]  # exp(-(k/8)^2)
    a = [stokes(N, i, "implicit_pc", "correlated", C=C) for i, (N, C) in enumerate(zip(sizes, Cs))]
    b = [stokes(N, i, "implicit_pc", "correlated", C=C) for i, (N, C) in enumerate(zip(sizes, Cs))]
    ens = Ensemble(a)
    ens.capture(25)
    for _ in range(3):
        ens.replay()
    ens.synchronize()
    for s in b:
        s.space_solver.step(75)
    for x, y in zip(a, b):
        assert rel_l2(x.space_solver.u_hat, y.space_solver.u_hat) < 1e-6
        assert x.space_solver.time()[1] == 75 and x.step == 75


@pytest.mark.parametrize("N", [(32, 32, 32), (64, 64)])
def test_graph_replay_equals_stepping(N):
    import torch
    from periodicflow import simulation as sim
    from periodicflow.serving import Request, make_solver
    r = Request(0, 0.0, "tgv", N, 30)
    a, b = make_solver(r), make_solver(r)
    st = torch.cuda.Stream()
    a.space_solver.set_stream(st)
    a.space_solver.capture(10)
    for _ in range(3):
        a.space_solver.replay()
    b.space_solver.step(30)
    torch.cuda.synchronize()
    assert rel_l2(a.space_solver.u_hat, b.space_solver.u_hat) == 0.0
    assert a.space_solver.time()[1] == 30
    noisy = stokes((32, 32), 1)
    noisy.space_solver.set_stream(st)
    with pytest.raises(NotImplementedError):
        noisy.space_solver.capture(5)


def test_ensemble_rejects_nonlinear_members():
    from periodicflow import simulation as sim
    from periodicflow.ensemble import Ensemble
    s = sim.Solver([32, 32], 0.01, 1.0, dealias="2/3")
    with pytest.raises(NotImplementedError):
        Ensemble([s])


def test_served_results_equal_alone():
    from periodicflow.serving import Request, Server
    reqs = [Request(0, 0.00, "thermal", (64, 64), 120, seed=1),
            Request(1, 0.00, "tgv", (32, 32, 32), 60),
            Request(2, 0.01, "thermal", (32, 32, 32), 90, seed=2),
            Request(3, 0.02, "tgv", (64, 64), 80),
            Request(4, 0.02, "thermal", (128, 128), 300, seed=3),
            Request(5, 0.03, "tgv", (16, 16, 16), 40)]
    srv = Server(chunk_nonlinear=15, chunk_linear=50, keep_results=True)
    m = srv.run(reqs, "continuous")
    mixed = {r.rid: r.result for r in reqs}
    assert m["requests"] == 6 and m["p99_latency_s"] >= m["p50_latency_s"] > 0
    srv.run(reqs, "serial")
    for r in reqs:
        assert rel_l2(mixed[r.rid], r.result) < 1e-6, r


def test_nonlinear_points_cap():
    """With the cap at one request's points, the pool of one grid (requests 0
    and 3, batched together) runs alone: the other grid's pool starts after
    it is done, a linear request passes both, and results equal the serial
    run's."""
    from periodicflow.serving import Request, Server
    reqs = [Request(0, 0.0, "tgv", (32, 32, 32), 60),
            Request(1, 0.0, "tgv", (64, 64), 60),
            Request(2, 0.0, "thermal", (64, 64), 100, seed=1),
            Request(3, 0.0, "tgv", (32, 32, 32), 40)]
    srv = Server(chunk_nonlinear=15, chunk_linear=50, keep_results=True,
                 nl_points_cap=32 ** 3)
    m = srv.run(reqs, "continuous")
    assert m["requests"] == 4
    mixed = {r.rid: r.result for r in reqs}
    assert reqs[3].started == reqs[0].started  # one pool, one chunk
    assert reqs[1].started >= reqs[0].finished
    assert reqs[2].started < reqs[0].finished
    srv.run(reqs, "serial")
    for r in reqs:
        assert rel_l2(mixed[r.rid], r.result) < 1e-6, r


def test_pool_join_and_leave_equal_alone():
    """Requests of one grid arriving at different times with different step
    counts share a pool: they join at chunk boundaries and leave as they
    finish (the last occupied slot moves into the freed one); each result
    equals the request solved alone."""
    from periodicflow.serving import Request, Server
    reqs = [Request(0, 0.000, "tgv", (32, 32, 32), 60),
            Request(1, 0.005, "tgv", (32, 32, 32), 45),
            Request(2, 0.010, "tgv", (32, 32, 32), 17),
            Request(3, 0.020, "tgv", (32, 32, 32), 75),
            Request(4, 0.020, "tgv", (64, 64), 50),
            Request(5, 0.030, "tgv", (64, 64), 33),
            Request(6, 0.040, "tgv", (32, 32, 32), 20)]
    srv = Server(chunk_nonlinear=10, keep_results=True)
    m = srv.run(reqs, "continuous")
    assert m["requests"] == 7
    mixed = {r.rid: r.result for r in reqs}
    srv.run(reqs, "serial")
    for r in reqs:
        assert rel_l2(mixed[r.rid], r.result) < 1e-6, r


def test_admission_respects_budget():
    from periodicflow.serving import Request, Server
    reqs = [Request(i, 0.0, "thermal", (128, 128), 20, seed=i) for i in range(4)]
    srv = Server(chunk_linear=10)
    one = srv.footprint(reqs[0])
    srv.budget = 2 * one  # at most two resident at a time
    m = srv.run(reqs, "continuous")
    assert m["requests"] == 4
    admitted = sorted(r.admitted for r in reqs)
    finished = sorted(r.finished for r in reqs)
    assert admitted[2] >= finished[0]  # the third waited for memory


def test_kernel_timer_inside_captured_graph():
    """With the per-launch timer on, pf_graph_capture records its events as
    graph nodes: one replay of the captured steps times every launch of the
    pass (three RK3 stages per step), and the state equals plain stepping."""
    import ctypes as C
    import torch
    from periodicflow import _native as N
    from periodicflow import simulation as sim
    import oracle as O
    Nn = (64, 64, 64)
    uh = O.spectral_random_field(O.Grid(Nn), 2)
    kw = dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp32", cfl=0.5)
    a = sim.Solver(list(Nn), 1e-3, 1.0, **kw)
    b = sim.Solver(list(Nn), 1e-3, 1.0, **kw)
    a.initialize(uh, "fourier")
    b.initialize(uh, "fourier")
    st = torch.cuda.Stream()
    ss = a.space_solver
    ss.set_stream(st)
    lib = N.lib()
    N.check(lib.pf_kernel_timer(ss._h, N.PF_PASS_FUSED[5]), ss._h, "timer")
    ss.capture(4)
    ss.replay()
    st.synchronize()
    tot, cnt = C.c_double(), C.c_longlong()
    N.check(lib.pf_kernel_timer_read(ss._h, C.byref(tot), C.byref(cnt)), ss._h, "timer read")
    assert cnt.value == 12 and tot.value > 0.0
    b.space_solver.step(4)
    assert np.array_equal(ss.u_hat, b.space_solver.u_hat)
