"""Realisations (pf_create_members): many nonlinear boxes of one configuration
advanced by one launch per fused pass must equal the same boxes solved one at
a time.

A member runs the arithmetic of its single solver, but in separately compiled
kernels (the member offsets are compile-time), whose multiply-add contraction
may differ; the band-energy sum of the forcing is an FP64 atomic sum in any
order.  Members therefore agree with their single solvers to rounding:
relative L2 1e-6 in FP32, 1e-13 in FP64.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _single(N, dt, kw, uh, steps, seed=0):
    from periodicflow import simulation as sim
    s = sim.Solver(list(N), dt, 1.0, seed=seed, **kw)
    s.initialize(uh, "fourier")
    s.space_solver.step(steps)
    t, _, d = s.space_solver.time()
    return s.space_solver.u_hat, t, d


CASES = [
    # id, N, members, solver keywords, steps
    ("3d_fp32_rk3_forcing_cfl", (32, 32, 32), 3,
     dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp32",
          forcing=(0.1, 2.5), cfl=0.5), 4),
    ("3d_fp32_rk4", (32, 16, 64), 4,
     dict(time_integrator="rk4", viscosity=1e-2, dealias="2/3", precision="fp32"), 3),
    ("3d_fp64_rk3_cfl", (32, 32, 32), 2,
     dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp64", cfl=0.5), 3),
    ("3d_fp32_pad_implicit_pc", (16, 32, 32), 2,
     dict(time_integrator="implicit_pc", viscosity=1e-2, dealias="3/2", precision="fp32"), 3),
    ("3d_fp64_pad_rk3", (16, 16, 32), 2,
     dict(time_integrator="rk3", viscosity=1e-2, dealias="3/2", precision="fp64"), 2),
    ("3d_fp32_three_pow2", (48, 48, 96), 2,
     dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp32", cfl=0.5), 2),
    ("3d_fp32_256_line", (32, 32, 256), 3,
     dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp32", cfl=0.5,
          forcing=(0.1, 2.5)), 2),
    ("2d_fp32_rk3_forcing_cfl", (64, 64), 5,
     dict(time_integrator="rk3", viscosity=1e-3, dealias="2/3", precision="fp32",
          forcing=(0.1, 2.5), cfl=0.5), 5),
    ("2d_fp64_rk4", (128, 64), 3,
     dict(time_integrator="rk4", viscosity=1e-3, dealias="2/3", precision="fp64"), 4),
    ("2d_fp32_512", (512, 512), 2,
     dict(time_integrator="rk3", viscosity=1e-3, dealias="2/3", precision="fp32", cfl=0.5), 3),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_members_equal_single_solvers(case):
    from periodicflow.ensemble import Realisations
    name, N, M, kw, steps = case
    dt = 1e-3
    g = O.Grid(N)
    ics = [O.spectral_random_field(g, 11 + m) for m in range(M)]
    R = Realisations(N, dt, M, **kw)
    for m, uh in enumerate(ics):
        R.set_state(m, uh)
    R.project()
    R.step(steps)
    got = R.states()
    tol = 1e-6 if kw["precision"] == "fp32" else 1e-13
    for m, uh in enumerate(ics):
        ref, t, d = _single(N, dt, kw, uh, steps)
        assert np.array_equal(got[m], R.state(m))
        err = rel_l2(got[m], ref)
        assert err <= tol, (m, err)
        tm, dm = R.time(m)
        assert abs(tm - t) <= max(tol, 1e-15) * t and abs(dm - d) <= max(tol, 1e-15) * d
        e, z = R.energy(m)
        eo, zo = O.energy(g, ref), O.enstrophy(g, ref)
        assert abs(e - eo) <= 1e-5 * eo and abs(z - zo) <= 1e-5 * zo


def test_members_philox_noise_seed_per_member():
    """Member m draws with key seed + m: equal to a solver created with it."""
    from periodicflow.ensemble import Realisations
    N, M, base = (32, 32, 32), 3, 40
    kw = dict(time_integrator="implicit_pc", viscosity=0.05, dealias="2/3", precision="fp32",
              noise_type="thermal", noise_mag=0.02)
    g = O.Grid(N)
    ics = [O.spectral_random_field(g, 21 + m) for m in range(M)]
    R = Realisations(N, 1e-3, M, seed=base, **kw)
    for m, uh in enumerate(ics):
        R.set_state(m, uh)
    R.project()
    R.step(3)
    for m, uh in enumerate(ics):
        ref, _, _ = _single(N, 1e-3, kw, uh, 3, seed=base + m)
        assert rel_l2(R.state(m), ref) < 1e-6, m


def test_members_vs_oracle():
    """A member against the FP64 oracle (forcing + CFL, FP32, 1e-5)."""
    from periodicflow.ensemble import Realisations
    N, M = (64, 32, 32), 3
    g = O.Grid(N)
    R = Realisations(N, 1e-3, M, time_integrator="rk3", viscosity=2e-3, dealias="2/3",
                     precision="fp32", forcing=(0.1, 2.5), cfl=0.5)
    ics = [O.spectral_random_field(g, 31 + m) for m in range(M)]
    for m, uh in enumerate(ics):
        R.set_state(m, uh)
    R.step(2)
    for m in (0, M - 1):
        o = O.OracleSolver(N, 1e-3, time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5),
                           cfl=0.5)
        o.initialize(ics[m], "fourier", project=False)
        o.advance(2)
        assert rel_l2(R.state(m), o.u_hat) < 1e-5


def test_members_graph_replay_and_autotune():
    import torch
    from periodicflow.ensemble import Realisations
    N, M = (32, 32, 64), 4
    kw = dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp32", cfl=0.5)
    g = O.Grid(N)
    ics = [O.spectral_random_field(g, 41 + m) for m in range(M)]
    a = Realisations(N, 1e-3, M, **kw)
    b = Realisations(N, 1e-3, M, **kw)
    for m, uh in enumerate(ics):
        a.set_state(m, uh)
        b.set_state(m, uh)
    before = a.states()
    a.autotune()
    assert np.array_equal(a.states(), before)
    st = torch.cuda.Stream()
    a.set_stream(st)
    a.capture(3)
    a.replay()
    a.replay()
    st.synchronize()
    b.step(6)
    assert np.array_equal(a.states(), b.states())
    assert a.steps == 6


def test_members_api_errors():
    from periodicflow.ensemble import Realisations
    with pytest.raises(NotImplementedError):  # linear ensembles go through pf_batch
        _linear_members()
    R = Realisations((16, 16, 16), 1e-3, 2, dealias="2/3", time_integrator="rk3")
    with pytest.raises(IndexError):
        R.state(2)
    assert R.footprint() > 0


def _linear_members():
    from periodicflow import _native as N
    from periodicflow.space_solver import build_config
    import ctypes as C
    cfg = build_config((16, 16), [(0, 6.283), (0, 6.283)], False, N.PF_IMPLICIT_PC, 0.1,
                       "thermal", 0.0, False, "fp32", 1e-3, 0, "philox", None, None, True)
    h = C.c_void_p()
    N.check(N.lib().pf_create_members(C.byref(cfg), 2, C.byref(h)), None, "pf_create_members")


@pytest.mark.parametrize("N", [(32, 32, 32), (64, 64)])
def test_active_members_and_copy(N):
    """Only members [0, active) advance; a finished member's slot is refilled
    by copying the last active member (state, time, dt) into it."""
    from periodicflow.ensemble import Realisations
    kw = dict(time_integrator="rk3", viscosity=2e-3, dealias="2/3", precision="fp32", cfl=0.5)
    g = O.Grid(N)
    ics = [O.spectral_random_field(g, 51 + m) for m in range(4)]
    R = Realisations(N, 1e-3, 4, **kw)
    for m, uh in enumerate(ics):
        R.set_state(m, uh)
    R.project()                    # as Solver.initialize does
    R.step(2)                      # all four
    R.set_active(2)
    parked = [R.state(2), R.state(3)]
    t3 = R.time(3)
    R.step(3)                      # members 0, 1 only
    assert np.array_equal(R.state(2), parked[0]) and np.array_equal(R.state(3), parked[1])
    assert R.time(3) == t3
    for m in (0, 1):
        ref, t, d = _single(N, 1e-3, kw, ics[m], 5)
        assert rel_l2(R.state(m), ref) < 1e-6
        assert abs(R.time(m)[0] - t) < 1e-6 * t
    # member 1 leaves; member 3 (parked after 2 steps) takes its slot and joins
    R.copy_member(1, 3)
    assert np.array_equal(R.state(1), parked[1]) and R.time(1) == t3
    R.set_member_time(0, 0.25, 2e-3)
    assert R.time(0) == (0.25, 2e-3)
    R.step(2)
    ref, _, _ = _single(N, 1e-3, kw, ics[3], 4)
    assert rel_l2(R.state(1), ref) < 1e-6
