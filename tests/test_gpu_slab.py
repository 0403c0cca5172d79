"""Slab decomposition of one box (pf_slab_*, periodicflow.slab) against the
whole-box solver and the FP64 oracle.

The slabs of a group live on one device; their exchanges are the same
stores into the destination slab's buffers that a one-slab-per-GPU run sends
over NVLink, so a group checks the decomposition's arithmetic and data
movement.  A slab advances the arithmetic of the whole-box fused schedule in
separately compiled kernels (multiply-add contraction may differ) and sums
the forcing band energy over the slabs in another order: agreement is to
rounding, relative L2 1e-6 in FP32 and 1e-13 in FP64.

The one-slab-per-process form runs here with one rank (its NCCL communicator,
barriers and reductions on one GPU); runs over several GPUs need a GPU per
rank.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-6, "fp64": 1e-13}

CASES = [
    # id, N, slabs, solver keywords, steps
    ("fp64_rk3_forcing_cfl_s2", (32, 32, 32), 2,
     dict(time_integrator="rk3", viscosity=2e-3, precision="fp64", forcing=(0.1, 2.5), cfl=0.5), 3),
    ("fp32_rk3_cfl_s4", (32, 32, 32), 4,
     dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", cfl=0.5), 3),
    ("fp32_rk4_s2", (64, 32, 48), 2,
     dict(time_integrator="rk4", viscosity=1e-2, precision="fp32"), 2),
    ("fp32_three_pow2_s2", (48, 48, 96), 2,
     dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", cfl=0.5), 2),
    ("fp64_implicit_pc_thermal_s2", (32, 16, 32), 2,
     dict(time_integrator="implicit_pc", viscosity=0.05, precision="fp64", noise_type="thermal",
          noise_mag=0.02, seed=9), 3),
    ("fp32_explicit_pc_nyquist_s8", (64, 64, 64), 8,
     dict(time_integrator="explicit_pc", viscosity=1e-2, precision="fp32", mask_nyquist=True), 2),
    ("fp32_rk2_forcing_s4", (128, 64, 128), 4,
     dict(time_integrator="rk2", viscosity=2e-3, precision="fp32", forcing=(0.1, 2.5)), 2),
    ("fp32_256cubed_rk3_s2", (256, 256, 256), 2,
     dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", cfl=0.5), 1),
]


def _whole(N, dt, kw, uh, steps):
    from periodicflow import simulation as sim
    kw = dict(kw)
    seed = kw.pop("seed", 0)
    s = sim.Solver(list(N), dt, 1.0, dealias="2/3", seed=seed, **kw)
    s.initialize(uh, "fourier", project=False)
    s.space_solver.step(steps)
    t, n, d = s.space_solver.time()
    return s.space_solver.u_hat, (t, n, d), s.space_solver


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_slab_group_equals_whole_box(case):
    from periodicflow.slab import SlabGroup
    name, N, S, kw, steps = case
    dt = 1e-3
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 5)
    G = SlabGroup(N, dt, S, **kw)
    G.set_state(uh)
    assert np.array_equal(G.state(), uh.astype(np.complex64 if kw["precision"] == "fp32"
                                                 else np.complex128).astype(np.complex128))
    G.step(steps)
    ref, (t, n, d), ss = _whole(N, dt, kw, uh, steps)
    got = G.state()
    tol = TOL[kw["precision"]]
    assert rel_l2(got, ref) <= tol, rel_l2(got, ref)
    tg, ng, dg = G.time()
    assert ng == n == steps
    assert abs(tg - t) <= max(tol, 1e-15) * t and abs(dg - d) <= max(tol, 1e-15) * d
    e, z = G.energy()
    eo, zo = O.energy(g, ref), O.enstrophy(g, ref)
    assert abs(e - eo) <= 1e-5 * eo and abs(z - zo) <= 1e-5 * zo


def test_slab_group_vs_oracle_fp64():
    """Four slabs, FP64, forcing and CFL dt, two RK3 steps: within 1e-11 of the oracle."""
    from periodicflow.slab import SlabGroup
    N = (32, 32, 32)
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 7)
    G = SlabGroup(N, 1e-3, 4, time_integrator="rk3", viscosity=2e-3, precision="fp64",
                  forcing=(0.1, 2.5), cfl=0.5)
    G.set_state(uh)
    G.step(2)
    o = O.OracleSolver(N, 1e-3, time_integrator="rk3", viscosity=2e-3, forcing=(0.1, 2.5),
                       cfl=0.5)
    o.initialize(uh, "fourier", project=False)
    o.advance(2)
    assert rel_l2(G.state(), o.u_hat) < 1e-11


def test_slab_group_fp32_256cubed_vs_oracle():
    """The headline box in two slabs against the FP64 oracle (one RK3 step, 1e-5)."""
    from periodicflow.slab import SlabGroup
    N = (256, 256, 256)
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 1)
    G = SlabGroup(N, 1e-3, 2, time_integrator="rk3", viscosity=2e-3, precision="fp32")
    G.set_state(uh)
    G.step(1)
    o = O.OracleSolver(N, 1e-3, time_integrator="rk3", viscosity=2e-3)
    o.initialize(uh, "fourier", project=False)
    o.advance(1)
    assert rel_l2(G.state(), o.u_hat) < 1e-5


def test_slab_solver_one_rank_through_nccl():
    """The one-slab-per-process form with one rank: IPC export, NCCL
    communicator, barriers and reductions; equals the whole box."""
    from periodicflow.slab import SlabSolver
    N = (32, 32, 32)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp64", forcing=(0.1, 2.5),
              cfl=0.5)
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 3)
    s = SlabSolver(N, 1e-3, **kw)
    assert s.slabs == 1 and s.rank == 0
    s.set_local_state(uh)
    s.step(3)
    ref, (t, n, d), _ = _whole(N, 1e-3, kw, uh, 3)
    assert rel_l2(s.local_state(), ref) <= 1e-13
    assert s.time()[1] == 3
    s.close()


def test_slab_group_graph_replay_equals_plain_steps():
    """step(n >= 2) of a noise-free group replays one recorded step."""
    from periodicflow.slab import SlabGroup
    N = (64, 32, 32)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", forcing=(0.1, 2.5),
              cfl=0.5)
    uh = O.spectral_random_field(O.Grid(N), 8)
    a, b = SlabGroup(N, 1e-3, 2, **kw), SlabGroup(N, 1e-3, 2, **kw)
    a.set_state(uh)
    b.set_state(uh)
    for _ in range(4):
        a.step(1)
    b.step(2)
    b.step(2)
    assert np.array_equal(a.state(), b.state())
    assert a.time() == b.time()


def test_slab_group_local_layout():
    """Slab r holds rows k1 in [r n1/S, (r+1) n1/S) of the whole-box array."""
    from periodicflow.slab import SlabGroup, slab_layout
    N, S = (32, 64, 32), 4
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 2)
    G = SlabGroup(N, 1e-3, S, time_integrator="rk3", precision="fp64")
    G.set_state(uh)
    for r in range(S):
        L = slab_layout(N, S, r)
        k0, w = L["k1_first"], L["n1_per_slab"]
        assert np.array_equal(G.slab_state(r), uh[:, :, k0:k0 + w, :])


def test_slab_api_errors():
    from periodicflow.slab import SlabGroup
    with pytest.raises(ValueError):
        SlabGroup((32, 48, 32), 1e-3, 5)             # 5 does not divide the sides
    with pytest.raises(NotImplementedError):
        SlabGroup((32, 32, 32), 1e-3, 2, noise_type="correlated", noise_mag=0.1)
    with pytest.raises(NotImplementedError):
        SlabGroup((32, 32), 1e-3, 2)                  # 2D
    G = SlabGroup((32, 32, 32), 1e-3, 2)
    with pytest.raises(ValueError):
        G.set_state(np.zeros((3, 32, 16, 17), dtype=np.complex128))
