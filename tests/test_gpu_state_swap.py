"""The state buffers of a one-box fused solver swap roles every step: the
first stage writes the new state into the u0 buffer and the old state stays
where it is as the step's u0, instead of being copied.  The kernels and their
arithmetic are the same either way, so a run equals the same run with the
swap off (PF_STATE_SWAP=0) bit for bit -- through plain steps, the recorded
one-step graphs (one per buffer), captured graphs of odd and even length
with steps in between, state changes and the E / Z readers."""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _solver(N, kw, uh, swap):
    from periodicflow import simulation as sim
    old = os.environ.get("PF_STATE_SWAP")
    os.environ["PF_STATE_SWAP"] = "1" if swap else "0"
    try:
        s = sim.Solver(list(N), 1e-3, 1.0, **kw)
    finally:
        if old is None:
            os.environ.pop("PF_STATE_SWAP")
        else:
            os.environ["PF_STATE_SWAP"] = old
    s.initialize(uh, "fourier", project=False)
    return s


CASES = [
    # (no forcing: its band energy is an FP64 sum in any order, so runs with
    # it agree to rounding only, the swap aside)
    ("3d_fp32_rk3_cfl", (64, 64, 64),
     dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", dealias="2/3", cfl=0.5)),
    ("3d_fp64_rk4", (32, 32, 64),
     dict(time_integrator="rk4", viscosity=1e-2, precision="fp64", dealias="2/3")),
    ("3d_fp32_pad_implicit_pc_thermal", (32, 32, 32),
     dict(time_integrator="implicit_pc", viscosity=0.05, precision="fp32", dealias="3/2",
          noise_type="thermal", noise_mag=0.02, seed=3)),
    ("2d_fp32_rk3_cfl", (128, 128),
     dict(time_integrator="rk3", viscosity=1e-3, precision="fp32", dealias="2/3", cfl=0.5)),
    ("2d_fp64_explicit_pc_nyquist", (64, 128),
     dict(time_integrator="explicit_pc", viscosity=1e-2, precision="fp64", dealias="2/3",
          mask_nyquist=True)),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_swapped_buffers_equal_in_place(case):
    name, N, kw = case
    g = O.Grid(N)
    uh = O.spectral_random_field(g, 12)
    a = _solver(N, kw, uh, True)
    b = _solver(N, kw, uh, False)
    for s in (a, b):
        s.space_solver.step(1)       # odd number of plain steps: a's state in its u0 buffer
        s.space_solver.step(4)       # recorded graphs of both buffers (noise-free cases)
        s.space_solver.step(3)
    assert np.array_equal(a.space_solver.u_hat, b.space_solver.u_hat)
    assert a.space_solver.time() == b.space_solver.time()
    # E and Z are FP64 sums over blocks in any order: equal to rounding
    ea, eb = a.space_solver.energy(), b.space_solver.energy()
    assert np.allclose(ea, eb, rtol=1e-13, atol=0.0)
    uh2 = O.spectral_random_field(g, 13)
    for s in (a, b):
        s.initialize(uh2, "fourier")  # writes the current buffer, projects
        s.space_solver.step(2)
    assert np.array_equal(a.space_solver.u_hat, b.space_solver.u_hat)


@pytest.mark.parametrize("nsteps", [3, 4])
def test_swapped_buffers_captured_graph(nsteps):
    """Graphs of odd and even length replayed with plain steps in between."""
    import torch
    N = (64, 64, 64)
    kw = dict(time_integrator="rk3", viscosity=2e-3, precision="fp32", dealias="2/3", cfl=0.5)
    uh = O.spectral_random_field(O.Grid(N), 14)
    a = _solver(N, kw, uh, True)
    b = _solver(N, kw, uh, False)
    st = torch.cuda.Stream()
    a.space_solver.set_stream(st)
    a.space_solver.step(1)
    a.space_solver.capture(nsteps)
    a.space_solver.replay()
    a.space_solver.step(1)           # leaves the state in the other buffer
    a.space_solver.replay()          # moves it back first
    a.space_solver.replay()
    st.synchronize()
    b.space_solver.step(2 + 3 * nsteps)
    assert np.array_equal(a.space_solver.u_hat, b.space_solver.u_hat)
