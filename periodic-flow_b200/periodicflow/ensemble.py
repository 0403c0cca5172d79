"""Ensembles of independent realisations.

The reference runs one realisation per process (simulation.py:189-225).
Here:

* ``Ensemble``: many linear (fluctuating Stokes) ``Solver`` objects of mixed
  grid sizes and dimensions (Philox or no noise) advance together: one kernel
  launch per call covers every member and every step, and a fixed number of
  steps can be captured once as a CUDA graph and replayed;
* ``Realisations``: many nonlinear realisations of one configuration whose
  fused passes each run as one launch over all members.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N

_nat = N  # for code whose grid argument is named N


class Ensemble:
    def __init__(self, solvers):
        self.solvers = list(solvers)
        handles = (C.c_void_p * len(self.solvers))(
            *[s.space_solver._h.value for s in self.solvers])
        b = C.c_void_p()
        N.check(N.lib().pf_batch_create(handles, len(self.solvers), C.byref(b)), None,
                "pf_batch_create")
        self._b = b
        self._stream = None
        self._graph_steps = 0

    def __del__(self):
        b = getattr(self, "_b", None)
        if b:
            try:
                N.lib().pf_batch_destroy(b)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._b = None

    def _check(self, rc, what):
        if rc != N.PF_OK:
            msg = N.lib().pf_batch_last_error(self._b)
            raise N.NativeError(f"{what} failed (status {rc}): {msg.decode() if msg else ''}")

    def _advance_hosts(self, nsteps):
        for s in self.solvers:
            dt = s.time_integrator.dt
            for _ in range(nsteps):
                s.t += dt
            s.step += nsteps

    def step(self, nsteps: int):
        """Advance every member ``nsteps`` steps (one launch, synchronous)."""
        self._check(N.lib().pf_batch_step(self._b, int(nsteps)), "pf_batch_step")
        self._advance_hosts(int(nsteps))

    def capture(self, nsteps: int, stream=None):
        """Record "advance ``nsteps``" as a CUDA graph on ``stream`` (a
        torch.cuda.Stream; one is created when omitted)."""
        import torch
        self._stream = stream or torch.cuda.Stream()
        self._check(N.lib().pf_batch_set_stream(self._b, C.c_void_p(self._stream.cuda_stream)),
                    "pf_batch_set_stream")
        self._check(N.lib().pf_batch_capture(self._b, int(nsteps)), "pf_batch_capture")
        self._graph_steps = int(nsteps)

    def replay(self):
        """Launch the captured graph (asynchronous on the capture stream)."""
        self._check(N.lib().pf_batch_replay(self._b), "pf_batch_replay")
        self._advance_hosts(self._graph_steps)

    def synchronize(self):
        self._check(N.lib().pf_batch_sync(self._b), "pf_batch_sync")


class Realisations:
    """``count`` realisations of one nonlinear configuration in one launch per pass.

    The reference runs one realisation per process (simulation.py:189-225).
    Here the states of ``count`` boxes of one configuration -- the keyword
    arguments of ``Solver`` (grid, dt, integrator, viscosity, noise, domain,
    dealias, precision, seed, forcing, cfl) -- sit one after another on the
    device, and every fused pass of a stage is a single kernel launch over all
    of them (C-ABI ``pf_create_members``).  Each member keeps its own dt (CFL),
    time and forcing-band energy; member ``m`` draws Philox noise with key
    ``seed + m``, so it equals a ``Solver`` created with that seed.
    ``step(n)`` replays a recorded one-step CUDA graph for
    noise-free runs, as a single solver does.
    """

    def __init__(self, N, dt: float, count: int, *, time_integrator: str = "rk2",
                 viscosity: float = 1e-3, noise_type: str = "thermal", noise_mag: float = 0.0,
                 domain=2 * math.pi, dealias: str = "3/2", mask_nyquist: bool = False,
                 precision: str = "fp32", seed: int = 0, forcing=None, cfl=None):
        from . import _comm
        from .basis import FourierSpace
        from .space_solver import build_config
        from .time_integrator import DICT_TIME_INTEGRATORS
        if time_integrator not in DICT_TIME_INTEGRATORS:
            raise ValueError(f"Time integrator '{time_integrator}' not found.")
        space = FourierSpace(_comm.COMM_WORLD, 0, list(N), domain=domain, dealias=dealias,
                             mask_nyquist=mask_nyquist)
        self.N = tuple(space.N)
        self.dim = len(self.N)
        self.shape_spectral = space.shape_spectral
        self.count = int(count)
        self._cfg = build_config(self.N, space.domain, True,
                                 DICT_TIME_INTEGRATORS[time_integrator].native_id, viscosity,
                                 noise_type, noise_mag, mask_nyquist, precision, dt, seed,
                                 "philox", forcing, cfl, True, dealias=space.dealias_rule)
        h = C.c_void_p()
        _nat.check(_nat.lib().pf_create_members(C.byref(self._cfg), self.count, C.byref(h)),
                   None, "pf_create_members")
        self._h = h
        self.steps = 0
        self.active = self.count

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().pf_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._h = None

    @staticmethod
    def footprint_of(cfg, count: int) -> int:
        """Device bytes of ``count`` members of the pf_config ``cfg``."""
        b = C.c_ulonglong()
        N.check(N.lib().pf_footprint_members(C.byref(cfg), int(count), C.byref(b)), None,
                "pf_footprint_members")
        return int(b.value)

    def footprint(self) -> int:
        return self.footprint_of(self._cfg, self.count)

    def _member(self, m):
        if not 0 <= m < self.count:
            raise IndexError(f"member {m} of {self.count}")
        return int(m)

    def set_state(self, m: int, u_hat):
        """Spectral state of member m (complex, (dim,) + spectral shape)."""
        a = np.ascontiguousarray(np.broadcast_to(u_hat, (self.dim,) + self.shape_spectral),
                                 dtype=np.complex128)
        N.check(N.lib().pf_set_fourier_member(self._h, self._member(m), a.ctypes.data, 0),
                self._h, "set member state")

    def state(self, m: int) -> np.ndarray:
        out = np.empty((self.dim,) + self.shape_spectral, dtype=np.complex128)
        N.check(N.lib().pf_get_fourier_member(self._h, self._member(m), out.ctypes.data, 0),
                self._h, "get member state")
        return out

    def states(self) -> np.ndarray:
        out = np.empty((self.count, self.dim) + self.shape_spectral, dtype=np.complex128)
        N.check(N.lib().pf_get_fourier(self._h, out.ctypes.data, 0), self._h, "get states")
        return out

    def project(self):
        """Leray projection of every member's state (Solver.initialize(project=True))."""
        N.check(N.lib().pf_project(self._h), self._h, "project")

    def step(self, nsteps: int):
        N.check(N.lib().pf_step(self._h, int(nsteps)), self._h, "step")
        self.steps += int(nsteps)

    def time(self, m: int = 0):
        """(t, dt) of member m."""
        t, dt = C.c_double(), C.c_double()
        N.check(N.lib().pf_get_time_member(self._h, self._member(m), C.byref(t), C.byref(dt)),
                self._h, "member time")
        return t.value, dt.value

    def set_time(self, t: float, step: int = 0):
        N.check(N.lib().pf_set_time(self._h, float(t), int(step)), self._h, "set_time")

    def energy(self, m: int = 0):
        e, z = C.c_double(), C.c_double()
        N.check(N.lib().pf_energy_member(self._h, self._member(m), C.byref(e), C.byref(z)),
                self._h, "member energy")
        return e.value, z.value

    def set_active(self, active: int):
        """Advance only members [0, active) from now on (continuous batching)."""
        N.check(N.lib().pf_set_active_members(self._h, int(active)), self._h, "set_active")
        self.active = int(active)

    def copy_member(self, dst: int, src: int):
        """Member src's state, time and dt onto member dst (on the device)."""
        N.check(N.lib().pf_copy_member(self._h, self._member(dst), self._member(src)), self._h,
                "copy_member")

    def set_member_time(self, m: int, t: float, dt: float):
        N.check(N.lib().pf_set_time_member(self._h, self._member(m), float(t), float(dt)),
                self._h, "set_member_time")

    def autotune(self) -> dict:
        picks = (C.c_int * 12)()
        N.check(N.lib().pf_autotune(self._h, picks), self._h, "autotune")
        return {"axes_256": list(picks[:6]), "axes_384": list(picks[6:])}

    def set_stream(self, stream):
        ptr = getattr(stream, "cuda_stream", stream)
        N.check(N.lib().pf_set_stream(self._h, C.c_void_p(ptr) if ptr else None), self._h,
                "set_stream")

    def capture(self, nsteps: int):
        """Record "advance ``nsteps``" as a CUDA graph (set a stream first)."""
        N.check(N.lib().pf_graph_capture(self._h, int(nsteps)), self._h, "graph capture")
        self._graph_steps = int(nsteps)

    def replay(self):
        N.check(N.lib().pf_graph_replay(self._h), self._h, "graph replay")
        self.steps += self._graph_steps
