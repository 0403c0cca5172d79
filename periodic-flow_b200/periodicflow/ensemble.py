"""Ensembles of independent linear (fluctuating Stokes) realisations.

The reference runs one realisation per process (simulation.py:189-225).  Here
many ``Solver`` objects of mixed grid sizes and dimensions (linear runs:
``is_nonlinear=False``, Philox or no noise) advance together: one kernel
launch per call covers every member and every step, and a fixed number of
steps can be captured once as a CUDA graph and replayed.
"""
from __future__ import annotations

import ctypes as C

from . import _native as N


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
