"""Continuous-batching request loop for many independent solves on one GPU.

Requests (a grid, a kind of run, a number of steps) arrive over time.  The
server admits a waiting request as soon as its device footprint fits the HBM
budget and a slot is free, keeps its state on the device, and advances all
admitted requests together in rounds:

* linear requests (fluctuating Stokes) go through one ensemble launch per
  round (``pf_batch_step``): all of them, of any size, in one kernel;
* nonlinear requests (Taylor-Green) each run a chunk of steps on their own
  CUDA stream, so their kernels overlap on the device; the ones running at
  once stay under a cap on their total grid points (``nl_points_cap``);

requests that finish leave at the end of the round, freeing memory and a
slot for the next arrivals.  ``mode='serial'`` is the one-at-a-time baseline:
each request is created, solved to the end and freed before the next starts.
Latency = finish - arrival; throughput = points x steps over the makespan.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .space_solver import build_config, device_footprint

KINDS = ("tgv", "thermal")


@dataclass
class Request:
    rid: int
    arrival: float       # seconds after the start of the run
    kind: str            # 'tgv' (nonlinear Taylor-Green) or 'thermal' (fluctuating Stokes)
    N: tuple
    steps: int
    seed: int = 0
    admitted: float | None = None
    finished: float | None = None
    result: np.ndarray | None = field(default=None, repr=False)

    @property
    def linear(self) -> bool:
        return self.kind == "thermal"

    @property
    def points(self) -> int:
        return int(np.prod(self.N))


# physical set-up of the two kinds of request.  Thermal runs use the implicit
# predictor-corrector: the explicit one (amplification 1 + z + z^2/2, z =
# -nu |k|^2 dt) is unstable once nu |k|^2 dt > 2, i.e. |k| > sqrt(2 / (nu dt))
# = 44.7 at nu = 0.1, dt = 0.01, which every grid from 128^2 up contains.
TGV = dict(dt=0.005, integrator="rk4", nu=1 / 1600)
THERMAL = dict(dt=0.01, integrator="implicit_pc", nu=0.1, kT=1e-3)


def _integrator_id(name):
    from .time_integrator import DICT_TIME_INTEGRATORS
    return DICT_TIME_INTEGRATORS[name].native_id


def request_config(r: Request, precision="fp32"):
    d = len(r.N)
    dom = [(0.0, 2 * np.pi)] * d
    if r.linear:
        mag = math.sqrt(2 * THERMAL["nu"] * THERMAL["kT"])
        return build_config(r.N, dom, False, _integrator_id(THERMAL["integrator"]), THERMAL["nu"],
                            "thermal", mag, False, precision, THERMAL["dt"], r.seed, "philox",
                            None, None, True)
    return build_config(r.N, dom, True, _integrator_id(TGV["integrator"]), TGV["nu"], "thermal",
                        0.0, False, precision, TGV["dt"], r.seed, "philox", None, None, True)


def make_solver(r: Request, precision="fp32"):
    """Solver with the request's initial state (Taylor-Green velocity, or rest
    for the thermal-noise runs)."""
    from .simulation import Solver
    d = len(r.N)
    if r.linear:
        s = Solver(list(r.N), THERMAL["dt"], 1.0, is_nonlinear=False,
                   time_integrator=THERMAL["integrator"], viscosity=THERMAL["nu"],
                   noise_type="thermal", noise_mag=math.sqrt(2 * THERMAL["nu"] * THERMAL["kT"]),
                   dealias="2/3", precision=precision, seed=r.seed)
        return s
    s = Solver(list(r.N), TGV["dt"], 1.0, time_integrator=TGV["integrator"], viscosity=TGV["nu"],
               dealias="2/3", precision=precision)
    x = s.space_solver.x
    u = np.zeros((d,) + tuple(r.N))
    if d == 3:
        u[0] = np.sin(x[0]) * np.cos(x[1]) * np.cos(x[2])
        u[1] = -np.cos(x[0]) * np.sin(x[1]) * np.cos(x[2])
    else:
        u[0] = np.sin(x[0]) * np.cos(x[1])
        u[1] = -np.cos(x[0]) * np.sin(x[1])
    s.initialize(u)
    # the first request of each geometry tunes the fused passes' launch
    # variants; later ones start from the library's cached picks
    key = (tuple(r.N), precision)
    if key not in _TUNED:
        s.space_solver.autotune()
        _TUNED.add(key)
    return s


_TUNED: set = set()


def poisson_requests(n, rate=50.0, seed=2, min_steps=100, max_steps=5000,
                     sizes2d=(64, 128, 256, 512, 1024), sizes3d=(32, 64, 128)):
    """Poisson arrivals; grid sides log-uniform over the built sizes; steps
    log-uniform in [min_steps, max_steps]; kinds and dimensions equally likely."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        d = 2 if rng.random() < 0.5 else 3
        side = int(rng.choice(sizes2d if d == 2 else sizes3d))
        kind = KINDS[int(rng.integers(0, 2))]
        steps = int(round(math.exp(rng.uniform(math.log(min_steps), math.log(max_steps)))))
        out.append(Request(i, t, kind, (side,) * d, steps, seed=1000 + i))
    return out


class Server:
    def __init__(self, hbm_budget=150e9, max_slots=64, chunk_nonlinear=25, chunk_linear=500,
                 precision="fp32", keep_results=False, nl_points_cap=1 << 21):
        self.budget = float(hbm_budget)
        self.max_slots = max_slots
        # grid points of the nonlinear requests running at once (None: no
        # cap).  A nonlinear request waits while the running ones and it
        # together pass the cap (one always runs); nonlinear requests keep
        # their arrival order, linear ones may pass a waiting one.  Nonlinear
        # steps of grids up to 1024^2 / 128^3 work largely out of the 126 MB
        # L2: running more of them at once evicts each other's fields (on the
        # serving mix 2^21 points gave 1.35-1.45x the serial throughput,
        # no cap 0.76-1.12x)
        self.nl_points_cap = nl_points_cap
        self.chunk_nl = chunk_nonlinear
        self.chunk_lin = chunk_linear
        self.precision = precision
        self.keep_results = keep_results

    def footprint(self, r: Request) -> int:
        return device_footprint(request_config(r, self.precision))

    # ------------------------------------------------------------------ runs
    def run(self, requests, mode="continuous"):
        import torch
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            r.admitted = r.finished = None
            r.result = None
        if mode == "serial":
            return self._run_serial(reqs, torch)
        return self._run_continuous(reqs, torch)

    def _finish(self, r, sol, t0):
        if self.keep_results:
            r.result = sol.space_solver.u_hat
        r.finished = time.perf_counter() - t0

    def _run_serial(self, reqs, torch):
        t0 = time.perf_counter()
        for r in reqs:
            wait = r.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            r.admitted = time.perf_counter() - t0
            sol = make_solver(r, self.precision)
            sol.space_solver.step(r.steps)
            torch.cuda.synchronize()
            self._finish(r, sol, t0)
            del sol
        return self._metrics(reqs, "serial")

    def _run_continuous(self, reqs, torch):
        """Event-driven continuous batching: every nonlinear request advances
        on its own stream by graph-replayed chunks and gets its next chunk as
        soon as its previous one has completed (polled with CUDA events), so
        small requests are not held back by large ones; all linear requests
        advance together as one captured ensemble graph on a stream of its
        own, re-captured at a chunk boundary when its membership changes.
        Arrivals are admitted against the memory budget and slot limit as
        they come."""
        from .ensemble import Ensemble
        t0 = time.perf_counter()
        pending = list(reqs)
        nl = []            # [request, solver, remaining, footprint, stream, event]
        lin = []           # [request, solver, remaining, footprint]
        lin_wait = []      # admitted linear requests waiting for the next chunk boundary
        ens = None
        ens_chunk = 0
        ens_event = None
        ens_stream = torch.cuda.Stream()
        used = 0

        def admit(now):
            nonlocal used
            i = 0
            nl_blocked = False
            nl_points = sum(a[0].points for a in nl)
            while i < len(pending) and pending[i].arrival <= now and \
                    len(nl) + len(lin) + len(lin_wait) < self.max_slots:
                r = pending[i]
                if not r.linear and self.nl_points_cap is not None and (
                        nl_blocked or (nl and nl_points + r.points > self.nl_points_cap)):
                    nl_blocked = True  # later nonlinear arrivals wait behind it
                    i += 1
                    continue
                fp = self.footprint(r)
                if used + fp > self.budget and (nl or lin or lin_wait):
                    break  # wait for memory to free up
                pending.pop(i)
                if not r.linear:
                    nl_points += r.points
                r.admitted = time.perf_counter() - t0
                sol = make_solver(r, self.precision)
                used += fp
                if r.linear:
                    lin_wait.append([r, sol, r.steps, fp])
                    continue
                stream = torch.cuda.Stream()
                sol.space_solver.set_stream(stream)
                torch.cuda.current_stream().synchronize()  # set-up copies done
                if r.steps >= self.chunk_nl:
                    sol.space_solver.capture(self.chunk_nl)
                a = [r, sol, r.steps, fp, stream, torch.cuda.Event()]
                launch_nl(a)
                nl.append(a)

        def launch_nl(a):
            c = min(self.chunk_nl, a[2])
            if c == self.chunk_nl:
                a[1].space_solver.replay()
            else:
                a[1].space_solver.step(c)
            a[2] -= c
            a[5].record(a[4])

        def relaunch_linear():
            nonlocal ens, ens_chunk, ens_event
            lin.extend(lin_wait)
            lin_wait.clear()
            if not lin:
                ens = None
                return
            torch.cuda.current_stream().synchronize()
            ens_chunk = min(self.chunk_lin, min(a[2] for a in lin))
            ens = Ensemble([a[1] for a in lin])
            ens.capture(ens_chunk, ens_stream)
            ens.replay()
            ens_event = torch.cuda.Event()
            ens_event.record(ens_stream)

        while pending or nl or lin or lin_wait:
            admit(time.perf_counter() - t0)
            progressed = False
            keep = []
            for a in nl:
                if not a[5].query():
                    keep.append(a)
                    continue
                progressed = True
                if a[2] == 0:
                    self._finish(a[0], a[1], t0)
                    used -= a[3]
                else:
                    launch_nl(a)
                    keep.append(a)
            nl[:] = keep
            if ens is None:
                if lin_wait:
                    relaunch_linear()
                    progressed = True
            elif ens_event.query():
                progressed = True
                for a in lin:
                    a[2] -= ens_chunk
                done = [a for a in lin if a[2] == 0]
                for a in done:
                    self._finish(a[0], a[1], t0)
                    used -= a[3]
                left = [a for a in lin if a[2] > 0]
                # a new chunk length (or membership) needs a new capture
                if done or lin_wait or (left and min(a[2] for a in left) < ens_chunk):
                    lin[:] = left
                    ens = None
                    relaunch_linear()
                else:
                    ens.replay()
                    ens_event.record(ens_stream)
            if not progressed:
                if not (nl or lin or lin_wait) and pending:
                    time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))
                else:
                    time.sleep(5e-5)
        torch.cuda.synchronize()
        return self._metrics(reqs, "continuous")

    @staticmethod
    def _metrics(reqs, mode):
        lat = np.array([r.finished - r.arrival for r in reqs])
        svc = np.array([r.finished - r.admitted for r in reqs])
        span = max(r.finished for r in reqs) - min(r.arrival for r in reqs)
        pts_steps = sum(r.points * r.steps for r in reqs)
        steps = sum(r.steps for r in reqs)
        return {"mode": mode, "requests": len(reqs), "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_service_s": float(svc.mean()), "makespan_s": float(span),
                "steps_per_s": steps / span, "mpts_steps_per_s": pts_steps / 1e6 / span}
