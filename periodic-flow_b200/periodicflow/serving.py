"""Continuous-batching request loop for many independent solves on one GPU.

Requests (a grid, a kind of run, a number of steps) arrive over time.  The
server admits a waiting request as soon as its device footprint fits the HBM
budget and a slot is free, keeps its state on the device, and advances all
admitted requests together in rounds:

* linear requests (fluctuating Stokes) go through one ensemble launch per
  round (``pf_batch_step``): all of them, of any size, in one kernel;
* nonlinear requests (Taylor-Green) of one grid share a pool: a
  ``Realisations`` handle whose fused passes are one launch over every
  request in it; pools run chunks of steps on their own CUDA streams, so
  their kernels overlap on the device, under a cap on the grid points of the
  chunks in flight (``nl_points_cap``);

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
    started: float | None = None   # first chunk (a pool's join) or admission (linear)
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


def tgv_spectrum(N):
    """Normalised half spectrum of the Taylor-Green velocity (u = sin x cos y
    cos z, v = -cos x sin y cos z, w = 0; in 2D u = sin x cos y, v = -cos x
    sin y) on [0, 2 pi)^d: the sampled field's forward transform, which has
    only the modes |k_i| = 1, written directly."""
    d = len(N)
    shape = (d,) + tuple(N[:-1]) + (N[-1] // 2 + 1,)
    uh = np.zeros(shape, dtype=np.complex128)
    if d == 3:
        for s0 in (1, -1):
            for s1 in (1, -1):
                uh[0, s0 % N[0], s1 % N[1], 1] = -0.125j * s0
                uh[1, s0 % N[0], s1 % N[1], 1] = 0.125j * s1
    else:
        for s0 in (1, -1):
            uh[0, s0 % N[0], 1] = -0.25j * s0
            uh[1, s0 % N[0], 1] = 0.25j
    return uh


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
    s.initialize(tgv_spectrum(r.N), "fourier")
    # the first request of each geometry tunes the fused passes' launch
    # variants; later ones start from the library's cached picks
    key = (tuple(r.N), precision)
    if key not in _TUNED:
        s.space_solver.autotune()
        _TUNED.add(key)
    return s


_TUNED: set = set()


class Pool:
    """Nonlinear requests of one grid advancing together: a Realisations
    handle of `cap` slots on its own stream.  Occupied slots are [0, active);
    a request joins at slot `active`; one that finishes leaves by moving the
    last occupied slot into its place.  Every chunk of steps is one launch
    sequence over all occupied slots."""

    def __init__(self, N, cap, precision, torch):
        from .ensemble import Realisations
        self.N = tuple(N)
        self.cap = cap
        self.R = Realisations(self.N, TGV["dt"], cap, time_integrator=TGV["integrator"],
                              viscosity=TGV["nu"], dealias="2/3", precision=precision)
        key = (self.N, precision)
        if key not in _TUNED:
            self.R.autotune()
            _TUNED.add(key)
        self.stream = torch.cuda.Stream()
        self.R.set_stream(self.stream)
        self.event = torch.cuda.Event()
        self.slots = []      # [request, remaining steps] of slots 0 .. active-1
        self.waiting = []    # admitted requests joining at the next chunk boundary
        self.chunk = 0       # steps of the chunk in flight (0: idle)
        self.ic = tgv_spectrum(self.N)

    def free(self) -> int:
        return self.cap - len(self.slots) - len(self.waiting)

    def points(self) -> int:
        return len(self.slots) * int(np.prod(self.N))

    def absorb(self):
        """Waiting requests take the next slots (between chunks only: the
        uploads are ordered on the pool's stream)."""
        for r in self.waiting:
            m = len(self.slots)
            self.R.set_state(m, self.ic)
            self.R.set_member_time(m, 0.0, TGV["dt"])
            self.slots.append([r, r.steps])
        self.waiting.clear()

    def launch(self, chunk_max, now):
        if not self.slots:
            self.chunk = 0
            return
        for a in self.slots:
            if a[0].started is None:
                a[0].started = now
        self.R.set_active(len(self.slots))
        self.chunk = min(chunk_max, min(a[1] for a in self.slots))
        self.R.step(self.chunk)
        self.event.record(self.stream)

    def collect(self, keep_results):
        """After a chunk: the requests that finished (their results read out
        when wanted), their slots refilled from the end."""
        done = []
        for a in self.slots:
            a[1] -= self.chunk
        m = 0
        while m < len(self.slots):
            if self.slots[m][1] == 0:
                r = self.slots[m][0]
                if keep_results:
                    r.result = self.R.state(m)
                done.append(r)
                last = len(self.slots) - 1
                if m != last:
                    self.R.copy_member(m, last)
                    self.slots[m] = self.slots[last]
                self.slots.pop()
            else:
                m += 1
        self.chunk = 0
        return done


def poisson_requests(n, rate=50.0, seed=2, min_steps=100, max_steps=5000,
                     sizes2d=(64, 128, 256, 512, 1024), sizes3d=(32, 48, 64, 96, 128, 192)):
    """Poisson arrivals; grid sides log-uniform over the built sizes (2D:
    powers of two 64..1024; 3D: the ladder 32..192 of 2^b and 3 * 2^b sides,
    ratios 1.5 and 4/3); steps log-uniform in [min_steps, max_steps]; kinds
    and dimensions equally likely."""
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
                 precision="fp32", keep_results=False, nl_points_cap=1 << 24,
                 pool_points=1 << 24, max_members=64):
        self.budget = float(hbm_budget)
        self.max_slots = max_slots
        # a pool of nonlinear requests of one grid holds up to pool_points
        # grid points (at most max_members requests)
        self.pool_points = int(pool_points)
        self.max_members = int(max_members)
        # grid points of the nonlinear chunks in flight at once (None: no
        # cap); a pool waits while the running ones and it together pass the
        # cap (one always runs).  Without batching, concurrent requests of
        # grids up to 1024^2 / 128^3 evicted each other's fields from the 126
        # MB L2 (on the serving mix 2^21 points gave 1.35-1.45x the serial
        # throughput, no cap 0.76-1.12x); pools stream their members through
        # HBM in one launch, so the cap is per chunk of all members.
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
            r.admitted = r.started = r.finished = None
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
            r.admitted = r.started = time.perf_counter() - t0
            sol = make_solver(r, self.precision)
            sol.space_solver.step(r.steps)
            torch.cuda.synchronize()
            self._finish(r, sol, t0)
            del sol
        return self._metrics(reqs, "serial")

    def pool_cap(self, r: Request) -> int:
        """Slots of a new pool for r's grid: up to pool_points grid points in
        all, at most max_members."""
        return int(max(1, min(self.max_members, self.pool_points // r.points)))

    def _run_continuous(self, reqs, torch):
        """Event-driven continuous batching.  Nonlinear requests of one grid
        share a pool (one Realisations handle on its own stream) and advance
        together, one launch sequence per chunk over all occupied slots; a
        request joins its pool at the next chunk boundary and leaves at the
        one where its steps are done.  Pools run concurrently and each gets
        its next chunk as soon as a CUDA event shows the previous one done.
        All linear requests advance together as one captured ensemble graph on
        a stream of its own, re-captured at a chunk boundary when its
        membership changes.  Arrivals are admitted against the memory budget
        (a pool counts its full capacity) and the slot limit as they come."""
        from .ensemble import Ensemble, Realisations
        t0 = time.perf_counter()
        pending = list(reqs)
        pools = {}         # grid -> Pool
        lin = []           # [request, solver, remaining, footprint]
        lin_wait = []      # admitted linear requests waiting for the next chunk boundary
        ens = None
        ens_chunk = 0
        ens_event = None
        ens_stream = torch.cuda.Stream()
        used = 0

        def busy():
            return any(p.slots or p.waiting for p in pools.values()) or lin or lin_wait

        def pool_for(r):
            nonlocal used
            p = pools.get(r.N)
            if p is not None:
                return p if p.free() > 0 else None
            cap = self.pool_cap(r)
            fp = Realisations.footprint_of(request_config(r, self.precision), cap)
            if used + fp > self.budget and busy():
                return None
            used += fp
            p = Pool(r.N, cap, self.precision, torch)
            pools[r.N] = p
            return p

        def admit(now):
            nonlocal used
            i = 0
            while i < len(pending) and pending[i].arrival <= now:
                r = pending[i]
                if not r.linear:
                    p = pool_for(r)
                    if p is None:
                        i += 1  # pool full or no memory yet: wait
                        continue
                    pending.pop(i)
                    r.admitted = time.perf_counter() - t0
                    p.waiting.append(r)
                    continue
                if len(lin) + len(lin_wait) >= self.max_slots:
                    i += 1
                    continue
                fp = self.footprint(r)
                if used + fp > self.budget and busy():
                    break  # wait for memory to free up
                pending.pop(i)
                r.admitted = r.started = time.perf_counter() - t0
                lin_wait.append([r, make_solver(r, self.precision), r.steps, fp])
                used += fp

        def running_points():
            return sum(p.points() for p in pools.values() if p.chunk)

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

        while pending or busy():
            admit(time.perf_counter() - t0)
            progressed = False
            for p in pools.values():
                if p.chunk and p.event.query():
                    now = time.perf_counter() - t0
                    for r in p.collect(self.keep_results):
                        r.finished = now
                    progressed = True
            # idle pools with work start their next chunk, within the cap on
            # the grid points of nonlinear chunks in flight (one always runs)
            for p in pools.values():
                if p.chunk or not (p.slots or p.waiting):
                    continue
                p.absorb()
                run = running_points()
                if self.nl_points_cap is not None and run and run + p.points() > self.nl_points_cap:
                    continue
                p.launch(self.chunk_nl, time.perf_counter() - t0)
                progressed = True
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
                if not busy() and pending:
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
