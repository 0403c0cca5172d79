#!/usr/bin/env python
"""Benchmark of the periodicflow B200 backend.

Workload (N=1): 3D forced isotropic turbulence on a 256^3 box, FP32, TVD RK3
with CFL 0.5, linear band forcing (|k| <= 2.5, eps = 0.1), nu = 2e-3, 2/3
dealiasing, random solenoidal initial field E(k) ~ k^4 exp(-2 (k/4)^2) (seed 1),
synthetic (no dataset is involved).  One step = one full RK3 time step (three
stages) on the device.  Metric: Mpts * RK-steps / s = 256^3 / 1e6 * steps / s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank advances its own
independent box (seed 1 + rank): weak scaling, no data-path collective; the
time is the max over ranks.  ``--impl reference`` times the CPU oracle (the
FP64 NumPy/SciPy restatement of the reference's path) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "periodic-flow_b200"))

METRIC = "Mpts*RK-steps/s at 256^3 FP32"
UNIT = "Mpts*steps/s"

CFG = dict(n=256, nu=2e-3, integrator="rk3", cfl=0.5, forcing=(0.1, 2.5), seed=1, dt0=1e-3)

# Algorithmic bytes per launch of each timed pass, in units of one FP32 complex
# half-spectrum field U = n0 n1 (n2/2+1) 8 B, for the 2/3-rule fused schedule
# (c = 2 kmax + 1 kept indices of a complex axis, c2 = kmax + 1 of the last one).


def pass_bytes(n):
    nh = n // 2 + 1
    kmax = (n - 1) // 3
    c1, c2 = 2 * kmax + 1, kmax + 1
    cb = 8
    U = n * n * nh * cb
    return {
        "P1": (3 * c1 * c1 * c2 + 5 * n * c1 * c2) * cb,
        "P2": (5 * n * c1 * c2 + 6 * n * n * c2) * cb,
        "P3": (6 * n * n * c2) * cb + 3 * U,
        "P4": 6 * U,
        # nl (3) + u_hat (3) + u0 (3) read, u_hat (3) written; RK3's first
        # stage reads no u0 and writes the new state into the u0 buffer (the
        # state buffers swap roles): 9 U, mean over the three stages 11 U
        "P5": 11 * U,
        "U": U,
    }


# DRAM bytes (read + write) per launch at n = 256 from one ncu --set full
# capture per kernel of k_p3 / k_p5 (default launch forms) under
# "bench.py --mode case --n 256 --steps 2".
NCU_TRAFFIC_256 = {3: 270.720256e6 + 161.286400e6, 5: 608.809472e6 + 171.203072e6}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        lr = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(lr)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", lr))
        return dist, dist.get_rank(), ws
    return None, 0, 1


class ClockSampler:
    """SM clock, power and clock-event reasons during the timed region, read
    (never set) through NVML every 5 ms from a thread -- the timed region can
    be a few tens of ms -- or, without the NVML bindings, from nvidia-smi
    every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.gpu)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            nv = None
        if nv is not None:
            self.stop_flag = threading.Event()

            def poll():
                while not self.stop_flag.is_set():
                    try:
                        reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    except Exception:
                        reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                    self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), smax,
                                      nv.nvmlDeviceGetPowerUsage(h) / 1e3, reasons))
                    time.sleep(0.005)
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join()
            rows = self.rows
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
            reasons = sorted({k for r in rows for k, b in self.REASONS.items() if r[3] & b})
            return {"sm_mhz": float(np.median([r[0] for r in rows])),
                    "sm_max_mhz": float(max(r[1] for r in rows)), "reasons": reasons,
                    "samples": len(rows), "source": "nvml, every 5 ms",
                    "power_w_max": float(max(r[2] for r in rows))}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")
        sm = np.array([num(r[1]) for r in rows])
        smax = np.array([num(r[2]) for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.nanmedian(sm)), "sm_max_mhz": float(np.nanmax(smax)),
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, every 200 ms",
                "power_w_max": float(np.nanmax([num(r[3]) for r in rows]))}


def initial_field(n, seed):
    """Product-side initial field (host NumPy set-up)."""
    from periodicflow import _comm
    from periodicflow.basis import FourierSpace
    from periodicflow.initial import spectral_random_field
    return spectral_random_field(FourierSpace(_comm.COMM_WORLD, 0, [n] * 3, dealias="2/3"), seed)


def oracle_initial_field(n, seed):
    import oracle as O
    return O.spectral_random_field(O.Grid((n, n, n)), seed)


def make_solver(n, precision="fp32", dealias="2/3", fused=True):
    from periodicflow import simulation as sim
    return sim.Solver([n] * 3, CFG["dt0"], 1.0, time_integrator=CFG["integrator"],
                      viscosity=CFG["nu"], dealias=dealias, precision=precision,
                      forcing=CFG["forcing"], cfl=CFG["cfl"], fused=fused)


def run_ours(args, dist, rank, world):
    import torch
    from periodicflow import _native as N
    import ctypes as C
    n = args.n
    dev = torch.cuda.current_device()
    uh0 = initial_field(n, CFG["seed"] + rank)
    pad = args.dealias == "3/2"
    sol = make_solver(n, dealias=args.dealias)
    ss = sol.space_solver
    ss.initialize_velocity(uh0, "fourier")
    # launch variants of the fused passes picked by the library's autotuner
    variants = ss.autotune() if not args.no_autotune else ss.fused_variants()
    ss.step(args.warmup)
    torch.cuda.synchronize()
    lib = N.lib()
    # The K timed steps are captured as one CUDA graph (outside the timed
    # region) and replayed once.  The per-launch times of the dominant pass
    # come from a second replay of K steps captured with that pass's timer
    # inside as event nodes (which add gaps between the launches, so the
    # whole-step time is not taken from it).
    stream = torch.cuda.Stream()
    ss.set_stream(stream)
    dominant = N.PF_PASS_FUSED[args.timed_pass]
    ss.capture(args.steps)
    # ------------------------------------------------------------ timed region
    c0 = C.c_longlong()
    lib.pf_launch_count(C.byref(c0))
    clocks = ClockSampler(dev)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record()
        ss.replay()
        ev1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ck = clocks.stop()
    c1 = C.c_longlong()
    lib.pf_launch_count(C.byref(c1))
    ms = ev0.elapsed_time(ev1)
    # ------------------------------------------- per-launch time of the pass
    N.check(lib.pf_kernel_timer(ss._h, dominant), ss._h, "timer")
    ss.capture(args.steps)
    with torch.cuda.stream(stream):
        ss.replay()
    torch.cuda.synchronize()
    tot_ms, nl = C.c_double(), C.c_longlong()
    N.check(lib.pf_kernel_timer_read(ss._h, C.byref(tot_ms), C.byref(nl)), ss._h, "timer")
    lib.pf_kernel_timer(ss._h, -1)
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    pts = n ** 3 / 1e6
    value = world * pts * args.steps / (ms / 1e3)
    _, _, dt_now = ss.time()
    # ---------------------------------------------------------------- roofline
    pb = padded_pass_bytes(n) if pad else pass_bytes(n)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    avg_s = tot_ms.value / max(nl.value, 1) / 1e3
    alg = pb[f"P{args.timed_pass}"]
    achieved = alg / avg_s / 1e9 if avg_s > 0 else None
    traffic, traffic_src = args.traffic, "--traffic"
    if traffic is None and n == 256 and not pad and args.timed_pass in NCU_TRAFFIC_256:
        traffic, traffic_src = NCU_TRAFFIC_256[args.timed_pass], "ncu capture at 256^3"
    roofline = {"bound": "hbm", "kernel": f"fused pass P{args.timed_pass}",
                "achieved": achieved, "peak": peak, "peak_source": peak_src, "unit": "GB/s",
                "frac": achieved / peak if achieved else None,
                "traffic": traffic, "traffic_source": traffic_src if traffic else None,
                "alg_bytes_per_launch": alg,
                "avg_launch_ms": avg_s * 1e3, "launches_timed": nl.value}
    step_bytes = 3 * sum(pb[f"P{i}"] for i in range(1, 6))
    step_model = "75.5 U per stage (3/2 fused schedule)" if pad else "33.4 U per stage"
    step_roof = {"alg_bytes_per_step": step_bytes, "model": step_model,
                 "achieved_gbs": step_bytes / (ms / args.steps / 1e3) / 1e9 * 1.0,
                 "frac": step_bytes / (ms / args.steps / 1e3) / 1e9 / peak}
    if not pad:
        # the five-pass model without the 2/3 rule's truncation (every pass
        # reads and writes whole fields): 46 U per stage
        full = 3 * 46 * pb["U"]
        step_roof["untruncated_model"] = "46 U per stage (whole fields in every pass)"
        step_roof["frac_untruncated"] = full / (ms / args.steps / 1e3) / 1e9 / peak
    # --------------------------------------------------------------------- e2e
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, uh0, rank, dist, args.dealias)
    # ------------------------------------------------------------ cpu baseline
    cpu = None
    check = None
    if rank == 0 and world == 1 and not args.no_cpu and not pad:
        cpu, oracle_state = cpu_baseline(n, args.cpu_steps, uh0)
        check = oracle_check(n, uh0, oracle_state, args.cpu_steps)
        del oracle_state
        check["config2_stokes_256sq"] = {
            "workload": "2D thermal Stokes 256^2, explicit PC dt 0.01, injected NumPy noise "
                        "(seed 0), 10 steps, relative L2 vs FP64 oracle",
            "fp32_rel_l2": oracle_check_stokes("fp32"), "fp64_rel_l2": oracle_check_stokes("fp64")}
    ensemble = None
    if rank == 0 and not args.no_ensemble and not pad:
        ensemble = run_ensemble(args)
    nlbatch = None
    if rank == 0 and not args.no_nlbatch and not pad:
        nlbatch = run_batched_nonlinear(args)
    slabs = None
    if rank == 0 and not args.no_slab and not pad:
        slabs = run_slab_group(args, uh0)
    served = None
    if rank == 0 and not args.no_serving and not pad:
        served = run_serving(args)
    padded = None
    if rank == 0 and not args.no_padded and not pad:
        padded = run_padded(args, uh0, peak)
    fp64 = None
    if rank == 0 and not args.no_fp64 and not pad:
        fp64 = run_fp64(args, uh0)
    cufft = None
    if rank == 0 and not args.no_cufft and not pad:
        cufft = run_cufft_comparison(args, uh0)
        cufft["fused_speedup"] = cufft["ms_per_step"] / (ms / args.steps)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32", "data": "synthetic",
            "config": {"workload": f"3D forced isotropic turbulence {n}^3, RK3 CFL 0.5, "
                                   f"linear forcing |k|<=2.5 eps=0.1, nu=2e-3, {args.dealias} dealias"
                                   + (f" (padded transforms of {3 * n // 2} points)" if pad else ""),
                       "grid": [n, n, n], "integrator": "rk3", "replicas_per_gpu": 1,
                       "parallelism": f"replicas x{world} (one box per GPU)",
                       "l2": "working set > L2 (state 3x67.6 MB + intermediates)",
                       "timed_launch": f"{args.steps} steps captured as one CUDA graph, replayed once; "
                                       "the roofline pass's launch times from a second such "
                                       "replay with timer event nodes",
                       "launch_variants": variants,
                       "autotuned": not args.no_autotune,
                       "dt_after_run": dt_now},
            "gpu_launches": int(c1.value - c0.value),
            "clocks": ck, "roofline": roofline, "step_roofline": step_roof,
            "e2e": e2e, "cpu_baseline": cpu, "oracle_check": check,
            "batched": ensemble, "batched_nonlinear": nlbatch, "served": served,
            "slab_group": slabs,
            "padded_3_2": padded,
            "cufft_comparison": cufft, "fp64": fp64,
        }
        print(json.dumps(line), flush=True)


def run_e2e(args, uh0, rank, dist, dealias="2/3"):
    """Same metric through the public API with host buffers: upload the state
    from pinned host memory, then per step one step and an E, Z read-back,
    then download the final state; copies inside the timed region."""
    import torch
    n = args.n
    pinned = torch.empty(uh0.shape, dtype=torch.complex128, pin_memory=True)
    pinned.numpy()[...] = uh0
    host_in = pinned.numpy()
    out_pinned = torch.empty(uh0.shape, dtype=torch.complex128, pin_memory=True)
    sol = make_solver(n, dealias=dealias)
    ss = sol.space_solver
    ss.initialize_velocity(host_in, "fourier")
    ss.step(args.warmup)
    torch.cuda.synchronize()
    import ctypes as C
    from periodicflow import _native as N
    K = args.e2e_steps
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    ss.initialize_velocity(host_in, "fourier")
    ez = []
    for _ in range(K):
        ss.step(1)
        ez.append(ss.energy())
    N.check(N.lib().pf_get_fourier(ss._h, C.c_void_p(out_pinned.data_ptr()), 0), ss._h, "get")
    t1 = time.perf_counter()
    sec = t1 - t0
    if dist:
        t = torch.tensor([sec], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
    world = dist.get_world_size() if dist else 1
    state_b = int(np.prod(uh0.shape)) * 16
    return {"value": world * n ** 3 / 1e6 * K / sec, "unit": UNIT, "steps": K,
            "h2d_bytes_per_step": state_b / K, "d2h_bytes_per_step": (state_b + 16 * K) / K,
            "note": "one whole run of the configuration's length: state upload (complex128), "
                    "then per step pf_step(1) + E,Z read-back (16 B), then state download; "
                    "wall clock"}


def ensemble_members(scale=1.0, precision="fp32"):
    """Configuration 4: 128 x 128^2 + 32 x 256^2 (2D) + 8 x 64^3 (3D) correlated
    fluctuating Stokes realisations, C(k) = exp(-(k/8)^2), seeds 0..167,
    implicit predictor-corrector, dt = 0.02 (nu = 0.1, kT = 1e-3)."""
    import math
    from periodicflow import simulation as sim
    sizes = ([(128, 128)] * max(1, int(128 * scale)) + [(256, 256)] * max(1, int(32 * scale))
             + [(64, 64, 64)] * max(1, int(8 * scale)))
    nu, kT = 0.1, 1e-3
    out = []
    for seed, N in enumerate(sizes):
        s = sim.Solver(list(N), 0.02, 1.0, is_nonlinear=False, time_integrator="implicit_pc",
                       viscosity=nu, noise_type="correlated", noise_mag=math.sqrt(2 * nu * kT),
                       dealias="2/3", precision=precision, seed=seed)
        s.set_correlation_function(np.exp(-s.space_solver.k2 / 64.0))
        out.append(s)
    return out


def cufft_step_factory(n, uh0, dev="cuda"):
    """The headline step written with torch.fft (cuFFT) and torch element-wise
    kernels, for comparison only: 2/3 mask, curl, inverse transforms,
    u x omega, forward transform, Leray projection, viscous term, band forcing,
    CFL time step and the TVD RK3 stage rule -- the oracle's arithmetic in
    FP32 on the GPU, with no fusion."""
    import torch
    nh = n // 2 + 1
    ki = torch.fft.fftfreq(n, d=1.0 / n, device=dev)
    kl = torch.arange(nh, device=dev, dtype=torch.float32)
    k = [ki.view(n, 1, 1).expand(n, n, nh), ki.view(1, n, 1).expand(n, n, nh),
         kl.view(1, 1, nh).expand(n, n, nh)]
    k = torch.stack(k).to(torch.float32)
    k2 = (k * k).sum(0)
    kok2 = k / torch.where(k2 == 0, torch.ones_like(k2), k2)
    keep = ((3 * k.abs()) < n).all(0).to(torch.float32)
    band = ((k2 > 0) & (k2 <= CFG["forcing"][1] ** 2)).to(torch.float32)
    w = torch.full((nh,), 2.0, device=dev)
    w[0] = 1.0
    w[-1] = 1.0
    eps, nu, cfl = CFG["forcing"][0], CFG["nu"], CFG["cfl"]
    dxinv = n / (2 * np.pi)
    ab = ((0.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0))
    uh = torch.from_numpy(uh0).to(dev).to(torch.complex64)

    def curl(v):
        return 1j * torch.stack([k[1] * v[2] - k[2] * v[1], k[2] * v[0] - k[0] * v[2],
                                 k[0] * v[1] - k[1] * v[0]])

    def step(uh):
        u0 = uh
        dt = None
        for s_, (a, b) in enumerate(ab):
            um = uh * keep
            u = torch.fft.irfftn(um, s=(n, n, n), dim=(1, 2, 3), norm="forward")
            om = torch.fft.irfftn(curl(um), s=(n, n, n), dim=(1, 2, 3), norm="forward")
            if s_ == 0:
                dt = cfl / (u.abs().sum(0) * dxinv).max()
            c = torch.stack([u[1] * om[2] - u[2] * om[1], u[2] * om[0] - u[0] * om[2],
                             u[0] * om[1] - u[1] * om[0]])
            nl = torch.fft.rfftn(c, dim=(1, 2, 3), norm="forward")
            nl = nl - k * (kok2 * nl).sum(0, keepdim=True)
            ef = 0.5 * (w * band * (uh.abs() ** 2).sum(0)).sum()
            f = (eps / (2 * ef)) * band * uh
            uh = a * u0 + b * (uh + dt * (nl - nu * k2 * uh + f))
        return uh

    return step, uh


def run_cufft_comparison(args, uh0):
    """torch.fft (cuFFT) step vs the fused path: time K steps each, and the
    agreement of the two states after 5 steps from the same initial field."""
    import torch
    n = args.n
    step, uh = cufft_step_factory(n, uh0)
    k = args.cufft_steps
    for _ in range(2):
        uh = step(uh)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(k):
        uh = step(uh)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / k
    # agreement: 5 steps each from uh0
    step, ua = cufft_step_factory(n, uh0)
    for _ in range(5):
        ua = step(ua)
    sol = make_solver(n)
    sol.space_solver.initialize_velocity(uh0, "fourier")
    sol.space_solver.step(5)
    ub = sol.space_solver.u_hat
    ua = ua.cpu().numpy()
    rel = float(np.linalg.norm(ua - ub) / np.linalg.norm(ub))
    del sol
    torch.cuda.empty_cache()
    return {"workload": "the headline step with torch.fft (cuFFT) and torch element-wise ops, "
                        "FP32, unfused (comparison only; not a product path)",
            "ms_per_step": ms, "value": n ** 3 / 1e6 / (ms / 1e3), "unit": UNIT,
            "steps": k, "rel_l2_vs_fused_after_5_steps": rel}


def padded_pass_bytes(n):
    """Algorithmic bytes per launch of each pass of the fused 3/2 schedule
    (t = 3n/2; see padded_stage_bytes)."""
    nh = n // 2 + 1
    t = 3 * n // 2
    cb = 8
    U = n * n * nh * cb
    A = 5 * t * n * nh * cb
    B = 6 * t * t * nh * cb
    NL = 3 * t * t * nh * cb
    F = 3 * t * n * nh * cb
    # P5: mean over RK3's stages (the first writes the new state, reads no u0)
    return {"P1": 3 * U + A, "P2": A + B, "P3": B + NL, "P4": NL + F, "P5": F + 8 * U, "U": U}


def padded_stage_bytes(n):
    """Algorithmic bytes per stage of the fused 3/2 schedule (t = 3n/2):
    P1 u_hat (3 U) in, A (5 t n nh) out; P2 A in, B (6 t^2 nh) out; P3 B in,
    nl (3 t^2 nh) out; P4 nl in, folded (3 t n nh) out; P5 that in, u_hat and
    u0 in, u_hat out (the first RK3 stage reads no u0: 75.5 U per stage on
    average)."""
    nh = n // 2 + 1
    t = 3 * n // 2
    cb = 8
    U = n * n * nh * cb
    A = 5 * t * n * nh * cb
    B = 6 * t * t * nh * cb
    NL = 3 * t * t * nh * cb
    F = 3 * t * n * nh * cb
    return (3 * U + A) + (A + B) + (B + NL) + (NL + F) + (F + 8 * U)


def run_fp64(args, uh0):
    """The headline workload in FP64 (the reference's precision) through the
    fused FP64 schedule, and the FP32 state's error against it after the same
    steps from the same initial field (both runs step-by-step identical in
    dt: the CFL step is taken in each precision)."""
    import torch
    n = args.n
    k = args.fp64_steps
    out = {"workload": f"{n}^3 headline workload in FP64 (fused FP64 schedule)"}
    states = {}
    for prec in ("fp64", "fp32"):
        sol = make_solver(n, precision=prec)
        ss = sol.space_solver
        ss.initialize_velocity(uh0, "fourier")
        ss.step(3)  # warm-up: first launches (module loading) and the step graph's recording
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ss.step(k)
        e1.record()
        torch.cuda.synchronize()
        if prec == "fp64":
            ms = e0.elapsed_time(e1) / k
            out["ms_per_step"] = ms
            out["value"] = n ** 3 / 1e6 / (ms / 1e3)
            out["unit"] = UNIT
        states[prec] = ss.u_hat
        del ss, sol
        torch.cuda.synchronize()
    a, b = states["fp32"], states["fp64"]
    out["steps"] = k
    out["warmup_steps"] = 3
    out["fp32_rel_l2_vs_fp64"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return out


def run_padded(args, uh0, peak):
    """The reference's default dealias rule (3/2 padding) on the headline
    workload: fused padded passes, with the generic padded path beside it."""
    import torch
    n = args.n
    out = {"workload": f"{n}^3 FP32 RK3 CFL 0.5, forcing as the headline, 3/2 padding "
                       f"(transforms of {3 * n // 2} points)"}
    for key, fused in (("fused", True), ("generic", False)):
        sol = make_solver(n, dealias="3/2", fused=fused)
        ss = sol.space_solver
        ss.initialize_velocity(uh0, "fourier")
        if fused and not args.no_autotune:
            out["launch_variants"] = ss.autotune()
        ss.step(2)
        torch.cuda.synchronize()
        k = args.padded_steps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ss.step(k)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / k
        out[f"{key}_ms_per_step"] = ms
        out[f"{key}_value"] = n ** 3 / 1e6 / (ms / 1e3)
        del ss, sol
        torch.cuda.synchronize()
    step_bytes = 3 * padded_stage_bytes(n)
    out["unit"] = UNIT
    out["alg_bytes_per_step"] = step_bytes
    out["fused_frac_of_hbm"] = step_bytes / (out["fused_ms_per_step"] / 1e3) / 1e9 / peak
    out["speedup_fused_vs_generic"] = out["generic_ms_per_step"] / out["fused_ms_per_step"]
    return out


def run_ensemble(args):
    """Batched (one graph-captured launch for all realisations and steps) vs
    the plain path: the same realisations solved one at a time (Solver.solve
    per realisation; and a per-step loop, pf_step(1) per step, on a sample)."""
    import torch
    from periodicflow.ensemble import Ensemble
    steps = args.ens_steps
    plain = ensemble_members(args.ens_scale)
    batch = ensemble_members(args.ens_scale)
    pts = sum(int(np.prod(s.space_solver.N)) for s in plain)
    nreal = len(plain)
    torch.cuda.synchronize()
    # plain, whole solves one after the other
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in plain:
        s.space_solver.step(steps)
    e1.record()
    torch.cuda.synchronize()
    plain_s = e0.elapsed_time(e1) / 1e3
    probe = (0, nreal // 2, nreal - 1)
    plain_states = {i: plain[i].space_solver.u_hat for i in probe}
    # plain, stepwise loop (one time step per call) on a sample of steps
    samp = min(steps, args.ens_stepwise_sample)
    t0 = time.perf_counter()
    for s in plain:
        for _ in range(samp):
            s.space_solver.step(1)
    torch.cuda.synchronize()
    stepwise_s = (time.perf_counter() - t0) * steps / samp
    # batched: capture once, replay once
    ens = Ensemble(batch)
    ens.capture(steps)
    torch.cuda.synchronize()
    e0.record(ens._stream)
    ens.replay()
    e1.record(ens._stream)
    ens.synchronize()
    batch_s = e0.elapsed_time(e1) / 1e3
    check = max(float(np.linalg.norm(batch[i].space_solver.u_hat - plain_states[i])
                      / np.linalg.norm(plain_states[i])) for i in probe)
    return {"workload": f"{nreal} correlated-noise Stokes realisations (2D 128^2, 2D 256^2, "
                        f"3D 64^3), implicit PC, {steps} steps",
            "realisations": nreal, "steps": steps,
            "batched_s": batch_s, "plain_s": plain_s, "plain_stepwise_s_est": stepwise_s,
            "batched_realisation_steps_per_s": nreal * steps / batch_s,
            "plain_realisation_steps_per_s": nreal * steps / plain_s,
            "batched_mpts_steps_per_s": pts * steps / 1e6 / batch_s,
            "plain_mpts_steps_per_s": pts * steps / 1e6 / plain_s,
            "speedup_vs_plain": plain_s / batch_s, "speedup_vs_stepwise": stepwise_s / batch_s,
            "max_rel_diff_batched_vs_plain": check,
            "stepwise_sample_steps": samp}


def run_serving(args):
    """The serving configuration (continuous batching vs one request at a
    time through the public API), and a mix of small requests only, where a
    single solve leaves most of the GPU idle.  serial_in_service is the sum of
    the serial requests' service times (set-up included) over the serial
    makespan."""
    from periodicflow.serving import Request, Server, poisson_requests

    def warm(reqs):
        # one short request per distinct (grid, kind): the kernels' first
        # launches (module loading) happen before either timed run
        seen = {}
        for r in reqs:
            seen.setdefault((r.N, r.kind), r)
        return [Request(i, 0.0, r.kind, r.N, 60, seed=r.seed) for i, r in enumerate(seen.values())]

    def one(reqs, label):
        kw = {} if args.serve_nl_points is None else {"nl_points_cap": args.serve_nl_points or None}
        srv = Server(hbm_budget=150e9, **kw)
        srv.run(warm(reqs), "continuous")
        srv.run(warm(reqs), "serial")
        cont = srv.run(reqs, "continuous")
        ser = srv.run(reqs, "serial")
        busy = sum(r.finished - r.admitted for r in reqs) / ser["makespan_s"]  # serial run's times
        return {"workload": label, "continuous": cont, "serial": ser,
                "serial_in_service": busy,
                "throughput_ratio": cont["mpts_steps_per_s"] / ser["mpts_steps_per_s"],
                "p50_ratio": ser["p50_latency_s"] / cont["p50_latency_s"],
                "p99_ratio": ser["p99_latency_s"] / cont["p99_latency_s"]}

    reqs = poisson_requests(args.serve_requests, rate=50.0, seed=2,
                            max_steps=args.serve_max_steps)
    out = one(reqs, f"{len(reqs)} Poisson requests (50/s, seed 2): 2D 64^2-1024^2 and 3D "
                    f"32^3-192^3 log-uniform, Taylor-Green or thermal noise, "
                    f"100-{args.serve_max_steps} steps, 150 GB budget")
    small = poisson_requests(120, rate=200.0, seed=3, min_steps=100, max_steps=2000,
                             sizes2d=(64, 128, 256), sizes3d=(16, 32, 64))
    out["small_requests"] = one(small, "120 Poisson requests (200/s, seed 3): 2D 64^2-256^2 and "
                                       "3D 16^3-64^3, Taylor-Green or thermal noise, 100-2000 steps")
    return out


def run_case(args):
    """One solver of the forced-turbulence configuration on a grid of side
    args.n in args.dim dimensions (FP32, 2/3 rule, RK3, CFL 0.5, band
    forcing, seed-1 field) advanced args.steps steps with the library's
    default launch forms: the command profiles are captured on."""
    import torch
    from periodicflow import _comm, simulation as sim
    from periodicflow.basis import FourierSpace
    from periodicflow.initial import spectral_random_field
    torch.cuda.set_device(0)
    N = [args.n] * args.dim
    s = sim.Solver(N, CFG["dt0"], 1.0, time_integrator=CFG["integrator"], viscosity=CFG["nu"],
                   dealias="2/3", precision="fp32", forcing=CFG["forcing"], cfl=CFG["cfl"])
    uh = spectral_random_field(FourierSpace(_comm.COMM_WORLD, 0, N, dealias="2/3"), CFG["seed"])
    s.space_solver.initialize_velocity(uh, "fourier")
    s.space_solver.step(args.steps)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "case", "grid": N, "steps": args.steps,
                      "launch_variants": s.space_solver.fused_variants()}), flush=True)


def run_batched_nonlinear(args):
    """Realisations of a nonlinear configuration in one launch per fused pass
    (pf_create_members) against the same boxes solved one at a time through
    the plain solver (its one-step graph replayed per step), from the same
    random initial fields; aggregate Mpts*steps/s, CUDA events."""
    import torch
    from periodicflow import _comm, simulation as sim
    from periodicflow.basis import FourierSpace
    from periodicflow.ensemble import Realisations
    from periodicflow.initial import spectral_random_field
    out = {}
    cases = [("2D Taylor-Green-like random fields 256^2, RK4 dt 0.005, nu 1/1600, FP32",
              (256, 256), 64, args.nlb_steps),
             ("3D random fields 64^3, RK4 dt 0.005, nu 1/1600, FP32", (64, 64, 64), 32,
              args.nlb_steps // 2)]
    for label, N, M, steps in cases:
        kw = dict(time_integrator="rk4", viscosity=1 / 1600, dealias="2/3", precision="fp32")
        space = FourierSpace(_comm.COMM_WORLD, 0, list(N), dealias="2/3")
        ics = [spectral_random_field(space, 100 + m) for m in range(M)]
        R = Realisations(N, 0.005, M, **kw)
        R.autotune()
        for m, uh in enumerate(ics):
            R.set_state(m, uh)
        R.project()  # as Solver.initialize does
        singles = []
        for uh in ics:
            s = sim.Solver(list(N), 0.005, 1.0, **kw)
            s.initialize(uh, "fourier")
            singles.append(s)
        R.step(3)
        for s in singles:
            s.space_solver.step(3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        R.step(steps)
        e1.record()
        torch.cuda.synchronize()
        tb = e0.elapsed_time(e1) / 1e3
        e0.record()
        for s in singles:
            s.space_solver.step(steps)
        e1.record()
        torch.cuda.synchronize()
        tp = e0.elapsed_time(e1) / 1e3
        diff = max(float(np.linalg.norm(R.state(m) - singles[m].space_solver.u_hat)
                         / np.linalg.norm(singles[m].space_solver.u_hat)) for m in (0, M // 2, M - 1))
        pts = M * float(np.prod(N)) / 1e6 * steps
        out["2d" if len(N) == 2 else "3d"] = {
            "workload": f"{M} x {label}, {steps} steps", "members": M, "steps": steps,
            "batched_s": tb, "plain_s": tp, "batched_mpts_steps_per_s": pts / tb,
            "plain_mpts_steps_per_s": pts / tp, "speedup_vs_plain": tp / tb,
            "max_rel_diff_batched_vs_plain": diff}
        del R, singles
    return out


def slab_exchange_bytes(n, S, cb=8):
    """NVLink bytes one GPU sends per RK3 step when the n^3 box is split over S
    GPUs: P1's planes for the other slabs (5 fields of the slab's kept
    columns) and P4's rows for the other slabs (3 fields of its planes), per
    stage."""
    nh = n // 2 + 1
    kmax = (n - 1) // 3
    c1, c2 = 2 * kmax + 1, kmax + 1
    frac = (S - 1) / S
    e1 = 5 * n * (c1 / S) * c2 * cb * frac
    e2 = 3 * (n / S) * n * nh * cb * frac
    return 3 * (e1 + e2)


def run_slab_group(args, uh0):
    """The headline box split into S slabs held on this one GPU (pf_slab
    group): ms per RK3 step of all slabs' kernels against the whole-box step
    with the same plain launches, and the state difference.  The cross-slab
    stores stay in this GPU's memory here; on S GPUs they cross NVLink
    (bytes per GPU and step, and their time at the measured 770 GB/s peer
    bandwidth, reported beside)."""
    import torch
    from periodicflow.slab import SlabGroup
    n = args.n
    steps = args.slab_steps
    kw = dict(time_integrator=CFG["integrator"], viscosity=CFG["nu"], precision="fp32",
              forcing=CFG["forcing"], cfl=CFG["cfl"])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sol = make_solver(n)
    ss = sol.space_solver
    ss.initialize_velocity(uh0, "fourier")
    ss.step(3)
    torch.cuda.synchronize()
    e0.record()
    ss.step(steps)
    e1.record()
    torch.cuda.synchronize()
    whole_ms = e0.elapsed_time(e1) / steps
    ref = ss.u_hat
    out = {"workload": f"{n}^3 forced RK3 CFL 0.5 FP32, {steps} steps after 3 warm-up, "
                       "one recorded step replayed per step (both), every slab on this GPU",
           "whole_box_ms_per_step": whole_ms, "slabs": {}}
    for S in (2, 4, 8):
        G = SlabGroup((n, n, n), CFG["dt0"], S, **kw)
        G.set_state(uh0)
        G.step(3)
        torch.cuda.synchronize()
        e0.record()
        G.step(steps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        diff = float(np.linalg.norm(G.state() - ref) / np.linalg.norm(ref))
        b = slab_exchange_bytes(n, S)
        out["slabs"][str(S)] = {"ms_per_step": ms, "vs_whole_box": whole_ms / ms,
                                "rel_l2_vs_whole_box": diff,
                                "nvlink_bytes_per_gpu_step": b,
                                "nvlink_ms_at_770GBs": b / 770e9 * 1e3}
        G.close()
        del G
    return out


def cpu_baseline(n, steps, uh0):
    """The oracle (FP64 NumPy + scipy.fft on all host cores) on the same box,
    from the benchmark's initial field.  Returns the baseline record and the
    oracle, whose state the FP32 check below compares against."""
    import scipy.fft  # noqa: F401
    import oracle as O
    import oracle.pf_oracle as P
    P.FFT_WORKERS = os.cpu_count()
    o = O.OracleSolver((n, n, n), CFG["dt0"], time_integrator=CFG["integrator"],
                       viscosity=CFG["nu"], forcing=CFG["forcing"], cfl=CFG["cfl"])
    o.initialize(uh0, "fourier")
    t0 = time.perf_counter()
    o.advance(steps)
    sec = time.perf_counter() - t0
    return {"value": n ** 3 / 1e6 * steps / sec, "unit": UNIT, "cores": os.cpu_count(),
            "kind": "port", "sample": f"{steps} full RK3 steps of the {n}^3 workload, FP64 "
            f"oracle (NumPy pointwise single-threaded, scipy.fft workers={os.cpu_count()}), "
            f"{sec:.1f} s"}, o


def spectrum_errors(got, ref):
    """Max relative error over shells holding >= 1e-10 of the peak shell
    energy (the initial spectrum underflows to 0 at high k), and the relative
    L2 error of the whole spectrum."""
    got, ref = np.asarray(got, float), np.asarray(ref, float)
    m = min(len(got), len(ref))
    got, ref = got[:m], ref[:m]
    sel = ref >= 1e-10 * ref.max()
    rel = np.abs(got[sel] - ref[sel]) / ref[sel]
    return float(rel.max()), float(np.linalg.norm(got - ref) / np.linalg.norm(ref)), int(sel.sum())


def oracle_check(n, uh0, o, steps):
    """The headline workload in FP32 through the fused schedule, advanced from
    the same initial field by the oracle's steps, against the FP64 oracle."""
    import oracle as O
    sol = make_solver(n)
    ss = sol.space_solver
    ss.initialize_velocity(uh0, "fourier")
    ss.step(steps)
    got = ss.u_hat
    rel = float(np.linalg.norm(got - o.u_hat) / np.linalg.norm(o.u_hat))
    nb = int(np.sqrt(3 * (n // 2) ** 2)) + 2
    smax, sl2, nsel = spectrum_errors(ss.spectrum(nb), O.spectrum(o.grid, o.u_hat, nb))
    _, _, dt = ss.time()
    out = {"workload": f"{n}^3 forced turbulence (seed-1 field, RK3 CFL 0.5, band forcing), "
                       "FP32 fused schedule vs FP64 oracle from the same initial field",
           "steps": steps, "rel_l2": rel, "tolerance": 1e-5,
           "spectrum_max_rel_err": smax, "spectrum_shells_compared": nsel,
           "spectrum_rel_l2": sl2, "dt_rel_err": abs(dt - o.dt) / o.dt}
    del sol
    return out


def oracle_check_stokes(precision, steps=10):
    """Configuration 2 (2D thermal Stokes 256^2, nu 0.1, kT 1e-3, explicit PC,
    dt 0.01) for `steps` steps with the reference's NumPy draws (seed 0)
    injected into both codes.  The explicit scheme is unstable at 256^2
    (nu |k|^2 dt up to 33 > 2), so the state grows each step; the check is of
    the arithmetic, relative L2 over all modes."""
    import oracle as O
    from periodicflow import simulation as sim
    n, nu, kT, dt = 256, 0.1, 1e-3, 0.01
    mag = float(np.sqrt(2 * nu * kT))
    g = O.Grid((n, n))
    rng = np.random.RandomState(0)
    fields = [O.numpy_noise_fields(g, "thermal", rng) for _ in range(steps)]
    o = O.OracleSolver((n, n), dt, is_nonlinear=False, time_integrator="explicit_pc",
                       viscosity=nu, noise_type="thermal", noise_mag=mag,
                       noise=lambda step: fields[step - 1])
    o.initialize(np.zeros((2,) + g.spec_shape, complex), "fourier")
    o.advance(steps)
    s = sim.Solver([n, n], dt, 1.0, is_nonlinear=False, time_integrator="explicit_pc",
                   viscosity=nu, noise_type="thermal", noise_mag=mag, precision=precision,
                   noise_source="injected")
    ss = s.space_solver
    for w1, w2 in fields:
        ss.inject_noise(w1, w2)
        ss.step(1)
    got = ss.u_hat
    return float(np.linalg.norm(got - o.u_hat) / np.linalg.norm(o.u_hat))


def run_reference(args, rank, world):
    if rank != 0:
        return
    n = args.n
    import oracle as O
    import oracle.pf_oracle as P
    P.FFT_WORKERS = os.cpu_count()
    o = O.OracleSolver((n, n, n), CFG["dt0"], time_integrator=CFG["integrator"],
                       viscosity=CFG["nu"], forcing=CFG["forcing"], cfl=CFG["cfl"])
    o.initialize(oracle_initial_field(n, CFG["seed"]), "fourier")
    warm = min(args.warmup, 1)
    o.advance(warm)
    budget = args.ref_budget_s
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        o.advance(1)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    sec = time.perf_counter() - t0
    value = n ** 3 / 1e6 * done / sec
    sample = (f"{done} of {args.steps} requested full RK3 steps (time box {budget:.0f} s) of the "
              f"{n}^3 workload after {warm} warm-up step(s); FP64 oracle (NumPy + scipy.fft, "
              f"{os.cpu_count()} workers)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": done, "warmup": warm, "ms_per_step": sec / done * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic",
            "config": {"workload": f"3D forced isotropic turbulence {n}^3, RK3 CFL 0.5, "
                                   "linear forcing |k|<=2.5 eps=0.1, nu=2e-3, 2/3 dealias",
                       "grid": [n, n, n]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(),
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--timed-pass", type=int, default=5, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--traffic", type=float, default=None,
                    help="DRAM bytes per launch of the timed pass from an ncu capture")
    ap.add_argument("--no-e2e", action="store_true")
    # the forced-turbulence configuration's full run: 2000 steps, E and Z every step
    ap.add_argument("--e2e-steps", type=int, default=2000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--ref-budget-s", type=float, default=120.0)
    ap.add_argument("--mode", choices=["headline", "ensemble", "serving", "case"],
                    default="headline",
                    help="case: run the forced-turbulence step on a --dim-dimensional "
                         "grid of side --n for --steps steps, untimed (the case profiles "
                         "are captured on)")
    ap.add_argument("--dim", type=int, default=3, choices=[2, 3])
    ap.add_argument("--dealias", choices=["2/3", "3/2"], default="2/3",
                    help="3/2: the reference's default rule on the same workload (fused padded "
                         "passes); the line then times pass --timed-pass of that schedule")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-nlbatch", action="store_true")
    ap.add_argument("--nlb-steps", type=int, default=200)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-slab", action="store_true")
    ap.add_argument("--slab-steps", type=int, default=10)
    ap.add_argument("--no-padded", action="store_true")
    ap.add_argument("--no-cufft", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=10)
    ap.add_argument("--cufft-steps", type=int, default=20)
    ap.add_argument("--padded-steps", type=int, default=10)
    ap.add_argument("--ens-steps", type=int, default=5000)
    ap.add_argument("--ens-scale", type=float, default=1.0)
    ap.add_argument("--ens-stepwise-sample", type=int, default=50)
    ap.add_argument("--serve-requests", type=int, default=60)
    ap.add_argument("--serve-max-steps", type=int, default=5000)
    ap.add_argument("--serve-nl-points", type=int, default=None,
                    help="cap on grid points of concurrently running nonlinear requests "
                         "(0: none; default: the server's)")
    args = ap.parse_args()
    if args.mode == "case":
        run_case(args)
        return
    if args.mode in ("ensemble", "serving"):
        import torch
        torch.cuda.set_device(0)
        out = run_ensemble(args) if args.mode == "ensemble" else run_serving(args)
        print(json.dumps({"mode": args.mode, **out}), flush=True)
        return
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank, world)
        return
    dist, rank, world = _dist()
    try:
        run_ours(args, dist, rank, world)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
