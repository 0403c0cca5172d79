"""Solver: the reference's public API (simulation.py:12-225) over the CUDA backend.

Extensions beyond the reference's keyword set (all optional):
  precision      'fp32' (default; env PERIODICFLOW_PRECISION) or 'fp64'
  seed           Philox key of the device noise (default: the value the
                 constructor reseeds NumPy's global generator with)
  noise_source   'philox' (device, Hermitian-symmetric), 'numpy' (host draws in
                 the reference's RNG order, uploaded every step) or 'injected'
                 (caller calls inject_noise before each step)
  forcing        (eps, kf): linear band forcing at constant injection eps
  cfl            CFL number for an adaptive dt (nonlinear runs)
  diagnostics    record E and Z after every step (``history``)
  fused          use the fused pencil passes where built (default True)
  nonlinear      alias of is_nonlinear (examples/tgv3d.py passes it)
"""
from __future__ import annotations

import os
import traceback

import numpy as np

from . import _comm
from . import logger
from .io import HDF5Writer
from .space_solver import SpaceSolver
from .time_integrator import DICT_TIME_INTEGRATORS
from .utils import Timer


class Solver:
    def __init__(self, N, dt: float, end_time: float, is_nonlinear: bool = True,
                 time_integrator: str = "rk2", viscosity: float = 1e-3,
                 noise_type: str = "thermal", noise_mag: float = 0.0, domain=2 * np.pi,
                 check_interval: int = np.iinfo(np.int64).max, verbose: bool = False,
                 write_solution: bool = False, file_name: str = None, file_mode: str = "w",
                 write_interval: int = np.iinfo(np.int64).max, periodic: bool = False,
                 dealias: str = "3/2", mask_nyquist: bool = False, fft_plan: str = "FFTW_MEASURE",
                 decomposition: str = "slab", optimization: bool = True, *,
                 precision: str | None = None, seed: int | None = None,
                 noise_source: str = "philox", forcing=None, cfl: float | None = None,
                 diagnostics: bool = False, fused: bool = True, nonlinear: bool | None = None):
        self.comm = _comm.COMM_WORLD
        self.mpi_rank = self.comm.Get_rank()
        self.mpi_size = self.comm.Get_size()
        if nonlinear is not None:
            is_nonlinear = nonlinear
        if time_integrator not in DICT_TIME_INTEGRATORS:
            raise ValueError(f"Time integrator '{time_integrator}' not found.")
        integ_cls = DICT_TIME_INTEGRATORS[time_integrator]
        if integ_cls.native_id is None:
            raise NotImplementedError(f"integrator '{time_integrator}' has no device rule")
        # simulation.py:100 -- the reference reseeds NumPy's global generator
        s = np.random.randint(0, 2 ** 32 - 1)
        np.random.seed(s)
        if precision is None:
            precision = os.environ.get("PERIODICFLOW_PRECISION", "fp32")
        self.space_solver = SpaceSolver(
            self.comm, self.mpi_rank, N, is_nonlinear=is_nonlinear, viscosity=viscosity,
            noise_type=noise_type, noise_mag=noise_mag, domain=domain, dealias=dealias,
            mask_nyquist=mask_nyquist, fft_plan=fft_plan, decomposition=decomposition,
            dt=dt, integrator_id=integ_cls.native_id, precision=precision,
            seed=int(s) if seed is None else int(seed), noise_source=noise_source,
            forcing=forcing, cfl=cfl, fused=fused)
        self.end_time = end_time
        self.write_solution = write_solution
        self.write_interval = write_interval
        self.check_interval = check_interval
        self.verbose = verbose
        self.step = 0
        self.t = 0.0
        self.file_mode = file_mode
        self.cfl = cfl
        self.diagnostics = diagnostics
        self.history = np.zeros((0, 2))
        self._init_integrator(time_integrator, dt, optimization)
        self._init_writer(file_name, periodic)
        self._timer = Timer(self.comm, verbose)
        if diagnostics:
            self.space_solver.record_history(True)

    def __getattr__(self, name):
        # simulation.py:116-120: pass-through to the space solver
        if name == "space_solver":
            raise AttributeError(name)
        ss = self.__dict__.get("space_solver")
        if ss is not None and hasattr(ss, name):
            return getattr(ss, name)
        raise AttributeError(f"'{type(self).__name__}' object has no attribute '{name}'")

    def _init_integrator(self, time_integrator, dt, optimization=False):
        try:
            self.time_integrator = DICT_TIME_INTEGRATORS[time_integrator](
                dt, self.space_solver.linear_operator, optimization)
            self.time_integrator._on_update = self.space_solver.set_linear_operator
        except Exception as e:
            if self.mpi_rank == 0:
                logger.error(f"Failed to initialize time integrator: {e}\n{traceback.format_exc()}")
            raise

    def _init_writer(self, file_name, periodic):
        if self.write_solution:
            if file_name is None:
                raise ValueError("write_solution=True needs a file_name")
            ss = self.space_solver
            names = ["u", "v", "w"][:ss.dim]
            self.solution_writer = HDF5Writer(
                self.comm, self.mpi_rank, self.mpi_size, file_name, solver=ss,
                component_names=names, time_points=[0.0, self.end_time],
                end_points=[b for _, b in ss.domain], periodic=periodic)

    @classmethod
    def read_config(cls, config: dict):
        """simulation.py:156-159."""
        return cls(**config)

    def initialize(self, u0, space: str = "physical", project: bool = True,
                   mask_zero_mode: bool = True):
        """simulation.py:161-180."""
        self.space_solver.initialize_velocity(u0, space, mask_zero_mode)
        if project:
            self.space_solver.project()
        if self.write_solution:
            self.solution_writer.write(self.step)

    def set_linear_operator(self, L):
        """simulation.py:182-184 (also refreshes (1 - dt/2 L)^-1 on the device)."""
        self.time_integrator.update_linear_operator(L)

    def set_correlation_function(self, C):
        """simulation.py:186-187."""
        self.space_solver.set_correlation_function(C)

    def inject_noise(self, w1, w2):
        self.space_solver.inject_noise(w1, w2)

    def _advance(self, nsteps: int):
        ss = self.space_solver
        if ss.noise_source == "numpy" and ss.noise_mag != 0.0:
            for _ in range(nsteps):
                ss.random_fields()
                ss.step(1)
        else:
            ss.step(nsteps)

    def _steps_to_end(self, t: float, dt: float):
        """Steps the reference loop takes from t (simulation.py:205-207)."""
        n = 0
        limit = int(np.ceil((self.end_time - t) / dt)) + 2
        while not np.isclose(t, self.end_time, atol=1e-10):
            t += dt
            n += 1
            if n > limit:
                raise RuntimeError("time loop would not end: end_time is not a multiple of dt "
                                   "(np.isclose(t, end_time) is never reached)")
        return n

    def solve(self, nsteps: int | None = None):
        """simulation.py:189-225.  ``nsteps`` (extension) runs a fixed number of
        steps instead of stopping at end_time (needed with an adaptive dt)."""
        self.comm.Barrier()
        self._timer.start()
        dt = self.time_integrator.dt
        if nsteps is None:
            if self.cfl:
                raise ValueError("an adaptive dt (cfl) needs solve(nsteps=...)")
            nsteps = self._steps_to_end(self.t, dt)
        done = 0
        while done < nsteps:
            chunk = nsteps - done
            for iv in (self.write_interval if self.write_solution else None, self.check_interval):
                if iv is not None and 0 < iv < np.iinfo(np.int64).max:
                    chunk = min(chunk, iv - (self.step % iv))
            self._advance(chunk)
            done += chunk
            if self.cfl:
                self.t, self.step, _ = self.space_solver.time()
            else:
                for _ in range(chunk):
                    self.t += dt
                self.step += chunk
            if self.write_solution and self.step % self.write_interval == 0:
                self.solution_writer.write(self.step)
            if self.step % self.check_interval == 0:
                self._timer(self.t, self.step)
        if self.diagnostics:
            self.history = np.concatenate([self.history, self.space_solver.history()])
        if self.write_solution:
            self.solution_writer.close()
        self._timer.final()
