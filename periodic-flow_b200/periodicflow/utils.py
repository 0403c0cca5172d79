"""Timing helpers with the behaviour of the reference's utils.py:7-98."""
from __future__ import annotations

import time

import numpy as np

from . import logger
from ._comm import SUM


def periodic_bc(u: np.ndarray) -> np.ndarray:
    """Append the first slice along every axis (utils.py:7-14)."""
    for axis in range(u.ndim):
        first = np.take(u, indices=0, axis=axis)
        u = np.concatenate((u, np.expand_dims(first, axis=axis)), axis=axis)
    return u


class Timer:
    """Wall clock between checks, averaged over ranks (utils.py:17-72)."""

    def __init__(self, comm, verbose: bool = False):
        self.comm = comm
        self.mpi_rank = comm.Get_rank()
        self.mpi_size = comm.Get_size()
        self.verbose = verbose
        self.start_time = time.time()
        self.t0 = self.start_time

    def __call__(self, simulation_time: float, step: int):
        t1 = time.time()
        dt = t1 - self.t0
        self.t0 = t1
        dt_avg = self.comm.allreduce(dt, op=SUM) / self.mpi_size
        if self.verbose and self.mpi_rank == 0:
            logger.info(f"Step = {step:08d}, time = {simulation_time:.2e}, runtime since last "
                        f"check = {self._format_time(dt_avg, 'hh:mm:ss')}")
        self.comm.Barrier()

    def start(self):
        if self.mpi_rank == 0:
            logger.info("Simulation started")

    def final(self):
        runtime = time.time() - self.start_time
        runtime_avg = self.comm.allreduce(runtime, op=SUM) / self.mpi_size
        if self.mpi_rank == 0:
            logger.info(f"Simulation completed. Total run time: {self._format_time(runtime_avg)}")

    @staticmethod
    def _format_time(seconds: float, format: str = "dd-hh:mm:ss") -> str:
        days, rem = divmod(seconds, 86400)
        hours, rem = divmod(rem, 3600)
        minutes, secs = divmod(rem, 60)
        f = format.casefold()
        if f == "mm:ss":
            return f"{int(minutes):02d}:{int(secs):02d}"
        if f == "hh:mm:ss":
            return f"{int(hours):02d}:{int(minutes):02d}:{int(secs):02d}"
        if f == "dd-hh:mm:ss":
            return f"{int(days):02d}-{int(hours):02d}:{int(minutes):02d}:{int(secs):02d}"
        raise ValueError("Invalid format. Choose 'dd-hh:mm:ss', 'hh:mm:ss', or 'mm:ss'.")
