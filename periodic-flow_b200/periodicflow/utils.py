"""Run-time helpers of the solver loop: the periodic closure of snapshot arrays
and the progress timer (interfaces of the reference's utils.py:7-98; the log
texts are the reference's so its users see the same lines)."""
from __future__ import annotations

import time

import numpy as np

from . import logger

# Duration layouts: (wrap, fields).  The seconds are first reduced modulo
# `wrap` (None: kept whole), then each field, from the largest to the
# smallest, is (unit seconds, separator written before it).
_LAYOUTS = {
    "dd-hh:mm:ss": (None, ((86400, ""), (3600, "-"), (60, ":"), (1, ":"))),
    "hh:mm:ss": (86400, ((3600, ""), (60, ":"), (1, ":"))),
    "mm:ss": (3600, ((60, ""), (1, ":"))),
}


def periodic_bc(u: np.ndarray) -> np.ndarray:
    """Close a periodic array: every axis gains one trailing entry equal to
    its first one (corners included), as snapshot files store x = L."""
    return np.pad(u, [(0, 1)] * u.ndim, mode="wrap")


def format_duration(seconds: float, layout: str = "dd-hh:mm:ss") -> str:
    """Whole seconds as two-digit fields in ``layout``; the shorter layouts
    drop the larger units (days, then hours) as the reference does."""
    spec = _LAYOUTS.get(layout.casefold())
    if spec is None:
        raise ValueError("Invalid format. Choose 'dd-hh:mm:ss', 'hh:mm:ss', or 'mm:ss'.")
    wrap, fields = spec
    rest = seconds if wrap is None else seconds % wrap
    out = []
    for unit, sep in fields:
        n, rest = divmod(rest, unit)
        out.append(f"{sep}{int(n):02d}")
    return "".join(out)


class Timer:
    """Wall-clock progress of a run, averaged over the ranks of ``comm``.

    ``start()`` announces the run, calling the timer with (time, step) logs
    the lap since the previous call when ``verbose``, ``final()`` logs the
    whole run.  Every rank must make the same calls (the lap and total are
    reduced over the communicator)."""

    def __init__(self, comm, verbose: bool = False):
        self.comm = comm
        self.mpi_rank = comm.Get_rank()
        self.mpi_size = comm.Get_size()
        self.verbose = verbose
        self.start_time = time.time()
        self._lap_from = self.start_time

    def _mean_over_ranks(self, value: float) -> float:
        return self.comm.allreduce(value) / self.mpi_size

    def _lap(self) -> float:
        now = time.time()
        lap, self._lap_from = now - self._lap_from, now
        return lap

    def start(self):
        if self.mpi_rank == 0:
            logger.info("Simulation started")

    def __call__(self, simulation_time: float, step: int):
        lap = self._mean_over_ranks(self._lap())
        if self.verbose and self.mpi_rank == 0:
            logger.info(f"Step = {step:08d}, time = {simulation_time:.2e}, runtime since last "
                        f"check = {format_duration(lap, 'hh:mm:ss')}")
        self.comm.Barrier()

    def final(self):
        total = self._mean_over_ranks(time.time() - self.start_time)
        if self.mpi_rank == 0:
            logger.info(f"Simulation completed. Total run time: {format_duration(total)}")

    # name used by the reference's callers
    _format_time = staticmethod(format_duration)
