"""Snapshot writer with the reference's interface (io.py:15-196).

Snapshots of the physical velocity are taken from the device at write time.
``reconfigure_dataset`` produces the reference's flat layout
{x, y[, z], t, <var>/<zero-padded step>} with the optional periodic point;
it is written as HDF5 when h5py is importable, else as ``<file>.npz`` with the
same keys.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from . import logger
from .utils import periodic_bc


class HDF5Writer:
    def __init__(self, comm, rank, size, file_name, solver=None, component_names=("u", "v", "w"),
                 time_points=(0.0, 1.0), end_points=(2 * np.pi, 2 * np.pi), periodic=False):
        self.comm = comm
        self.mpi_rank = rank
        self.mpi_size = size
        self.file_name = str(file_name)
        self.solver = solver
        self.names = list(component_names)
        self.time_points = list(time_points)
        self.end_points = list(end_points)
        self.periodic = periodic
        self.snapshots = {}  # step -> (d, N...) float64
        self.closed = False

    def write(self, step: int):
        self.snapshots[int(step)] = self.solver.u

    def close(self):
        self.closed = True

    def _layout(self):
        steps = sorted(self.snapshots)
        nd = len(str(steps[-1])) if steps else 1
        out = {}
        for ax, (label, x_end) in enumerate(zip(["x", "y", "z"], self.end_points)):
            if ax >= self.solver.dim:
                break
            coord = np.ravel(self.solver.x[ax])
            if self.periodic:
                coord = np.append(coord, x_end)
            out[label] = coord
        out["t"] = np.linspace(self.time_points[0], self.time_points[-1], len(steps))
        for s in steps:
            for i, name in enumerate(self.names):
                data = self.snapshots[s][i]
                if self.periodic:
                    data = periodic_bc(data)
                out[f"{name}/{str(s).zfill(nd)}"] = data
        return out

    def reconfigure_dataset(self):
        if self.mpi_rank == 0:
            logger.info("HDF5Writer.reconfigure_dataset: Start reconfiguring dataset.")
        data = self._layout()
        path = Path(self.file_name).with_suffix(".h5")
        try:
            import h5py
        except ImportError:
            h5py = None
        if h5py is not None:
            with h5py.File(path, "w") as f:
                for k, v in data.items():
                    f.create_dataset(k, data=v)
        else:
            path = path.with_suffix(".npz")
            np.savez(path, **data)
        if self.mpi_rank == 0:
            logger.info(f"HDF5Writer.reconfigure_dataset: Dataset written to {path}.")
        return path
