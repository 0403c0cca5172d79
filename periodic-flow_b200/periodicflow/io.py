"""Snapshot writer with the reference's interface (io.py:15-196).

``write(step)`` takes the physical velocity off the device and streams it to
``<file>.snapshots/<step>.npy`` (memory stays flat however many snapshots a
run writes).  ``reconfigure_dataset`` produces the reference's flat layout
{x, y[, z], t, <var>/<zero-padded step>} with the optional periodic point
(io.py:97-196): HDF5 when h5py is importable, else ``<file>.npz`` with the
same keys, written member by member.
"""
from __future__ import annotations

import os
import shutil
import zipfile
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
        self.snapdir = Path(self.file_name + ".snapshots")
        if self.snapdir.exists():
            shutil.rmtree(self.snapdir)
        self.snapdir.mkdir(parents=True)
        self.steps = []
        self.closed = False

    def write(self, step: int):
        np.save(self.snapdir / f"{int(step)}.npy", self.solver.u)
        self.steps.append(int(step))

    def close(self):
        self.closed = True

    def _coords(self):
        out = {}
        for ax, (label, x_end) in enumerate(zip(["x", "y", "z"], self.end_points)):
            if ax >= self.solver.dim:
                break
            coord = np.ravel(self.solver.x[ax])
            if self.periodic:
                coord = np.append(coord, x_end)
            out[label] = coord
        out["t"] = np.linspace(self.time_points[0], self.time_points[-1], len(self.steps))
        return out

    def _fields(self):
        """Yield (key, array) one snapshot component at a time."""
        steps = sorted(set(self.steps))
        nd = len(str(steps[-1])) if steps else 1
        for s in steps:
            data = np.load(self.snapdir / f"{s}.npy")
            for i, name in enumerate(self.names):
                arr = data[i]
                if self.periodic:
                    arr = periodic_bc(arr)
                yield f"{name}/{str(s).zfill(nd)}", arr

    def reconfigure_dataset(self):
        if self.mpi_rank == 0:
            logger.info("HDF5Writer.reconfigure_dataset: Start reconfiguring dataset.")
        path = Path(self.file_name).with_suffix(".h5")
        try:
            import h5py
        except ImportError:
            h5py = None
        if h5py is not None:
            with h5py.File(path, "w") as f:
                for k, v in self._coords().items():
                    f.create_dataset(k, data=v)
                for k, v in self._fields():
                    f.create_dataset(k, data=v)
        else:
            path = path.with_suffix(".npz")
            with zipfile.ZipFile(path, "w", allowZip64=True) as zf:
                items = list(self._coords().items())
                for k, v in items:
                    with zf.open(k + ".npy", "w", force_zip64=True) as fh:
                        np.lib.format.write_array(fh, np.asarray(v))
                for k, v in self._fields():
                    with zf.open(k + ".npy", "w", force_zip64=True) as fh:
                        np.lib.format.write_array(fh, np.asarray(v))
        shutil.rmtree(self.snapdir, ignore_errors=True)
        if self.mpi_rank == 0:
            logger.info(f"HDF5Writer.reconfigure_dataset: Dataset written to {path}.")
        return path
