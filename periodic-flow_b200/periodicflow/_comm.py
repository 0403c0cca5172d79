"""Communicator with the mpi4py methods the solver and the examples call.

The backend runs one box per GPU and needs no MPI.  Without an initialised
``torch.distributed`` process group this is a single-rank communicator; with
one, rank/size/barrier/allreduce/bcast go through it (gloo or nccl), which is
how ensembles of independent boxes are spread over several GPUs.
"""
from __future__ import annotations

import sys


class SUM:  # mirrors mpi4py.MPI.SUM as an op tag
    pass


class Comm:
    def _dist(self):
        try:
            import torch.distributed as dist
            if dist.is_available() and dist.is_initialized():
                return dist
        except Exception:  # pragma: no cover
            pass
        return None

    def Get_rank(self) -> int:
        d = self._dist()
        return d.get_rank() if d else 0

    def Get_size(self) -> int:
        d = self._dist()
        return d.get_world_size() if d else 1

    def Barrier(self) -> None:
        d = self._dist()
        if d:
            d.barrier()

    def allreduce(self, value, op=SUM):
        d = self._dist()
        if not d:
            return value
        out = [None] * d.get_world_size()
        d.all_gather_object(out, value)
        return sum(out)

    def allgather(self, obj):
        d = self._dist()
        if not d:
            return [obj]
        out = [None] * d.get_world_size()
        d.all_gather_object(out, obj)
        return out

    def bcast(self, obj, root: int = 0):
        d = self._dist()
        if not d:
            return obj
        box = [obj]
        d.broadcast_object_list(box, src=root)
        return box[0]

    def Abort(self, code: int = 1) -> None:
        sys.exit(code)


COMM_WORLD = Comm()
