"""One periodic box split into slabs: the reference's ``decomposition='slab'``.

The reference builds its spaces over MPI's COMM_WORLD with shenfun's
``TensorProductSpace(..., slab=True)`` (basis.py:64, simulation.py:81-83):
physical arrays are split along axis 0, spectral arrays along axis 1, and
alltoall transposes move between them.  Here slab ``r`` of ``S`` holds the
spectral rows ``k1`` in ``[r n1/S, (r+1) n1/S)`` -- its local ``u_hat`` is
``(3, n0, n1/S, n2/2+1)`` -- and the two transposes of every evaluation of
the nonlinear term are stores of the fused passes into the destination slab's
buffers (C-ABI ``pf_slab_*``).

* ``SlabGroup`` holds all slabs of one box in this process, on one device.
* ``SlabSolver`` holds one slab per process and GPU: the processes share
  their exchange buffers by CUDA IPC and an NCCL communicator (made from an id
  that rank 0 draws) that carries the exchange barriers and the CFL / forcing
  reductions.  The handshake goes over a communicator with ``allgather`` and
  ``bcast`` (mpi4py's, or this package's torch.distributed one).

Built for the 3D nonlinear problem with the 2/3 rule (FP32 / FP64), every
integrator, CFL dt, band forcing, Nyquist mask and thermal Philox noise.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as _nat

__all__ = ["slab_layout", "SlabGroup", "SlabSolver", "exchange_handshake"]


def slab_layout(N, slabs: int, slab: int) -> dict:
    """Extents of slab ``slab`` of ``slabs`` of an (n0, n1, n2) box (host logic)."""
    out = (C.c_int * 6)()
    _nat.check(_nat.lib().pf_slab_layout(int(N[0]), int(N[1]), int(slabs), int(slab), out),
               None, "pf_slab_layout", _nat.lib().pf_slab_last_error)
    keys = ("n0_per_slab", "n1_per_slab", "x0_first", "k1_first", "kept_first", "kept_count")
    return dict(zip(keys, [int(v) for v in out]))


def _config(N, dt, time_integrator, viscosity, noise_type, noise_mag, domain, mask_nyquist,
            precision, seed, forcing, cfl):
    from . import _comm
    from .basis import FourierSpace
    from .space_solver import build_config
    from .time_integrator import DICT_TIME_INTEGRATORS
    if time_integrator not in DICT_TIME_INTEGRATORS:
        raise ValueError(f"Time integrator '{time_integrator}' not found.")
    space = FourierSpace(_comm.COMM_WORLD, 0, list(N), domain=domain, dealias="2/3",
                         mask_nyquist=mask_nyquist)
    cfg = build_config(tuple(space.N), space.domain, True,
                       DICT_TIME_INTEGRATORS[time_integrator].native_id, viscosity, noise_type,
                       noise_mag, mask_nyquist, precision, dt, seed, "philox", forcing, cfl, True,
                       dealias="truncate")
    return space, cfg


def exchange_handshake(comm, export: bytes, make_id):
    """Every rank's export blocks (rank order) and rank 0's NCCL id.

    ``comm`` has mpi4py's ``Get_rank``, ``allgather`` and ``bcast``;
    ``make_id()`` draws the id (called on rank 0 only)."""
    exports = comm.allgather(bytes(export))
    nid = make_id() if comm.Get_rank() == 0 else None
    nid = comm.bcast(nid, root=0)
    if any(len(e) != len(export) for e in exports):
        raise ValueError("slab exports differ in size across ranks")
    return b"".join(exports), nid


class _Slabs:
    _err = None

    def _check(self, rc, what):
        _nat.check(rc, self._h, what, _nat.lib().pf_slab_last_error)

    def _setup(self, N, kw):
        self.space, self._cfg = _config(N, **kw)
        self.N = tuple(self.space.N)
        if len(self.N) != 3:
            raise NotImplementedError("slab decomposition is built for 3D boxes")
        self.shape_spectral = self.space.shape_spectral

    def _local_shape(self):
        n0, n1 = self.N[0], self.N[1]
        return (3, n0, n1 // self.slabs, self.N[2] // 2 + 1)

    def _set(self, r, uh):
        a = np.ascontiguousarray(uh, dtype=np.complex128)
        if a.shape != self._local_shape():
            raise ValueError(f"slab state has shape {a.shape}, expected {self._local_shape()}")
        self._check(_nat.lib().pf_slab_set_fourier(self._h, r, a.ctypes.data, 0),
                    "pf_slab_set_fourier")

    def _get(self, r):
        a = np.empty(self._local_shape(), dtype=np.complex128)
        self._check(_nat.lib().pf_slab_get_fourier(self._h, r, a.ctypes.data, 0),
                    "pf_slab_get_fourier")
        return a

    def _energy(self, r):
        e, z = C.c_double(), C.c_double()
        self._check(_nat.lib().pf_slab_energy(self._h, r, C.byref(e), C.byref(z)),
                    "pf_slab_energy")
        return e.value, z.value

    def step(self, nsteps: int = 1) -> None:
        """Advance every slab held here ``nsteps`` steps (collective across ranks)."""
        self._check(_nat.lib().pf_slab_step(self._h, int(nsteps)), "pf_slab_step")
        self._check(_nat.lib().pf_slab_sync(self._h), "pf_slab_sync")

    def time(self):
        """(t, steps, dt) of the box."""
        t, n, dt = C.c_double(), C.c_longlong(), C.c_double()
        self._check(_nat.lib().pf_slab_get_time(self._h, C.byref(t), C.byref(n), C.byref(dt)),
                    "pf_slab_get_time")
        return t.value, n.value, dt.value

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            _nat.lib().pf_slab_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass


class SlabGroup(_Slabs):
    """All ``slabs`` slabs of one box in this process, on the current device.

    Keywords as ``Solver`` (time_integrator, viscosity, noise_type, noise_mag,
    domain, mask_nyquist, precision, seed, forcing, cfl); the rule is 2/3."""

    def __init__(self, N, dt: float, slabs: int, *, time_integrator: str = "rk2",
                 viscosity: float = 1e-3, noise_type: str = "thermal", noise_mag: float = 0.0,
                 domain=2 * math.pi, mask_nyquist: bool = False, precision: str = "fp32",
                 seed: int = 0, forcing=None, cfl=None):
        self._h = None
        self._setup(N, dict(dt=dt, time_integrator=time_integrator, viscosity=viscosity,
                            noise_type=noise_type, noise_mag=noise_mag, domain=domain,
                            mask_nyquist=mask_nyquist, precision=precision, seed=seed,
                            forcing=forcing, cfl=cfl))
        self.slabs = int(slabs)
        h = C.c_void_p()
        _nat.check(_nat.lib().pf_slab_create_group(C.byref(self._cfg), self.slabs, C.byref(h)),
                   None, "pf_slab_create_group", _nat.lib().pf_slab_last_error)
        self._h = h

    def set_state(self, u_hat) -> None:
        """Whole-box spectral state (3, n0, n1, n2/2+1), split over the slabs."""
        u = np.asarray(u_hat)
        if u.shape != tuple([3] + list(self.shape_spectral)):
            raise ValueError(f"state has shape {u.shape}")
        w = self.N[1] // self.slabs
        for r in range(self.slabs):
            self._set(r, u[:, :, r * w:(r + 1) * w, :])

    def state(self) -> np.ndarray:
        """Whole-box spectral state gathered from the slabs."""
        return np.concatenate([self._get(r) for r in range(self.slabs)], axis=2)

    def slab_state(self, r: int) -> np.ndarray:
        return self._get(r)

    def energy(self):
        """(E, Z) of the box: the slabs' parts summed."""
        parts = [self._energy(r) for r in range(self.slabs)]
        return sum(p[0] for p in parts), sum(p[1] for p in parts)


class SlabSolver(_Slabs):
    """Slab ``comm.Get_rank()`` of a box split over ``comm.Get_size()`` processes,
    one GPU each (the reference's one-field-per-communicator run)."""

    def __init__(self, N, dt: float, *, comm=None, time_integrator: str = "rk2",
                 viscosity: float = 1e-3, noise_type: str = "thermal", noise_mag: float = 0.0,
                 domain=2 * math.pi, mask_nyquist: bool = False, precision: str = "fp32",
                 seed: int = 0, forcing=None, cfl=None):
        from . import _comm
        self._h = None
        self.comm = comm if comm is not None else _comm.COMM_WORLD
        self.rank = self.comm.Get_rank()
        self.slabs = self.comm.Get_size()
        self._setup(N, dict(dt=dt, time_integrator=time_integrator, viscosity=viscosity,
                            noise_type=noise_type, noise_mag=noise_mag, domain=domain,
                            mask_nyquist=mask_nyquist, precision=precision, seed=seed,
                            forcing=forcing, cfl=cfl))
        h = C.c_void_p()
        _nat.check(_nat.lib().pf_slab_create(C.byref(self._cfg), self.slabs, self.rank,
                                             C.byref(h)),
                   None, "pf_slab_create", _nat.lib().pf_slab_last_error)
        self._h = h
        used = C.c_size_t()
        buf = (C.c_char * 256)()
        self._check(_nat.lib().pf_slab_export(h, buf, 256, C.byref(used)), "pf_slab_export")
        exports, nid = exchange_handshake(self.comm, bytes(buf)[:used.value], self._nccl_id)
        ex = C.create_string_buffer(exports, len(exports))
        idb = C.create_string_buffer(nid, len(nid))
        self._check(_nat.lib().pf_slab_connect(h, ex, idb), "pf_slab_connect")

    @staticmethod
    def _nccl_id() -> bytes:
        buf = (C.c_char * 128)()
        _nat.check(_nat.lib().pf_slab_nccl_id(buf, 128), None, "pf_slab_nccl_id",
                   _nat.lib().pf_slab_last_error)
        return bytes(buf)

    def set_local_state(self, u_hat_local) -> None:
        """This slab's spectral rows (3, n0, n1/S, n2/2+1)."""
        self._set(self.rank, u_hat_local)

    def local_state(self) -> np.ndarray:
        return self._get(self.rank)

    def energy(self):
        """(E, Z) of the box (reduced over the ranks)."""
        e, z = self._energy(self.rank)
        return self.comm.allreduce(e), self.comm.allreduce(z)
