"""Spatial operator of the solver (the reference's space_solver.py:67-310).

The state lives on the GPU inside a C-ABI solver handle; ``u_hat`` and ``u``
are host (NumPy, FP64) views materialised on access, and assignments upload.
The right-hand side (nonlinear term, Leray projection, linear term, noise,
forcing) is computed fused with the stage update on the device;
``compute_rhs`` also writes its parts to arrays for callers that read them.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from . import logger
from .basis import FourierSpace

NOISE_SOURCES = ("philox", "numpy", "injected")


def build_config(Ns, domain, is_nonlinear, integrator_id, viscosity, noise_type, noise_mag,
                 mask_nyquist, precision, dt, seed, noise_source, forcing, cfl, fused,
                 dealias="truncate"):
    """The pf_config of a solver (include/periodicflow_b200.h)."""
    dim = len(Ns)
    cfg = N.PfConfig()
    N.lib().pf_config_default(C.byref(cfg))
    cfg.dim = dim
    for a in range(3):
        cfg.n[a] = Ns[a] if a < dim else 1
        lo, hi = domain[a] if a < dim else (0.0, 2 * np.pi)
        cfg.domain[a][0] = lo
        cfg.domain[a][1] = hi
    cfg.is_nonlinear = int(bool(is_nonlinear))
    cfg.integrator = integrator_id
    cfg.viscosity = viscosity
    cfg.noise_type = N.PF_NOISE_THERMAL if noise_type == "thermal" else N.PF_NOISE_CORRELATED
    cfg.noise_mag = noise_mag
    cfg.dealias = N.PF_DEALIAS_PAD if dealias == "pad" else N.PF_DEALIAS_TRUNCATE
    cfg.mask_nyquist = int(bool(mask_nyquist))
    cfg.precision = N.PF_FP64 if precision == "fp64" else N.PF_FP32
    cfg.dt = dt
    cfg.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    cfg.noise_source = N.PF_NOISE_SRC_PHILOX if noise_source == "philox" else N.PF_NOISE_SRC_INJECTED
    if forcing is not None:
        cfg.forcing_eps, cfg.forcing_kf = float(forcing[0]), float(forcing[1])
    cfg.cfl = float(cfl) if cfl else 0.0
    cfg.fused = int(bool(fused))
    return cfg


def device_footprint(cfg) -> int:
    """Device bytes a solver with this config allocates (no device use)."""
    b = C.c_ulonglong()
    N.check(N.lib().pf_footprint(C.byref(cfg), C.byref(b)), None, "pf_footprint")
    return int(b.value)


class SpaceSolver(FourierSpace):
    def __init__(self, comm, mpi_rank, N_, is_nonlinear: bool = True, viscosity: float = 1e-3,
                 noise_type: str = "thermal", noise_mag: float = 0.0, *, dt: float = 1e-3,
                 integrator_id: int = N.PF_RK2, precision: str = "fp32", seed: int = 0,
                 noise_source: str = "philox", forcing=None, cfl=None, fused: bool = True,
                 **kwargs):
        super().__init__(comm, mpi_rank, N_, **kwargs)
        if self.dim not in (2, 3):
            raise ValueError("NS solver only supports 2D and 3D problems.")
        if noise_type not in ("thermal", "correlated"):
            raise ValueError(f"Invalid noise type '{noise_type}'. Options are 'thermal' or 'correlated'.")
        if noise_source not in NOISE_SOURCES:
            raise ValueError(f"noise_source must be one of {NOISE_SOURCES}")
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be 'fp32' or 'fp64'")
        self._is_nonlinear = is_nonlinear
        self.viscosity = viscosity
        self.noise_type = noise_type
        self.noise_mag = noise_mag
        self.noise_source = noise_source
        self.precision = precision
        self.shape_local_physical = (self.dim,) + self.shape_physical
        self.shape_local_fourier = (self.dim,) + self.shape_spectral
        self.ncomp = self.dim ** 2 if noise_type == "thermal" else self.dim
        # space_solver.py:143-148
        self._k0_mask_0 = np.where(self.k2 == 0, 0, 1)
        self._noise_normal_factor = self._k0_mask_0 / np.sqrt(np.prod(self.N)) / np.sqrt(
            2 - 2 / self.dim)
        self.linear_operator = -viscosity * self.k2
        self.correlation_func = np.zeros(self.shape_spectral)
        self.forcing_cfg = forcing
        cfg = build_config(self.N, self.domain, is_nonlinear, integrator_id, viscosity,
                           noise_type, noise_mag, self.nyquist_mask is not None, precision, dt,
                           seed, noise_source, forcing, cfl, fused, dealias=self.dealias_rule)
        self._u_host = None
        self._rhs_ready = False
        h = C.c_void_p()
        N.check(N.lib().pf_create(C.byref(cfg), C.byref(h)), None, "pf_create")
        self._h = h
        self._cfg = cfg

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                N.lib().pf_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._h = None

    # ------------------------------------------------------------ state views
    @property
    def u_hat(self) -> np.ndarray:
        out = np.empty(self.shape_local_fourier, dtype=np.complex128)
        N.check(N.lib().pf_get_fourier(self._h, out.ctypes.data, 0), self._h, "get u_hat")
        return out

    @u_hat.setter
    def u_hat(self, value):
        a = np.ascontiguousarray(np.broadcast_to(value, self.shape_local_fourier),
                                 dtype=np.complex128)
        N.check(N.lib().pf_set_fourier(self._h, a.ctypes.data, 0), self._h, "set u_hat")

    @property
    def u(self) -> np.ndarray:
        """Physical velocity: the backward transform of the current state,
        written into this solver's host array (the same array object on every
        access), so in-place edits of it reach the state through forward()."""
        if self._u_host is None:
            self._u_host = np.empty(self.shape_local_physical, dtype=np.float64)
        N.check(N.lib().pf_get_physical(self._h, self._u_host.ctypes.data, 0), self._h, "get u")
        return self._u_host

    @u.setter
    def u(self, value):
        a = np.ascontiguousarray(np.broadcast_to(value, self.shape_local_physical),
                                 dtype=np.float64)
        N.check(N.lib().pf_set_physical(self._h, a.ctypes.data, 0), self._h, "set u")
        if self._u_host is None:
            self._u_host = np.empty(self.shape_local_physical, dtype=np.float64)
        self._u_host[...] = a

    # space_solver.py:180-213
    def initialize_velocity(self, u0, space: str = "physical", mask_zero_mode: bool = True):
        if space.casefold() == "physical":
            if tuple(np.shape(u0)) != self.shape_local_physical:
                raise ValueError(
                    "SpaceSolver.initialize_velocity: Invalid shape for the input physical "
                    f"velocity. Expected {self.shape_local_physical}, got {np.shape(u0)}.")
            self.u = u0
        elif space.casefold() == "fourier":
            if tuple(np.shape(u0)) != self.shape_local_fourier:
                raise ValueError(
                    "SpaceSolver.initialize_velocity: Invalid shape for the input Fourier "
                    f"velocity. Expected {self.shape_local_fourier}, got {np.shape(u0)}.")
            self.u_hat = u0
            if mask_zero_mode:
                N.check(N.lib().pf_mask_zero_mode(self._h), self._h, "mask zero mode")
        else:
            raise ValueError("SpaceSolver.initialize_velocity: Invalid space type. Options are "
                             "'physical' or 'fourier'.")

    def project(self):
        """Leray projection of the state in place (math.leray_projection on u_hat)."""
        N.check(N.lib().pf_project(self._h), self._h, "project")

    def forward(self, u=None):
        """V.forward (space_solver.py:215-219): the physical field -- ``u`` if
        given, else this solver's host array ``self.u`` as last read or
        edited in place -- transformed into the state."""
        if u is None:
            u = self._u_host if self._u_host is not None else self.u
        self.u = u

    def backward(self):
        """V.backward (space_solver.py:221-225): returns the physical field."""
        return self.u

    def set_linear_operator(self, L):
        L = np.ascontiguousarray(np.broadcast_to(L, self.shape_spectral), dtype=np.float64)
        self.linear_operator[...] = L
        N.check(N.lib().pf_set_linear_operator(self._h, L.ctypes.data, 0), self._h,
                "set_linear_operator")

    def set_correlation_function(self, Cf):
        Cf = np.ascontiguousarray(np.broadcast_to(np.real(Cf), self.shape_spectral),
                                  dtype=np.float64)
        self.correlation_func[...] = Cf
        N.check(N.lib().pf_set_correlation(self._h, Cf.ctypes.data, 0), self._h,
                "set_correlation_function")

    # ---------------------------------------------------------------- noise
    def random_fields(self):
        """Draw w1, w2 for the next step with NumPy's global generator in the
        reference's order (space_solver.py:227-238) and hand them to the device."""
        shape = (self.ncomp,) + self.shape_spectral
        w1 = np.random.randn(*shape) + 1j * np.random.randn(*shape)
        w2 = np.random.randn(*shape) + 1j * np.random.randn(*shape)
        w1 *= self._noise_normal_factor
        w2 *= self._noise_normal_factor
        self.inject_noise(w1, w2)
        return w1, w2

    def inject_noise(self, w1, w2):
        shape = (self.ncomp,) + self.shape_spectral
        a = np.ascontiguousarray(np.broadcast_to(w1, shape), dtype=np.complex128)
        b = np.ascontiguousarray(np.broadcast_to(w2, shape), dtype=np.complex128)
        N.check(N.lib().pf_inject_noise(self._h, a.ctypes.data, b.ctypes.data, 0), self._h,
                "inject_noise")

    def compute_rhs(self, a: float = 0.0):
        """Assemble the right-hand side of the current state with noise factor
        ``a`` (space_solver.py:302-310) into ``rhs_linear``, ``rhs_nonlinear``,
        ``noise``, ``forcing`` and ``p_hat``.  The time step does not need
        this call: on the device each stage computes these terms per mode
        inside its update.  The noise uses the fields of the next step."""
        N.check(N.lib().pf_compute_rhs(self._h, float(a)), self._h, "compute_rhs")
        self._rhs_ready = True

    def _rhs_array(self, name):
        shape = self.shape_spectral if name == "p_hat" else self.shape_local_fourier
        out = np.zeros(shape, dtype=np.complex128)
        if self._rhs_ready:
            N.check(N.lib().pf_get_rhs(self._h, N.PF_RHS[name], out.ctypes.data, 0), self._h,
                    f"get {name}")
        return out

    # arrays of the reference's SpaceSolver (space_solver.py:152-178) as host
    # copies of the last compute_rhs (zeros before it)
    rhs_linear = property(lambda self: self._rhs_array("rhs_linear"))
    rhs_nonlinear = property(lambda self: self._rhs_array("rhs_nonlinear"))
    noise = property(lambda self: self._rhs_array("noise"))
    forcing = property(lambda self: self._rhs_array("forcing"))
    p_hat = property(lambda self: self._rhs_array("p_hat"))

    # ------------------------------------------------------------ diagnostics
    def energy(self):
        e, z = C.c_double(), C.c_double()
        N.check(N.lib().pf_energy(self._h, C.byref(e), C.byref(z)), self._h, "energy")
        return e.value, z.value

    def spectrum(self, nbins: int | None = None):
        if nbins is None:
            nbins = int(np.sqrt(sum((n // 2) ** 2 for n in self.N))) + 2
        out = np.zeros(nbins)
        N.check(N.lib().pf_spectrum(self._h, out.ctypes.data, nbins), self._h, "spectrum")
        return out

    def step(self, nsteps: int):
        N.check(N.lib().pf_step(self._h, int(nsteps)), self._h, "step")

    def set_stream(self, stream):
        """Order this solver's device work on ``stream`` (torch.cuda.Stream,
        raw cudaStream_t as int, or None for the legacy default stream)."""
        ptr = getattr(stream, "cuda_stream", stream)
        N.check(N.lib().pf_set_stream(self._h, C.c_void_p(ptr) if ptr else None), self._h,
                "set_stream")

    def footprint(self) -> int:
        return device_footprint(self._cfg)

    def capture(self, nsteps: int):
        """Record "advance ``nsteps``" as a CUDA graph (needs a stream set with
        set_stream and a noise-free run); replay() then costs one launch."""
        N.check(N.lib().pf_graph_capture(self._h, int(nsteps)), self._h, "graph capture")
        self._graph_steps = int(nsteps)

    def replay(self):
        N.check(N.lib().pf_graph_replay(self._h), self._h, "graph replay")

    def autotune(self) -> dict:
        """Time the launch variants of the fused passes on this solver's
        buffers and keep the fastest (later solvers of the same geometry in
        this process start from them).  The state is unchanged."""
        picks = (C.c_int * 12)()
        N.check(N.lib().pf_autotune(self._h, picks), self._h, "autotune")
        return {"axes_256": list(picks[:6]), "axes_384": list(picks[6:])}

    def fused_variants(self) -> dict:
        out = (C.c_int * 12)()
        N.check(N.lib().pf_fused_variants(self._h, out), self._h, "fused variants")
        return {"axes_256": list(out[:6]), "axes_384": list(out[6:])}

    def time(self):
        t, s, dt = C.c_double(), C.c_longlong(), C.c_double()
        N.check(N.lib().pf_get_time(self._h, C.byref(t), C.byref(s), C.byref(dt)), self._h, "time")
        return t.value, s.value, dt.value

    def set_time(self, t: float, step: int):
        N.check(N.lib().pf_set_time(self._h, float(t), int(step)), self._h, "set_time")

    def record_history(self, enable: bool = True):
        N.check(N.lib().pf_record_history(self._h, int(bool(enable))), self._h, "record_history")

    def history(self):
        cap = 1 << 20
        out = np.zeros((cap, 2))
        cnt = C.c_int()
        N.check(N.lib().pf_history(self._h, out.ctypes.data, cap, C.byref(cnt)), self._h, "history")
        return out[:cnt.value].copy()


__all__ = ["SpaceSolver", "logger"]
