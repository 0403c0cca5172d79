"""ctypes binding of libpfb200.so (the C ABI declared in include/periodicflow_b200.h).

The library is the only compute path of this package: importing a module that
needs it fails loudly when it is missing, and no CPU fallback exists.
"""
from __future__ import annotations

import ctypes as C
import os

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libpfb200.so")

PF_OK = 0
PF_EXPLICIT_PC, PF_IMPLICIT_PC, PF_RK2, PF_RK3, PF_RK4 = range(5)
PF_NOISE_THERMAL, PF_NOISE_CORRELATED = 0, 1
PF_NOISE_SRC_PHILOX, PF_NOISE_SRC_INJECTED = 1, 2
PF_DEALIAS_TRUNCATE, PF_DEALIAS_PAD = 0, 1
PF_FP32, PF_FP64 = 0, 1
PF_PASS_UPDATE, PF_PASS_FFT_STRIDED, PF_PASS_FFT_LAST, PF_PASS_STOKES = 0, 1, 2, 4
PF_PASS_FUSED = {1: 11, 2: 12, 3: 13, 4: 14, 5: 15}
PF_RHS = {"rhs_linear": 0, "rhs_nonlinear": 1, "noise": 2, "forcing": 3, "p_hat": 4}


class PfConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("n", C.c_int * 3),
        ("domain", (C.c_double * 2) * 3),
        ("is_nonlinear", C.c_int),
        ("integrator", C.c_int),
        ("viscosity", C.c_double),
        ("noise_type", C.c_int),
        ("noise_mag", C.c_double),
        ("dealias", C.c_int),
        ("mask_nyquist", C.c_int),
        ("precision", C.c_int),
        ("dt", C.c_double),
        ("seed", C.c_ulonglong),
        ("noise_source", C.c_int),
        ("forcing_eps", C.c_double),
        ("forcing_kf", C.c_double),
        ("cfl", C.c_double),
        ("fused", C.c_int),
    ]


class NativeError(RuntimeError):
    pass


_lib = None

# (name, restype, argtypes)
_SIGS = [
    ("pf_config_default", C.c_int, [C.POINTER(PfConfig)]),
    ("pf_create", C.c_int, [C.POINTER(PfConfig), C.POINTER(C.c_void_p)]),
    ("pf_destroy", C.c_int, [C.c_void_p]),
    ("pf_footprint", C.c_int, [C.POINTER(PfConfig), C.POINTER(C.c_ulonglong)]),
    ("pf_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pf_last_error", C.c_char_p, [C.c_void_p]),
    ("pf_sizes", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                           C.POINTER(C.c_int)]),
    ("pf_set_fourier", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_get_fourier", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_set_physical", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_get_physical", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_mask_zero_mode", C.c_int, [C.c_void_p]),
    ("pf_project", C.c_int, [C.c_void_p]),
    ("pf_set_linear_operator", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_set_correlation", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_inject_noise", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_step", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_graph_capture", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_graph_replay", C.c_int, [C.c_void_p]),
    ("pf_autotune", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("pf_fused_variants", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("pf_get_time", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                              C.POINTER(C.c_double)]),
    ("pf_set_time", C.c_int, [C.c_void_p, C.c_double, C.c_longlong]),
    ("pf_energy", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    ("pf_history", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    ("pf_record_history", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_spectrum", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    ("pf_create_members", C.c_int, [C.POINTER(PfConfig), C.c_int, C.POINTER(C.c_void_p)]),
    ("pf_footprint_members", C.c_int, [C.POINTER(PfConfig), C.c_int, C.POINTER(C.c_ulonglong)]),
    ("pf_members", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("pf_set_fourier_member", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    ("pf_get_fourier_member", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    ("pf_get_time_member", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]),
    ("pf_energy_member", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)]),
    ("pf_set_active_members", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_copy_member", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("pf_set_time_member", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
    ("pf_compute_rhs", C.c_int, [C.c_void_p, C.c_double]),
    ("pf_get_rhs", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    ("pf_kernel_timer", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_kernel_timer_read", C.c_int, [C.c_void_p, C.POINTER(C.c_double),
                                       C.POINTER(C.c_longlong)]),
    ("pf_launch_count", C.c_int, [C.POINTER(C.c_longlong)]),
    ("pf_backward_noalloc", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
    ("pf_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    ("pf_batch_destroy", C.c_int, [C.c_void_p]),
    ("pf_batch_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pf_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("pf_batch_step", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_batch_capture", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_batch_replay", C.c_int, [C.c_void_p]),
    ("pf_batch_sync", C.c_int, [C.c_void_p]),
    ("pf_slab_layout", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    ("pf_slab_create_group", C.c_int, [C.POINTER(PfConfig), C.c_int, C.POINTER(C.c_void_p)]),
    ("pf_slab_create", C.c_int, [C.POINTER(PfConfig), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("pf_slab_export", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("pf_slab_nccl_id", C.c_int, [C.c_void_p, C.c_size_t]),
    ("pf_slab_connect", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("pf_slab_destroy", C.c_int, [C.c_void_p]),
    ("pf_slab_last_error", C.c_char_p, [C.c_void_p]),
    ("pf_slab_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("pf_slab_sizes", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_longlong)]),
    ("pf_slab_set_fourier", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    ("pf_slab_get_fourier", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    ("pf_slab_step", C.c_int, [C.c_void_p, C.c_int]),
    ("pf_slab_sync", C.c_int, [C.c_void_p]),
    ("pf_slab_get_time", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong),
                                   C.POINTER(C.c_double)]),
    ("pf_slab_energy", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]),
    ("pf_op_cross", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_longlong)] + [C.c_void_p] * 4),
    ("pf_op_curl", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_longlong)] + [C.c_void_p] * 4),
    ("pf_op_apply_linear_operator", C.c_int,
     [C.c_int, C.c_int, C.POINTER(C.c_longlong)] + [C.c_void_p] * 4),
    ("pf_op_leray_projection", C.c_int,
     [C.c_int, C.c_int, C.POINTER(C.c_longlong)] + [C.c_void_p] * 5),
    ("pf_op_symmetrize", C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_longlong)] + [C.c_void_p] * 3),
    ("pf_op_noise_divergence", C.c_int,
     [C.c_int, C.c_int, C.POINTER(C.c_longlong)] + [C.c_void_p] * 4),
    ("pf_op_stepping", C.c_int,
     [C.c_int, C.c_int, C.c_int, C.c_double, C.c_longlong] + [C.c_void_p] * 7
     + [C.c_longlong, C.c_void_p]),
]

EXPORTED = [s[0] for s in _SIGS]


def library_path() -> str:
    return _LIB_PATH


def lib():
    """Load the C-ABI library (once); raise if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(
                f"periodicflow CUDA backend library not found at {_LIB_PATH}; build it with "
                "`python periodic-flow_b200/csrc/build.py` (there is no CPU fallback)")
        L = C.CDLL(_LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, handle=None, what: str = "", errfn=None):
    if rc != PF_OK:
        msg = (errfn or lib().pf_last_error)(handle)
        msg = msg.decode() if msg else ""
        if rc == 1:
            raise ValueError(f"{what}: {msg}")
        if rc == 3:
            raise NotImplementedError(f"{what}: {msg}")
        raise NativeError(f"{what} failed (status {rc}): {msg}")
