"""Pointwise spectral / physical operators (the reference's math.py:4-100) as
CUDA kernels behind the C ABI.  Arguments are CUDA tensors (complex64/float32
or complex128/float64) or NumPy arrays; outputs are written in place."""
from __future__ import annotations

import ctypes as C

from . import _native as N
from ._dev import Arg, precision_of, real_dtype, stream_ptr


def _shape(a, lead: int):
    s = tuple(a.shape[lead:]) if lead else tuple(a.shape)
    return (C.c_longlong * len(s))(*s), len(s)


def cross(c, a, b):
    """u x w; 2D: (a1 b, -a0 b) with scalar b (math.py:4-28)."""
    prec = precision_of(a)
    rd = real_dtype(prec)
    A, B, Cc = Arg(a, rd, False), Arg(b, rd, False), Arg(c, rd, False)
    shp, dim = _shape(a, 1)
    N.check(N.lib().pf_op_cross(prec, dim, shp, Cc.ptr, A.ptr, B.ptr, stream_ptr()), None, "cross")
    Cc.write_back()


def curl(c, k, a):
    """c = i k x a; 2D gives the scalar i (k0 a1 - k1 a0) (math.py:31-49)."""
    prec = precision_of(a)
    rd = real_dtype(prec)
    A, K, Cc = Arg(a, rd, True), Arg(k, rd, False), Arg(c, rd, True)
    shp, dim = _shape(a, 1)
    N.check(N.lib().pf_op_curl(prec, dim, shp, Cc.ptr, K.ptr, A.ptr, stream_ptr()), None, "curl")
    Cc.write_back()


def apply_linear_operator(Lu, L, u):
    """Lu[i] = L * u[i] (math.py:52-68)."""
    prec = precision_of(u)
    rd = real_dtype(prec)
    U, Lr, Out = Arg(u, rd, True), Arg(L, rd, False), Arg(Lu, rd, True)
    shp, dim = _shape(u, 1)
    N.check(N.lib().pf_op_apply_linear_operator(prec, dim, shp, Out.ptr, Lr.ptr, U.ptr,
                                                stream_ptr()), None, "apply_linear_operator")
    Out.write_back()


def leray_projection(u, k, k_k2, p_hat):
    """p = (k/k^2).u ; u -= p k, in place; p stored in p_hat (math.py:71-100)."""
    prec = precision_of(u)
    rd = real_dtype(prec)
    U, K, KK, P = Arg(u, rd, True), Arg(k, rd, False), Arg(k_k2, rd, False), Arg(p_hat, rd, True)
    shp, dim = _shape(u, 1)
    N.check(N.lib().pf_op_leray_projection(prec, dim, shp, U.ptr, K.ptr, KK.ptr, P.ptr,
                                           stream_ptr()), None, "leray_projection")
    U.write_back()
    P.write_back()


def symmetrize(w_sym, w):
    """(W + W^T) sqrt(1/2) of a d x d tensor field (space_solver.py:15-42)."""
    prec = precision_of(w)
    rd = real_dtype(prec)
    W, S = Arg(w, rd, True), Arg(w_sym, rd, True)
    shp, dim = _shape(w, 1)
    N.check(N.lib().pf_op_symmetrize(prec, dim, shp, S.ptr, W.ptr, stream_ptr()), None,
            "symmetrize")
    S.write_back()


def noise_divergence(noise, w_sym, k):
    """noise_a = i sum_b k_b W_sym[a, b] (space_solver.py:45-64)."""
    prec = precision_of(w_sym)
    rd = real_dtype(prec)
    W, K, Nz = Arg(w_sym, rd, True), Arg(k, rd, False), Arg(noise, rd, True)
    shp, dim = _shape(w_sym, 1)
    N.check(N.lib().pf_op_noise_divergence(prec, dim, shp, Nz.ptr, W.ptr, K.ptr, stream_ptr()),
            None, "noise_divergence")
    Nz.write_back()
