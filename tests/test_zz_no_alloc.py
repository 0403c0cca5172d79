"""pf_backward_noalloc: the backward transform for callers that cannot
allocate device memory (a fixed budget handed over by an embedding
application, a context where the allocator must not be entered).  Its work
copy lives in the library's fixed 32 MiB device array instead of memory the
call allocates.

Called through the C ABI on device arrays and checked against the existing
entry point (pf_get_physical on a solver handle) within the tolerances the
other parity tests use, on two calls in a row with different inputs, so a
call that read stale scratch contents from the previous one would fail.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 1e-5}


def _solver(N, precision):
    from periodicflow import simulation as sim
    return sim.Solver(list(N), 0.01, 1.0, is_nonlinear=False, dealias="2/3",
                      precision=precision)


def _spectral(s, seed):
    """A Hermitian-consistent random spectrum: forward transform of noise."""
    rng = np.random.default_rng(seed)
    ss = s.space_solver
    ss.u = rng.standard_normal(ss.shape_local_physical)
    return ss.u_hat


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("N", [(32, 32, 32), (16, 64, 32), (64, 64), (256, 128)])
def test_noalloc_backward_matches_get_physical(precision, N):
    import torch
    from periodicflow import _native as nat
    lib = nat.lib()
    s = _solver(N, precision)
    ss = s.space_solver
    cdt = torch.complex128 if precision == "fp64" else torch.complex64
    rdt = torch.float64 if precision == "fp64" else torch.float32
    prec = nat.PF_FP64 if precision == "fp64" else nat.PF_FP32
    n = (C.c_int * len(N))(*N)
    for seed in (1, 2):  # two calls in a row
        uh = _spectral(s, seed)
        ref = ss.u  # existing entry point: pf_get_physical
        uh_dev = torch.from_numpy(uh).to(cdt).cuda()
        u_dev = torch.empty(ss.shape_local_physical, dtype=rdt, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = lib.pf_backward_noalloc(prec, len(N), n, C.c_void_p(uh_dev.data_ptr()),
                                     C.c_void_p(u_dev.data_ptr()), C.c_void_p(stream))
        assert rc == nat.PF_OK, lib.pf_last_error(None)
        torch.cuda.synchronize()
        got = u_dev.cpu().numpy().astype(np.float64)
        assert rel_l2(got, ref) < TOL[precision], (seed, rel_l2(got, ref))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from periodicflow import _native as nat
    lib = nat.lib()
    n = (C.c_int * 3)(256, 256, 256)  # 3 * 256*256*129 complex128 > 32 MiB
    rc = lib.pf_backward_noalloc(nat.PF_FP64, 3, n, C.c_void_p(16), C.c_void_p(16), None)
    assert rc == 1
    assert b"32 MiB" in lib.pf_last_error(None) or b"33554432" in lib.pf_last_error(None)
