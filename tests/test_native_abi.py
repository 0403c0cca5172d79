"""CPU checks of the C-ABI library: it loads, exports every declared symbol,
and the ctypes mirror of pf_config has the C layout (measured with gcc)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "periodicflow_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(pf_\w+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    from periodicflow import _native as N
    lib = N.lib()
    decl = declared_symbols()
    assert len(decl) >= 29
    for name in decl:
        assert hasattr(lib, name), name
    assert set(decl) == set(N.EXPORTED)


def test_config_layout_matches_c():
    from periodicflow import _native as N
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "periodicflow_b200.h"
int main(void) {
  printf("%zu", sizeof(pf_config));
#define O(f) printf(" %zu", offsetof(pf_config, f));
  O(dim) O(n) O(domain) O(is_nonlinear) O(integrator) O(viscosity) O(noise_type)
  O(noise_mag) O(dealias) O(mask_nyquist) O(precision) O(dt) O(seed) O(noise_source)
  O(forcing_eps) O(forcing_kf) O(cfl) O(fused)
  printf("\n");
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write(src)
        subprocess.check_call(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    fields = ["dim", "n", "domain", "is_nonlinear", "integrator", "viscosity", "noise_type",
              "noise_mag", "dealias", "mask_nyquist", "precision", "dt", "seed", "noise_source",
              "forcing_eps", "forcing_kf", "cfl", "fused"]
    assert vals[0] == ctypes.sizeof(N.PfConfig)
    for f, off in zip(fields, vals[1:]):
        assert getattr(N.PfConfig, f).offset == off, f


def test_config_default_without_gpu():
    from periodicflow import _native as N
    cfg = N.PfConfig()
    assert N.lib().pf_config_default(ctypes.byref(cfg)) == 0
    assert cfg.dim == 3 and cfg.integrator == N.PF_RK2 and abs(cfg.viscosity - 1e-3) < 1e-18
    assert cfg.fused == 1 and cfg.noise_source == N.PF_NOISE_SRC_PHILOX


def test_create_fails_loudly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from periodicflow import _native as N
    cfg = N.PfConfig()
    N.lib().pf_config_default(ctypes.byref(cfg))
    h = ctypes.c_void_p()
    rc = N.lib().pf_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc != 0 and not h.value
    with pytest.raises(N.NativeError):
        N.check(rc, None, "pf_create")


def test_invalid_config_rejected_before_device_use():
    from periodicflow import _native as N
    cfg = N.PfConfig()
    N.lib().pf_config_default(ctypes.byref(cfg))
    cfg.dim = 4
    h = ctypes.c_void_p()
    rc = N.lib().pf_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == N.PF_OK + 1
    assert b"2D and 3D" in N.lib().pf_last_error(None)
    cfg.dim = 3
    cfg.n[1] = 40  # 5 * 8: only 2^b and 3 * 2^b lengths are built
    assert N.lib().pf_create(ctypes.byref(cfg), ctypes.byref(h)) == 3
    cfg.n[1] = 48
    cfg.dealias = N.PF_DEALIAS_PAD  # padded side 72 = 9 * 8 is not built
    assert N.lib().pf_create(ctypes.byref(cfg), ctypes.byref(h)) == 3
    cfg.dealias = 7
    assert N.lib().pf_create(ctypes.byref(cfg), ctypes.byref(h)) == 1


@pytest.mark.parametrize("dim,dealias,precision", [(3, "truncate", "fp32"), (3, "pad", "fp64"),
                                                   (2, "truncate", "fp32")])
def test_member_footprint_is_affine_in_members(dim, dealias, precision):
    """pf_footprint_members: shared scratch once, per-member buffers times the
    member count; one member equals pf_footprint (no device use)."""
    import ctypes as C
    import math
    from periodicflow import _native as N
    from periodicflow.space_solver import build_config
    Ns = (64, 32, 64)[:dim]
    cfg = build_config(Ns, [(0.0, 2 * math.pi)] * dim, True, N.PF_RK3, 2e-3, "thermal", 0.0,
                       False, precision, 1e-3, 0, "philox", None, 0.5, True, dealias=dealias)

    def fp(m):
        b = C.c_ulonglong()
        N.check(N.lib().pf_footprint_members(C.byref(cfg), m, C.byref(b)), None, "footprint")
        return b.value
    one = C.c_ulonglong()
    N.check(N.lib().pf_footprint(C.byref(cfg), C.byref(one)), None, "footprint")
    assert fp(1) == one.value
    assert fp(3) - fp(2) == fp(2) - fp(1) > 0
    assert fp(1) > fp(2) - fp(1)  # the shared scratch is counted once
    with pytest.raises(ValueError):
        fp(0)
