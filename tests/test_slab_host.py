"""Host logic of the slab decomposition (no GPU): the partition of a box into
slabs (pf_slab_layout) against a restatement of the shenfun slab split
(basis.py:64: spectral arrays split along axis 1 in equal blocks), the
checks applied before any device use, and the cross-process handshake
(exports in rank order, rank 0's NCCL id) over two gloo ranks."""
import ctypes
import multiprocessing as mp
import os

import pytest

from periodicflow import _native as N


def _kfreq(i, n):
    return i if i <= (n - 1) // 2 else i - n


def _layout(n0, n1, S, r):
    """Slab r of S: equal blocks of planes x0 and rows k1; its kept 2/3-rule
    rows (|k1| <= (n1-1)//3) as a range of compact indices."""
    kmax = (n1 - 1) // 3
    c1 = 2 * kmax + 1
    rows = range(r * (n1 // S), (r + 1) * (n1 // S))
    comp = [i if i <= kmax else i - (n1 - c1) for i in rows if abs(_kfreq(i, n1)) <= kmax]
    assert comp == list(range(comp[0], comp[0] + len(comp))) if comp else True
    return [n0 // S, n1 // S, r * (n0 // S), r * (n1 // S), comp[0] if comp else 0, len(comp)]


@pytest.mark.parametrize("n0,n1", [(16, 16), (32, 48), (64, 256), (256, 256), (96, 384), (512, 64)])
@pytest.mark.parametrize("S", [1, 2, 4, 8])
def test_slab_layout_matches_restatement(n0, n1, S):
    if n0 % S or n1 % S:
        pytest.skip("slabs must divide the sides")
    total = 0
    for r in range(S):
        out = (ctypes.c_int * 6)()
        assert N.lib().pf_slab_layout(n0, n1, S, r, out) == 0
        assert list(out) == _layout(n0, n1, S, r)
        total += out[5]
    assert total == 2 * ((n1 - 1) // 3) + 1  # every kept row in exactly one slab


def test_slab_layout_rejects_bad_arguments():
    out = (ctypes.c_int * 6)()
    assert N.lib().pf_slab_layout(32, 48, 5, 0, out) == 1   # 5 divides neither side
    assert N.lib().pf_slab_layout(32, 32, 9, 0, out) == 1   # more than 8 slabs
    assert N.lib().pf_slab_layout(32, 32, 2, 2, out) == 1   # no slab 2 of 2


def _cfg(**kw):
    cfg = N.PfConfig()
    N.lib().pf_config_default(ctypes.byref(cfg))
    cfg.dim = 3
    for a, n in enumerate(kw.pop("n", (32, 32, 32))):
        cfg.n[a] = n
    cfg.dealias = N.PF_DEALIAS_TRUNCATE
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def test_slab_checks_before_device_use():
    h = ctypes.c_void_p()
    lib = N.lib()
    assert lib.pf_slab_create_group(ctypes.byref(_cfg(n=(32, 48, 32))), 5, ctypes.byref(h)) == 1
    assert b"divide" in lib.pf_slab_last_error(None)
    assert lib.pf_slab_create_group(ctypes.byref(_cfg(dealias=N.PF_DEALIAS_PAD)), 2,
                                    ctypes.byref(h)) == 3
    assert lib.pf_slab_create_group(ctypes.byref(_cfg(is_nonlinear=0)), 2, ctypes.byref(h)) == 3
    assert lib.pf_slab_create_group(
        ctypes.byref(_cfg(noise_mag=0.1, noise_type=N.PF_NOISE_CORRELATED)), 2,
        ctypes.byref(h)) == 3
    assert lib.pf_slab_create_group(ctypes.byref(_cfg(n=(16, 16, 16))), 8, ctypes.byref(h)) == 3
    assert lib.pf_slab_create(ctypes.byref(_cfg()), 2, 2, ctypes.byref(h)) == 1
    assert not h.value


def test_slab_create_fails_loudly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from periodicflow.slab import SlabGroup
    with pytest.raises(N.NativeError):
        SlabGroup((32, 32, 32), 1e-3, 2, time_integrator="rk3")


def _handshake_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from periodicflow import _comm
    from periodicflow.slab import exchange_handshake
    calls = []

    def make_id():
        calls.append(rank)
        return bytes([7]) * 128

    exports, nid = exchange_handshake(_comm.COMM_WORLD, bytes([rank + 1]) * 128, make_id)
    out.put((rank, exports, nid, calls))
    dist.destroy_process_group()


def test_handshake_over_gloo():
    """Two ranks: every rank gets all exports in rank order and rank 0's id
    (drawn once, on rank 0)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_handshake_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    for rank, exports, nid, calls in res:
        assert exports == bytes([1]) * 128 + bytes([2]) * 128
        assert nid == bytes([7]) * 128
        assert calls == ([0] if rank == 0 else [])
