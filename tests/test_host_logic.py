"""CPU tests of host-side logic: geometry, initial fields, loop bookkeeping,
writer layout, the communicator stand-in (gloo, world size 2)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O


def test_fourier_space_matches_oracle_grid():
    from periodicflow import _comm
    from periodicflow.basis import FourierSpace
    for N, dom in [((8, 16), 2 * np.pi), ((16, 8, 32), [(0, 2 * np.pi), (0, np.pi), (0, 4 * np.pi)])]:
        fs = FourierSpace(_comm.COMM_WORLD, 0, N, domain=dom, dealias="2/3", mask_nyquist=True)
        g = O.Grid(N, domain=dom, mask_nyquist=True)
        np.testing.assert_array_equal(fs.k, g.k)
        np.testing.assert_array_equal(fs.k2, g.k2)
        np.testing.assert_array_equal(fs.k_over_k2, g.k_over_k2)
        np.testing.assert_array_equal(fs.nyquist_mask, g.nyquist_mask)
        for a, b in zip(fs.x, g.x):
            np.testing.assert_array_equal(a, b)


def test_domain_parsing_and_errors():
    from periodicflow import _comm
    from periodicflow.basis import FourierSpace
    fs = FourierSpace(_comm.COMM_WORLD, 0, (8, 8), domain=(0.0, 1.0))
    assert fs.domain == [(0.0, 1.0), (0.0, 1.0)]
    with pytest.raises(ValueError):
        FourierSpace(_comm.COMM_WORLD, 0, (8, 8), domain=3)
    with pytest.raises(ValueError):
        FourierSpace(_comm.COMM_WORLD, 0, (8, 8), dealias="1/2")


def test_initial_fields_match_oracle():
    from periodicflow import _comm
    from periodicflow.basis import FourierSpace
    from periodicflow.initial import spectral_random_field, taylor_green
    N = (32, 32, 32)
    fs = FourierSpace(_comm.COMM_WORLD, 0, N, dealias="2/3")
    g = O.Grid(N)
    np.testing.assert_allclose(spectral_random_field(fs, 1), O.spectral_random_field(g, 1),
                               rtol=1e-12, atol=1e-15)
    np.testing.assert_array_equal(taylor_green(fs.x), O.taylor_green(g))
    uh = spectral_random_field(fs, 1)
    assert abs(O.energy(g, uh) - 0.5) < 1e-12
    assert np.max(np.abs(np.sum(g.k * uh, axis=0))) < 1e-12


def test_steps_to_end_matches_reference_loop():
    from periodicflow.simulation import Solver
    class S:  # only the fields _steps_to_end reads
        end_time = 10
    for dt, end in [(1e-3, 10), (0.01, 10), (0.02, 1.0), (0.005, 2.0)]:
        S.end_time = end
        t, n = 0.0, 0
        while not np.isclose(t, end, atol=1e-10):
            t += dt
            n += 1
        assert Solver._steps_to_end(S, 0.0, dt) == n
    S.end_time = 1.0
    with pytest.raises(RuntimeError):
        Solver._steps_to_end(S, 0.0, 0.3)


def test_periodic_bc_and_timer_format():
    from periodicflow.utils import Timer, periodic_bc
    a = np.arange(6.0).reshape(2, 3)
    b = periodic_bc(a)
    assert b.shape == (3, 4) and b[2, 0] == a[0, 0] and b[0, 3] == a[0, 0]
    assert Timer._format_time(3723.0, "hh:mm:ss") == "01:02:03"
    assert Timer._format_time(90061.0) == "01-01:01:01"
    with pytest.raises(ValueError):
        Timer._format_time(1.0, "x")


def test_writer_layout_without_h5py(tmp_path):
    from periodicflow.io import HDF5Writer
    class Fake:
        dim = 2
        x = [np.arange(4.0).reshape(4, 1), np.arange(4.0).reshape(1, 4)]
        u = np.ones((2, 4, 4))
    w = HDF5Writer(None, 0, 1, str(tmp_path / "sol"), solver=Fake(), component_names=["u", "v"],
                   time_points=[0.0, 1.0], end_points=[4.0, 4.0], periodic=True)
    for s in (0, 5, 10):
        w.write(s)
    path = w.reconfigure_dataset()
    z = np.load(path)
    assert set(z.files) == {"x", "y", "t", "u/00", "u/05", "u/10", "v/00", "v/05", "v/10"}
    assert z["u/05"].shape == (5, 5) and z["x"][-1] == 4.0
    np.testing.assert_allclose(z["t"], [0.0, 0.5, 1.0])


def _comm_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from periodicflow import _comm
    c = _comm.COMM_WORLD
    res = (c.Get_rank(), c.Get_size(), c.allreduce(rank + 1.0), c.bcast({"L": 0.5} if rank == 0 else None))
    c.Barrier()
    out.put(res)
    dist.destroy_process_group()


def test_comm_stand_in_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    ps = [ctx.Process(target=_comm_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 2 and r[2] == 3.0 and r[3] == {"L": 0.5} for r in res)
