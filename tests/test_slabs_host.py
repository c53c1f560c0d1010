"""z-slab decomposition and the halo exchange of one box over ranks: the
plane bookkeeping on the host, and the exchange and MIN reduction as two
gloo ranks on CPU with a host stand-in for the device box."""
import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from isothermal_mhd_b200.slabs import Decomposition, RankSlab, halo_width


def test_decomposition_scatter_gather_round_trip():
    dec = Decomposition((4, 3, 23), 3, 5)
    assert dec.counts == [8, 8, 7] and dec.starts == [0, 8, 16]
    a = np.random.default_rng(0).random((2, 23, 3, 4))
    parts = [dec.scatter(a, r) for r in range(3)]
    assert parts[0].shape == (2, 18, 3, 4)
    # halo planes are the periodic neighbours' planes
    np.testing.assert_array_equal(parts[0][:, :5], a[:, 18:23])
    np.testing.assert_array_equal(parts[2][:, -5:], a[:, 0:5])
    np.testing.assert_array_equal(dec.gather(parts), a)


def test_halo_width_and_too_thin_slabs():
    assert halo_width("plm", 0) == 5 and halo_width("ppm", 2) == 7
    with pytest.raises(ValueError):
        Decomposition(16, 4, 6)


class HostSlab:
    """Stand-in for a device slab: planes of a (nf, nz, ny, nx) float64 array."""

    def __init__(self, a, dt_local, sums=None):
        self.a = a
        self.dt_local = dt_local
        self.sums = sums
        self.global_sums = None

    def pack_planes(self, z0, n):
        return torch.from_numpy(np.ascontiguousarray(self.a[:, z0:z0 + n]).reshape(-1).copy())

    def unpack_planes(self, z0, n, t):
        self.a[:, z0:z0 + n] = t.numpy().reshape(self.a.shape[0], n, *self.a.shape[2:])

    def force_sums(self):
        return self.sums

    def set_force_sums(self, s):
        self.global_sums = np.asarray(s)

    def step(self, dt, drive=False):
        return self.dt_local


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    dec = Decomposition((3, 2, 14), world, 3)
    g = np.arange(2 * 14 * 2 * 3, dtype=np.float64).reshape(2, 14, 2, 3)
    local = dec.scatter(g, rank).copy()
    h = dec.halo
    local[:, :h] = -1.0                      # stale halos
    local[:, -h:] = -1.0
    slab = RankSlab(dec, rank, HostSlab(local, 0.1 * (rank + 1)), dist)
    dt = slab.step(1.0)
    ok = np.array_equal(local, dec.scatter(g, rank)) and dt == 0.1
    q.put((rank, ok))
    dist.destroy_process_group()


def _drive_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    dec = Decomposition((3, 2, 14), world, 3)
    local = np.zeros((2, dec.local_nz(rank), 2, 3))
    box = HostSlab(local, 0.1, sums=np.arange(1.0, 6.0) * (rank + 1))
    RankSlab(dec, rank, box, dist).step(1.0, drive=True)
    expect = np.arange(1.0, 6.0) * sum(r + 1 for r in range(world))
    q.put((rank, box.global_sums is not None and np.array_equal(box.global_sums, expect)))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_add_up_forcing_sums_on_drive_steps(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + world + (os.getpid() % 1000)
    procs = [ctx.Process(target=_drive_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] for r in range(world)), res


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_halos_and_reduce_dt(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + world + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert all(res[r] for r in range(world)), res
