"""Radial slabs on CPU: the row split, slab states and their reassembly, and
the rank protocol of fargo3d_b200.slabs.RankSlab (MIN of the CFL minimum,
halo exchange with both neighbours) on two gloo ranks with a host engine."""
import ctypes as C
import os
import socket

import numpy as np
import pytest


def test_split_rows_and_reassembly():
    from fargo3d_b200 import config_fargo2d, initial_state
    from fargo3d_b200.slabs import assemble, slab_configs, slab_rows, split_rows
    assert split_rows(128, 3) == [(0, 43), (43, 43), (86, 42)]
    assert split_rows(10, 4) == [(0, 3), (3, 3), (6, 2), (8, 2)]
    cfg = config_fargo2d(16, 10, seed=1)
    cs = slab_configs(cfg, 3)
    assert [c.ny for c in cs] == [4, 3, 3] and [c.slab_y0 for c in cs] == [0, 4, 7]
    assert all(c.slab_ny_global == 10 for c in cs)
    rho = initial_state(cfg)[0]
    rows = split_rows(10, 3)
    parts = [slab_rows(rho, y0, n) for y0, n in rows]
    assert parts[1].shape == (1, 3 + 6, 16)
    assert np.array_equal(parts[1][:, 3:6], rho[:, 7:10])      # active rows 4..6 of the whole disk
    assert np.array_equal(assemble(parts, rows), rho)


class HostSlab:
    """A stand-in slab engine on host arrays: a field of rows, a 'step' that
    adds the time step to the active rows."""

    def __init__(self, rank, ny=5, nx=8):
        self.ny, self.nx = ny, nx
        self.f = np.full((3, 1, ny + 6, nx), -1.0)
        self.f[:, :, 3:ny + 3, :] = rank * 100 + np.arange(ny)[None, None, :, None] + 0.01 * np.arange(nx)
        self.rank = rank

    def halo_bytes(self, which):
        return 3 * 1 * 3 * self.nx * 8

    def halo(self, which, side, unpack, ptr, on_host):
        assert on_host
        buf = np.ctypeslib.as_array((C.c_double * (3 * 3 * self.nx)).from_address(ptr)).reshape(3, 1, 3, self.nx)
        j0 = (0 if side == 0 else self.ny + 3) if unpack else (3 if side == 0 else self.ny)
        if unpack:
            self.f[:, :, j0:j0 + 3, :] = buf
        else:
            buf[...] = self.f[:, :, j0:j0 + 3, :]

    def initialize(self):
        pass

    def step_begin(self):
        return 0.5 + self.rank          # rank 0 holds the minimum

    def step_advance(self, dt_interval, cfl):
        self.dt = cfl
        return cfl

    def step_transport(self):
        self.f[:, :, 3:self.ny + 3, :] += self.dt


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from fargo3d_b200.slabs import RankSlab
    eng = HostSlab(rank)
    rs = RankSlab(eng, rank, world, on_host=True)
    rs.initialize()
    dts = [rs.step() for _ in range(2)]
    q.put((rank, dts, eng.f.copy()))
    dist.barrier()
    dist.destroy_process_group()


def test_rank_slabs_exchange_and_min_on_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (dts, f)) for r, dts, f in (q.get(timeout=120) for _ in ps))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (dt0, f0), (dt1, f1) = res[0], res[1]
    assert dt0 == dt1 == [0.5, 0.5]                       # MIN over the ranks
    ny = 5
    # after the last exchange: rank 0's outer ghosts = rank 1's first rows, and back
    assert np.array_equal(f0[:, :, ny + 3:ny + 6], f1[:, :, 3:6])
    assert np.array_equal(f1[:, :, 0:3], f0[:, :, ny:ny + 3])
    # the mesh's own edges (rank 0 inner, rank 1 outer) are not touched by the exchange
    assert np.all(f0[:, :, 0:3] == -1.0) and np.all(f1[:, :, ny + 3:] == -1.0)
