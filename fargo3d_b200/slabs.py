"""One disk split into radial slabs over several GPUs.

The reference runs a large disk on several processes by cutting its mesh
into radial (and colatitude) slabs, each with NGHY = 3 ghost rows per side
that neighbouring slabs fill with their edge rows (split.c:76-213,
comm.c:197-363); every ring stays whole, so the azimuthal means and the FARGO
shift stay local, and the collective work of a step is a MIN of the time
step over the slabs (cfl_fluids_min.c:14-17).  Here a slab is an fb_disk of
the rows [y0, y0 + ny) of the whole mesh (fb_params.slab_y0 /
slab_ny_global): its mesh edges come from the global row index, its
boundary templates apply on the mesh's own edges only.  A step is

    begin (ComputeVmed + cfl)  ->  MIN of the CFL minimum over the slabs
    advance (planets + Sources) ->  exchange the V_temp halos
    transport (+ NewVelocity, Stockholm) -> exchange the state halos

the same two ghost fills per step as the reference (algogas.c:116-118,
main.c:431), so a disk stepped in slabs gives the whole disk's result bit for
bit.  Slabs are FP64 disks of one fluid whose planets do not feel the disk.

`LocalSlabs` keeps every slab in this process (one GPU or several; halos
through device buffers); `RankSlab` is one slab per rank of a
torch.distributed group: NCCL point-to-point sends of the halo buffers into
the neighbour's own buffers and an all-reduce MIN of the time step (gloo
with host buffers where there is no GPU).  The slab engine is anything with
the Disk methods step_begin / step_advance / step_transport / halo_bytes /
halo, so the rank logic runs on CPU with a host-side engine in the tests.
"""
from __future__ import annotations

import dataclasses
from typing import List, Sequence, Tuple

import numpy as np

from .setups import NGH, DiskConfig

HALO_STATE, HALO_VTEMP = 0, 1


def split_rows(ny: int, nslabs: int) -> List[Tuple[int, int]]:
    """(y0, ny) of each slab: the reference's round-robin split (split.c:
    103-113): the first ny % n slabs get one row more."""
    if nslabs < 1 or nslabs > ny:
        raise ValueError("need 1 <= slabs <= ny")
    q, r = divmod(ny, nslabs)
    out, y0 = [], 0
    for k in range(nslabs):
        n = q + 1 if k < r else q
        out.append((y0, n))
        y0 += n
    return out


def slab_configs(cfg: DiskConfig, nslabs: int) -> List[DiskConfig]:
    if cfg.nfluids != 1 or any(p.feel_disk for p in cfg.planets):
        raise ValueError("slabs carry one fluid and planets that do not feel the disk")
    return [dataclasses.replace(cfg, ny=n, slab_y0=y0, slab_ny_global=cfg.ny) for y0, n in split_rows(cfg.ny, nslabs)]


def slab_rows(arr: np.ndarray, y0: int, ny: int) -> np.ndarray:
    """A slab's stored rows (ghosts included) of a whole-disk array: its local
    row jl is the whole disk's stored row jl + y0."""
    return np.ascontiguousarray(arr[:, y0:y0 + ny + 2 * NGH, :])


def assemble(parts: Sequence[np.ndarray], rows: Sequence[Tuple[int, int]]) -> np.ndarray:
    """The whole disk's array from the slabs' arrays (active rows from each,
    the mesh's ghost rows from the first and the last slab)."""
    nz, _, nx = parts[0].shape
    ny = sum(n for _, n in rows)
    out = np.empty((nz, ny + 2 * NGH, nx))
    for a, (y0, n) in zip(parts, rows):
        out[:, y0 + NGH:y0 + NGH + n, :] = a[:, NGH:NGH + n, :]
    out[:, :NGH, :] = parts[0][:, :NGH, :]
    out[:, ny + NGH:, :] = parts[-1][:, rows[-1][1] + NGH:, :]
    return out


class LocalSlabs:
    """Every slab of one disk in this process (slab k on devices[k % len])."""

    def __init__(self, cfg: DiskConfig, nslabs: int, precision: str = "fp64", devices=(0,)):
        import torch
        from .disk import Disk
        self.cfg, self.rows = cfg, split_rows(cfg.ny, nslabs)
        self.disks = [Disk(c, precision, device=devices[k % len(devices)])
                      for k, c in enumerate(slab_configs(cfg, nslabs))]
        # one halo buffer per slab edge and kind, on the slab's device
        self.buf = {}
        for k, d in enumerate(self.disks):
            dev = torch.device("cuda", devices[k % len(devices)])
            for which in (HALO_STATE, HALO_VTEMP):
                self.buf[k, which] = torch.empty(d.halo_bytes(which), dtype=torch.uint8, device=dev)

    def set_state(self, rho, vx, vy, vz, cs):
        for d, (y0, n) in zip(self.disks, self.rows):
            d.set_state(*[None if a is None else slab_rows(np.asarray(a), y0, n) for a in (rho, vx, vy, vz, cs)])

    def initialize(self):
        for d in self.disks:
            d.initialize()
        self.exchange(HALO_STATE)

    def exchange(self, which: int):
        """Each internal edge: the lower slab's last rows into the upper's
        ghosts and the upper's first rows into the lower's ghosts."""
        for k in range(len(self.disks) - 1):
            lo, hi = self.disks[k], self.disks[k + 1]
            b = self.buf[k, which]
            lo.halo(which, 1, False, b.data_ptr(), False)
            if b.device != self.buf[k + 1, which].device:
                self.buf[k + 1, which].copy_(b)
                b = self.buf[k + 1, which]
            hi.halo(which, 0, True, b.data_ptr(), False)
            b = self.buf[k + 1, which]
            hi.halo(which, 0, False, b.data_ptr(), False)
            if b.device != self.buf[k, which].device:
                self.buf[k, which].copy_(b)
                b = self.buf[k, which]
            lo.halo(which, 1, True, b.data_ptr(), False)

    def step(self, dt_interval: float = 1e30) -> float:
        cfl = min(d.step_begin() for d in self.disks)
        dts = [d.step_advance(dt_interval, cfl) for d in self.disks]
        self.exchange(HALO_VTEMP)
        for d in self.disks:
            d.step_transport()
        self.exchange(HALO_STATE)
        return dts[0]

    def run(self, nsteps: int, dt_interval: float = 1e30):
        return [self.step(dt_interval) for _ in range(nsteps)]

    def state(self):
        parts = [d.state() for d in self.disks]
        return {k: assemble([p[k] for p in parts], self.rows) for k in ("rho", "vx", "vy", "vz")}

    def close(self):
        for d in self.disks:
            d.close()


class RankSlab:
    """This rank's slab of a disk split over the ranks of the default
    torch.distributed group: NCCL sends of device halo buffers (gloo: host
    buffers), all-reduce MIN of the CFL minimum."""

    def __init__(self, engine, rank: int, world: int, on_host: bool, device=None):
        import torch
        self.engine, self.rank, self.world, self.on_host = engine, rank, world, on_host
        dev = torch.device("cpu") if on_host else device
        self.send, self.recv = {}, {}
        for which in (HALO_STATE, HALO_VTEMP):
            nb = engine.halo_bytes(which)
            for side in (0, 1):
                self.send[which, side] = torch.empty(nb, dtype=torch.uint8, device=dev)
                self.recv[which, side] = torch.empty(nb, dtype=torch.uint8, device=dev)
        self.dev = dev

    def exchange(self, which: int):
        import torch.distributed as dist
        ops = []
        nbr = {0: self.rank - 1, 1: self.rank + 1}
        for side in (0, 1):
            if 0 <= nbr[side] < self.world:
                self.engine.halo(which, side, False, self.send[which, side].data_ptr(), self.on_host)
                ops.append(dist.P2POp(dist.irecv, self.recv[which, side], nbr[side]))
                ops.append(dist.P2POp(dist.isend, self.send[which, side], nbr[side]))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for side in (0, 1):
            if 0 <= nbr[side] < self.world:
                self.engine.halo(which, side, True, self.recv[which, side].data_ptr(), self.on_host)

    def cfl_min(self, local: float) -> float:
        import torch
        import torch.distributed as dist
        t = torch.tensor([local], dtype=torch.float64, device=self.dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        return float(t.item())

    def initialize(self):
        self.engine.initialize()
        self.exchange(HALO_STATE)

    def step(self, dt_interval: float = 1e30) -> float:
        cfl = self.cfl_min(self.engine.step_begin())
        dt = self.engine.step_advance(dt_interval, cfl)
        self.exchange(HALO_VTEMP)
        self.engine.step_transport()
        self.exchange(HALO_STATE)
        return dt
