"""Continuous-batching server of disk-planet solves (C-ABI fb_server_*).

A request is one disk (a DiskConfig and its initial state) to be advanced
until a physical end time.  `Server.submit` queues it and returns at once;
the library's worker thread admits queued requests in arrival order while a
batch slot is free and their device bytes fit the HBM budget, runs every
admitted disk together (one batched launch per stage), and retires each one
as soon as it reaches its end time.  Requests that arrive while others run
join at the next chunk of steps.

`serving_requests` draws the serving workload: disk sizes {256x64, 512x128,
1024x256, 2048x512} with weights {.4, .3, .2, .1}, Poisson arrivals, one
planet each, the physics of the batched workload, seeded numpy default_rng.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List

import numpy as np

from . import _abi
from .setups import DiskConfig, Planet, initial_state

_D = C.POINTER(C.c_double)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_D)


class Server:
    def __init__(self, precision: str = "fp32", device: int = 0, is3d: bool = False, hbm_budget: int = 0,
                 max_disks: int = 64, chunk_steps: int = 10, tiles="table"):
        L = _abi.bind_server(_abi.lib())
        h = C.c_void_p()
        prec = _abi.FB_FP64 if precision == "fp64" else _abi.FB_FP32
        _abi.check(L.fb_server_create(prec, device, int(is3d), int(hbm_budget), max_disks, chunk_steps,
                                      C.byref(h)))
        self._h = h
        self.precision = precision
        self._shapes = {}
        if tiles == "table":   # the autotuner's choices for every shape it lists
            from .autotune import TileTable
            for key, e in TileTable.default().entries.items():
                shape, prec = key.split(":")
                nx, ny, nz = (int(v) for v in shape.split("x"))
                if prec == precision and (nz > 1) == is3d:
                    _abi.check(L.fb_server_set_tiles(h, nx, ny, nz, e["sweep_x_cells"], e["col_segment"]))

    def submit(self, cfg: DiskConfig, t_end: float, state=None) -> int:
        """Queue one disk; `state` = (rho, vx, vy, vz, cs) or the setup's
        initial state.  Returns the request id."""
        st = state if state is not None else initial_state(cfg)
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(cfg.shape) for a in st]
        rid = C.c_longlong()
        p = _abi.params_of(cfg)
        _abi.check(_abi.lib().fb_server_submit(self._h, C.byref(p), *[_ptr(a) for a in arrs], float(t_end),
                                               C.byref(rid)))
        self._shapes[rid.value] = cfg.shape
        return rid.value

    def status(self, rid: int) -> int:
        s = C.c_int()
        _abi.check(_abi.lib().fb_server_status(self._h, rid, C.byref(s)))
        return s.value

    def wait(self, rid: int, timeout: float = 3600.0) -> int:
        s = C.c_int()
        _abi.check(_abi.lib().fb_server_wait(self._h, rid, float(timeout), C.byref(s)))
        return s.value

    def fetch(self, rid: int):
        """Final state and info of a finished request (forgotten afterwards).
        info: submitted, admitted, finished (server clock, s), steps, time,
        status, bytes, cells; latency = finished - submitted."""
        shape = self._shapes.pop(rid)
        out = [np.empty(shape) for _ in range(4)]
        info = np.zeros(8)
        _abi.check(_abi.lib().fb_server_fetch(self._h, rid, *[_ptr(a) for a in out], _ptr(info)))
        names = ("submitted", "admitted", "finished", "steps", "time", "status", "bytes", "cells")
        return ({"rho": out[0], "vx": out[1], "vy": out[2], "vz": out[3]},
                dict(zip(names, info.tolist())))

    def stats(self) -> dict:
        o = np.zeros(8)
        _abi.check(_abi.lib().fb_server_stats(self._h, _ptr(o)))
        names = ("queued", "running", "finished", "bytes_reserved", "budget", "chunks", "cell_updates", "clock")
        return dict(zip(names, o.tolist()))

    def clock(self) -> float:
        return _abi.lib().fb_server_clock(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().fb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Request:
    cfg: DiskConfig
    t_end: float
    arrival: float   # seconds after the start of the arrival process


SERVING_SIZES = ((256, 64), (512, 128), (1024, 256), (2048, 512))
SERVING_WEIGHTS = (0.4, 0.3, 0.2, 0.1)


def serving_requests(n: int, rate: float = 20.0, orbits: float = 50.0, seed: int = 0) -> List[Request]:
    """n requests: Poisson arrivals at `rate` per second, sizes drawn from
    SERVING_SIZES with SERVING_WEIGHTS, each run for `orbits` orbits of the
    planet at r = 1 (t_end = 2 pi orbits)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate))
        nx, ny = SERVING_SIZES[int(rng.choice(len(SERVING_SIZES), p=SERVING_WEIGHTS))]
        q = float(np.exp(rng.uniform(np.log(1e-5), np.log(3e-3))))
        alpha = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        h = float(rng.uniform(0.03, 0.08))
        p = float(rng.uniform(0.0, 1.5))
        cfg = DiskConfig(nx=nx, ny=ny, aspectratio=h, sigmaslope=p, alpha=alpha, alpha_visc=True, nu=0.0,
                         planets=[Planet(1.0, q)], seed=seed * 100000 + k)
        out.append(Request(cfg, 2.0 * math.pi * orbits, t))
    return out
