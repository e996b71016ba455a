"""Many independent disks advanced together (C-ABI fb_batch_*).

Each stage of a hydro step is one launch over the tiles of every disk; the
scalar work of a step runs on the device and sequences of steps replay from a
captured CUDA graph, so `run` enqueues work without host round trips.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .disk import _out_arrays
from .setups import initial_state


class _Member:
    """A disk owned by a batch (state access through the one-disk C-ABI)."""

    def __init__(self, h, shape):
        self._h, self.shape = h, shape


def _ptr_array(addr):
    """A C array of double pointers from addresses (None: NULL), or None when
    every entry is NULL."""
    if all(a is None for a in addr):
        return None
    arr = (C.c_void_p * len(addr))(*addr)
    return C.cast(arr, C.POINTER(C.POINTER(C.c_double)))


class Batch:
    """`tiles`: "table" applies the autotuner's table (fargo3d_b200/autotune.py)
    to every member whose shape it lists, None keeps the defaults."""

    def __init__(self, cfgs, precision: str = "fp32", device: int = 0, tiles="table"):
        L = _abi.bind_batch(_abi.lib())
        self.cfgs = list(cfgs)
        arr = (_abi.FbParams * len(self.cfgs))(*[_abi.params_of(c) for c in self.cfgs])
        h = C.c_void_p()
        prec = _abi.FB_FP64 if precision == "fp64" else _abi.FB_FP32
        _abi.check(L.fb_batch_create(arr, len(self.cfgs), prec, device, C.byref(h)))
        self._h = h
        self.precision = precision
        self._members = []
        for i, c in enumerate(self.cfgs):
            dh = C.c_void_p()
            _abi.check(L.fb_batch_disk(h, i, C.byref(dh)))
            self._members.append(_Member(dh, c.shape))
        if tiles == "table":
            from .autotune import TileTable
            TileTable.default().apply(self)

    def __len__(self):
        return len(self.cfgs)

    def set_state(self, i, rho, vx, vy, vz, cs, fluid: int = 0):
        m = self._members[i]
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(m.shape)
                for a in (rho, vx, vy, vz, cs)]
        p = [None if a is None else a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        _abi.check(_abi.lib().fb_disk_set_state(m._h, fluid, *p))

    def load_initial_states(self):
        for i, c in enumerate(self.cfgs):
            for f in range(c.nfluids):
                self.set_state(i, *initial_state(c, f), fluid=f)
        self.initialize()

    def initialize(self):
        _abi.check(_abi.lib().fb_batch_initialize(self._h))

    def run(self, nsteps: int, dt_interval: float = 1e30):
        _abi.check(_abi.lib().fb_batch_run(self._h, nsteps, dt_interval))

    def sync(self):
        _abi.check(_abi.lib().fb_batch_sync(self._h))

    def set_states(self, states, fluid: int = 0):
        """Every member's state of `fluid` in one library call: one
        (rho, vx, vy, vz, cs) per member, FARGO3D layout (None skips a field
        or a member).  Page-locked arrays move by DMA back to back."""
        n = len(self.cfgs)
        keep, cols = [], []
        for q in range(5):
            addr = [None] * n
            for i, st in enumerate(states):
                a = None if st is None else st[q]
                if a is None:
                    continue
                a = np.ascontiguousarray(a, dtype=np.float64).reshape(self._members[i].shape)
                keep.append(a)
                addr[i] = a.__array_interface__["data"][0]
            cols.append(_ptr_array(addr))
        _abi.check(_abi.lib().fb_batch_set_states(self._h, fluid, *cols))

    def states(self, fluid: int = 0, out=None):
        """Every member's fields of `fluid` (``out``: one dict of
        preallocated arrays per member, as for :meth:`state`), read in one
        library call."""
        self.sync()
        n = len(self.cfgs)
        res = [_out_arrays(self._members[i].shape, self.cfgs[i].nz > 1, None if out is None else out[i])
               for i in range(n)]
        cols = [_ptr_array([res[i][k].__array_interface__["data"][0] if (k != "vz" or self.cfgs[i].nz > 1) else None
                            for i in range(n)]) for k in ("rho", "vx", "vy", "vz")]
        _abi.check(_abi.lib().fb_batch_get_states(self._h, fluid, *cols))
        return res

    def state(self, i, fluid: int = 0, out: dict | None = None):
        """Disk i's current fields as float64 arrays (``out``: preallocated
        arrays to fill, as for :meth:`Disk.state`)."""
        self.sync()
        m = self._members[i]
        is3d = self.cfgs[i].nz > 1
        res = _out_arrays(m.shape, is3d, out)
        p = [res[k].ctypes.data_as(C.POINTER(C.c_double)) if (k != "vz" or is3d) else None
             for k in ("rho", "vx", "vy", "vz")]
        _abi.check(_abi.lib().fb_disk_get_state(m._h, fluid, *p))
        return res

    def scalars(self, i):
        o = np.zeros(8)
        st = C.c_int()
        _abi.check(_abi.lib().fb_batch_get_scalars(self._h, i, o.ctypes.data_as(C.POINTER(C.c_double)),
                                                   C.byref(st)))
        return o, st.value

    def mass(self, i, fluid: int = 0) -> float:
        """Total mass of disk i's fluid (compensated FP64 sum on the device)."""
        self.sync()
        m = C.c_double()
        _abi.check(_abi.lib().fb_disk_mass(self._members[i]._h, fluid, C.byref(m)))
        return m.value

    def set_chains(self, chains: int):
        """Step the disks as this many concurrent groups (streams); 1..8."""
        _abi.check(_abi.lib().fb_batch_set_chains(self._h, chains))

    def chains(self) -> int:
        return _abi.lib().fb_batch_get_chains(self._h)

    def set_tiles(self, i, sweep_x_cells: int = 0, col_segment: int = 0):
        _abi.check(_abi.lib().fb_batch_set_tiles(self._h, i, sweep_x_cells, col_segment))

    def tiles(self, i):
        cx, ns = C.c_int(), C.c_int()
        _abi.check(_abi.lib().fb_disk_get_tiles(self._members[i]._h, C.byref(cx), C.byref(ns)))
        return cx.value, ns.value

    def profile_step(self, dt_interval: float = 1e30) -> dict:
        """One eager step with per-launch-group device times (ms)."""
        ms = (C.c_float * 40)()
        names = (C.c_char_p * 40)()
        n = _abi.lib().fb_batch_profile_step(self._h, dt_interval, ms, names, 40)
        if n < 0:
            _abi.check(n)
        return {names[i].decode(): float(ms[i]) for i in range(n)}

    @property
    def stream(self) -> int:
        return _abi.lib().fb_batch_stream(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().fb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
