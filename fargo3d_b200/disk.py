"""Python mirror of the reference's run loop over the C-ABI.

`Disk` plays the part of one FARGO3D run (main.c): it owns a disk's device
state, applies the initial boundaries and Stockholm profiles (main.c:311-316)
and advances hydro steps (main.c:361-448) on the GPU.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi
from .setups import DiskConfig, initial_state


def _out_arrays(shape, is3d: bool, out):
    """Result arrays: the caller's (``out``) or new ones.  The vz of a 2D
    disk, when the caller gives none, is a read-only zero view (no
    allocation)."""
    res = {}
    size = math.prod(shape)
    for k in ("rho", "vx", "vy", "vz"):
        a = None if out is None else out.get(k)
        if a is None:
            a = np.empty(shape) if (k != "vz" or is3d) else np.broadcast_to(np.float64(0.0), shape)
        elif not (a.dtype == np.float64 and a.flags.c_contiguous and a.size == size):
            raise ValueError("out[%r] must be a C-contiguous float64 array of %d values" % (k, size))
        elif k == "vz" and not is3d:
            a.fill(0.0)
        res[k] = a.reshape(shape)
    return res


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class Disk:
    def __init__(self, cfg: DiskConfig, precision: str = "fp64", device: int = 0, tiles="table"):
        """`tiles`: "table" applies the autotuner's choice for this shape
        (fargo3d_b200/autotune.py), None keeps the defaults."""
        self.cfg = cfg
        self.precision = precision
        L = _abi.lib()
        self._p = _abi.params_of(cfg)
        h = C.c_void_p()
        prec = _abi.FB_FP64 if precision == "fp64" else _abi.FB_FP32
        _abi.check(L.fb_disk_create(C.byref(self._p), prec, device, C.byref(h)))
        self._h = h
        if tiles == "table":
            from .autotune import TileTable, cx_candidates
            t = TileTable.default().get(cfg, precision)
            if t and t[0] in cx_candidates(cfg.nx, precision, cfg.is3d):
                _abi.check(L.fb_disk_set_tiles(h, t[0], t[1]))
        self.shape = cfg.shape

    # ------------------------------------------------------------------ state
    def set_state(self, rho, vx, vy, vz, cs, fluid: int = 0):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(self.shape)
                for a in (rho, vx, vy, vz, cs)]
        _abi.check(_abi.lib().fb_disk_set_state(self._h, fluid, *[_ptr(a) for a in arrs]))

    def state(self, fluid: int = 0, out: dict | None = None):
        """Current fields as float64 arrays.  ``out`` may hold preallocated
        C-contiguous float64 arrays (page-locked ones move by DMA) for any of
        rho / vx / vy / vz; vz of a 2D disk is zero and not read back."""
        res = _out_arrays(self.shape, self.cfg.nz > 1, out)
        p = [_ptr(res[k]) if (k != "vz" or self.cfg.nz > 1) else None for k in ("rho", "vx", "vy", "vz")]
        _abi.check(_abi.lib().fb_disk_get_state(self._h, fluid, *p))
        return res

    def initialize(self):
        _abi.check(_abi.lib().fb_disk_initialize(self._h))

    def load_initial_state(self):
        for f in range(self.cfg.nfluids):
            self.set_state(*initial_state(self.cfg, f), fluid=f)
        self.initialize()

    # ------------------------------------------------------------------ steps
    def step(self, dt_interval: float = 1e30) -> float:
        dt = C.c_double()
        _abi.check(_abi.lib().fb_disk_step(self._h, dt_interval, C.byref(dt)))
        return dt.value

    def run(self, nsteps: int, dt_interval: float = 1e30):
        return [self.step(dt_interval) for _ in range(nsteps)]

    # the step in three parts (a radial slab of a disk split over GPUs)
    def step_begin(self) -> float:
        """ComputeVmed + cfl: this disk's CFL minimum."""
        m = C.c_double()
        _abi.check(_abi.lib().fb_disk_step_begin(self._h, C.byref(m)))
        return m.value

    def step_advance(self, dt_interval: float, cfl_min: float) -> float:
        """DT clip and planets with the (global) CFL minimum, Sources."""
        dt = C.c_double()
        _abi.check(_abi.lib().fb_disk_step_advance(self._h, dt_interval, cfl_min, C.byref(dt)))
        return dt.value

    def step_transport(self):
        """Transport, NewVelocity, Stockholm, the mesh-edge ghosts."""
        _abi.check(_abi.lib().fb_disk_step_transport(self._h))

    def halo_bytes(self, which: int) -> int:
        n = C.c_size_t()
        _abi.check(_abi.lib().fb_disk_halo_bytes(self._h, which, C.byref(n)))
        return n.value

    def halo(self, which: int, side: int, unpack: bool, ptr: int, on_host: bool):
        """Copy the halo rows of one edge between the disk and a buffer at
        `ptr` (device or host memory)."""
        _abi.check(_abi.lib().fb_disk_halo(self._h, which, side, int(unpack), C.c_void_p(ptr), int(on_host)))

    def scalars(self):
        o = np.zeros(8)
        _abi.check(_abi.lib().fb_disk_get_scalars(self._h, _ptr(o)))
        return o

    def device_fields(self, fluid: int = 0):
        ptrs = (C.c_void_p * 5)()
        esz = C.c_size_t()
        _abi.check(_abi.lib().fb_disk_device_fields(self._h, fluid, ptrs, C.byref(esz)))
        return [p for p in ptrs], esz.value

    def energy(self, fluid: int = 0):
        """The fluid's Energy field: the internal energy of an adiabatic disk,
        the sound speed of an isothermal one."""
        e = np.empty(self.shape)
        _abi.check(_abi.lib().fb_disk_get_energy(self._h, fluid, _ptr(e)))
        return e

    def mass(self, fluid: int = 0) -> float:
        """Total mass of a fluid (compensated FP64 sum of rho * Vol over the
        active cells, on the device)."""
        m = C.c_double()
        _abi.check(_abi.lib().fb_disk_mass(self._h, fluid, C.byref(m)))
        return m.value

    def background(self, fluid: int = 0):
        """The per-ring azimuthal background an FP32 disk stores vx relative
        to, shape (Nz+6 or 1, Ny+6); zeros for FP64 disks."""
        nz, ny, _ = self.shape
        o = np.zeros((nz, ny))
        _abi.check(_abi.lib().fb_disk_get_background(self._h, fluid, _ptr(o)))
        return o

    @property
    def stream(self) -> int:
        return _abi.lib().fb_disk_stream(self._h)

    @staticmethod
    def fluid_name(fluid: int) -> str:
        """FARGO3D's fluid names (setups/fargo_multifluid/condinit.c): gas, dust1, ..."""
        return "gas" if fluid == 0 else "dust%d" % fluid

    def write_dat(self, outdir: str, n: int):
        """Every fluid's merged output files <outdir>/<fluid><field><n>.dat
        (FARGO3D's WriteMerging layout) and the planet files' next line."""
        L = _abi.lib()
        for f in range(self.cfg.nfluids):
            _abi.check(L.fb_disk_write_dat(self._h, f, outdir.encode(), self.fluid_name(f).encode(), n))
        _abi.check(L.fb_disk_write_planets(self._h, outdir.encode(), n))

    def read_dat(self, outdir: str, n: int):
        """Replace the active cells of every fluid with output number n."""
        L = _abi.lib()
        for f in range(self.cfg.nfluids):
            _abi.check(L.fb_disk_read_dat(self._h, f, outdir.encode(), self.fluid_name(f).encode(), n))

    def close(self):
        if getattr(self, "_h", None):
            _abi.lib().fb_disk_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
