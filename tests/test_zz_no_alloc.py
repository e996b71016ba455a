"""fb_cfl_dt_static: the CFL time step for callers that cannot allocate.

Callers that own all device memory (FARGO3D's own GPU build, whose Fields are
allocated once by CreateField; applications running from a fixed pool) may
not let a library call cudaMalloc.  fb_cfl_dt_static computes the time step
of a state held in the caller's device buffers with its scratch in a fixed
device array.  This test drives it through the C-ABI on a disk's own device
fields -- and on pitched copies of them, laid out as FARGO3D's
cudaMallocPitch Fields are -- and checks it against the time step the regular
entry point (fb_disk_step) takes from the same state, on two calls in a row,
with no change in the device's free memory around the second call.
"""
import ctypes as C
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-12  # FP64 bar of the parity tests (identical in practice)


class CflStaticArgs(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("spherical", C.c_int),
                ("alpha_visc", C.c_int),
                ("rho", C.c_void_p), ("cs", C.c_void_p), ("vx", C.c_void_p), ("vy", C.c_void_p),
                ("vz", C.c_void_p), ("xmin", C.c_void_p), ("ymin", C.c_void_p), ("zmin", C.c_void_p),
                ("sin_zmed", C.c_void_p),
                ("cfl", C.c_double), ("nu", C.c_double), ("alpha", C.c_double),
                ("mindx", C.c_double), ("xlen", C.c_double),
                ("pitch", C.c_int), ("stride", C.c_longlong)]


def _mesh(cfg):
    """Mesh edges computed by the oracle's C code (the same libm expressions
    as the library's host side), so the device copies are bit-identical."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    pyoracle.build()
    d = pyoracle.Disk(cfg, "oracle")
    xa, ya, za = d.geometry()
    d.close()
    return xa, ya, za


def _pitched_copy(arr, pitch, dev):
    """A device copy of a [z][y][x] field with rows of `pitch` elements; the
    row tails hold NaN, which a correct kernel never reads."""
    import torch
    nz, ny, nx = arr.shape
    t = torch.full((nz, ny, pitch), float("nan"), dtype=torch.float64, device=dev)
    t[:, :, :nx] = torch.from_numpy(np.ascontiguousarray(arr)).to(dev)
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cyl2d", "sph3d", "cyl2d_pitched", "sph3d_pitched"])
def test_cfl_dt_static_matches_step(which):
    import torch
    from fargo3d_b200 import Disk, config_fargo2d, config_p3disof, initial_state
    from fargo3d_b200 import _abi
    L = _abi.lib()
    L.fb_cfl_dt_static.argtypes = [C.POINTER(CflStaticArgs), C.c_void_p, C.c_void_p]
    L.fb_cfl_dt_static.restype = C.c_int
    pitched = which.endswith("_pitched")
    if which.startswith("cyl2d"):
        # Nx = 60: FARGO3D's cudaMallocPitch pads a 480-byte row to 512 bytes
        cfg = config_fargo2d(60 if pitched else 64, 32, seed=21).replace(noise=1e-2)
    else:
        cfg = config_p3disof(36 if pitched else 32, 16, 8, seed=22)
    xa, ya, za = _mesh(cfg)
    dev = torch.device("cuda", 0)
    xmin = torch.from_numpy(xa).to(dev)
    ymin = torch.from_numpy(ya).to(dev)
    zmin = torch.from_numpy(za).to(dev)
    zmed = 0.5 * (za[1:] + za[:-1])
    sinz = torch.tensor([math.sin(z) for z in zmed] + [0.0], dtype=torch.float64, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)

    init = initial_state(cfg)
    d = Disk(cfg, "fp64", device=0)
    d.set_state(*init)
    d.initialize()
    ptrs, esz = d.device_fields()
    assert esz == 8
    a = CflStaticArgs()
    a.nx, a.ny, a.nz = cfg.nx, cfg.ny, cfg.nz
    a.spherical, a.alpha_visc = int(cfg.spherical), int(cfg.alpha_visc)
    a.xmin, a.ymin, a.zmin, a.sin_zmed = xmin.data_ptr(), ymin.data_ptr(), zmin.data_ptr(), sinz.data_ptr()
    a.cfl, a.nu, a.alpha = cfg.cfl, cfg.nu, cfg.alpha
    a.mindx = float(np.min(xa[1:] - xa[:-1]))
    a.xlen = cfg.xmax - cfg.xmin
    pitch = 64 if pitched else 0
    keep = []
    for call in range(2):  # two calls in a row, each on the state the last step left
        if pitched:
            st = d.state()
            keep = [_pitched_copy(x, pitch, dev) for x in (st["rho"], init[4], st["vx"], st["vy"], st["vz"])]
            a.rho, a.cs, a.vx, a.vy, a.vz = [t.data_ptr() for t in keep]
            a.pitch, a.stride = pitch, pitch * (cfg.ny + 6)
        else:
            a.rho, a.vx, a.vy, a.vz, a.cs = ptrs
        torch.cuda.synchronize()
        if call == 1:  # the first call looked the scratch up; from here on nothing is allocated
            free0, alloc0 = torch.cuda.mem_get_info(0)[0], torch.cuda.memory_allocated(0)
        rc = L.fb_cfl_dt_static(C.byref(a), C.c_void_p(out.data_ptr()), C.c_void_p(d.stream))
        assert rc == 0, _abi.lib().fb_last_error()
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info(0)[0] == free0
            assert torch.cuda.memory_allocated(0) == alloc0
        dt_static = float(out.item())
        dt_step = d.step(1e30)
        assert abs(dt_static - dt_step) <= TOL * dt_step, (call, dt_static, dt_step)
    # meshes beyond the fixed scratch are refused, nothing is launched
    big = CflStaticArgs.from_buffer_copy(a)
    big.ny = 70000  # (Ny + 6) rings > FB_NOALLOC_MAX_RINGS
    assert L.fb_cfl_dt_static(C.byref(big), C.c_void_p(out.data_ptr()), C.c_void_p(d.stream)) == -6
    assert b"FB_NOALLOC_MAX_RINGS" in _abi.lib().fb_last_error()
    # a pitch shorter than a row is refused
    if pitched:
        short = CflStaticArgs.from_buffer_copy(a)
        short.pitch = cfg.nx - 1
        assert L.fb_cfl_dt_static(C.byref(short), C.c_void_p(out.data_ptr()), C.c_void_p(d.stream)) == -1
    d.close()


@pytest.mark.gpu
def test_cfl_dt_static_flags_a_bad_state():
    """A density planted non-positive on the host gives a NaN time step (the
    regular step refuses the same state with FB_ERR_NONFINITE)."""
    import torch
    from fargo3d_b200 import Disk, FargoError, config_fargo2d, initial_state
    from fargo3d_b200 import _abi
    L = _abi.lib()
    L.fb_cfl_dt_static.argtypes = [C.POINTER(CflStaticArgs), C.c_void_p, C.c_void_p]
    L.fb_cfl_dt_static.restype = C.c_int
    cfg = config_fargo2d(64, 32, seed=23)
    xa, ya, za = _mesh(cfg)
    dev = torch.device("cuda", 0)
    xmin, ymin, zmin = (torch.from_numpy(x).to(dev) for x in (xa, ya, za))
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    st = list(initial_state(cfg))
    st[0] = st[0].copy()
    st[0][0, 9, 5] = -1.0
    d = Disk(cfg, "fp64", device=0)
    d.set_state(*st)
    d.initialize()
    ptrs, _ = d.device_fields()
    a = CflStaticArgs()
    a.nx, a.ny, a.nz = cfg.nx, cfg.ny, cfg.nz
    a.rho, a.vx, a.vy, a.vz, a.cs = ptrs
    a.xmin, a.ymin, a.zmin = xmin.data_ptr(), ymin.data_ptr(), zmin.data_ptr()
    a.cfl, a.nu, a.alpha = cfg.cfl, cfg.nu, cfg.alpha
    a.mindx = float(np.min(xa[1:] - xa[:-1]))
    a.xlen = cfg.xmax - cfg.xmin
    torch.cuda.synchronize()
    assert L.fb_cfl_dt_static(C.byref(a), C.c_void_p(out.data_ptr()), C.c_void_p(d.stream)) == 0
    torch.cuda.synchronize()
    assert math.isnan(float(out.item()))
    with pytest.raises(FargoError):
        d.step(1e30)
    d.close()
