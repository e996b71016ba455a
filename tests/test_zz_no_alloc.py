"""fb_cfl_dt_static: the CFL time step for callers that cannot allocate.

Callers that own all device memory (FARGO3D's own GPU build, whose Fields are
allocated once by CreateField; applications running from a fixed pool) may
not let a library call cudaMalloc.  fb_cfl_dt_static computes the time step
of a state held in the caller's device buffers with its scratch in a fixed
device array.  This test drives it through the C-ABI on a disk's own device
fields and checks it against the time step the regular entry point
(fb_disk_step) takes from the same state, on two calls in a row.
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
                ("mindx", C.c_double), ("xlen", C.c_double)]


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


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cyl2d", "sph3d"])
def test_cfl_dt_static_matches_step(which):
    import torch
    from fargo3d_b200 import Disk, config_fargo2d, config_p3disof, initial_state
    from fargo3d_b200 import _abi
    L = _abi.lib()
    L.fb_cfl_dt_static.argtypes = [C.POINTER(CflStaticArgs), C.c_void_p, C.c_void_p]
    L.fb_cfl_dt_static.restype = C.c_int
    if which == "cyl2d":
        cfg = config_fargo2d(64, 32, seed=21).replace(noise=1e-2)
    else:
        cfg = config_p3disof(32, 16, 8, seed=22)
    xa, ya, za = _mesh(cfg)
    dev = torch.device("cuda", 0)
    xmin = torch.from_numpy(xa).to(dev)
    ymin = torch.from_numpy(ya).to(dev)
    zmin = torch.from_numpy(za).to(dev)
    zmed = 0.5 * (za[1:] + za[:-1])
    sinz = torch.tensor([math.sin(z) for z in zmed] + [0.0], dtype=torch.float64, device=dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)

    d = Disk(cfg, "fp64", device=0)
    d.set_state(*initial_state(cfg))
    d.initialize()
    ptrs, esz = d.device_fields()
    assert esz == 8
    a = CflStaticArgs()
    a.nx, a.ny, a.nz = cfg.nx, cfg.ny, cfg.nz
    a.spherical, a.alpha_visc = int(cfg.spherical), int(cfg.alpha_visc)
    a.rho, a.vx, a.vy, a.vz, a.cs = ptrs
    a.xmin, a.ymin, a.zmin, a.sin_zmed = xmin.data_ptr(), ymin.data_ptr(), zmin.data_ptr(), sinz.data_ptr()
    a.cfl, a.nu, a.alpha = cfg.cfl, cfg.nu, cfg.alpha
    a.mindx = float(np.min(xa[1:] - xa[:-1]))
    a.xlen = cfg.xmax - cfg.xmin
    torch.cuda.synchronize()
    for call in range(2):  # two calls in a row, each on the state the last step left
        rc = L.fb_cfl_dt_static(C.byref(a), C.c_void_p(out.data_ptr()), C.c_void_p(d.stream))
        assert rc == 0, _abi.lib().fb_last_error()
        torch.cuda.synchronize()
        dt_static = float(out.item())
        dt_step = d.step(1e30)
        assert abs(dt_static - dt_step) <= TOL * dt_step, (call, dt_static, dt_step)
    # meshes beyond the fixed scratch are refused, nothing is launched
    big = CflStaticArgs.from_buffer_copy(a)
    big.ny = 70000  # (Ny + 6) rings > FB_NOALLOC_MAX_RINGS
    assert L.fb_cfl_dt_static(C.byref(big), C.c_void_p(out.data_ptr()), C.c_void_p(d.stream)) == -6
    d.close()
