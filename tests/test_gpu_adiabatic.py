"""The adiabatic equation of state: SubStep3, the
adiabatic pressure and sound speed, the artificial viscosity's heating and
the energy's transport, on the CUDA FP64 path, against the reference's own C
sources compiled with ADIABATIC (oracle/_ref/libfargo_ref_cyl2d_ad.so: the
fargo setup's flags with ADIABATIC and ALPHAVISCOSITY, energy boundaries
SYMMETRIC).  The FP64 kernels keep the reference's operation order, so the
fields and the time steps agree to the FP64 bar (1e-12 relative L-infinity),
bit for bit over the first steps.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
TOL = 1e-12


def rel_linf(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def run_both(cfg, n):
    import pyoracle
    from fargo3d_b200 import Disk, initial_state
    init = initial_state(cfg)
    d = Disk(cfg, "fp64")
    d.set_state(*init)
    d.initialize()
    dts = np.array(d.run(n))
    got = d.state()
    got["energy"] = d.energy()
    d.close()
    r = pyoracle.Disk(cfg, "ref")
    r.set_state(*init)
    r.initialize()
    dtr = np.array([r.step() for _ in range(n)])
    want = r.state()
    want["energy"] = r.energy()
    r.close()
    return got, dts, want, dtr


@pytest.mark.gpu
def test_adiabatic_bit_exact_short():
    from fargo3d_b200 import config_adiabatic2d
    got, dts, want, dtr = run_both(config_adiabatic2d(48, 20, seed=71), 3)
    assert np.array_equal(dts, dtr)
    for k in ("rho", "vx", "vy", "energy"):
        assert np.array_equal(got[k][:, 3:-3], want[k][:, 3:-3]), (k, rel_linf(got[k], want[k]))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,n", [((48, 20), 40), ((384, 128), 200)])
def test_adiabatic_matches_reference(shape, n):
    from fargo3d_b200 import config_adiabatic2d
    got, dts, want, dtr = run_both(config_adiabatic2d(*shape, seed=72), n)
    assert np.max(np.abs(dts - dtr) / dtr) <= TOL
    for k in ("rho", "vx", "vy", "energy"):
        e = rel_linf(got[k][:, 3:-3], want[k][:, 3:-3])
        assert e <= TOL, (k, e)


@pytest.mark.gpu
def test_adiabatic_restricted_to_the_fp64_one_disk_path():
    from fargo3d_b200 import Batch, Disk, FargoError, config_adiabatic2d
    cfg = config_adiabatic2d(32, 16, seed=73)
    with pytest.raises(FargoError):
        Disk(cfg, "fp32")
    with pytest.raises(FargoError):
        Batch([cfg], "fp64")
