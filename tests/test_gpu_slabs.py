"""A disk stepped as radial slabs (fargo3d_b200/slabs.py)
gives the whole disk's result bit for bit: every slab here runs on one GPU
with its halos exchanged through device buffers; the
multi-process form (one slab per GPU, NCCL) uses the same library calls and
is tested on CPU ranks in tests/test_slabs.py."""
import numpy as np
import pytest


def whole_and_slabs(cfg, nslabs, n):
    from fargo3d_b200 import Disk, initial_state
    from fargo3d_b200.slabs import LocalSlabs
    init = initial_state(cfg)
    d = Disk(cfg, "fp64")
    d.set_state(*init)
    d.initialize()
    dts = np.array(d.run(n))
    want = d.state()
    d.close()
    s = LocalSlabs(cfg, nslabs)
    s.set_state(*init)
    s.initialize()
    dts2 = np.array(s.run(n))
    got = s.state()
    s.close()
    return dts, want, dts2, got


@pytest.mark.gpu
@pytest.mark.parametrize("which,nslabs", [("cyl2d", 2), ("cyl2d", 3), ("sph3d", 2), ("adiabatic", 3)])
def test_slabs_equal_the_whole_disk(which, nslabs):
    from fargo3d_b200 import config_adiabatic2d, config_fargo2d, config_p3disof
    cfg, n = {"cyl2d": (config_fargo2d(64, 48, seed=101), 20),
              "sph3d": (config_p3disof(32, 24, 8, seed=102), 6),
              "adiabatic": (config_adiabatic2d(48, 30, seed=103), 12)}[which]
    dts, want, dts2, got = whole_and_slabs(cfg, nslabs, n)
    assert np.array_equal(dts, dts2)
    keys = ("rho", "vx", "vy", "vz") if cfg.is3d else ("rho", "vx", "vy")
    for k in keys:
        a, b = got[k][:, 3:-3], want[k][:, 3:-3]
        if cfg.is3d:
            a, b = got[k][3:-3, 3:-3], want[k][3:-3, 3:-3]
        assert np.array_equal(a, b), (k, np.max(np.abs(a - b)))


@pytest.mark.gpu
def test_slab_refusals():
    from fargo3d_b200 import Disk, FargoError, Planet, config_fargo2d, config_multifluid
    from fargo3d_b200.slabs import slab_configs
    with pytest.raises(ValueError):
        slab_configs(config_multifluid(32, 16), 2)
    bad = config_fargo2d(32, 16).replace(slab_y0=10, slab_ny_global=20)   # rows past the mesh
    with pytest.raises(FargoError):
        Disk(bad, "fp64")
    feel = config_fargo2d(32, 16).replace(planets=[Planet(1.0, 1e-3, True, True)], slab_y0=0, slab_ny_global=32)
    with pytest.raises(FargoError):
        Disk(feel, "fp64")
