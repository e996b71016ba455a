"""Mass conservation on the CUDA path, with the device's compensated mass
reduction (fb_disk_mass, the analogue of ComputeMass, LowTasks.c:709-748).

With Stockholm damping off, no mass crosses the radial edges: the ghost
boundaries put v_r = 0 on the first and last active faces
(std/boundaries.txt ANTISYMMETRIC with the edge face nulled), so the upwind
fluxes there vanish, and the FARGO shift is a permutation.  The total mass of
every fluid must then stay constant to round-off:
  FP64: the state is rounded in double every step, and the relative change
        of a sum of ~1e5 cells is ~1e-16 / sqrt(N) per step; the bar, 2e-14
        after 100 steps, is the compensated sum's own accuracy with margin.
  FP32: every stored density is rounded to float every sweep (relative
        2^-24 per cell, unbiased), which moves the total by ~6e-8 / sqrt(N)
        per sweep; the bar is 2e-8 after 100 steps (three sweeps a step).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

BAR = {"fp64": 2e-14, "fp32": 2e-8}


def closed(cfg):
    return cfg.replace(stockholm=False)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("which", ["fargo2d", "multifluid", "p3disof"])
def test_mass_conserved_to_roundoff(which, precision):
    from fargo3d_b200 import Disk, config_fargo2d, config_multifluid, config_p3disof
    if which == "fargo2d":
        cfg, n = closed(config_fargo2d(384, 128, seed=61)), 100
    elif which == "multifluid":
        cfg, n = closed(config_multifluid(256, 128, seed=62)), 100
    else:
        cfg, n = closed(config_p3disof(64, 32, 16, seed=63)), 40
    d = Disk(cfg, precision)
    d.load_initial_state()
    m0 = np.array([d.mass(f) for f in range(cfg.nfluids)])
    worst = np.zeros(cfg.nfluids)
    for _ in range(n):
        d.step()
        m = np.array([d.mass(f) for f in range(cfg.nfluids)])
        worst = np.maximum(worst, np.abs(m / m0 - 1.0))
    d.close()
    assert np.all(worst <= BAR[precision]), (which, precision, worst)


@pytest.mark.gpu
def test_device_mass_matches_oracle_mass():
    """The device reduction against the oracle's compensated host sum of the
    same FP64 state (both to round-off of a compensated sum)."""
    import pyoracle
    from fargo3d_b200 import Disk, config_fargo2d, initial_state
    pyoracle.build()
    cfg = config_fargo2d(96, 48, seed=64)
    d = Disk(cfg, "fp64")
    d.load_initial_state()
    d.run(5)
    st = d.state()
    o = pyoracle.Disk(cfg, "oracle")
    o.set_state(st["rho"], st["vx"], st["vy"], st["vz"], initial_state(cfg)[4])
    assert abs(d.mass() / o.mass() - 1.0) <= 1e-15
    o.close()
    d.close()


@pytest.mark.gpu
def test_batch_mass_equals_member_disk_mass():
    """A batch member's mass (FP32, the batched step) is conserved as the
    one-disk path's is, and is read after the batch's queued steps."""
    from fargo3d_b200 import Batch, config_fargo2d
    cfgs = [closed(config_fargo2d(128, 64, seed=65)), closed(config_fargo2d(256, 96, seed=66))]
    b = Batch(cfgs, "fp32")
    b.load_initial_states()
    m0 = [b.mass(i) for i in range(2)]
    b.run(50)
    m1 = [b.mass(i) for i in range(2)]
    b.close()
    for a, c in zip(m0, m1):
        assert abs(c / a - 1.0) <= BAR["fp32"], (a, c)
