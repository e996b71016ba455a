"""Dust diffusion (DustDiffusion_Main, dust_diffusion_main.c,
dust_diffusion_core.c, dust_diffusion_coefficients.c) on the CUDA FP64 path,
against the reference's own C sources compiled with the stock
fargo_multifluid flags including DUSTDIFFUSION (oracle/_ref/
libfargo_ref_mf5_dd.so): gas + 4 dust species, implicit drag, diffusion of
every dust density after the drag.  FP64 bar: 1e-12 relative L-infinity per
field and fluid, bit for bit over the first steps."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
TOL = 1e-12


def run_both(cfg, n):
    import pyoracle
    from fargo3d_b200 import Disk, initial_state
    init = [initial_state(cfg, f) for f in range(cfg.nfluids)]
    d = Disk(cfg, "fp64")
    for f, st in enumerate(init):
        d.set_state(*st, fluid=f)
    d.initialize()
    dts = np.array(d.run(n))
    got = [d.state(f) for f in range(cfg.nfluids)]
    d.close()
    want, dtr, _ = pyoracle.run(cfg, n, "ref", 1e30, state=init)
    return got, dts, want, dtr


@pytest.mark.gpu
def test_dust_diffusion_bit_exact_short():
    from fargo3d_b200 import config_multifluid
    got, dts, want, dtr = run_both(config_multifluid(64, 32, seed=81, dust_diffusion=True), 3)
    assert np.array_equal(dts, dtr)
    for f in range(5):
        for k in ("rho", "vx", "vy"):
            assert np.array_equal(got[f][k][:, 3:-3], want[f][k][:, 3:-3]), (f, k)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,n", [((64, 32), 40), ((768, 256), 20)])
def test_dust_diffusion_matches_reference(shape, n):
    from fargo3d_b200 import config_multifluid
    got, dts, want, dtr = run_both(config_multifluid(*shape, seed=82, dust_diffusion=True), n)
    assert np.max(np.abs(dts - dtr) / dtr) <= TOL
    for f in range(5):
        for k in ("rho", "vx", "vy"):
            a, b = got[f][k][:, 3:-3], want[f][k][:, 3:-3]
            e = np.max(np.abs(a - b)) / np.max(np.abs(b))
            assert e <= TOL, (f, k, e)


@pytest.mark.gpu
def test_dust_diffusion_conserves_dust_mass():
    """Diffusion moves dust between cells: with Stockholm damping off and no
    flux through the radial edges, every dust fluid's mass stays at its
    round-off level (the compensated device sum)."""
    from fargo3d_b200 import Disk, config_multifluid
    cfg = config_multifluid(128, 64, seed=83, dust_diffusion=True).replace(stockholm=False)
    d = Disk(cfg, "fp64")
    d.load_initial_state()
    m0 = np.array([d.mass(f) for f in range(5)])
    d.run(50)
    m1 = np.array([d.mass(f) for f in range(5)])
    d.close()
    assert np.all(np.abs(m1 / m0 - 1.0) <= 1e-13), m1 / m0 - 1.0
