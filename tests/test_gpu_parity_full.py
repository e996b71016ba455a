"""FP64 parity at the benchmark configurations' own sizes and step counts,
against the reference's own C sources (oracle/_ref, compiled from the
reference tree by oracle/ref/Makefile), same initial state, native CFL steps.

  fargo2d     384 x 128, 1000 steps (the 2D cylindrical configuration)
  multifluid  768 x 256 x 5 fluids, 100 steps (gas + 4 dust, implicit drag)
  p3disof     512 x 256 x 48, 10 steps (the 3D spherical configuration)

Bar: <= 1e-12 relative L-infinity per field (the FP64 path keeps the
reference's operation order and is bit-exact in practice), and the same time
steps.  The reference side runs on the host and takes most of the time.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
TOL = 1e-12


def rel_linf(a, b):
    den = np.max(np.abs(b))
    return np.max(np.abs(a - b)) / (den if den > 0 else 1.0)


def _ref_available(cfg):
    import pyoracle
    path = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libfargo_ref_%s.so" % pyoracle.ref_variant(cfg))
    return os.path.exists(path)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["fargo2d", "multifluid", "p3disof"])
def test_fp64_full_size_matches_reference(which):
    import pyoracle
    from fargo3d_b200 import Disk, config_fargo2d, config_multifluid, config_p3disof, initial_state
    if which == "fargo2d":
        cfg, n = config_fargo2d(384, 128, seed=0), 1000
    elif which == "multifluid":
        cfg, n = config_multifluid(768, 256, seed=0), 100
    else:
        cfg, n = config_p3disof(512, 256, 48, seed=0), 10
    assert _ref_available(cfg), "the reference-source oracle (oracle/_ref) is not built"
    init = [initial_state(cfg, f) for f in range(cfg.nfluids)]
    d = Disk(cfg, "fp64")
    for f, st in enumerate(init):
        d.set_state(*st, fluid=f)
    d.initialize()
    dts = np.array(d.run(n))
    got = [d.state(f) for f in range(cfg.nfluids)]
    d.close()
    ref, dtr, _ = pyoracle.run(cfg, n, "ref", 1e30, state=init)
    assert np.max(np.abs(dts - dtr) / dtr) <= TOL
    keys = ("rho", "vx", "vy", "vz") if cfg.is3d else ("rho", "vx", "vy")
    for f in range(cfg.nfluids):
        for k in keys:
            e = rel_linf(got[f][k], ref[f][k])
            assert e <= TOL, (which, f, k, e)
