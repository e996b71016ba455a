"""The drop-in binding (fargo3d_b200/integration/b200_hydro.c) compiled into
the reference's own build: the reference's step loop, Fields, .par globals
and planetary system, with the hydro step handed to the B200 library, must
reproduce the unmodified reference run."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import cases, golden_init, golden_out  # noqa: E402

GOLD = os.path.join(HERE, "golden")


def _dropin_built(cfg):
    import pyoracle
    return os.path.exists(os.path.join(pyoracle.HERE, "_ref", "libfargo_ref_dropin_%s.so" % pyoracle.ref_variant(cfg)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cyl2d", "mf5"])
def test_dropin_reproduces_reference(name):
    import pyoracle
    cfg, nsteps, dti = cases()[name]
    if not _dropin_built(cfg):
        pytest.fail("drop-in build missing: run __graft_entry__.build() where the reference tree is present")
    g = np.load(os.path.join(GOLD, name + ".npz"))
    init = golden_init(g, cfg)
    # bit for bit over the first steps against the reference's own sources
    out, dts, sc = pyoracle.run(cfg, 3, "dropin", dti, state=init)
    ref, rdts, rsc = pyoracle.run(cfg, 3, "ref", dti, state=init)
    assert np.array_equal(dts, rdts)
    for f in range(cfg.nfluids):
        for k in ("rho", "vx", "vy"):
            assert np.array_equal(out[f][k], ref[f][k]), (f, k)
    assert np.array_equal(sc[:7], rsc[:7])   # time, frame, dt, planet 0 (through Sys and OMEGAFRAME)
    # the full golden run to FP64 round-off
    out, dts, _ = pyoracle.run(cfg, nsteps, "dropin", dti, state=init)
    assert np.max(np.abs(dts - g["dts"]) / g["dts"]) <= 1e-12
    for f in range(cfg.nfluids):
        want = golden_out(g, f)
        for k in ("rho", "vx", "vy"):
            d = np.max(np.abs(out[f][k] - want[k])) / np.max(np.abs(want[k]))
            assert d <= 1e-12, (f, k, d)
