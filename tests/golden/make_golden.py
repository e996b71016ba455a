"""Generate the golden vectors in this directory from the reference's OWN
hot-path sources (oracle/_ref/libfargo_ref_*.so, built by oracle/ref/Makefile
from the reference tree).  Run in a container that has the reference:

    python tests/golden/make_golden.py

Each <case>.npz holds the initial state, the state after N hydro steps, the
N time steps and the final scalars, as computed by the reference's code
(fluid 0 under rho0, vx0, ..., rho, vx, ...; fluid f > 0 under f<f>_rho0 ...).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import pyoracle  # noqa: E402
from cases import cases, golden_arrays  # noqa: E402
from fargo3d_b200.setups import initial_state  # noqa: E402


def main():
    """Writes the cases that have no file yet (--force: all of them)."""
    pyoracle.build()
    for name, (cfg, nsteps, dti) in cases().items():
        path = os.path.join(HERE, name + ".npz")
        if os.path.exists(path) and "--force" not in sys.argv:
            continue
        init = [initial_state(cfg, f) for f in range(cfg.nfluids)]
        out, dts, sc = pyoracle.run(cfg, nsteps, "ref", dti, state=init)
        np.savez_compressed(path, dts=dts, scalars=sc, nsteps=nsteps, dt_interval=dti,
                            **golden_arrays(init, out))
        print(name, "steps", nsteps, "dt0", dts[0])


if __name__ == "__main__":
    main()
