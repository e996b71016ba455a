"""Generate the golden vectors in this directory from the reference's OWN
hot-path sources (oracle/_ref/libfargo_ref_*.so, built by oracle/ref/Makefile
from the reference tree).  Run in a container that has the reference:

    python tests/golden/make_golden.py

Each <case>.npz holds the initial state, the state after N hydro steps, the
N time steps and the final scalars, as computed by the reference's code.
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
from cases import cases  # noqa: E402
from fargo3d_b200.setups import initial_state  # noqa: E402


def main():
    pyoracle.build()
    for name, (cfg, nsteps, dti) in cases().items():
        init = [initial_state(cfg, f) for f in range(cfg.nfluids)]
        out, dts, sc = pyoracle.run(cfg, nsteps, "ref", dti, state=init)
        np.savez_compressed(os.path.join(HERE, name + ".npz"),
                            rho0=init[0][0], vx0=init[0][1], vy0=init[0][2], vz0=init[0][3], cs=init[0][4],
                            rho=out[0]["rho"], vx=out[0]["vx"], vy=out[0]["vy"], vz=out[0]["vz"],
                            dts=dts, scalars=sc, nsteps=nsteps, dt_interval=dti)
        print(name, "steps", nsteps, "dt0", dts[0])


if __name__ == "__main__":
    main()
