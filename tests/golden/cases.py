"""Small parity cases shared by the golden-vector generator and the tests.

The `*_par` cases are read from FARGO3D setup files (setups/<name>/<name>.par
and .opt, planets/*.cfg beside them) by fargo3d_b200.parfile, with the mesh
made small by a parameter redefinition, as FARGO3D's command line does."""
import math
import os

from fargo3d_b200.setups import (DiskConfig, Planet, config_adiabatic2d, config_fargo2d, config_multifluid,
                                  config_p3disof)


SETUPS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "setups")


def _setup(name, redefine, seed):
    from fargo3d_b200.parfile import load_setup
    return load_setup(os.path.join(SETUPS, name), redefine=redefine, seed=seed).config


def cases():
    return {
        # setups/fargo flags, 2D cylindrical, constant nu, one planet, guiding-centre frame
        "cyl2d": (config_fargo2d(32, 16, seed=1), 20, 1e30),
        # same mesh, DT interval shorter than a few CFL steps: exercises main.c:394-395
        "cyl2d_dtclip": (config_fargo2d(32, 16, seed=2), 12, 0.3),
        # ALPHAVISCOSITY, steeper profile, thinner disk
        "cyl2d_alpha": (config_fargo2d(48, 20, seed=3).replace(
            alpha_visc=True, alpha=3e-3, nu=0.0, sigmaslope=1.0, aspectratio=0.04,
            planets=[Planet(1.0, 2e-3)]), 20, 1e30),
        # fixed frame, no indirect term, two planets feeling each other (N-body RK5)
        "cyl2d_twoplanets": (config_fargo2d(32, 16, seed=4).replace(
            frame="F", omegaframe=1.0, indirect_term=False,
            planets=[Planet(1.0, 1e-3, False, True), Planet(1.6, 5e-4, False, True)]), 15, 1e30),
        # setups/p3disof flags, 3D spherical
        "sph3d": (config_p3disof(16, 12, 6, seed=5), 6, 1e30),
        # setups/fargo_multifluid flags: gas + 4 dust species, implicit drag
        "mf5": (config_multifluid(32, 16, seed=6), 12, 1e30),
        # planets that feel the disk (AdvanceSystemFromDisk + ComputeAccel) and each other
        "cyl2d_feeldisk": (config_fargo2d(32, 16, seed=8).replace(
            frame="F", omegaframe=1.0, indirect_term=False,
            planets=[Planet(1.0, 1e-3, True, True), Planet(1.4, 3e-4, True, True)]), 15, 1e30),
        # ADIABATIC equation of state (the fargo flags with ADIABATIC and alpha viscosity)
        "cyl2d_ad": (config_adiabatic2d(48, 20, seed=9), 20, 0.2),
        # the multifluid flags with DUSTDIFFUSION
        "mf5_dd": (config_multifluid(32, 16, seed=10, dust_diffusion=True), 12, 1e30),
        # read from setup files: the fargo disk (linear spacing, flat Sigma)
        "fargo_par": (_setup("fargo_par", "Nx:32,Ny:16", 11), 20, 1e30),
        # the p3disof disk: flared (FlaringIndex 0.5), Sigma ~ r^-1, q = 1e-5
        "p3disof_par": (_setup("p3disof_par", "Nx:16,Ny:12,Nz:6", 12), 6, 1e30),
        # the fargo_multifluid disk: 3 dust species as dense as the gas, diffusing
        "mf4_par": (_setup("mf4_par", "Nx:32,Ny:16", 13), 12, 1e30),
    }


def _key(f, k):
    return k if f == 0 else "f%d_%s" % (f, k)


def golden_init(g, cfg):
    """Per-fluid initial states (rho, vx, vy, vz, cs) stored in a golden file."""
    return [tuple(g[_key(f, k)] for k in ("rho0", "vx0", "vy0", "vz0", "cs")) for f in range(cfg.nfluids)]


def golden_out(g, f=0):
    """Fluid f's state after the golden run (with its energy "e" where the
    file holds it)."""
    return {k: g[_key(f, k)] for k in ("rho", "vx", "vy", "vz", "e") if _key(f, k) in g}


def golden_arrays(init, out):
    """npz arrays of every fluid's initial and final state."""
    d = {}
    for f, (st, o) in enumerate(zip(init, out)):
        for k, v in zip(("rho0", "vx0", "vy0", "vz0", "cs"), st):
            d[_key(f, k)] = v
        for k in ("rho", "vx", "vy", "vz", "e"):
            if k in o:
                d[_key(f, k)] = o[k]
    return d
