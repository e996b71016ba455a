"""Small parity cases shared by the golden-vector generator and the tests."""
import math

from fargo3d_b200.setups import DiskConfig, Planet, config_fargo2d, config_p3disof


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
    }
