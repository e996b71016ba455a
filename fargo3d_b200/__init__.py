"""fargo3d_b200 -- FARGO3D's hydro time step on NVIDIA B200 (sm_100a).

The per-cell work runs in hand-written CUDA kernels behind a C-ABI
(include/fargo_b200.h, libfargo_b200.so built in-tree); this package is the
Python host mirror of the reference's run loop over that ABI.
"""
from .setups import (DiskConfig, Planet, config_batched, config_fargo2d, config_multifluid, config_p3disof, config_adiabatic2d,
                     geometry, initial_state)
from .disk import Disk
from .batch import Batch
from .serving import Server, serving_requests
from ._abi import FargoError

__all__ = ["DiskConfig", "Planet", "config_batched", "config_fargo2d", "config_multifluid", "config_p3disof",
           "initial_state",
           "geometry", "Disk", "Batch", "Server", "serving_requests", "FargoError"]
