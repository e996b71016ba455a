"""ctypes binding of the C-ABI in include/fargo_b200.h (libfargo_b200.so)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfargo_b200.so")

FB_MAXPLANETS = 8
FB_MAXFLUIDS = 8
FB_FP64, FB_FP32 = 0, 1
FB_OK = 0
ERRORS = {-1: "FB_ERR_ARG", -2: "FB_ERR_CUDA", -3: "FB_ERR_NULL_DT", -4: "FB_ERR_NONFINITE",
          -5: "FB_ERR_NOMEM", -6: "FB_ERR_TOO_LARGE"}
FB_DONE, FB_SLOT_EMPTY, FB_SLOT_RESERVED = 1, 2, 3
FB_REQ_QUEUED, FB_REQ_RUNNING, FB_REQ_DONE, FB_REQ_FAILED = 0, 1, 2, 3


class FbParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("spherical", C.c_int), ("log_spacing", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("aspectratio", C.c_double), ("sigmaslope", C.c_double), ("flaringindex", C.c_double),
        ("nu", C.c_double), ("alpha", C.c_double), ("alpha_visc", C.c_int),
        ("cfl", C.c_double), ("omegaframe", C.c_double), ("frame", C.c_int),
        ("indirect_term", C.c_int),
        ("thickness_smoothing", C.c_double), ("roche_smoothing", C.c_double), ("mass_taper", C.c_double),
        ("damping_zone", C.c_double), ("tau_damp", C.c_double), ("killing_bc_colatitude", C.c_double),
        ("nplanets", C.c_int),
        ("pl_dist", C.c_double * FB_MAXPLANETS), ("pl_mass", C.c_double * FB_MAXPLANETS),
        ("pl_feeldisk", C.c_int * FB_MAXPLANETS), ("pl_feelothers", C.c_int * FB_MAXPLANETS),
        ("eccentricity", C.c_double), ("inclination", C.c_double),
        ("nfluids", C.c_int), ("invstokes", C.c_double * FB_MAXFLUIDS),
        ("stockholm", C.c_int),
        ("adiabatic", C.c_int), ("gamma", C.c_double), ("dust_diffusion", C.c_int),
        ("slab_y0", C.c_int), ("slab_ny_global", C.c_int),
    ]


def params_of(cfg) -> FbParams:
    p = FbParams()
    p.nx, p.ny, p.nz = cfg.nx, cfg.ny, cfg.nz
    p.spherical, p.log_spacing = int(cfg.spherical), int(cfg.log_spacing)
    for k in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "aspectratio", "sigmaslope",
              "flaringindex", "nu", "alpha", "cfl", "omegaframe", "thickness_smoothing",
              "roche_smoothing", "mass_taper", "damping_zone", "tau_damp",
              "killing_bc_colatitude", "eccentricity", "inclination"):
        setattr(p, k, float(getattr(cfg, k)))
    p.alpha_visc = int(cfg.alpha_visc)
    p.frame = {"F": 0, "C": 1, "G": 2}[cfg.frame]
    p.indirect_term = int(cfg.indirect_term)
    if len(cfg.planets) > FB_MAXPLANETS:
        raise ValueError("at most %d planets" % FB_MAXPLANETS)
    p.nplanets = len(cfg.planets)
    for i, pl in enumerate(cfg.planets):
        p.pl_dist[i], p.pl_mass[i] = pl.distance, pl.mass
        p.pl_feeldisk[i], p.pl_feelothers[i] = int(pl.feel_disk), int(pl.feel_others)
    p.nfluids = cfg.nfluids
    for i, v in enumerate(cfg.invstokes):
        p.invstokes[i] = v
    p.stockholm = int(cfg.stockholm)
    p.adiabatic = int(cfg.adiabatic)
    p.gamma = float(cfg.gamma)
    p.dust_diffusion = int(cfg.dust_diffusion)
    p.slab_y0 = int(getattr(cfg, "slab_y0", 0))
    p.slab_ny_global = int(getattr(cfg, "slab_ny_global", 0))
    return p


_lib = None

_D = C.POINTER(C.c_double)


def lib():
    """Load libfargo_b200.so (building it first if it is missing/stale).
    Raises if the shared library cannot be loaded: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _b
        _b.build()
    L = C.CDLL(LIB_PATH)
    L.fb_last_error.restype = C.c_char_p
    L.fb_disk_create.argtypes = [C.POINTER(FbParams), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.fb_disk_destroy.argtypes = [C.c_void_p]
    L.fb_disk_set_state.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _D, _D]
    L.fb_disk_get_state.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _D]
    L.fb_disk_initialize.argtypes = [C.c_void_p]
    L.fb_disk_step.argtypes = [C.c_void_p, C.c_double, _D]
    L.fb_disk_get_scalars.argtypes = [C.c_void_p, _D]
    L.fb_disk_device_fields.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]
    L.fb_disk_get_background.argtypes = [C.c_void_p, C.c_int, _D]
    L.fb_disk_set_wait_limit.argtypes = [C.c_void_p, C.c_longlong]
    L.fb_disk_mass.argtypes = [C.c_void_p, C.c_int, _D]
    L.fb_disk_get_energy.argtypes = [C.c_void_p, C.c_int, _D]
    L.fb_disk_step_begin.argtypes = [C.c_void_p, _D]
    L.fb_disk_step_advance.argtypes = [C.c_void_p, C.c_double, C.c_double, _D]
    L.fb_disk_step_transport.argtypes = [C.c_void_p]
    L.fb_disk_halo_bytes.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
    L.fb_disk_halo.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int]
    L.fb_disk_stream.restype = C.c_void_p
    L.fb_disk_stream.argtypes = [C.c_void_p]
    L.fb_params_bytes.argtypes = [C.POINTER(FbParams), C.c_int, C.POINTER(C.c_size_t)]
    L.fb_disk_set_tiles.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.fb_disk_get_tiles.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.fb_disk_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
    _lib = L
    return L


class FargoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (ERRORS.get(code, code), msg))
        self.code = code


def check(rc: int):
    if rc != FB_OK:
        raise FargoError(rc, lib().fb_last_error().decode(errors="replace"))
    return rc


def bind_batch(L):
    if getattr(L, "_batch_bound", False):
        return L
    L.fb_batch_create.argtypes = [C.POINTER(FbParams), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.fb_batch_destroy.argtypes = [C.c_void_p]
    L.fb_batch_disk.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
    L.fb_batch_initialize.argtypes = [C.c_void_p]
    L.fb_batch_run.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.fb_batch_sync.argtypes = [C.c_void_p]
    L.fb_batch_get_scalars.argtypes = [C.c_void_p, C.c_int, _D, C.POINTER(C.c_int)]
    L.fb_batch_stream.restype = C.c_void_p
    L.fb_batch_stream.argtypes = [C.c_void_p]
    L.fb_batch_profile_step.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_float), C.POINTER(C.c_char_p), C.c_int]
    L.fb_batch_create_slots.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.fb_batch_add.argtypes = [C.c_void_p, C.POINTER(FbParams), C.c_double, C.POINTER(C.c_int)]
    L.fb_batch_activate.argtypes = [C.c_void_p, C.c_int]
    L.fb_batch_remove.argtypes = [C.c_void_p, C.c_int]
    L.fb_batch_capacity.argtypes = [C.c_void_p]
    L.fb_batch_poll.argtypes = [C.c_void_p, C.POINTER(C.c_int), _D, C.POINTER(C.c_longlong)]
    L.fb_batch_set_tiles.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.fb_batch_set_chains.argtypes = [C.c_void_p, C.c_int]
    L.fb_batch_get_chains.argtypes = [C.c_void_p]
    _PP = C.POINTER(C.POINTER(C.c_double))
    L.fb_batch_set_states.argtypes = [C.c_void_p, C.c_int, _PP, _PP, _PP, _PP, _PP]
    L.fb_batch_get_states.argtypes = [C.c_void_p, C.c_int, _PP, _PP, _PP, _PP]
    L.fb_disk_set_tiles.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.fb_disk_get_tiles.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L._batch_bound = True
    return L


def bind_server(L):
    if getattr(L, "_server_bound", False):
        return L
    bind_batch(L)
    L.fb_server_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.fb_server_submit.argtypes = [C.c_void_p, C.POINTER(FbParams), _D, _D, _D, _D, _D, C.c_double,
                                   C.POINTER(C.c_longlong)]
    L.fb_server_status.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(C.c_int)]
    L.fb_server_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double, C.POINTER(C.c_int)]
    L.fb_server_fetch.argtypes = [C.c_void_p, C.c_longlong, _D, _D, _D, _D, _D]
    L.fb_server_stats.argtypes = [C.c_void_p, _D]
    L.fb_server_clock.argtypes = [C.c_void_p]
    L.fb_server_clock.restype = C.c_double
    L.fb_server_destroy.argtypes = [C.c_void_p]
    L.fb_server_set_tiles.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L._server_bound = True
    return L


def params_bytes(cfg, precision: str) -> int:
    """Upper bound of the device bytes one disk of this configuration takes."""
    out = C.c_size_t()
    p = params_of(cfg)
    check(lib().fb_params_bytes(C.byref(p), FB_FP64 if precision == "fp64" else FB_FP32, C.byref(out)))
    return out.value
