"""ctypes driver for the oracle (TEST INFRASTRUCTURE ONLY).

Loads either the C restatement (oracle/_build/libfargo_oracle.so) or one of
the libraries built from the reference's own sources (oracle/_ref/
libfargo_ref_<variant>.so) and runs hydro steps on a given initial state.
Both expose the same entry points (fo_* / ref_*), so the same driver serves
both.  Only tests, the smoke check and the CPU leg of bench.py use this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAXP = 8
MAXF = 8


class FoParams(C.Structure):
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
        ("pl_dist", C.c_double * MAXP), ("pl_mass", C.c_double * MAXP),
        ("pl_feeldisk", C.c_int * MAXP), ("pl_feelothers", C.c_int * MAXP),
        ("eccentricity", C.c_double), ("inclination", C.c_double),
        ("nfluids", C.c_int), ("invstokes", C.c_double * MAXF),
        ("stockholm", C.c_int),
        ("adiabatic", C.c_int), ("gamma", C.c_double), ("dust_diffusion", C.c_int),
        ("slab_y0", C.c_int), ("slab_ny_global", C.c_int),
    ]


def make_params(cfg) -> FoParams:
    p = FoParams()
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
    p.nplanets = len(cfg.planets)
    for i, pl in enumerate(cfg.planets):
        p.pl_dist[i], p.pl_mass[i] = pl.distance, pl.mass
        p.pl_feeldisk[i], p.pl_feelothers[i] = int(pl.feel_disk), int(pl.feel_others)
    p.nfluids = cfg.nfluids
    for i, v in enumerate(cfg.invstokes):
        p.invstokes[i] = v
    p.stockholm = int(cfg.stockholm)
    p.adiabatic = int(getattr(cfg, "adiabatic", False))
    p.gamma = float(getattr(cfg, "gamma", 1.66666667))
    p.dust_diffusion = int(getattr(cfg, "dust_diffusion", False))
    return p


def build(ref: str | None = None):
    """Compile the oracle restatement and, when the reference tree is given
    (`ref`, or FARGO_REFERENCE in the environment), the reference's own
    sources; without one, the previously built oracle/_ref libraries stay."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    ref = ref or os.environ.get("FARGO_REFERENCE")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), "REF=" + ref], check=True)


def build_dropin(ref: str | None = None):
    """The drop-in variants of the reference build -- the step loop's body
    handed to the library ('dropin') and the stock step loop with the
    setup-directory files of fargo3d_b200/integration/setup ('shadow') --
    (needs libfargo_b200.so and the reference tree, as for build())."""
    ref = ref or os.environ.get("FARGO_REFERENCE")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), "REF=" + ref, "dropin", "shadow"], check=True)


def ref_variant(cfg) -> str:
    if getattr(cfg, "adiabatic", False):
        if cfg.is3d or not cfg.alpha_visc or cfg.nfluids > 1:
            raise ValueError("the compiled reference has one adiabatic variant: 2D, one fluid, alpha viscosity")
        return "cyl2d_ad"
    if cfg.nfluids > 1:
        dd = getattr(cfg, "dust_diffusion", False)
        if cfg.is3d or cfg.alpha_visc or not (cfg.nfluids == 5 or (cfg.nfluids == 4 and dd)):
            raise ValueError("the compiled reference's multifluid variants are 2D with constant nu: "
                             "5 fluids, or 4 fluids with dust diffusion")
        return "mf%d%s" % (cfg.nfluids, "_dd" if dd else "")
    if cfg.is3d:
        return "sph3d"
    return "cyl2d_alpha" if cfg.alpha_visc else "cyl2d"


_D = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_D) if a is not None else None


class Disk:
    """One disk advanced by the oracle ('oracle'), the reference ('ref'), or
    the reference's step loop handed to the B200 library through the
    FARGO3D-side drop-in binding ('dropin')."""

    _libs = {}

    def __init__(self, cfg, kind: str = "oracle"):
        """kind: 'oracle' (the C restatement), 'ref' (the reference's sources
        as the parity tests build them), 'ref_o3' (the same sources with the
        reference's stock -O3, for timing), 'dropin' or 'shadow' (the
        reference's build with its hydro step on the B200 library)."""
        self.cfg, self.kind = cfg, kind
        if kind == "oracle":
            path = os.path.join(HERE, "_build", "libfargo_oracle.so")
        elif kind in ("dropin", "shadow"):
            path = os.path.join(HERE, "_ref", "libfargo_ref_%s_%s.so" % (kind, ref_variant(cfg)))
        elif kind == "ref_o3":
            path = os.path.join(HERE, "_ref", "libfargo_ref_%s_o3.so" % ref_variant(cfg))
        else:
            path = os.path.join(HERE, "_ref", "libfargo_ref_%s.so" % ref_variant(cfg))
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        if kind in ("ref", "ref_o3", "dropin", "shadow"):
            # Each reference library holds one disk in its globals (and in
            # function-level statics such as potential.c's alreadycalculated):
            # load a fresh private copy per Disk.  dlopen identifies a library
            # by its inode, so the copy must be a new file, not a link.
            import shutil
            import tempfile
            tmp = tempfile.mkdtemp(prefix="fargo_ref_")
            copy = os.path.join(tmp, os.path.basename(path))
            shutil.copyfile(path, copy)
            lib = C.CDLL(copy, mode=os.RTLD_NOW | os.RTLD_LOCAL)
            shutil.rmtree(tmp, ignore_errors=True)
        else:
            lib = Disk._libs.get(path)
            if lib is None:
                lib = Disk._libs[path] = C.CDLL(path)
        self.lib = lib
        self.params = make_params(cfg)
        self.shape = cfg.shape
        if kind == "oracle":
            lib.fo_create.restype = C.c_void_p
            lib.fo_create.argtypes = [C.POINTER(FoParams)]
            lib.fo_step.restype = C.c_double
            lib.fo_step.argtypes = [C.c_void_p, C.c_double]
            lib.fo_mass.restype = C.c_double
            lib.fo_mass.argtypes = [C.c_void_p, C.c_int]
            for n in ("fo_set_state", "fo_get_state", "fo_initialize", "fo_get_scalars",
                      "fo_destroy", "fo_get_geometry"):
                getattr(lib, n).restype = None
            lib.fo_get_energy.restype = None
            self.h = lib.fo_create(C.byref(self.params))
            if not self.h:
                raise ValueError("the oracle restatement has the adiabatic EOS and dust diffusion for 2D "
                                 "cylindrical disks only (not together)")
        else:
            lib.ref_create.restype = C.c_int
            lib.ref_create.argtypes = [C.POINTER(FoParams)]
            lib.ref_step.restype = C.c_double
            lib.ref_step.argtypes = [C.c_double]
            rc = lib.ref_create(C.byref(self.params))
            if rc != 0:
                raise RuntimeError("ref_create failed: %d" % rc)
            self.h = None

    def _call(self, name, *args):
        if self.kind == "oracle":
            return getattr(self.lib, "fo_" + name)(C.c_void_p(self.h), *args)
        return getattr(self.lib, "ref_" + name)(*args)

    def set_state(self, rho, vx, vy, vz, cs, fluid: int = 0):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (rho, vx, vy, vz, cs)]
        self._keep = arrs
        self._call("set_state", C.c_int(fluid), *[_ptr(a) for a in arrs])

    def initialize(self):
        self._call("initialize")

    def step(self, dt_interval: float = 1e30) -> float:
        if self.kind == "oracle":
            return self.lib.fo_step(C.c_void_p(self.h), C.c_double(dt_interval))
        return self.lib.ref_step(C.c_double(dt_interval))

    def state(self, fluid: int = 0):
        out = [np.zeros(self.shape) for _ in range(4)]
        self._call("get_state", C.c_int(fluid), *[_ptr(a) for a in out])
        return {"rho": out[0], "vx": out[1], "vy": out[2], "vz": out[3]}

    def scalars(self):
        o = np.zeros(8)
        self._call("get_scalars", _ptr(o))
        return o

    def geometry(self):
        nz, ny, nx = self.shape
        xa, ya, za = np.zeros(nx + 1), np.zeros(ny + 1), np.zeros(nz + 1)
        self._call("get_geometry", _ptr(xa), _ptr(ya), _ptr(za))
        return xa, ya, za

    def energy(self, fluid: int = 0):
        """The fluid's Energy field (the internal energy of an adiabatic
        disk, the sound speed of an isothermal one)."""
        out = np.zeros(self.shape)
        if self.kind == "oracle":
            self.lib.fo_get_energy(C.c_void_p(self.h), C.c_int(fluid), _ptr(out))
            return out
        self.lib.ref_get_energy.restype = None
        self.lib.ref_get_energy(C.c_int(fluid), _ptr(out))
        return out

    def write_outputs(self, outdir: str, n: int, fluid: int = 0):
        """The reference's own output writers ('ref' kinds): fluid's merged
        <outdir>/<name><field><n>.dat files (WriteMerging) and, for fluid 0,
        the planet files' next line (WritePlanetSystemFile)."""
        if self.kind not in ("ref", "ref_o3", "shadow"):
            raise NotImplementedError("only the reference-source libraries write FARGO3D outputs")
        self.lib.ref_write_outputs.restype = C.c_int
        self.lib.ref_write_outputs.argtypes = [C.c_int, C.c_char_p, C.c_int]
        rc = self.lib.ref_write_outputs(fluid, outdir.encode(), n)
        if rc != 0:
            raise RuntimeError("ref_write_outputs failed: %d" % rc)

    def mass(self, fluid: int = 0) -> float:
        if self.kind != "oracle":
            raise NotImplementedError
        return self.lib.fo_mass(C.c_void_p(self.h), C.c_int(fluid))

    def close(self):
        if self.kind == "oracle" and self.h:
            self.lib.fo_destroy(C.c_void_p(self.h))
            self.h = None


def run(cfg, nsteps: int, kind: str = "oracle", dt_interval: float = 1e30, state=None):
    """Initial state -> nsteps hydro steps; returns (per fluid the state dict
    with its energy "e", dts, scalars)."""
    from fargo3d_b200.setups import initial_state
    d = Disk(cfg, kind)
    for f in range(cfg.nfluids):
        st = state[f] if state is not None else initial_state(cfg, f)
        d.set_state(*st, fluid=f)
    d.initialize()
    dts = [d.step(dt_interval) for _ in range(nsteps)]
    out = [dict(d.state(f), e=d.energy(f)) for f in range(cfg.nfluids)]
    sc = d.scalars()
    d.close()
    return out, np.array(dts), sc
