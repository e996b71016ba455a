"""Disk configurations and initial conditions.

`DiskConfig` carries the run-time parameters of one disk: what FARGO3D reads
from a setup's .opt flags and .par file (std/stdpar.par, setups/fargo/fargo.par,
setups/p3disof/p3disof.par) for the hot path this package implements.  The
initial-condition builders restate the setups' CondInit (setups/fargo/condinit.c,
setups/p3disof/condinit.c) with a seeded numpy noise source in place of
drand48, so the same initial state can be handed to every implementation.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

NGH = 3  # NGHY = NGHZ = 3 (define.h:57-63)
FRAMES = {"F": 0, "C": 1, "G": 2}


@dataclass
class Planet:
    distance: float = 1.0
    mass: float = 1e-3
    feel_disk: bool = False
    feel_others: bool = False


@dataclass
class DiskConfig:
    nx: int = 384
    ny: int = 128
    nz: int = 1                       # 1 -> 2D (X, Y) mesh
    spherical: bool = False           # False: CYLINDRICAL, True: SPHERICAL (3D)
    log_spacing: bool = True          # Spacing Log
    xmin: float = -math.pi
    xmax: float = math.pi
    ymin: float = 0.4
    ymax: float = 2.5
    zmin: float = 0.0
    zmax: float = 0.0
    aspectratio: float = 0.05
    sigmaslope: float = 0.5
    flaringindex: float = 0.0
    sigma0: float = 6.3661977237e-4
    nu: float = 1e-5
    alpha: float = 0.0
    alpha_visc: bool = False
    cfl: float = 0.44
    omegaframe: float = 1.0005
    frame: str = "G"
    indirect_term: bool = True
    thickness_smoothing: float = 0.6
    roche_smoothing: float = 0.0
    mass_taper: float = 0.0
    damping_zone: float = 1.15
    tau_damp: float = 0.3
    killing_bc_colatitude: float = -0.2
    planets: List[Planet] = field(default_factory=lambda: [Planet()])
    eccentricity: float = 0.0
    inclination: float = 0.0
    nfluids: int = 1
    invstokes: Tuple[float, ...] = ()
    epsilon: float = 0.0              # EPSILON, dust-to-gas ratio per dust fluid (0: 0.01 / (nfluids - 1))
    stockholm: bool = True
    dust_diffusion: bool = False      # DUSTDIFFUSION of the dust fluids (multifluid)
    adiabatic: bool = False           # ADIABATIC equation of state (else ISOTHERMAL)
    gamma: float = 1.66666667         # GAMMA
    noise: float = 1e-4
    seed: int = 0
    slab_y0: int = 0                  # radial slab of a larger disk: rows [slab_y0, slab_y0 + ny)
    slab_ny_global: int = 0           # of a mesh of slab_ny_global rows (0: the disk is whole)
    dt_output: float = 0.314159265359  # DT

    @property
    def is3d(self) -> bool:
        return self.nz > 1

    @property
    def shape(self) -> Tuple[int, int, int]:
        """Stored (z, y, x) shape, ghosts included: x fastest (define.h:455)."""
        return (self.nz + 2 * NGH if self.is3d else 1, self.ny + 2 * NGH, self.nx)

    @property
    def active_cells(self) -> int:
        return self.nx * self.ny * (self.nz if self.is3d else 1)

    def replace(self, **kw) -> "DiskConfig":
        return dataclasses.replace(self, **kw)


# --------------------------------------------------------------------------
# Named configurations (the hot path's benchmark shapes).
def config_fargo2d(nx: int = 384, ny: int = 128, seed: int = 0) -> DiskConfig:
    """2D cylindrical isothermal disk with one planet (setups/fargo with
    SigmaSlope 0.5 and log spacing): 384 x 128, r in [0.4, 2.5]."""
    return DiskConfig(nx=nx, ny=ny, seed=seed)


def config_multifluid(nx: int = 768, ny: int = 256, nfluids: int = 5,
                      invstokes=(1000.0, 100.0, 10.0, 1.0), seed: int = 0, dust_diffusion: bool = False) -> DiskConfig:
    """2D cylindrical gas disk with nfluids - 1 dust species coupled by
    implicit drag (setups/fargo_multifluid with DRAGFORCE + STOKESNUMBER):
    1/St per dust species `invstokes`, dust-to-gas ratio 0.01 / (nfluids - 1)
    per species, fixed frame, no indirect term, constant nu = 1e-5, planet
    q = 1e-3 at r = 1; with dust_diffusion, the dust densities also diffuse
    down their concentration gradients (DUSTDIFFUSION, the setup's stock
    flag)."""
    return DiskConfig(nx=nx, ny=ny, sigma0=1e-4, frame="F", omegaframe=0.0, indirect_term=False,
                      nfluids=nfluids, invstokes=tuple(invstokes[:nfluids - 1]), seed=seed,
                      dust_diffusion=dust_diffusion)


def config_adiabatic2d(nx: int = 384, ny: int = 128, seed: int = 0, gamma: float = 1.4) -> DiskConfig:
    """The 2D cylindrical disk of config_fargo2d with an ADIABATIC equation of
    state (internal energy e, P = (GAMMA - 1) e) and alpha viscosity
    (alpha = 1e-3): the initial energy gives the isothermal disk's pressure,
    and the energy's radial boundaries mirror the active cells."""
    return DiskConfig(nx=nx, ny=ny, adiabatic=True, gamma=gamma, alpha_visc=True, alpha=1e-3, nu=0.0, seed=seed)


def config_p3disof(nx: int = 512, ny: int = 256, nz: int = 48, seed: int = 0) -> DiskConfig:
    """3D spherical isothermal disk (setups/p3disof): colatitude pi/2 +- 0.15,
    rho ~ r^-1.5 with a vertical hydrostatic profile, h = 0.05, no flaring,
    planet q = 3e-4 at r = 1, fixed frame rotating at 1."""
    return DiskConfig(
        nx=nx, ny=ny, nz=nz, spherical=True, log_spacing=False,
        ymin=0.6, ymax=1.5, zmin=1.42079632679489661922, zmax=1.72079632679489661922,
        sigmaslope=0.5, flaringindex=0.0, nu=1e-5, omegaframe=1.0, frame="F",
        indirect_term=False, thickness_smoothing=0.1,
        planets=[Planet(1.0, 3e-4)], seed=seed)


# --------------------------------------------------------------------------
def geometry(cfg: DiskConfig):
    """Cell edges and centres as InitSpace computes them (LowTasks.c:300-383)."""
    nx, ny = cfg.nx, cfg.ny
    nz = cfg.nz if cfg.is3d else 1
    j = np.arange(ny + 2 * NGH + 1, dtype=np.float64)
    if cfg.log_spacing:
        dy = (math.log(cfg.ymax) - math.log(cfg.ymin)) / ny
        ymin = np.array([math.exp(math.log(cfg.ymin) + dy * (jj - NGH)) for jj in j])
    else:
        dy = (cfg.ymax - cfg.ymin) / ny
        ymin = cfg.ymin + dy * (j - NGH)
    dx = (cfg.xmax - cfg.xmin) / nx
    xmin = cfg.xmin + dx * np.arange(nx + 1, dtype=np.float64)
    if cfg.is3d:
        dz = (cfg.zmax - cfg.zmin) / nz
        zmin = cfg.zmin + dz * (np.arange(nz + 2 * NGH + 1, dtype=np.float64) - NGH)
    else:
        zmin = np.zeros(2)
    med = lambda e: 0.5 * (e[1:] + e[:-1])
    return xmin, ymin, zmin, med(xmin), med(ymin), med(zmin)


def initial_state(cfg: DiskConfig, fluid: int = 0):
    """Initial (rho, vx, vy, vz, cs) arrays of shape cfg.shape.

    2D: setups/fargo/condinit.c:23-45 with Sigma = Sigma0 r^-SigmaSlope
    (1 + noise U(-1,1)), v_phi from the pressure-supported rotation curve and
    v_r = 0.  3D: setups/p3disof/condinit.c:21-50 (both FlaringIndex
    branches), with the same multiplicative density noise.  Dust fluids (fluid > 0) get
    eps = epsilon (default 0.01 / (nfluids - 1)) times the gas density, the Keplerian velocity
    without pressure support (2D) and no pressure (cs = 0)."""
    rng = np.random.default_rng(cfg.seed * 1000 + fluid)
    nzs, nys, nxs = cfg.shape
    _, _, _, xmed, ymed, zmed = geometry(cfg)
    r = ymed[None, :, None] * np.ones(cfg.shape)
    h, ss, fi = cfg.aspectratio, cfg.sigmaslope, cfg.flaringindex
    omegaframe = cfg.omegaframe
    if cfg.frame != "F" and cfg.planets:
        p0 = cfg.planets[0]
        omegaframe = math.sqrt((1.0 + p0.mass) / p0.distance ** 3)
    omega = np.sqrt(1.0 / r ** 3)
    noise = 1.0 + cfg.noise * rng.uniform(-1.0, 1.0, size=cfg.shape)
    if not cfg.is3d:
        rho = cfg.sigma0 * r ** (-ss) * noise
        cs = h * r ** fi * omega * r
        vx = omega * r * np.sqrt(1.0 + h ** 2 * r ** (2 * fi) * (2.0 * fi - 1.0 - ss)) - omegaframe * r
        vy = np.zeros(cfg.shape)
        vz = np.zeros(cfg.shape)
    else:
        st = np.sin(zmed)[:, None, None] * np.ones(cfg.shape)
        xi = ss + 1.0 + fi
        beta = 1.0 - 2.0 * fi
        hh = h * r ** fi
        if fi == 0.0:
            rho = cfg.sigma0 / math.sqrt(2.0 * math.pi) / h * r ** (-xi) * st ** (-beta - xi + 1.0 / (hh * hh)) * noise
        else:
            rho = (cfg.sigma0 / math.sqrt(2.0 * math.pi) / h * r ** (-xi) * st ** (-xi - beta)
                   * np.exp((1.0 - st ** (-2.0 * fi)) / 2.0 / fi / (hh * hh)) * noise)
        vx = omega * r * np.sqrt(st ** (-2.0 * fi) - (beta + xi) * hh * hh) - omegaframe * r * st
        cs = hh * np.sqrt(1.0 / r)
        vy = np.zeros(cfg.shape)
        vz = np.zeros(cfg.shape)
    if cfg.adiabatic:
        # the internal energy whose pressure (GAMMA - 1) e is the isothermal
        # disk's rho cs^2 (FARGO3D's Energy field holds e)
        cs = rho * cs * cs / (cfg.gamma - 1.0)
    if fluid > 0:
        # dust (setups/fargo_multifluid/condinit.c:38-44): eps times the gas
        # density, Keplerian azimuthal velocity without pressure support, no
        # radial velocity, no sound speed
        eps = cfg.epsilon if cfg.epsilon > 0.0 else 0.01 / max(cfg.nfluids - 1, 1)
        rho = rho * eps
        cs = np.zeros(cfg.shape)
        if not cfg.is3d:
            vx = omega * r - omegaframe * r
    return (np.ascontiguousarray(rho), np.ascontiguousarray(vx), np.ascontiguousarray(vy),
            np.ascontiguousarray(vz), np.ascontiguousarray(cs))


def config_batched(ndisks: int = 64, seed: int = 0):
    """Independent 2D disks of uneven sizes (the batched workload): N_phi in
    {128, 256, 512, 1024}, N_r in {64, 128, 256, 512}, planet mass ratio
    log-uniform in [1e-5, 3e-3], alpha viscosity log-uniform in [1e-4, 1e-2],
    aspect ratio uniform in [0.03, 0.08], Sigma ~ r^-p with p uniform in
    [0, 1.5].  Seeded numpy default_rng."""
    rng = np.random.default_rng(seed)
    out = []
    for d in range(ndisks):
        nx = int(rng.choice([128, 256, 512, 1024]))
        ny = int(rng.choice([64, 128, 256, 512]))
        q = float(np.exp(rng.uniform(np.log(1e-5), np.log(3e-3))))
        alpha = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        h = float(rng.uniform(0.03, 0.08))
        p = float(rng.uniform(0.0, 1.5))
        out.append(DiskConfig(nx=nx, ny=ny, aspectratio=h, sigmaslope=p, alpha=alpha, alpha_visc=True, nu=0.0,
                              planets=[Planet(1.0, q)], seed=seed * 100000 + d))
    return out
