"""FARGO3D setup files -> DiskConfig, and DiskConfig -> FARGO3D setup files.

A FARGO3D run is described by three text files: the parameter file
(`setups/<name>/<name>.par`, read by ReadVarFile, src/param.c:97-200, over the
defaults of std/stdpar.par), the planet file named by its `PlanetConfig`
parameter (`planets/*.cfg`, read by InitPlanetarySystem, src/psys.c:140-200)
and the build options (`setups/<name>/<name>.opt`, the `-D` flags handed to
the compiler).  `load_setup` reads the three with the same rules and returns
the `DiskConfig` of the disk they describe, so a FARGO3D user can start a
`Disk` or a `Batch` from the setup directory they already have.
`write_setup` goes the other way and writes the three files for a
`DiskConfig`, so the same disk can be run by a stock FARGO3D build.

Rules restated from the reference's readers:

* parameter lines: the first whitespace-delimited word is the name (case
  does not matter); the value is the first word after the separators
  `\\t :=>`; everything after it is ignored; a line whose first word starts
  with `#` is a comment (param.c:129-146);
* a real is the longest leading decimal number of the value (`%lf`), an
  integer is that real truncated toward zero, a boolean is true when the
  value starts with `y` or `Y`, a string is the word itself (param.c:134-144);
* the first definition of a name wins, later ones are ignored; `Include
  <file>` reads another parameter file in place (param.c:147-168);
  redefinitions (the command line's `-name:value,...`, redefoptions.c) beat
  the file;
* a planet line starts with a letter: name, distance, mass, accretion rate,
  feels-disk and feels-others, where any word not starting with `n`/`N`
  means yes; `SemiMajorAxis` > 0 replaces the first planet's distance,
  `OrbitalRadius` > 1e-30 scales every distance and `PlanetMass` > 1e-18
  replaces the first planet's mass (psys.c:168-194);
* `Frame` `C`/`c` is corotating, `G`/`g` guiding-centre, anything else the
  fixed frame (param.c:236-240); `Spacing` starting with `Lo` is
  logarithmic (LowTasks.c:337);
* `ThicknessSmoothing` and `RocheSmoothing` may not both be non-zero
  (param.c:250).

Deviations, each one loud: a value that is not a number where a number is
needed raises ValueError (the reference keeps the previous line's number);
every `-D` option that changes the physics beyond what this library
integrates raises NotImplementedError naming the option; a planet with a
non-zero accretion rate or `ExcludeHill yes` raises NotImplementedError.
`Noise` perturbs the density only: the reference's fargo CondInit draws
`NOISE * (U[0,1) - 0.5)` (setups/fargo/condinit.c:33), which is
`DiskConfig.noise = NOISE / 2` of the seeded `1 + noise * U(-1, 1)` factor
`initial_state` applies; its velocity perturbations (condinit.c:46-48) are
not restated.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Mapping, Optional, Tuple, Union

from .setups import DiskConfig, Planet

PathLike = Union[str, "os.PathLike[str]"]

_SEPARATORS = "\t :=>"                # param.c:108
_PLANET_SEPARATORS = "\t :=>_"        # psys.c:174
_REDEF_SEPARATORS = "\t :=>,;"        # redefoptions.c

# Defaults of the parameters this library reads, restating std/stdpar.par
# (names upper-case, as the reader compares them).  DT has no standard
# default: a setup's .par defines it.
STD_DEFAULTS: Dict[str, str] = {
    "NX": "1", "NY": "1", "NZ": "1",
    "XMIN": "0.0", "XMAX": "1.0", "YMIN": "0.0", "YMAX": "1.0", "ZMIN": "0.0", "ZMAX": "1.0",
    "SIGMASLOPE": "0.0", "ECCENTRICITY": "0.0", "INCLINATION": "0.0",
    "THICKNESSSMOOTHING": "0.0", "ROCHESMOOTHING": "0.0",
    "ASPECTRATIO": "0.05", "SIGMA0": "1.0", "FLARINGINDEX": "0.0", "NU": "0.0",
    "FRAME": "fixed", "OMEGAFRAME": "0.0", "INDIRECTTERM": "no", "EXCLUDEHILL": "no",
    "MASSTAPER": "0.0", "NOISE": "0.0", "SPACING": "Lin", "GAMMA": "1.66666667", "ALPHA": "0.0",
    "PLANETCONFIG": "NONE", "DAMPINGZONE": "1.15", "TAUDAMP": "0.3", "KILLINGBCCOLATITUDE": "-0.2",
    "CFL": "0.44", "PLANETMASS": "0.0", "ORBITALRADIUS": "0.0", "SEMIMAJORAXIS": "0.0",
}

# Build options this library reads.
_HANDLED_OPTIONS = {"X", "Y", "Z", "CYLINDRICAL", "SPHERICAL", "ISOTHERMAL", "ADIABATIC", "VISCOSITY",
                    "ALPHAVISCOSITY", "POTENTIAL", "STOCKHOLM", "NFLUIDS", "DRAGFORCE", "STOKESNUMBER",
                    "DUSTDIFFUSION", "FLOAT"}
# Build options that change output, diagnostics or the CUDA launch shape of
# the reference, not the arithmetic of a hydro step.
_NEUTRAL_OPTIONS = {"LEGACY", "LONGSUMMARY", "DEBUG", "PROFILING", "WALLCLOCK", "MPIIO", "MATPLOTLIB",
                    "NOOUTPUTS", "NOFLUSH", "WRITEGHOSTS", "PINNED", "BIGMEM", "MPICUDA", "PARALLEL",
                    "GPU", "BLOCK_X", "BLOCK_Y", "BLOCK_Z"}

_NUMBER = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")


# --------------------------------------------------------------------------
# Parameter values (param.c:134-144)

def _value_word(rest: str) -> str:
    """The first word after the separators that follow a name."""
    words = rest.lstrip(_SEPARATORS).split()
    return words[0] if words else ""


def as_real(word: str, name: str = "value") -> float:
    m = _NUMBER.match(word)
    if not m:
        raise ValueError("%s: %r is not a number" % (name, word))
    return float(m.group(0))


def as_int(word: str, name: str = "value") -> int:
    return int(as_real(word, name))


def as_bool(word: str) -> bool:
    return word[:1].upper() == "Y"


# --------------------------------------------------------------------------
# Readers

def parse_redefinitions(text: str) -> Dict[str, str]:
    """`name:value,name:value` (the command line's parameter redefinition,
    redefoptions.c) -> {NAME: value}."""
    words = [w for w in re.split("[" + re.escape(_REDEF_SEPARATORS) + "]+", text) if w]
    if len(words) % 2:
        raise ValueError("parameter redefinition %r: names and values do not pair up" % text)
    return {words[i].upper(): words[i + 1] for i in range(0, len(words), 2)}


def read_par(path: PathLike, redefine: Optional[Mapping[str, str]] = None,
             _into: Optional[Dict[str, str]] = None, _depth: int = 0) -> Dict[str, str]:
    """Read a FARGO3D parameter file -> {NAME: value word} (defined names
    only, no defaults).  `redefine` entries win over the file."""
    out: Dict[str, str] = {} if _into is None else _into
    if _into is None and redefine:
        out.update({k.upper(): str(v) for k, v in redefine.items()})
    if _depth > 16:
        raise ValueError("%s: Include nested more than 16 deep" % path)
    path = os.fspath(path)
    with open(path, "r") as fh:
        for line in fh:
            words = line.split()
            if not words or words[0].startswith("#"):
                continue
            name = words[0]
            word = _value_word(line[line.index(name) + len(name):])
            name = name.upper()
            if name == "INCLUDE":
                read_par(_resolve(word, os.path.dirname(path)), None, out, _depth + 1)
            elif name != "END" and name not in out:
                out[name] = word
    return out


def read_planets(path: PathLike) -> List[Tuple[str, Planet, float]]:
    """Read a FARGO3D planet file -> [(name, Planet, accretion rate)]."""
    out = []
    with open(os.fspath(path), "r") as fh:
        for line in fh:
            if not line[:1].isalpha():
                continue
            name = line.split()[0]
            rest = line[len(name):].lstrip(_PLANET_SEPARATORS).split()
            if len(rest) < 2:
                raise ValueError("%s: planet %r needs a distance and a mass" % (path, name))
            dist, mass = as_real(rest[0], name), as_real(rest[1], name)
            accret = as_real(rest[2], name) if len(rest) > 2 else 0.0
            feel_disk = not rest[3][:1].lower() == "n" if len(rest) > 3 else True
            feel_others = not rest[4][:1].lower() == "n" if len(rest) > 4 else True
            out.append((name, Planet(dist, mass, feel_disk, feel_others), accret))
    return out


def read_opt(path: PathLike, make_vars: Optional[Mapping[str, str]] = None) -> Dict[str, Optional[str]]:
    """Read a FARGO3D setup's .opt (a makefile fragment) -> {OPTION: value or
    None} of its `-D` flags.  Variables (`NAME = v`, `:=`, `+=`) expand as
    `${NAME}` / `$(NAME)`; `ifeq`/`ifneq` blocks are evaluated with the
    file's variables over `make_vars` (an unset variable is empty, so the
    `ifeq (${GPU}, 1)` blocks of the stock setups are skipped by default)."""
    var: Dict[str, str] = {k: str(v) for k, v in (make_vars or {}).items()}
    expand = lambda s: re.sub(r"\$[({]([A-Za-z_0-9]+)[)}]", lambda m: var.get(m.group(1), ""), s)
    live: List[bool] = []
    with open(os.fspath(path), "r") as fh:
        for raw in fh:
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            head = line.split()[0]
            if head in ("ifeq", "ifneq"):
                cond = expand(line[len(head):].strip())
                m = re.match(r"^\((.*),(.*)\)$", cond)
                if not m:
                    raise ValueError("%s: cannot read %r" % (path, raw.strip()))
                same = m.group(1).strip() == m.group(2).strip()
                live.append(same if head == "ifeq" else not same)
                continue
            if head == "else":
                if not live:
                    raise ValueError("%s: else without ifeq" % path)
                live[-1] = not live[-1]
                continue
            if head == "endif":
                if not live:
                    raise ValueError("%s: endif without ifeq" % path)
                live.pop()
                continue
            if not all(live):
                continue
            m = re.match(r"^([A-Za-z_][A-Za-z_0-9]*)\s*(\+=|:=|\?=|=)\s*(.*)$", line)
            if not m:
                continue
            name, op, value = m.group(1), m.group(2), expand(m.group(3))
            if op == "+=":
                var[name] = (var.get(name, "") + " " + value).strip()
            elif op != "?=" or name not in var:
                var[name] = value
    if live:
        raise ValueError("%s: ifeq without endif" % path)
    opts: Dict[str, Optional[str]] = {}
    for word in var.get("FARGO_OPT", "").split():
        if word.startswith("-D"):
            k, _, v = word[2:].partition("=")
            opts[k] = v if _ else None
    return opts


# --------------------------------------------------------------------------
# Setup -> DiskConfig

@dataclass
class Setup:
    """A FARGO3D setup as read: the disk, its arithmetic precision ("fp32"
    under -DFLOAT, else "fp64"), the planet names and every parameter and
    option read."""
    config: DiskConfig
    precision: str = "fp64"
    planet_names: List[str] = field(default_factory=list)
    params: Dict[str, str] = field(default_factory=dict)
    options: Dict[str, Optional[str]] = field(default_factory=dict)


def _resolve(name: str, *dirs: str) -> str:
    """A file named in a setup: absolute, else found beside the naming file
    or one of its ancestors (the reference runs from its tree's root, where
    `planets/` and `setups/` sit), else relative to the working directory."""
    if os.path.isabs(name):
        return name
    for d in dirs:
        d = os.path.abspath(d)
        while True:
            cand = os.path.join(d, name)
            if os.path.exists(cand):
                return cand
            up = os.path.dirname(d)
            if up == d:
                break
            d = up
    return name


def config_from_params(params: Mapping[str, str], options: Mapping[str, Optional[str]],
                       planets: Optional[List[Tuple[str, Planet, float]]] = None,
                       **overrides) -> Tuple[DiskConfig, str]:
    """The DiskConfig (and precision) of parameter words `params` (defined
    names; std/stdpar.par defaults fill the rest), build options `options`
    and planets `planets`.  `overrides` are DiskConfig fields set last
    (e.g. seed)."""
    P = dict(STD_DEFAULTS)
    P.update({k.upper(): v for k, v in params.items()})

    def real(k):
        if k not in P:
            raise ValueError("parameter %s is not defined" % k)
        return as_real(P[k], k)

    opts = set(options)
    unknown = sorted(opts - _HANDLED_OPTIONS - _NEUTRAL_OPTIONS)
    if unknown:
        raise NotImplementedError("build option(s) outside the hydro step this library integrates: "
                                  + ", ".join("-D" + u for u in unknown))
    if not {"X", "Y"} <= opts:
        raise NotImplementedError("the disk needs both -DX (azimuth) and -DY (radius)")
    if ("SPHERICAL" in opts) == ("CYLINDRICAL" in opts):
        raise NotImplementedError("exactly one of -DCYLINDRICAL and -DSPHERICAL")
    if ("ISOTHERMAL" in opts) == ("ADIABATIC" in opts):
        raise NotImplementedError("exactly one of -DISOTHERMAL and -DADIABATIC")
    if "POTENTIAL" not in opts:
        raise NotImplementedError("the disk needs -DPOTENTIAL (the star's and planets' gravity)")
    if "VISCOSITY" in opts and "ALPHAVISCOSITY" in opts:
        raise NotImplementedError("-DVISCOSITY and -DALPHAVISCOSITY together")
    nfl = int(options.get("NFLUIDS") or 1)
    if nfl > 1 and not {"DRAGFORCE", "STOKESNUMBER"} <= opts:
        raise NotImplementedError("dust fluids couple to the gas through -DDRAGFORCE with -DSTOKESNUMBER")
    spacing = P["SPACING"]
    if spacing[:1].upper() in ("F", "N"):
        raise NotImplementedError("Spacing %s (a mesh read from a file)" % spacing)
    if as_bool(P["EXCLUDEHILL"]):
        raise NotImplementedError("ExcludeHill yes")
    if real("THICKNESSSMOOTHING") != 0.0 and real("ROCHESMOOTHING") != 0.0:
        raise ValueError("ThicknessSmoothing and RocheSmoothing cannot both be non-zero")
    pl: List[Planet] = []
    for i, (name, p, accret) in enumerate(planets or []):
        if accret != 0.0:
            raise NotImplementedError("planet %s accretes (rate %g)" % (name, accret))
        dist, mass = p.distance, p.mass
        if real("SEMIMAJORAXIS") > 0.0 and i == 0:
            dist = real("SEMIMAJORAXIS")
        if real("ORBITALRADIUS") > 1e-30:
            dist *= real("ORBITALRADIUS")
        if real("PLANETMASS") > 1e-18 and i == 0:
            mass = real("PLANETMASS")
        pl.append(Planet(dist, mass, p.feel_disk, p.feel_others))
    is3d = "Z" in opts
    frame = P["FRAME"][:1].upper()
    kw = dict(
        nx=as_int(P["NX"], "NX"), ny=as_int(P["NY"], "NY"), nz=as_int(P["NZ"], "NZ") if is3d else 1,
        spherical="SPHERICAL" in opts,
        log_spacing=spacing[:2].upper() == "LO",
        xmin=real("XMIN"), xmax=real("XMAX"), ymin=real("YMIN"), ymax=real("YMAX"),
        zmin=real("ZMIN") if is3d else 0.0, zmax=real("ZMAX") if is3d else 0.0,
        aspectratio=real("ASPECTRATIO"), sigmaslope=real("SIGMASLOPE"), flaringindex=real("FLARINGINDEX"),
        sigma0=real("SIGMA0"),
        nu=real("NU") if "VISCOSITY" in opts else 0.0,
        alpha=real("ALPHA"), alpha_visc="ALPHAVISCOSITY" in opts,
        cfl=real("CFL"), omegaframe=real("OMEGAFRAME"),
        frame=frame if frame in ("C", "G") else "F",
        indirect_term=as_bool(P["INDIRECTTERM"]),
        thickness_smoothing=real("THICKNESSSMOOTHING"), roche_smoothing=real("ROCHESMOOTHING"),
        mass_taper=real("MASSTAPER"), damping_zone=real("DAMPINGZONE"), tau_damp=real("TAUDAMP"),
        killing_bc_colatitude=real("KILLINGBCCOLATITUDE"),
        planets=pl, eccentricity=real("ECCENTRICITY"), inclination=real("INCLINATION"),
        nfluids=nfl,
        invstokes=tuple(real("INVSTOKES%d" % k) for k in range(1, nfl)),
        epsilon=real("EPSILON") if nfl > 1 and "EPSILON" in P else 0.0,
        stockholm="STOCKHOLM" in opts,
        dust_diffusion="DUSTDIFFUSION" in opts,
        adiabatic="ADIABATIC" in opts, gamma=real("GAMMA"),
        noise=0.5 * real("NOISE"),
    )
    if "DT" in P:
        kw["dt_output"] = real("DT")
    kw.update(overrides)
    return DiskConfig(**kw), ("fp32" if "FLOAT" in opts else "fp64")


def load_setup(par: PathLike, opt: Optional[PathLike] = None, planets: Optional[PathLike] = None,
               redefine: Union[None, str, Mapping[str, str]] = None,
               make_vars: Optional[Mapping[str, str]] = None, **overrides) -> Setup:
    """Read a FARGO3D setup.  `par` is the parameter file or a setup
    directory holding `<dir name>.par`; `opt` defaults to the .opt beside
    the .par with the same stem; `planets` to the file the `PlanetConfig`
    parameter names (NONE: no planet).  `redefine` is the command line's
    parameter redefinition (a `name:value,...` string or a mapping).
    `overrides` are DiskConfig fields set last (e.g. seed=3)."""
    par = os.fspath(par)
    if os.path.isdir(par):
        par = os.path.join(par, os.path.basename(os.path.normpath(par)) + ".par")
    if isinstance(redefine, str):
        redefine = parse_redefinitions(redefine)
    params = read_par(par, redefine)
    if opt is None:
        opt = os.path.splitext(par)[0] + ".opt"
    options = read_opt(opt, make_vars)
    pl: List[Tuple[str, Planet, float]] = []
    pc = params.get("PLANETCONFIG", STD_DEFAULTS["PLANETCONFIG"])
    if planets is None and pc.upper() != "NONE":
        planets = _resolve(pc, os.path.dirname(os.path.abspath(par)))
    if planets is not None:
        pl = read_planets(planets)
    cfg, precision = config_from_params(params, options, pl, **overrides)
    return Setup(cfg, precision, [n for n, _, _ in pl], params, options)


# --------------------------------------------------------------------------
# DiskConfig -> setup files

def write_setup(cfg: DiskConfig, directory: PathLike, name: str = "b200disk",
                precision: str = "fp64") -> Tuple[str, str, str]:
    """Write `<name>.par`, `<name>.opt` and `<name>.cfg` (the planets) for
    `cfg` into `directory` and return their paths.  `load_setup` of the
    .par gives `cfg` back (seed and slab fields aside; `epsilon` 0 is
    written as the dust-to-gas ratio it stands for)."""
    if precision not in ("fp64", "fp32"):
        raise ValueError("precision is 'fp64' or 'fp32'")
    if cfg.nfluids > 1 and len(cfg.invstokes) < cfg.nfluids - 1:
        raise ValueError("%d dust fluids need %d inverse Stokes numbers" % (cfg.nfluids - 1, cfg.nfluids - 1))
    directory = os.fspath(directory)
    os.makedirs(directory, exist_ok=True)
    par_path = os.path.join(directory, name + ".par")
    opt_path = os.path.join(directory, name + ".opt")
    cfg_path = os.path.abspath(os.path.join(directory, name + ".cfg"))
    r = repr
    yn = lambda b: "YES" if b else "NO"
    rows = [("Setup", name), ("Nx", cfg.nx), ("Ny", cfg.ny), ("Nz", cfg.nz if cfg.is3d else 1),
            ("Xmin", r(cfg.xmin)), ("Xmax", r(cfg.xmax)), ("Ymin", r(cfg.ymin)), ("Ymax", r(cfg.ymax))]
    if cfg.is3d:
        rows += [("Zmin", r(cfg.zmin)), ("Zmax", r(cfg.zmax))]
    rows += [("Spacing", "Log" if cfg.log_spacing else "Lin"),
             ("AspectRatio", r(cfg.aspectratio)), ("Sigma0", r(cfg.sigma0)), ("SigmaSlope", r(cfg.sigmaslope)),
             ("FlaringIndex", r(cfg.flaringindex)), ("Nu", r(cfg.nu)), ("Alpha", r(cfg.alpha)),
             ("CFL", r(cfg.cfl)), ("Frame", cfg.frame), ("OmegaFrame", r(cfg.omegaframe)),
             ("IndirectTerm", yn(cfg.indirect_term)),
             ("ThicknessSmoothing", r(cfg.thickness_smoothing)), ("RocheSmoothing", r(cfg.roche_smoothing)),
             ("MassTaper", r(cfg.mass_taper)), ("DampingZone", r(cfg.damping_zone)), ("TauDamp", r(cfg.tau_damp)),
             ("KillingBCColatitude", r(cfg.killing_bc_colatitude)),
             ("Eccentricity", r(cfg.eccentricity)), ("Inclination", r(cfg.inclination)),
             ("Gamma", r(cfg.gamma)), ("Noise", r(2.0 * cfg.noise)), ("DT", r(cfg.dt_output)),
             ("PlanetConfig", cfg_path if cfg.planets else "NONE")]
    if cfg.nfluids > 1:
        eps = cfg.epsilon if cfg.epsilon > 0.0 else 0.01 / (cfg.nfluids - 1)
        rows += [("Invstokes%d" % (k + 1), r(v)) for k, v in enumerate(cfg.invstokes[:cfg.nfluids - 1])]
        rows.append(("Epsilon", r(eps)))
    with open(par_path, "w") as fh:
        fh.writelines("%-24s %s\n" % (k, v) for k, v in rows)
    flags = ["X", "Y"] + (["Z"] if cfg.is3d else [])
    flags += ["SPHERICAL" if cfg.spherical else "CYLINDRICAL", "ADIABATIC" if cfg.adiabatic else "ISOTHERMAL",
              "POTENTIAL"]
    if cfg.alpha_visc:
        flags.append("ALPHAVISCOSITY")
    elif cfg.nu != 0.0:
        flags.append("VISCOSITY")
    if cfg.stockholm:
        flags.append("STOCKHOLM")
    if cfg.nfluids > 1:
        flags += ["DRAGFORCE", "STOKESNUMBER"]
    if cfg.dust_diffusion:
        flags.append("DUSTDIFFUSION")
    if precision == "fp32":
        flags.append("FLOAT")
    with open(opt_path, "w") as fh:
        fh.write("FLUIDS := %s\n" % " ".join(str(f) for f in range(cfg.nfluids)))
        fh.write("NFLUIDS = %d\n" % cfg.nfluids)
        fh.write("FARGO_OPT += -DNFLUIDS=${NFLUIDS}\n")
        fh.writelines("FARGO_OPT += -D%s\n" % f for f in flags)
    with open(cfg_path, "w") as fh:
        fh.write("# Planet Name  Distance  Mass  Accretion  Feels Disk  Feels Others\n")
        for i, p in enumerate(cfg.planets):
            fh.write("Planet%d %s %s 0.0 %s %s\n" % (i, r(p.distance), r(p.mass), yn(p.feel_disk),
                                                    yn(p.feel_others)))
    return par_path, opt_path, cfg_path
