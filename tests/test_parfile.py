"""FARGO3D setup files (.par, planet .cfg, .opt) -> DiskConfig and back.

The fixtures are written here in the reference's formats (std/stdpar.par,
setups/*/*.par, setups/*/*.opt, planets/*.cfg): the parsing rules of
src/param.c:97-200 and src/psys.c:140-200, the option blocks of a setup's
makefile fragment, and a round trip of every named configuration through
write_setup -> load_setup."""
import dataclasses
import math
import os

import pytest

from fargo3d_b200 import parfile as pf
from fargo3d_b200.setups import (Planet, config_adiabatic2d, config_batched, config_fargo2d, config_multifluid,
                                 config_p3disof)


def _write(path, text):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as fh:
        fh.write(text)
    return path


def test_values():
    assert pf.as_real("1.5e-3abc") == 1.5e-3
    assert pf.as_real("-.25") == -0.25
    assert pf.as_int("384.9") == 384 and pf.as_int("-2.7") == -2 and pf.as_int("1e3") == 1000
    assert pf.as_bool("yes") and pf.as_bool("Y") and pf.as_bool("yES")
    assert not pf.as_bool("no") and not pf.as_bool("True") and not pf.as_bool("")
    with pytest.raises(ValueError):
        pf.as_real("abc", "NX")


def test_read_par_rules(tmp_path):
    _write(str(tmp_path / "common.par"), "Sigma0 2.0\nCFL 0.3\n")
    p = _write(str(tmp_path / "a.par"), (
        "# comment line\n"
        "\n"
        "   # indented comment\n"
        "aspectratio\t0.07   Thickness over radius\n"
        "Nx :256\n"
        "Ny:32\n"                       # one word: the name is "NY:32"
        "Ny = 64 radial zones\n"
        "Ymin\t=>0.5\n"
        "AspectRatio 0.09\n"            # second definition: ignored
        "Include common.par\n"
        "Sigma0 5.0\n"                  # defined by the included file first
        "Frame  Guiding\n"
        "End\n"))
    par = pf.read_par(p)
    assert par["ASPECTRATIO"] == "0.07" and par["NX"] == "256" and par["NY"] == "64"
    assert par["YMIN"] == "0.5" and par["SIGMA0"] == "2.0" and par["CFL"] == "0.3" and par["FRAME"] == "Guiding"
    assert "END" not in par and "INCLUDE" not in par and par["NY:32"] == ""
    par = pf.read_par(p, pf.parse_redefinitions("nx:512,AspectRatio=0.04"))
    assert par["NX"] == "512" and par["ASPECTRATIO"] == "0.04" and par["NY"] == "64"
    with pytest.raises(ValueError):
        pf.parse_redefinitions("nx:512,ny")


def test_read_planets(tmp_path):
    p = _write(str(tmp_path / "p.cfg"), (
        "# Planet Name Distance Mass Accretion Feels Disk Feels Others\n"
        "Alpha\t1.0\t0.001\t0.0\tNO\tno\n"
        "  Indented 9.0 9.0 0.0 YES YES\n"
        "Beta :2.5 3e-4 0.0 yes Nope\n"
        "Gamma 4.0 1e-5\n"))
    pl = pf.read_planets(p)
    assert [n for n, _, _ in pl] == ["Alpha", "Beta", "Gamma"]
    assert pl[0][1] == Planet(1.0, 0.001, False, False)
    assert pl[1][1] == Planet(2.5, 3e-4, True, False)
    assert pl[2][1] == Planet(4.0, 1e-5, True, True) and pl[2][2] == 0.0


def test_read_opt(tmp_path):
    p = _write(str(tmp_path / "s.opt"), (
        "# options\n"
        "FLUIDS := 0 1 2\n"
        "NFLUIDS = 3\n"
        "FARGO_OPT += -DNFLUIDS=${NFLUIDS}\n"
        "FARGO_OPT +=  -DX -DY   # two on a line\n"
        "FARGO_OPT += -DCYLINDRICAL\n"
        "ifeq (${GPU}, 1)\n"
        "FARGO_OPT += -DBLOCK_X=16\n"
        "else\n"
        "FARGO_OPT += -DLONGSUMMARY\n"
        "endif\n"
        "ifneq ($(NFLUIDS), 1)\n"
        "FARGO_OPT += -DDRAGFORCE\n"
        "endif\n"))
    o = pf.read_opt(p)
    assert o == {"NFLUIDS": "3", "X": None, "Y": None, "CYLINDRICAL": None, "LONGSUMMARY": None, "DRAGFORCE": None}
    o = pf.read_opt(p, {"GPU": "1"})
    assert o["BLOCK_X"] == "16" and "LONGSUMMARY" not in o
    _write(str(tmp_path / "bad.opt"), "ifeq (a, a)\nFARGO_OPT += -DX\n")
    with pytest.raises(ValueError):
        pf.read_opt(str(tmp_path / "bad.opt"))


def _setup_tree(root, par_extra="", opt_extra="", planets="Jove 1.0 0.001 0.0 NO NO\n"):
    """A FARGO3D-style tree: setups/disk/disk.{par,opt} and planets/one.cfg."""
    _write(os.path.join(root, "planets", "one.cfg"), "# Name Dist Mass Acc FeelDisk FeelOthers\n" + planets)
    _write(os.path.join(root, "setups", "disk", "disk.par"), (
        "Setup\t\tdisk\n"
        "AspectRatio     \t0.05            Thickness over Radius in the disc\n"
        "Sigma0\t\t\t6.3661977237e-4\tSurface Density at r=1\n"
        "Nu\t\t\t1.0e-5\t\tUniform kinematic viscosity\n"
        "SigmaSlope\t\t0.5\n"
        "Spacing LOG\n"
        "PlanetConfig\t\tplanets/one.cfg\n"
        "ThicknessSmoothing \t0.6\n"
        "IndirectTerm\t\tYes\n"
        "Nx\t\t\t384\n"
        "Ny               \t128\n"
        "Nz 40\n"
        "Xmin\t\t\t-3.14159265358979323844\n"
        "Xmax\t\t\t3.14159265358979323844\n"
        "Ymin\t\t\t0.4\n"
        "Ymax\t\t\t2.5\n"
        "OmegaFrame     \t\t1.0005\n"
        "Frame\t\t\tG\n"
        "Noise 2e-4\n"
        "DT\t\t\t0.314159265359\n"
        "Ninterm 20\n" + par_extra))
    _write(os.path.join(root, "setups", "disk", "disk.opt"), (
        "FLUIDS := 0\nNFLUIDS = 1\nFARGO_OPT += -DNFLUIDS=${NFLUIDS}\n"
        "MONITOR_SCALAR = MASS | MOM_X | TORQ\n"
        "FARGO_OPT += -DSTOCKHOLM\nFARGO_OPT +=  -DX\nFARGO_OPT +=  -DY\nFARGO_OPT +=  -DISOTHERMAL\n"
        "FARGO_OPT +=  -DCYLINDRICAL\nFARGO_OPT += -DLEGACY\nFARGO_OPT += -DPOTENTIAL\nFARGO_OPT += -DVISCOSITY\n"
        + opt_extra +
        "ifeq (${GPU}, 1)\nFARGO_OPT += -DBLOCK_X=16\nendif\n"))
    return os.path.join(root, "setups", "disk")


def test_load_setup_matches_named_config(tmp_path):
    """The fargo-style tree above is config_fargo2d (Nz ignored without -DZ,
    default cfl, damping and gamma from the standard defaults)."""
    s = pf.load_setup(_setup_tree(str(tmp_path)))
    assert s.precision == "fp64" and s.planet_names == ["Jove"]
    ref = config_fargo2d()
    assert s.config == ref.replace(xmin=-math.pi, xmax=math.pi)
    assert s.config.xmin == -math.pi and s.config.nz == 1


def test_load_setup_overrides(tmp_path):
    d = _setup_tree(str(tmp_path), par_extra="SemiMajorAxis 1.5\nPlanetMass 3e-4\nOrbitalRadius 2.0\n",
                    opt_extra="FARGO_OPT += -DFLOAT\n",
                    planets="Jove 1.0 0.001 0.0 YES NO\nSat 3.0 1e-4 0.0 no yes\n")
    s = pf.load_setup(os.path.join(d, "disk.par"), redefine="Nx:512,frame:fixed", seed=7)
    c = s.config
    assert s.precision == "fp32" and c.nx == 512 and c.frame == "F" and c.seed == 7
    assert c.planets == [Planet(3.0, 3e-4, True, False), Planet(6.0, 1e-4, False, True)]
    assert c.noise == 1e-4 and c.log_spacing and c.stockholm and c.nu == 1e-5


@pytest.mark.parametrize("par_extra,opt_extra,planets,exc", [
    ("", "FARGO_OPT += -DMHD\n", None, NotImplementedError),
    ("", "FARGO_OPT += -DSTANDARD\n", None, NotImplementedError),
    ("", "FARGO_OPT += -DADIABATIC\n", None, NotImplementedError),
    ("", "FARGO_OPT += -DALPHAVISCOSITY\n", None, NotImplementedError),
    ("ExcludeHill yes\n", "", None, NotImplementedError),
    ("RocheSmoothing 0.1\n", "", None, ValueError),
    ("Spacing Fixed\n", "", None, NotImplementedError),
    ("", "", "Jove 1.0 0.001 0.1 NO NO\n", NotImplementedError),
    ("AspectRatio abc\n", "", None, ValueError),
])
def test_load_setup_refuses(tmp_path, par_extra, opt_extra, planets, exc):
    # the extra lines come first so that they are the definitions that count
    d = _setup_tree(str(tmp_path), opt_extra=opt_extra,
                    **({"planets": planets} if planets else {}))
    par = os.path.join(d, "disk.par")
    with open(par) as fh:
        body = fh.read()
    _write(par, par_extra + body)
    with pytest.raises(exc):
        pf.load_setup(d)


def test_option_rules():
    base = {"X": None, "Y": None, "CYLINDRICAL": None, "ISOTHERMAL": None, "POTENTIAL": None}
    pf.config_from_params({"NX": "8", "NY": "8"}, base)
    for drop in ("X", "CYLINDRICAL", "ISOTHERMAL", "POTENTIAL"):
        with pytest.raises(NotImplementedError):
            pf.config_from_params({}, {k: v for k, v in base.items() if k != drop})
    with pytest.raises(NotImplementedError):
        pf.config_from_params({}, dict(base, NFLUIDS="3"))
    with pytest.raises(NotImplementedError):
        pf.config_from_params({}, dict(base, SPHERICAL=None))
    c, _ = pf.config_from_params({"INVSTOKES1": "10", "INVSTOKES2": "1", "EPSILON": "0.5"},
                                 dict(base, NFLUIDS="3", DRAGFORCE=None, STOKESNUMBER=None))
    assert c.nfluids == 3 and c.invstokes == (10.0, 1.0) and c.epsilon == 0.5 and c.nu == 0.0
    with pytest.raises(ValueError):
        pf.config_from_params({"INVSTOKES1": "10"}, dict(base, NFLUIDS="3", DRAGFORCE=None, STOKESNUMBER=None))


def _named():
    yield "fargo2d", config_fargo2d(seed=3)
    yield "multifluid", config_multifluid(dust_diffusion=True)
    yield "adiabatic", config_adiabatic2d()
    yield "p3disof", config_p3disof()
    for i, c in enumerate(config_batched(6, seed=5)):
        yield "batched%d" % i, c


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_round_trip(tmp_path, precision):
    for name, cfg in _named():
        par, opt, cfgp = pf.write_setup(cfg, str(tmp_path / name), name, precision)
        assert all(os.path.exists(p) for p in (par, opt, cfgp))
        s = pf.load_setup(par, seed=cfg.seed)
        want = cfg
        if cfg.nfluids > 1 and cfg.epsilon == 0.0:
            want = cfg.replace(epsilon=0.01 / (cfg.nfluids - 1))
        assert s.precision == precision
        diff = {f.name for f in dataclasses.fields(want) if getattr(want, f.name) != getattr(s.config, f.name)}
        assert not diff, (name, diff)


@pytest.mark.skipif(not os.environ.get("FARGO_REFERENCE"), reason="FARGO_REFERENCE (a FARGO3D tree) not set")
def test_reference_setups():
    """The FARGO3D tree's own setups: the three this library integrates load
    with their stock values; the others stop on an option outside the hydro
    step."""
    root = os.environ["FARGO_REFERENCE"]
    s = pf.load_setup(os.path.join(root, "setups", "fargo"))
    c = s.config
    assert (c.nx, c.ny, c.frame, c.omegaframe, c.indirect_term, c.log_spacing) == (384, 128, "G", 1.0005, True, False)
    assert c.planets == [Planet(1.0, 0.001, False, False)] and c.nu == 1e-5 and c.stockholm
    s = pf.load_setup(os.path.join(root, "setups", "fargo_multifluid"))
    c = s.config
    assert c.nfluids == 4 and c.invstokes == (10.0, 1.0, 0.1) and c.epsilon == 1.0 and c.dust_diffusion
    s = pf.load_setup(os.path.join(root, "setups", "p3disof"))
    c = s.config
    assert c.is3d and c.spherical and (c.nx, c.ny, c.nz) == (100, 80, 40) and c.flaringindex == 0.5
    assert c.planets[0].mass == 1e-5
    for name in ("mri", "otvortex", "sod1d", "fargo_nu", "binary"):
        if os.path.isdir(os.path.join(root, "setups", name)):
            with pytest.raises(NotImplementedError):
                pf.load_setup(os.path.join(root, "setups", name))
