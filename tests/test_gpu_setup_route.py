"""The setup-directory route of the drop-in: no edit of main.c.

fargo3d_b200/integration/setup holds algogas.c, cfl.c, compute_vmed.c,
dust_diffusion_main.c and fresh.c; a FARGO3D setup directory that carries them
replaces the stock files of src/ (VPATH, src/makefile:306), and the stock DT
loop of main.c:361-448 then runs its hydro step on the B200 library.  Here
the reference's own build is linked the same way (oracle/ref/Makefile target
`shadow`), its step loop left as it is, and must reproduce the unmodified
reference bit for bit: fields, time steps, time, frame and planets, the
reference's own output writers after the steps (INPUT copies the state back
from the device), and a host write of the state between steps (OUTPUT marks
it for upload before the next step)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))


def configs():
    from fargo3d_b200 import Planet, config_adiabatic2d, config_fargo2d, config_multifluid, config_p3disof
    from fargo3d_b200.parfile import load_setup
    return {
        "cyl2d": config_fargo2d(64, 24, seed=111).replace(planets=[Planet(1.0, 1e-3), Planet(1.4, 3e-4)]),
        "sph3d": config_p3disof(24, 12, 6, seed=112),
        "mf5": config_multifluid(48, 20, seed=113),
        "cyl2d_ad": config_adiabatic2d(48, 20, seed=114),
        "mf5_dd": config_multifluid(48, 20, seed=115, dust_diffusion=True),
        # the fargo_multifluid disk as its setup files describe it (4 fluids, DUSTDIFFUSION)
        "mf4_par": load_setup(os.path.join(HERE, "golden", "setups", "mf4_par"), redefine="Nx:48,Ny:20",
                              seed=116).config,
    }


def _built(kind, cfg):
    import pyoracle
    path = os.path.join(pyoracle.HERE, "_ref", "libfargo_ref_%s_%s.so" % (kind, pyoracle.ref_variant(cfg)))
    if not os.path.exists(path):
        pytest.fail("setup-route build missing: run __graft_entry__.build() where the reference tree is present")


def _open(cfg, kind, init):
    import pyoracle
    d = pyoracle.Disk(cfg, kind)
    for f in range(cfg.nfluids):
        d.set_state(*init[f], fluid=f)
    d.initialize()
    return d


def _same(a, b, cfg):
    for f in range(cfg.nfluids):
        sa, sb = a.state(f), b.state(f)
        for k in ("rho", "vx", "vy") + (("vz",) if cfg.is3d else ()):
            assert np.array_equal(sa[k], sb[k]), (f, k, np.max(np.abs(sa[k] - sb[k])))
        assert np.array_equal(a.energy(f), b.energy(f)), (f, "energy")
    assert np.array_equal(a.scalars()[:7], b.scalars()[:7])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cyl2d", "sph3d", "mf5", "cyl2d_ad", "mf5_dd", "mf4_par"])
def test_stock_step_loop_on_the_b200(name):
    from fargo3d_b200 import initial_state
    cfg = configs()[name]
    _built("shadow", cfg)
    init = [initial_state(cfg, f) for f in range(cfg.nfluids)]
    dti = 0.0314159
    ours, ref = _open(cfg, "shadow", init), _open(cfg, "ref", init)
    for _ in range(4):
        assert ours.step(dti) == ref.step(dti)   # DT clipping included
    _same(ours, ref, cfg)
    ours.close()
    ref.close()


@pytest.mark.gpu
def test_outputs_and_host_writes_follow_the_freshness_protocol(tmp_path):
    from fargo3d_b200 import initial_state
    cfg = configs()["cyl2d"]
    _built("shadow", cfg)
    init = [initial_state(cfg, 0)]
    ours, ref = _open(cfg, "shadow", init), _open(cfg, "ref", init)
    for _ in range(3):
        ours.step()
        ref.step()
    # the reference's writers read the Fields after INPUT: the device's state
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    ours.write_outputs(str(a), 1)
    ref.write_outputs(str(b), 1)
    for nme in ("gasdens1.dat", "gasvx1.dat", "gasvy1.dat", "gasenergy1.dat", "planet0.dat"):
        assert (a / nme).read_bytes() == (b / nme).read_bytes(), nme
    # host code rewrites the state between steps (a restart): uploaded before the next step
    st = ref.state(0)
    new = (st["rho"] * 1.01, st["vx"], st["vy"], None, ref.energy(0))
    ours.set_state(*new, fluid=0)
    ref.set_state(*new, fluid=0)
    for _ in range(3):
        assert ours.step() == ref.step()
    _same(ours, ref, cfg)
    ours.close()
    ref.close()
