"""FARGO3D output files: merged .dat layout (active cells, x fastest, raw
doubles), write -> read round trip, planet files (output.c)."""
import os

import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cyl2d", "sph3d", "mf"])
def test_dat_layout_and_round_trip(tmp_path, which):
    from fargo3d_b200 import Disk, config_fargo2d, config_multifluid, config_p3disof, initial_state
    cfg = {"cyl2d": config_fargo2d(64, 32, seed=3), "sph3d": config_p3disof(32, 16, 8, seed=4),
           "mf": config_multifluid(32, 16, nfluids=3, seed=5)}[which]
    d = Disk(cfg, "fp64")
    for f in range(cfg.nfluids):
        d.set_state(*initial_state(cfg, f), fluid=f)
    d.initialize()
    d.run(3)
    out = str(tmp_path)
    d.write_dat(out, 7)
    nz = cfg.nz if cfg.is3d else 1
    g = 3
    for f in range(cfg.nfluids):
        st = d.state(f)
        name = Disk.fluid_name(f)
        for k in ("rho", "vx", "vy") + (("vz",) if cfg.is3d else ()):
            field = {"rho": "dens"}.get(k, k)
            a = np.fromfile(os.path.join(out, "%s%s7.dat" % (name, field)), dtype=np.float64)
            assert a.size == cfg.nx * cfg.ny * nz
            active = st[k][g:g + nz, g:g + cfg.ny, :] if cfg.is3d else st[k][0, g:g + cfg.ny, :]
            assert np.array_equal(a.reshape(active.shape), active), (f, k)
        assert os.path.exists(os.path.join(out, "%senergy7.dat" % name))
    # read back into a disk that ran further: the active cells return
    want = [d.state(f) for f in range(cfg.nfluids)]
    d.run(2)
    d.read_dat(out, 7)
    for f in range(cfg.nfluids):
        st = d.state(f)
        sl = (slice(g, g + nz), slice(g, g + cfg.ny)) if cfg.is3d else (0, slice(g, g + cfg.ny))
        for k in ("rho", "vx", "vy"):
            assert np.array_equal(st[k][sl], want[f][k][sl]), (f, k)
    d.close()


@pytest.mark.gpu
def test_planet_file_lines(tmp_path):
    from fargo3d_b200 import Disk, Planet, config_fargo2d
    cfg = config_fargo2d(32, 16, seed=6).replace(planets=[Planet(1.0, 1e-3), Planet(1.5, 2e-4)])
    d = Disk(cfg, "fp64")
    d.load_initial_state()
    out = str(tmp_path)
    for n in range(3):
        d.run(2)
        d.write_dat(out, n)
    sc = d.scalars()
    for k in range(2):
        rows = [ln.split("\t") for ln in open(os.path.join(out, "planet%d.dat" % k)).read().splitlines()]
        assert [int(r[0]) for r in rows] == [0, 1, 2]
        assert all(len(r) == 10 for r in rows)
    last = [float(v) for v in open(os.path.join(out, "planet0.dat")).read().splitlines()[-1].split("\t")]
    assert last[1] == sc[3] and last[2] == sc[4] and last[8] == sc[0] and last[9] == sc[1]
    d.close()


@pytest.mark.gpu
def test_fp32_state_transfer_rounds_like_a_host_cast():
    """FP32 disks take the caller's doubles over the bus and round them on the
    device: the stored values are the host's (float) casts, subnormals and
    ties to even included, across staging-chunk boundaries (a disk of more
    than 4 Mi values), into caller-supplied page-locked buffers too."""
    import torch
    from fargo3d_b200 import Disk, config_fargo2d
    cfg = config_fargo2d(2048, 2048, seed=5)
    n = int(np.prod(cfg.shape))
    assert n > 4 << 20
    rng = np.random.default_rng(7)
    vals = [rng.standard_normal(n) * 10.0 ** rng.integers(-46, 37, n) for _ in range(4)]
    vals[0][:8] = [0.0, -0.0, 1e-40, -3e-42, 1.5e-45, 3.0e38, 2.9e-39, 1.0 + 2.0 ** -24]
    vals[1][n - 3:] = [1.0 + 3 * 2.0 ** -24, -1e-44, 7.0]
    rho, vx, vy, cs = [v.reshape(cfg.shape) for v in vals]
    d = Disk(cfg, "fp32")
    d.set_state(rho, vx, vy, None, cs)
    got = d.state()
    for k, v in (("rho", rho), ("vy", vy)):
        assert np.array_equal(got[k], v.astype(np.float32).astype(np.float64)), k
    # vx is stored less its ring's background (the FP64 ring mean of the
    # first vx given): the float is the deviation's cast, read back plus it
    bg = d.background()[:, :, None]
    assert bg.shape[:2] == cfg.shape[:2]
    assert np.allclose(bg[0, :, 0], vx.mean(axis=2)[0], rtol=1e-12, atol=0.0)
    assert np.array_equal(got["vx"], (vx - bg).astype(np.float32).astype(np.float64) + bg)
    assert got["vz"].shape == cfg.shape and not got["vz"].any()
    out = {k: torch.empty(cfg.shape, dtype=torch.float64).pin_memory().numpy() for k in ("rho", "vx", "vy")}
    got2 = d.state(out=out)
    for k in out:
        assert np.shares_memory(got2[k], out[k])
        assert np.array_equal(got2[k], got[k]), k
    with pytest.raises(ValueError):
        d.state(out={"rho": np.empty(10)})
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cyl2d", "sph3d"])
def test_dat_files_equal_the_references_own_writer(which, tmp_path):
    """The same initial state advanced 10 FP64 steps by the library and by the
    reference's own C sources, each written by its own writer: the library's
    fb_disk_write_dat / fb_disk_write_planets and the reference's WriteMerging
    (output.c:283-315) / WritePlanetSystemFile (output.c:181-196), compiled
    from the reference tree into oracle/_ref.  The merged field files are
    byte-identical, the planet lines too; the library reads the reference's
    files back into the same state (the restart path)."""
    import pyoracle
    from fargo3d_b200 import Disk, config_fargo2d, config_p3disof, initial_state
    cfg = config_fargo2d(48, 20, seed=91) if which == "cyl2d" else config_p3disof(16, 12, 6, seed=92)
    init = initial_state(cfg)
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    ours.mkdir()
    theirs.mkdir()
    d = Disk(cfg, "fp64")
    d.set_state(*init)
    d.initialize()
    d.run(10)
    d.write_dat(str(ours), 3)
    r = pyoracle.Disk(cfg, "ref")
    r.set_state(*init)
    r.initialize()
    for _ in range(10):
        r.step()
    r.write_outputs(str(theirs), 3)
    names = ["gasdens3.dat", "gasenergy3.dat", "gasvx3.dat", "gasvy3.dat"] + (["gasvz3.dat"] if cfg.is3d else [])
    for nme in names:
        a, b = (ours / nme).read_bytes(), (theirs / nme).read_bytes()
        assert len(a) == 8 * cfg.active_cells and a == b, nme
    assert (ours / "planet0.dat").read_text() == (theirs / "planet0.dat").read_text()
    # the restart path: the reference's files into a fresh disk
    d2 = Disk(cfg, "fp64")
    d2.set_state(*init)
    d2.read_dat(str(theirs), 3)
    got, want = d2.state(), r.state()
    sl = (slice(3, -3) if cfg.is3d else slice(None), slice(3, -3), slice(None))
    for k in ("rho", "vx", "vy") + (("vz",) if cfg.is3d else ()):
        assert np.array_equal(got[k][sl], want[k][sl]), k
    d2.close()
    d.close()
    r.close()
