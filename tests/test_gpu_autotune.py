"""Tile autotuner: every tile choice computes the same step (FP64: bit for
bit), the tuner returns valid choices, and the table round-trips."""
import json
import os

import numpy as np
import pytest


def _mix():
    from fargo3d_b200 import Planet, config_fargo2d
    return [config_fargo2d(128, 64, seed=71),
            config_fargo2d(256, 64, seed=72).replace(alpha_visc=True, alpha=1e-3, nu=0.0, planets=[Planet(1.0, 1e-4)])]


@pytest.mark.gpu
def test_every_tile_choice_gives_the_same_fp64_step():
    from fargo3d_b200 import Batch, FargoError
    from fargo3d_b200.autotune import NS_CANDIDATES, cx_candidates
    cfgs = _mix()
    b = Batch(cfgs[:1], "fp64", tiles=None)
    with pytest.raises(FargoError):      # 32 rings of 128 cells per CTA: 360 KB of shared memory
        b.set_tiles(0, 16, 8)
    b.close()
    ref = Batch(cfgs, "fp64", tiles=None)
    ref.load_initial_states()
    ref.run(6)
    want = [ref.state(i) for i in range(len(cfgs))]
    ref.close()
    for cx in (1, 2, 4, 8, 16):
        for ns in NS_CANDIDATES:
            b = Batch(cfgs, "fp64", tiles=None)
            for i, c in enumerate(cfgs):
                if cx in cx_candidates(c.nx, "fp64"):
                    b.set_tiles(i, cx, ns)
            b.load_initial_states()
            b.run(6)
            for i in range(len(cfgs)):
                got = b.state(i)
                for k in ("rho", "vx", "vy"):
                    assert np.array_equal(got[k], want[i][k]), (cx, ns, i, k)
            b.close()


@pytest.mark.gpu
def test_tuner_returns_valid_choices(tmp_path):
    from fargo3d_b200 import config_fargo2d
    from fargo3d_b200.autotune import NS_CANDIDATES, TileTable, cx_candidates, shape_key, tune_shape
    cfg = config_fargo2d(256, 128)
    e = tune_shape(cfg, "fp32", min_cells=1e6, reps=2)
    assert e["sweep_x_cells"] in cx_candidates(256, "fp32")
    assert e["col_segment"] in NS_CANDIDATES
    assert set(e["ms"]["sweep_x"]) == {str(c) for c in cx_candidates(256, "fp32")}
    assert all(v > 0 for v in e["ms"]["sweep_cols"].values())
    t = TileTable({shape_key(cfg, "fp32"): e})
    p = os.path.join(str(tmp_path), "t.json")
    t.save(p)
    assert TileTable.load(p).get(cfg, "fp32") == (e["sweep_x_cells"], e["col_segment"])
    with open(p) as fh:
        assert shape_key(cfg, "fp32") in json.load(fh)
