"""Serving loop (fb_server_*) and slotted batches: requests that arrive
while others run join them, each result is the same alone and in the mix
(bit for bit: every disk's tiles compute the same arithmetic whatever else
shares the launch), a disk stops exactly at its end time, and the HBM budget
bounds what is admitted."""
import os
import sys
import time

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))


def _cfgs():
    from fargo3d_b200 import Planet, config_fargo2d
    return [
        config_fargo2d(128, 64, seed=51),
        config_fargo2d(256, 64, seed=52).replace(alpha_visc=True, alpha=1e-3, nu=0.0, planets=[Planet(1.0, 2e-4)]),
        config_fargo2d(128, 128, seed=53).replace(aspectratio=0.07),
        config_fargo2d(512, 128, seed=54).replace(sigmaslope=1.0),
    ]


@pytest.mark.gpu
def test_request_alone_equals_in_mix_and_matches_oracle():
    import pyoracle
    from fargo3d_b200 import Server
    cfgs = _cfgs()
    t_end = 1.5
    s = Server("fp32", max_disks=8, chunk_steps=10)
    a = s.submit(cfgs[0], t_end)
    assert s.wait(a, 300) == 2
    alone, info_alone = s.fetch(a)
    s.close()

    s = Server("fp32", max_disks=8, chunk_steps=10)
    first = [s.submit(cfgs[1], 3.0), s.submit(cfgs[2], 2.0)]
    t0 = time.time()
    while s.status(first[0]) != 1 and time.time() - t0 < 60:   # wait until it runs
        time.sleep(0.001)
    a = s.submit(cfgs[0], t_end)          # arrives while others are on the GPU
    late = s.submit(cfgs[3], 1.0)
    ids = first + [a, late]
    for r in ids:
        assert s.wait(r, 300) == 2
    mixed, info = s.fetch(a)
    for r in first + [late]:
        s.fetch(r)
    s.close()
    for k in ("rho", "vx", "vy"):
        assert np.array_equal(alone[k], mixed[k]), k
    assert info["steps"] == info_alone["steps"]
    assert abs(info["time"] - t_end) <= 1e-12 * t_end          # last step lands on the end time
    # against the FP64 oracle over the same steps (the DT interval = t_end clip)
    pyoracle.build()
    out, dts, _ = pyoracle.run(cfgs[0], int(info["steps"]), "oracle", dt_interval=t_end)
    assert abs(dts.sum() - t_end) <= 1e-12 * t_end
    ref = out[0]["rho"]
    l1 = np.sum(np.abs(mixed["rho"] - ref)) / np.sum(np.abs(ref))
    assert l1 <= 1e-5, l1


@pytest.mark.gpu
def test_hbm_budget_bounds_admission():
    from fargo3d_b200 import Server, config_fargo2d
    from fargo3d_b200._abi import FargoError, params_bytes
    cfgs = [config_fargo2d(256, 64, seed=60 + i) for i in range(3)]
    b = params_bytes(cfgs[0], "fp32")
    s = Server("fp32", hbm_budget=2 * b + b // 2, max_disks=8, chunk_steps=5)
    ids = [s.submit(c, 2.0) for c in cfgs]
    big = s.submit(config_fargo2d(1024, 512, seed=69), 1.0)   # can never fit
    seen = 0.0
    while s.stats()["running"] + s.stats()["queued"] > 0:
        st = s.stats()
        seen = max(seen, st["bytes_reserved"])
        time.sleep(0.0005)
    for r in ids:
        assert s.wait(r, 300) == 2
    infos = [s.fetch(r)[1] for r in ids]
    assert seen <= 2 * b + b // 2
    # the third request waited for one of the first two to leave
    assert infos[2]["admitted"] >= min(infos[0]["finished"], infos[1]["finished"])
    assert s.wait(big, 60) == 3
    with pytest.raises(FargoError) as e:
        s.fetch(big)
    assert "FB_ERR_TOO_LARGE" in str(e.value)
    s.close()


@pytest.mark.gpu
def test_params_bytes_bounds_actual_allocation():
    import ctypes as C
    from fargo3d_b200 import Disk, config_fargo2d, config_p3disof
    from fargo3d_b200._abi import lib, params_bytes
    for cfg in (config_fargo2d(384, 128), config_p3disof(64, 32, 16)):
        for prec in ("fp64", "fp32"):
            d = Disk(cfg, prec)
            got = C.c_size_t()
            assert lib().fb_disk_bytes(d._h, C.byref(got)) == 0
            est = params_bytes(cfg, prec)
            assert got.value <= est <= 1.1 * got.value, (cfg.nx, prec, got.value, est)
            d.close()
