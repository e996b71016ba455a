"""Batched disks (fb_batch_*): every member against the oracle, each result
the same alone and in the mix, and a failing member frozen while the others
continue.  The batched path runs the step's scalar work (planets, frame) on
the device with CUDA's libm, so FP64 agreement with the oracle is to
round-off (1e-10 relative), not bit for bit; FP32 meets the 1e-5 L1 bar."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))


def small_mix():
    from fargo3d_b200 import config_fargo2d, Planet
    return [
        config_fargo2d(32, 16, seed=31),
        config_fargo2d(64, 24, seed=32).replace(alpha_visc=True, alpha=2e-3, nu=0.0, sigmaslope=1.2,
                                                aspectratio=0.04, planets=[Planet(1.0, 2e-3)]),
        config_fargo2d(48, 20, seed=33).replace(aspectratio=0.07, sigmaslope=0.0, planets=[Planet(1.0, 3e-5)]),
        config_fargo2d(128, 64, seed=34).replace(alpha_visc=True, alpha=1e-4, nu=0.0),
    ]


def rel_linf(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def oracle_run(cfg, n):
    import pyoracle
    pyoracle.build()
    out, dts, sc = pyoracle.run(cfg, n, "oracle")
    return out[0], dts


@pytest.mark.gpu
def test_batch_fp64_members_match_oracle():
    from fargo3d_b200 import Batch
    cfgs = small_mix()
    b = Batch(cfgs, "fp64")
    b.load_initial_states()
    b.run(12)
    for i, c in enumerate(cfgs):
        st = b.state(i)
        ref, dts = oracle_run(c, 12)
        sc, status = b.scalars(i)
        assert status == 0
        assert abs(sc[0] - dts.sum()) <= 1e-10 * dts.sum()
        for k in ("rho", "vx", "vy"):
            assert rel_linf(st[k], ref[k]) <= 1e-10, (i, k, rel_linf(st[k], ref[k]))
    b.close()


@pytest.mark.gpu
def test_batch_fp32_members_match_oracle():
    from fargo3d_b200 import Batch
    cfgs = small_mix()
    b = Batch(cfgs, "fp32")
    b.load_initial_states()
    b.run(12)
    for i, c in enumerate(cfgs):
        st = b.state(i)
        ref, _ = oracle_run(c, 12)
        l1 = np.sum(np.abs(st["rho"] - ref["rho"])) / np.sum(np.abs(ref["rho"]))
        assert l1 <= 1e-5, (i, l1)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_member_alone_equals_in_mix(precision):
    from fargo3d_b200 import Batch
    cfgs = small_mix()
    mix = Batch(cfgs, precision)
    mix.load_initial_states()
    mix.run(10)
    for i in (1, 3):
        alone = Batch([cfgs[i]], precision)
        alone.load_initial_states()
        alone.run(10)
        a, m = alone.state(0), mix.state(i)
        for k in ("rho", "vx", "vy"):
            assert np.array_equal(a[k], m[k]), (i, k)
        alone.close()
    mix.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_concurrent_chains_give_the_same_bits(precision):
    """The disks stepped as 1, 3 or 8 concurrent chains (streams), through
    the captured graph (10 steps) and the eager remainder (3 steps): every
    member's state and scalars are the same bits."""
    from fargo3d_b200 import Batch
    cfgs = small_mix()
    out = {}
    for k in (1, 3, 8):
        b = Batch(cfgs, precision)
        b.load_initial_states()
        b.set_chains(k)
        b.run(13)
        b.sync()
        out[k] = [(b.state(i), list(b.scalars(i)[0])) for i in range(len(cfgs))]
        b.close()
    for k in (3, 8):
        for i in range(len(cfgs)):
            (a, sa), (r, sr) = out[k][i], out[1][i]
            assert sa == sr, (k, i)
            for key in ("rho", "vx", "vy"):
                assert np.array_equal(a[key], r[key]), (k, i, key)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_state_transfers_of_all_members(precision):
    """fb_batch_set_states / fb_batch_get_states move every member's state in
    one call and give the same bits as the per-member calls, into page-locked
    and ordinary buffers; a NULL entry leaves that member as it is."""
    import torch
    from fargo3d_b200 import Batch, initial_state
    cfgs = small_mix()
    sts = [initial_state(c) for c in cfgs]
    a, b = Batch(cfgs, precision), Batch(cfgs, precision)
    for i, st in enumerate(sts):
        a.set_state(i, *st)
    b.set_states([tuple(torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy() if x is not None else None
                        for x in st) for st in sts])
    a.initialize()
    b.initialize()
    a.run(4)
    b.run(4)
    outs = [{k: torch.empty(c.shape, dtype=torch.float64).pin_memory().numpy() for k in ("rho", "vx", "vy")}
            for c in cfgs]
    got = b.states(out=outs)
    for i in range(len(cfgs)):
        want = a.state(i)
        assert np.shares_memory(got[i]["rho"], outs[i]["rho"])
        for k in ("rho", "vx", "vy"):
            assert np.array_equal(got[i][k], want[k]), (i, k)
    # a NULL entry: member 1 keeps its state
    before = b.state(1)
    b.set_states([sts[0], None, sts[2], sts[3]])
    after = b.state(1)
    for k in ("rho", "vx", "vy"):
        assert np.array_equal(before[k], after[k]), k
    a.close()
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("pinned", [False, True])
def test_batch_transfers_through_one_host_block(pinned):
    """Members whose fields lie back to back in one host buffer, in the
    order of the call, cross in merged copies (more segments than one
    staging chunk holds, so the merging restarts at chunk boundaries); the
    state equals the one of per-member calls, and the fields read back into
    one block equal the per-member reads."""
    import torch
    from fargo3d_b200 import Batch, initial_state
    cfgs = [c.replace(seed=c.seed + 100 * k) for k in range(5) for c in small_mix()]
    sts = [initial_state(c) for c in cfgs]
    a, b = Batch(cfgs, "fp32"), Batch(cfgs, "fp32")
    for i, st in enumerate(sts):
        a.set_state(i, *st)
    n = [int(np.prod(c.shape)) for c in cfgs]
    blk = torch.empty(4 * sum(n), dtype=torch.float64)
    blk = blk.pin_memory() if pinned else blk
    blk = blk.numpy()
    views, o = [], 0
    for i, st in enumerate(sts):
        v = []
        for q in (0, 1, 2, 4):                  # rho, vx, vy, cs: the upload order of a 2D disk
            x = blk[o:o + n[i]].reshape(cfgs[i].shape)
            x[...] = st[q]
            v.append(x)
            o += n[i]
        views.append((v[0], v[1], v[2], None, v[3]))
    b.set_states(views)
    a.initialize()
    b.initialize()
    a.run(3)
    b.run(3)
    out = torch.empty(3 * sum(n), dtype=torch.float64)
    out = (out.pin_memory() if pinned else out).numpy()
    outs, o = [], 0
    for i, c in enumerate(cfgs):
        d = {}
        for k in ("rho", "vx", "vy"):
            d[k] = out[o:o + n[i]].reshape(c.shape)
            o += n[i]
        outs.append(d)
    got = b.states(out=outs)
    for i in range(len(cfgs)):
        want = a.state(i)
        for k in ("rho", "vx", "vy"):
            assert np.shares_memory(got[i][k], out)
            assert np.array_equal(got[i][k], want[k]), (i, k)
    a.close()
    b.close()


@pytest.mark.gpu
def test_batch_creation_refuses_a_bad_member():
    """Members are set up on several host threads; one member the library
    refuses fails the whole creation with that member's error text, and a
    batch created afterwards works."""
    from fargo3d_b200 import Batch, _abi
    cfgs = small_mix() * 3
    bad = cfgs[:5] + [cfgs[5].replace(planets=[], frame="G")] + cfgs[6:]
    with pytest.raises(_abi.FargoError, match="rotating frame needs a planet"):
        Batch(bad, "fp32")
    with pytest.raises(_abi.FargoError, match="one-disk path"):
        Batch(cfgs[:3] + [cfgs[3].replace(adiabatic=True, alpha_visc=True, alpha=1e-3, nu=0.0)], "fp64")
    b = Batch(cfgs, "fp32")
    b.load_initial_states()
    b.initialize()
    b.run(3)
    b.sync()
    for i in range(len(cfgs)):
        assert b.scalars(i)[1] == 0
    b.close()


@pytest.mark.gpu
def test_batch_failing_member_is_frozen_others_continue():
    """Fault injection on the host: one member starts with a NaN density.
    It is frozen with FB_ERR_NONFINITE; the others match their solo runs."""
    from fargo3d_b200 import Batch, initial_state
    cfgs = small_mix()
    b = Batch(cfgs, "fp64")
    for i, c in enumerate(cfgs):
        st = list(initial_state(c))
        if i == 2:
            st[0] = st[0].copy()
            st[0][0, 10, 7] = np.nan
        b.set_state(i, *st)
    b.initialize()
    b.run(8)
    _, status = b.scalars(2)
    assert status == -4
    for i in (0, 1, 3):
        _, s = b.scalars(i)
        assert s == 0
        solo = Batch([cfgs[i]], "fp64")
        solo.load_initial_states()
        solo.run(8)
        assert np.array_equal(solo.state(0)["rho"], b.state(i)["rho"])
        solo.close()
    b.close()


@pytest.mark.gpu
def test_fp32_accuracy_after_1000_steps():
    """North-star accuracy bar of the FP32 path: relative L1 density error
    against the FP64 oracle after 1000 hydro steps <= 1e-5 (batched FP32 with
    fast single-precision division, FP64 shift / means / planets)."""
    from fargo3d_b200 import Batch, config_fargo2d, Planet
    cfgs = [config_fargo2d(128, 64, seed=41),
            config_fargo2d(128, 64, seed=42).replace(alpha_visc=True, alpha=1e-3, nu=0.0,
                                                     planets=[Planet(1.0, 1e-3)])]
    b = Batch(cfgs, "fp32")
    b.load_initial_states()
    b.run(1000)
    for i, c in enumerate(cfgs):
        ref, _ = oracle_run(c, 1000)
        st = b.state(i)
        l1 = np.sum(np.abs(st["rho"] - ref["rho"])) / np.sum(np.abs(ref["rho"]))
        assert l1 <= 1e-5, (i, l1)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_multifluid_drag_matches_oracle(precision):
    """Gas + 4 dust species with implicit drag, two disks in one batch: every
    fluid of every member against the FP64 oracle."""
    import pyoracle
    from fargo3d_b200 import Batch, config_multifluid
    cfgs = [config_multifluid(64, 32, seed=81), config_multifluid(128, 48, seed=82)]
    b = Batch(cfgs, precision)
    b.load_initial_states()
    b.run(12)
    pyoracle.build()
    for i, c in enumerate(cfgs):
        out, dts, _ = pyoracle.run(c, 12, "oracle")
        for f in range(c.nfluids):
            st = b.state(i, fluid=f)
            if precision == "fp64":
                for k in ("rho", "vx", "vy"):
                    assert rel_linf(st[k], out[f][k]) <= 1e-10, (i, f, k, rel_linf(st[k], out[f][k]))
            else:
                l1 = np.sum(np.abs(st["rho"] - out[f]["rho"])) / np.sum(np.abs(out[f]["rho"]))
                assert l1 <= 1e-5, (i, f, l1)
    b.close()
