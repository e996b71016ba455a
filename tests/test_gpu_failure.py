"""Failure detection of the bounded waits, tested without a GPU fault.

The azimuthal sweep stages its ring rows with the bulk-copy engine and waits
for them on an mbarrier a bounded number of polls.  Setting the limit to
"no polls" makes every CTA give up at once: the copies still land (they are
valid), the CTA waits for them, writes nothing, flags the disk and returns,
and the host reads the flag with the next step's CFL minimum.
"""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_staged_load_timeout_is_reported(precision):
    from fargo3d_b200 import Disk, FargoError, config_fargo2d
    from fargo3d_b200 import _abi
    L = _abi.lib()
    cfg = config_fargo2d(64, 32, seed=51)
    d = Disk(cfg, precision)
    d.load_initial_state()
    d.step()
    _abi.check(L.fb_disk_set_wait_limit(d._h, -1))
    d.step()                         # the sweep gives up and flags the disk
    with pytest.raises(FargoError) as e:
        d.step()                     # reported with the next CFL readback
    assert "did not complete in time" in str(e.value)
    d.close()
    # a fresh disk with the default limit runs normally on the same device
    d2 = Disk(cfg, precision)
    d2.load_initial_state()
    dts = d2.run(3)
    assert all(np.isfinite(dts)) and min(dts) > 0
    d2.close()
