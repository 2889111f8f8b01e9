"""Failure reporting and zero-copy views, on the GPU.

A NaN injected into the host state before upload makes the next fn_sync
return FN_ERR_NONFINITE (the counter in fn_stats says how many bead-steps
saw it) instead of running on silently; the device views equal the
downloaded state in internal order."""
import numpy as np
import pytest

from fibrenet_b200 import generate as g

pytestmark = pytest.mark.gpu


def net():
    return g.plain_network(seed=61, fibres=20, beads=12, box=(16.0, 16.0, 6.0), z_range=(1.0, 5.0))


def test_nan_in_host_state_is_reported():
    from fibrenet_b200.native import ERRORS, NativeError, Simulation
    m = net()
    m.img = np.array(m.img, dtype=np.float64)
    m.img[17, 1] = np.nan
    s = Simulation(m, list_capacity=64)
    s.step(5)
    with pytest.raises(NativeError, match="non-finite") as e:
        s.sync()
    assert ERRORS.get(e.value.code, e.value.code) == ERRORS.get(6, 6)
    assert s.stats()["nonfinite"] > 0
    s.close()


def test_clean_run_syncs():
    from fibrenet_b200.native import Simulation
    with Simulation(net(), list_capacity=64) as s:
        s.step(20)
        s.sync()
        assert s.stats()["nonfinite"] == 0


def test_device_views_equal_downloads():
    from fibrenet_b200.native import Simulation
    with Simulation(net(), list_capacity=64) as s:
        s.step(7)
        perm = s.permutation()
        for field in ("pos", "img", "vel_old", "force"):
            v = s.device_view(field).cpu().numpy()
            host = s.get(field)
            np.testing.assert_array_equal(v[:, :3], host[perm].astype(v.dtype), err_msg=field)
