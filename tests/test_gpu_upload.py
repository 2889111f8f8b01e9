"""fn_upload's device path against its host path.

The device path copies the caller's arrays to the device as they are and
checks, orders and converts them there; the host path does the same work on
host threads.  For every model the device path takes, the two must leave the
same device state, bit for bit: same bead numbering, same packed bead
arrays, same bond statuses and the same trajectory afterwards.  Models
outside the device path (springs between non-consecutive beads) and invalid
models go to the host path, with the host path's errors.
"""
import numpy as np
import pytest

from fibrenet_b200 import generate as g
from gpu_util import FIELDS

pytestmark = pytest.mark.gpu


def sim(models, host, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("list_capacity", 64)
    return Simulation(models, host_upload=host, **kw)


def reversed_chains(m):
    m = m.normalised().copy()
    m.s_p1, m.s_p2 = m.s_p2.copy(), m.s_p1.copy()
    m.a_b1, m.a_b3 = m.a_b3.copy(), m.a_b1.copy()
    m.a_s1, m.a_s2 = m.a_s2.copy(), m.a_s1.copy()
    return m


def models():
    t = g.tensile_network(seed=31, fibres=120, beads=30, box=(80.0, 60.0, 10.0), z_range=(1.0, 9.0),
                          fail_mu=np.log(0.6), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=78.0, pull=0.5, cell=2.5)
    t_fl = t.copy()
    t_fl.a_type[:] = 1
    ens = [g.plain_network(seed=40 + k, fibres=8 + 5 * k, beads=12 + k, box=(20.0 + 3 * k, 20.0, 6.0),
                           z_range=(1.0, 5.0)) for k in range(5)]
    dense = g.dense_mat(seed=7, fibres=300, beads=40, box=(30.0, 30.0, 30.0))
    return {"tensile": t, "tensile_hrfl_angles": t_fl, "reversed": reversed_chains(t_fl), "ensemble": ens,
            "dense": dense}


def compare(a, b, nb):
    np.testing.assert_array_equal(a.permutation(), b.permutation())
    for f in FIELDS:
        np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)
    for x, y in zip(a.status(), b.status()):
        np.testing.assert_array_equal(x, y)
    for f in ("pos", "img"):  # packed fourth words (radius/type, 1/mass) included
        np.testing.assert_array_equal(a.device_view(f).cpu().numpy(), b.device_view(f).cpu().numpy(), err_msg=f)


@pytest.mark.parametrize("name", ["tensile", "tensile_hrfl_angles", "reversed", "ensemble", "dense"])
@pytest.mark.parametrize("reorder", [True, False])
def test_device_upload_equals_host_upload(name, reorder):
    m = models()[name]
    dev = sim(m, False, reorder=reorder)
    host = sim(m, True, reorder=reorder)
    assert dev.stats()["upload_on_device"] == 1
    assert host.stats()["upload_on_device"] == 0
    assert dev.stats()["bond_path"] == host.stats()["bond_path"] == 2
    compare(dev, host, dev.nb)
    for n in (9, 40):
        dev.step(n)
        host.step(n)
        compare(dev, host, dev.nb)
    # the host copies the device path fills on first need
    s_k = np.linspace(50.0, 150.0, dev.ns)
    dev.set_springs(k=s_k)
    host.set_springs(k=s_k)
    dev.step(10)
    host.step(10)
    compare(dev, host, dev.nb)
    c1, p1 = dev.lists()
    c2, p2 = host.lists()
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(p1, p2)


def test_non_chain_model_goes_to_the_host_path():
    """Cross-links between fibres: not fibres stored bead after bead."""
    m = g.plain_network(seed=6, fibres=30, beads=20, box=(20.0, 20.0, 6.0), z_range=(1.0, 5.0)).normalised().copy()
    m.s_type = np.concatenate([m.s_type, [0]]).astype(np.int32)
    m.s_tag = np.concatenate([m.s_tag, [-1]]).astype(np.int32)
    m.s_p1 = np.concatenate([m.s_p1, [0]]).astype(np.int32)
    m.s_p2 = np.concatenate([m.s_p2, [45]]).astype(np.int32)
    for f, v in (("s_rest", 1.5), ("s_k", 10.0), ("s_c1", 0.0), ("s_c2", 0.0)):
        setattr(m, f, np.concatenate([getattr(m, f), [v]]))
    dev = sim(m, False)
    host = sim(m, True)
    assert dev.stats()["upload_on_device"] == 0
    dev.step(20)
    host.step(20)
    compare(dev, host, dev.nb)


@pytest.mark.parametrize("fault", ["type", "mass", "spring", "angle", "hrfl_spring"])
def test_invalid_models_give_the_host_paths_errors(fault):
    from fibrenet_b200.native import NativeError
    m = g.plain_network(seed=3, fibres=10, beads=10, box=(12.0, 12.0, 6.0), z_range=(1.0, 5.0)).normalised().copy()
    if fault == "type":
        m.type = m.type.copy(); m.type[17] = 5
    elif fault == "mass":
        m.mass = m.mass.copy(); m.mass[23] = -1.0
    elif fault == "spring":
        m.s_p2 = m.s_p2.copy(); m.s_p2[7] = 10_000
    elif fault == "angle":
        m.a_b3 = m.a_b3.copy(); m.a_b3[4] = -3
    else:
        m.a_type = m.a_type.copy(); m.a_type[2] = 1
        m.a_s2 = m.a_s2.copy(); m.a_s2[2] = 99_999
    msgs = []
    for host in (False, True):
        with pytest.raises(NativeError) as e:
            sim(m, host)
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1]
