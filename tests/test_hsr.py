"""Pair kind 4 ("hsr"): a penalty spring on the overlap plus a soft harmonic
repulsion below rc on the same type pair (the dense-mat contact model).  The
reference has one pair kind per type pair, so this kind has no reference
kernel; it is pinned in two halves:

* with the soft term off it equals the reference's hs kind bit for bit (the
  oracle's REF mode, itself pinned to kernel.cl's golden vectors);
* with the penalty off, two beads feel k (rc - r) along the line of centres.

On the GPU it is bit-exact against the oracle's MIRROR mode and within 1e-5
(norm-wise) of the FP64 reference after one force evaluation.
"""
import numpy as np
import pytest

from fibrenet_b200 import generate as g
from fibrenet_b200.model import PAIR_HS, PAIR_HSR, Settings
from gpu_util import FIELDS, rel_norm


def small_mat(seed=5, fibres=200, beads=20, side=20.0, **kw):
    return g.dense_mat(seed=seed, fibres=fibres, beads=beads, box=(side, side, side), **kw)


def with_pair(m, kind, raw):
    m.pair_kind = np.array([kind], np.int32)
    m.pair_raw = np.array([raw], np.float64)
    return m


def test_hsr_without_soft_term_is_hs(oracle_built):
    po = oracle_built
    a = with_pair(small_mat(), PAIR_HS, [100.0, 0.0, 0.0, 0.0])
    b = with_pair(small_mat(), PAIR_HSR, [100.0, 0.0, 0.0, 0.0])
    ra, rb = po.OracleSim(a, po.MODE_REF), po.OracleSim(b, po.MODE_REF)
    for n in (1, 7, 12):
        ra.run(n)
        rb.run(n)
    for f in po.FIELD:
        np.testing.assert_array_equal(ra.get(f), rb.get(f), err_msg=f)


@pytest.mark.parametrize("r", [0.3, 0.9, 1.1, 1.25])
def test_hsr_two_beads_analytic(oracle_built, r):
    """Two free beads of radius 0.5 on the x axis: force on bead 0 is
    -(K max(1 - r, 0) + k max(rc - r, 0)) along x."""
    po = oracle_built
    K, k, rc = 100.0, 10.0, 1.2
    st = Settings(dt=0.001, lam=0.5, cutoff=1.2, box_unit_cell=1.0, box=(10.0, 10.0, 10.0),
                    bc_type=0, grid_update_freq=1)
    z = (0.0, 0.0, 0.0)
    beads = [(0, 0, 0, 0.5, 1.0, (4.0, 5.0, 5.0), z, (4.0, 5.0, 5.0)),
             (0, 1, 0, 0.5, 1.0, (4.0 + r, 5.0, 5.0), z, (4.0 + r, 5.0, 5.0))]
    m = g.explicit_model(st, ["C1"], {(0, 0): (PAIR_HSR, [K, k, rc])}, beads)
    o = po.OracleSim(m, po.MODE_REF)
    o.rebuild()
    o.forces_only(False, False, True)
    f = o.get("force")
    mag = K * max(1.0 - r, 0.0) + k * max(rc - r, 0.0)
    np.testing.assert_allclose(f[0], [-mag, 0.0, 0.0], atol=1e-12)
    np.testing.assert_allclose(f[1], [mag, 0.0, 0.0], atol=1e-12)


@pytest.mark.gpu
def test_soft_radius_beyond_cutoff_is_rejected():
    from fibrenet_b200 import native
    m = small_mat(fibres=4, beads=5)
    m.pair_raw = np.array([[100.0, 10.0, 1.5, 0.0]])
    with pytest.raises(native.NativeError, match="soft radius"):
        native.Simulation(m)


@pytest.mark.gpu
def test_dense_mat_bit_exact_vs_mirror(oracle_built):
    po = oracle_built
    from fibrenet_b200.native import Simulation
    m = small_mat()
    s = Simulation(m, reorder=False, list_capacity=64)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=64)
    for n in (1, 9, 30):
        s.step(n)
        o.run(n)
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f), o.get(f), err_msg=f)
    assert o.overflow() == (0, 0)


@pytest.mark.gpu
def test_dense_mat_forces_vs_fp64_reference(oracle_built):
    po = oracle_built
    from fibrenet_b200.native import Simulation
    m = small_mat(seed=8).fp32_representable()
    r = po.OracleSim(m, po.MODE_REF)
    r.rebuild()
    r.forces_only()
    s = Simulation(m, list_capacity=64, reorder=False)
    s.rebuild()
    s.forces_only()
    assert rel_norm(s.get("force"), r.get("force")) <= 1e-5
    r.forces_only(False, False, True)
    s.forces_only(False, False, True)
    assert rel_norm(s.get("force"), r.get("force")) <= 1e-5
