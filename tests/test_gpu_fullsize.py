"""Parity at the benchmarked sizes and for every contact kind, through the C ABI.

* The tensile network of the bench at full size (1,000,000 beads, LJ
  contacts with cut-off 2.5, HR_FL springs, finite x/z, periodic y, cell 2.5,
  64-entry lists, beads renumbered as the bench runs them): cell ids and the
  contact-pair set of one rebuild equal the oracle's restatement of
  FillGrid + BuildContactList (kernel.cl:487-789), with nothing dropped by
  the capacities; one 8-step segment is bit-exact against the mirror; the
  one-step forces are within 1e-5 (norm-wise) of the FP64 reference.
* One-step forces within 1e-5 of the FP64 reference for each term on its
  own (springs kernel.cl:366-441, angles :268-363, contacts :792-1011) on a
  60,000-bead tensile network (LJ, :875-919) and a 50,000-bead network with
  st contacts (:960-999).
"""
import numpy as np
import pytest

import pyoracle as po
from fibrenet_b200 import generate as g
from fibrenet_b200.model import PAIR_ST, permute_model
from gpu_util import FIELDS, rel_norm

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5  # relative, norm-wise, FP32 result vs FP64 reference (the per-step force bound)


def sim(model, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("list_capacity", 64)
    kw.setdefault("cell_capacity", 64)
    return Simulation(model, **kw)


def pair_keys(cnt, part, cap):
    """Sorted unique unordered pairs (as i * n + j, i < j) of per-bead lists."""
    n = cnt.shape[0]
    k = np.minimum(cnt, cap)
    i = np.repeat(np.arange(n, dtype=np.int64), k)
    mask = np.arange(part.shape[1])[None, :] < k[:, None]
    j = part[mask].astype(np.int64)
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    return np.unique(lo * n + hi)


def perturbed(m, sigma, seed):
    """FP32-representable copy with image positions jittered (so springs and
    angles carry force) and positions re-wrapped on the periodic axes."""
    m = m.fp32_representable()
    rng = np.random.default_rng(seed)
    img = (m.img + rng.normal(0.0, sigma, m.img.shape)).astype(np.float32).astype(np.float64)
    pos = img.copy()
    box = np.asarray(m.settings.box)
    for a in range(3):
        periodic = ((m.settings.periodic_mask >> a) & 1) if m.settings.periodic_mask >= 0 \
            else m.settings.bc_type == 0
        if periodic:
            pos[:, a] = np.mod(pos[:, a], box[a])
            pos[pos[:, a] >= box[a], a] = 0.0
    m.img, m.pos = img, pos
    return m


def check_terms(m, s_kw=None):
    r = po.OracleSim(m, po.MODE_REF, cell_cap=64, list_cap=64)
    r.rebuild()
    s = sim(m, **(s_kw or {}))
    s.rebuild()
    errs = {}
    for terms in [(1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1)]:
        r.forces_only(*terms)
        s.forces_only(*terms)
        fr = r.get("force")
        assert np.linalg.norm(fr) > 0.0, terms  # the term is active
        errs[terms] = rel_norm(s.get("force"), fr)
    s.close()
    r.close()
    for terms, e in errs.items():
        assert e <= FORCE_TOL, (terms, e)
    return errs


@pytest.fixture(scope="module")
def tensile_1m():
    return g.tensile_network(seed=1)


def test_tensile_1m_cells_pairs_and_segment(oracle_built, tensile_1m):
    m = tensile_1m
    s = sim(m, reorder=True)
    s.rebuild()
    bc, cc = s.cells()
    cnt, part = s.lists()
    st = s.stats()
    assert st["cell_overflow"] == 0 and st["list_overflow"] == 0

    r = po.OracleSim(m, po.MODE_REF, cell_cap=64, list_cap=64)
    r.rebuild()
    rbc, rcc = r.cells()
    rhead, rpart, _ = r.lists()
    assert r.overflow() == (0, 0)
    np.testing.assert_array_equal(bc, rbc)
    np.testing.assert_array_equal(cc, rcc)
    got = pair_keys(cnt, part, 64)
    want = pair_keys(rhead, rpart, 64)
    assert got.shape == want.shape and np.array_equal(got, want)
    assert 2 * len(want) == int(cnt.sum())  # full lists hold each pair once from each side
    r.close()

    # one rebuild segment, bit for bit against the mirror on the permuted model
    perm = s.permutation()
    o = po.OracleSim(permute_model(m, perm), po.MODE_MIRROR, cell_cap=64, list_cap=64)
    s.step(8)
    o.run(8)
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f)[perm], o.get(f), err_msg=f)
    np.testing.assert_array_equal(s.status()[0], o.status()[0])
    np.testing.assert_array_equal(s.status()[1], o.status()[1])
    assert o.overflow() == (0, 0)
    s.close()


def test_tensile_1m_one_step_forces(oracle_built, tensile_1m):
    m = perturbed(tensile_1m, 0.02, seed=11)
    check_terms(m, {"reorder": True})


def test_tensile_one_step_forces_each_term():
    """60,000 beads of the tensile geometry (box scaled to keep the fibre
    density): LJ contacts, HR_FL springs, finite x/z, periodic y."""
    F = 1200
    side = 1000.0 * np.sqrt(F / 20000.0)
    m = g.tensile_network(seed=6, fibres=F, box=(side, side, 20.0), clamp_lo=2.0, clamp_hi=side - 2.0)
    m = perturbed(m, 0.02, seed=12)
    for chain in (True, False):
        check_terms(m, {"chain": chain, "reorder": True})


def test_st_network_one_step_forces_each_term():
    """50,000 beads in a periodic box with st contacts (the reference's third
    pair kind: two harmonic arms, kernel.cl:960-999)."""
    m = g.plain_network(seed=23, fibres=1000, beads=50, box=(224.0, 224.0, 10.0), cell=1.25)
    m.pair_kind = np.array([PAIR_ST], np.int32)
    m.pair_raw = np.array([[2000.0, 500.0, 1.0, 1.03]])
    m.settings.cutoff = 1.2
    m.settings.dt = 0.0005
    m = perturbed(m, 0.05, seed=13)
    for chain in (True, False):
        check_terms(m, {"chain": chain, "reorder": True})
