"""Edge cases of the step loop on the GPU, each against the oracle's MIRROR
mode (bit for bit): networks without bonds, single beads, frozen (mass 0)
networks, ragged batches, and full cells / full contact lists, whose dropped
entries are counted the same way on both sides."""
import numpy as np
import pytest

import pyoracle as po
from fibrenet_b200 import generate as g
from fibrenet_b200.model import PAIR_HS, Settings
from gpu_util import FIELDS

pytestmark = pytest.mark.gpu


def sim(model, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("reorder", False)
    kw.setdefault("list_capacity", 64)
    return Simulation(model, **kw)


def gas(n=400, seed=3, side=8.0, k=50.0, vel=0.5):
    """Free beads (no springs, no angles) with penalty contacts."""
    rng = np.random.default_rng(seed)
    st = Settings(dt=0.001, lam=0.5, cutoff=1.0, box_unit_cell=1.0, box=(side, side, side), bc_type=0)
    beads = []
    for i in range(n):
        p = tuple(rng.uniform(0.0, side, 3))
        v = tuple(rng.normal(0.0, vel, 3))
        beads.append((0, i, 0, 0.5, 1.0, p, v, p))
    return g.explicit_model(st, ["A"], {(0, 0): (PAIR_HS, [k])}, beads)


def same_as_mirror(m, runs, cell_cap=64, list_cap=64, **kw):
    s = sim(m, cell_capacity=cell_cap, list_capacity=list_cap, **kw)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=cell_cap, list_cap=list_cap)
    for n in runs:
        s.step(n)
        o.run(n)
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f), o.get(f), err_msg=f)
    return s, o


def test_beads_without_bonds(oracle_built):
    m = gas()
    s, _ = same_as_mirror(m, [1, 17, 30])
    assert s.stats()["bond_path"] in (0, 1, 2)
    s.close()


def test_single_bead(oracle_built):
    m = gas(n=1)
    s, _ = same_as_mirror(m, [3, 9])
    s.close()


def test_frozen_network_does_not_move(oracle_built):
    m = g.plain_network(seed=5, fibres=10, beads=8, box=(12.0, 12.0, 6.0), z_range=(1.0, 5.0))
    m.mass = np.zeros(m.n_beads)
    s, _ = same_as_mirror(m, [12])
    np.testing.assert_array_equal(s.get("img"), np.asarray(m.img))
    s.close()


def test_ragged_batch_equals_separate_runs():
    ms = [gas(n=1, seed=1), g.plain_network(seed=2, fibres=60, beads=30, box=(30.0, 30.0, 6.0),
                                            z_range=(1.0, 5.0)), gas(n=37, seed=4)]
    with sim(ms) as b:
        b.step(23)
        img = b.get("img")
    base = 0
    for m in ms:
        with sim(m) as one:
            one.step(23)
            np.testing.assert_array_equal(img[base:base + m.n_beads], one.get("img"))
        base += m.n_beads


def test_full_cells_counted_like_the_mirror(oracle_built):
    """A crowded box with 2 beads per cell kept: the lowest-numbered beads of a
    full cell stay, the rest are listed nowhere, and both sides count the
    dropped beads identically."""
    m = gas(n=600, seed=9, side=6.0, vel=0.2)
    s, o = same_as_mirror(m, [8, 8], cell_cap=2)
    assert s.stats()["cell_overflow"] > 0
    assert s.stats()["cell_overflow"] == o.overflow()[0]
    s.close()


def test_full_lists_counted_like_the_mirror(oracle_built):
    m = gas(n=600, seed=10, side=6.0, vel=0.2)
    s, o = same_as_mirror(m, [8, 8], list_cap=3)
    assert s.stats()["list_overflow"] > 0
    assert s.stats()["list_overflow"] == o.overflow()[1]
    s.close()


@pytest.mark.parametrize("cap", [1, 2, 3])
def test_chain_path_under_tiny_list_capacity(oracle_built, cap):
    """Fibres on the chain bond path whose contact lists are cut to 1-3
    entries: the GPU drops exactly the entries the mirror drops, counts them
    alike, and the bits still agree."""
    m = g.tensile_network(seed=5, fibres=60, beads=30, box=(60.0, 40.0, 10.0), z_range=(1.0, 9.0),
                          clamp_lo=2.0, clamp_hi=58.0, placement="host")
    s, o = same_as_mirror(m, [8, 8, 3], list_cap=cap)
    assert s.stats()["bond_path"] == 2
    assert s.stats()["list_overflow"] > 0
    assert s.stats()["list_overflow"] == o.overflow()[1]
    s.close()


@pytest.mark.parametrize("cell_cap", [1, 3, 7, 8, 9, 64])
def test_cell_sort_paths_like_the_mirror(oracle_built, cell_cap):
    """Cells of up to eight beads are ordered in registers, larger or overfull
    ones by selection: a dense gas (up to ~10 beads per cell) at capacities
    below, at and above eight keeps the mirror's cells, lists and bits."""
    m = gas(n=2000, seed=12, side=6.0, vel=0.2)
    s, o = same_as_mirror(m, [8, 8, 5], cell_cap=cell_cap, list_cap=256)
    bc, cc = s.cells()
    obc, occ = o.cells()
    np.testing.assert_array_equal(cc, occ)
    np.testing.assert_array_equal(bc, obc)
    assert s.stats()["cell_overflow"] == o.overflow()[0]
    if cell_cap <= 8:
        assert s.stats()["cell_overflow"] > 0
    s.close()
