"""The C restatement (oracle/fibre_oracle.c) against the golden vectors the
reference's own kernels produced (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from fibrenet_b200.model import model_from_arrays


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d, model_from_arrays(d)


def run(sim, runs):
    for n in runs:
        if n < 0:
            sim.reset_energy()
        else:
            sim.run(int(n))


@pytest.mark.parametrize("name", golden_cases())
def test_ref_mode_bit_exact(oracle_built, name):
    po = oracle_built
    d, m = load(name)
    o = po.OracleSim(m, po.MODE_REF)
    run(o, d["runs"])
    for f in po.FIELD:
        np.testing.assert_array_equal(o.get(f), d["out_" + f], err_msg=f"{name}:{f}")
    s, a = o.status()
    np.testing.assert_array_equal(s, d["out_spring_status"])
    np.testing.assert_array_equal(a, d["out_angle_status"])
    o.rebuild()
    bc, cc = o.cells()
    np.testing.assert_array_equal(cc, d["out_grid_head"])
    grid = sorted((int(c), i) for i, c in enumerate(bc) if c >= 0)
    assert grid == [tuple(x) for x in d["out_grid"].tolist()]
    head, part, pair = o.lists()
    np.testing.assert_array_equal(head, d["out_list_head"])
    got = sorted(po.pair_set(head, part, pair))
    assert got == [tuple(x) for x in d["out_pairs"].tolist()]


@pytest.mark.parametrize("name", golden_cases())
def test_mirror_mode_close(oracle_built, name):
    """Mirror mode (FP32 storage of velocities/forces, per-bead gather order)
    stays within float rounding of the reference over the golden runs, and
    builds the same contact pair set from the same positions."""
    po = oracle_built
    d, m = load(name)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=256)
    run(o, d["runs"])
    ref_pos = d["out_img"]
    scale = max(1.0, float(np.abs(ref_pos).max()))
    np.testing.assert_allclose(o.get("img"), ref_pos, rtol=0, atol=2e-5 * scale)
    s, _ = o.status()
    assert (s != d["out_spring_status"]).sum() <= max(1, len(s) // 100)
    # list parity at the reference's final positions
    o.set("pos", d["out_pos"])
    o.rebuild()
    head, part, pair = o.lists()
    got = sorted(po.pair_set(head, part, pair))
    assert got == [tuple(x) for x in d["out_pairs"].tolist()]


def test_ref_build_matches_golden_when_present(oracle_built):
    """When the reference copy is built here, it still reproduces the golden
    vectors (guards the fixtures against drift of the build recipe)."""
    po = oracle_built
    if not po.ref_available():
        pytest.skip("reference copy not built on this machine")
    d, m = load("net_pbc_hs")
    r = po.RefSim(m, threads=1)
    run(r, d["runs"])
    np.testing.assert_array_equal(r.get("pos"), d["out_pos"])
