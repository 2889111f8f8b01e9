"""Parity of the CUDA path (through the C ABI) with the oracle.

* bit-exact against the oracle's MIRROR mode (same storage rounding and
  summation order) on every golden case, including bond statuses;
* within FP32 storage rounding of the reference's own results (golden
  vectors from kernel.cl) on the same cases;
* identical grid cells and contact-pair sets to the reference;
* one-step forces within 1e-5 (norm-wise) of the FP64 reference;
* bit-exact broken-spring sets over 1,000 steps of a tensile pull.
"""
import os

import numpy as np
import pytest

import pyoracle as po
from conftest import GOLDEN, golden_cases
from fibrenet_b200 import generate as g
from fibrenet_b200.model import model_from_arrays, permute_model
from gpu_util import FIELDS, rel_norm, run_seq

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5  # relative, norm-wise, FP32 result vs FP64 reference (the per-step force bound)


def sim(model, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("reorder", False)
    kw.setdefault("chain", True)
    kw.setdefault("list_capacity", 256)
    return Simulation(model, **kw)


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d, model_from_arrays(d)


@pytest.mark.parametrize("name", golden_cases())
def test_golden_bit_exact_vs_mirror(oracle_built, name):
    d, m = load(name)
    s = sim(m)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=256)
    run_seq(s, d["runs"])
    run_seq(o, d["runs"])
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f), o.get(f), err_msg=f"{name}: {f}")
    ss, sa = s.status()
    os_, oa = o.status()
    np.testing.assert_array_equal(ss, os_)
    np.testing.assert_array_equal(sa, oa)


@pytest.mark.parametrize("name", golden_cases())
def test_golden_close_to_reference(name):
    d, m = load(name)
    s = sim(m)
    run_seq(s, d["runs"])
    ref = d["out_img"]
    scale = max(1.0, float(np.abs(ref).max()))
    np.testing.assert_allclose(s.get("img"), ref, rtol=0, atol=2e-5 * scale)
    np.testing.assert_array_equal(s.status()[0], d["out_spring_status"])
    np.testing.assert_array_equal(s.status()[1], d["out_angle_status"])


@pytest.mark.parametrize("name", golden_cases())
def test_cells_and_pairs_match_reference(name):
    """Cell ids and the contact-pair set built from the reference's final
    positions equal the reference's own (kernel.cl FillGrid +
    BuildContactList), bit for bit."""
    d, m = load(name)
    m.pos = d["out_pos"]
    s = sim(m)
    s.rebuild()
    bc, cc = s.cells()
    np.testing.assert_array_equal(cc, d["out_grid_head"])
    grid = sorted((int(c), i) for i, c in enumerate(bc) if c >= 0)
    assert grid == [tuple(x) for x in d["out_grid"].tolist()]
    cnt, part = s.lists()
    got = sorted(po.pair_set(cnt, part))
    want = sorted({(int(a), int(b)) for a, b, _ in d["out_pairs"].tolist()})
    assert got == want


def test_one_step_forces_vs_fp64_reference(oracle_built):
    """Config-0 geometry (200 fibres x 50 beads), identical FP32-representable
    inputs: springs + angles + penalty contacts of one evaluation."""
    m = g.plain_network(seed=21).fp32_representable()
    # a perturbed state so every term is active
    rng = np.random.default_rng(0)
    m.img = m.img + rng.normal(0.0, 0.02, m.img.shape)
    m.img = m.img.astype(np.float32).astype(np.float64)
    box = np.asarray(m.settings.box)
    m.pos = np.mod(m.img, box)
    r = po.OracleSim(m, po.MODE_REF)
    r.rebuild()
    r.forces_only()
    fr = r.get("force")
    s = sim(m, list_capacity=64)
    s.rebuild()
    s.forces_only()
    fg = s.get("force")
    err = rel_norm(fg, fr)
    assert err <= FORCE_TOL, err
    # each term on its own
    for terms in [(1, 0, 0), (0, 1, 0), (0, 0, 1)]:
        r.forces_only(*terms)
        s.forces_only(*terms)
        e = rel_norm(s.get("force"), r.get("force"))
        assert e <= FORCE_TOL, (terms, e)


def test_reordered_run_matches_mirror_on_permuted_model(oracle_built):
    m = g.plain_network(seed=4, fibres=40, beads=25, box=(30.0, 30.0, 6.0), z_range=(1.0, 5.0))
    s = sim(m, reorder=True, list_capacity=64)
    perm = s.permutation()
    assert sorted(perm.tolist()) == list(range(m.n_beads))
    mp = permute_model(m, perm)
    o = po.OracleSim(mp, po.MODE_MIRROR, cell_cap=64, list_cap=64)
    s.step(37)
    o.run(37)
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f)[perm], o.get(f), err_msg=f)


def test_call_cadence_matches_mirror(oracle_built):
    """The rebuild counter restarts with every call (SimulationManager.cpp:152)."""
    m = g.plain_network(seed=9, fibres=30, beads=20, box=(25.0, 25.0, 6.0), z_range=(1.0, 5.0))
    s = sim(m, list_capacity=64)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=64)
    for n in [1, 5, 13, 2, 8]:
        s.step(n)
        o.run(n)
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f), o.get(f), err_msg=f)


def test_broken_set_1000_steps_bit_exact(oracle_built):
    """Tensile pull with HR_FL springs: the set of broken springs over 1,000
    steps equals the mirror oracle's exactly, checked every 100 steps."""
    m = g.tensile_network(seed=3, fibres=60, beads=30, box=(60.0, 40.0, 10.0), z_range=(1.0, 9.0),
                          fail_mu=np.log(0.8), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=58.0,
                          pull=0.5, cell=2.5, min_sep=1.0)
    s = sim(m, list_capacity=64)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=64)
    for _ in range(10):
        s.step(100)
        o.run(100)
        np.testing.assert_array_equal(s.status()[0], o.status()[0])
    np.testing.assert_array_equal(s.get("img"), o.get("img"))
    assert (s.status()[0] == 0).sum() > 0  # the pull does break springs


def test_batched_equals_separate_runs():
    ms = [g.plain_network(seed=30 + k, fibres=10 + 7 * k, beads=20, box=(20.0 + 4 * k, 20.0, 6.0),
                          z_range=(1.0, 5.0)) for k in range(4)]
    with sim(ms, list_capacity=64) as b:
        b.step(25)
        allpos = b.get("img")
        st = b.status()[0]
    off = 0
    soff = 0
    for m in ms:
        with sim(m, list_capacity=64) as one:
            one.step(25)
            np.testing.assert_array_equal(allpos[off:off + m.n_beads], one.get("img"))
            np.testing.assert_array_equal(st[soff:soff + m.n_springs], one.status()[0])
        off += m.n_beads
        soff += m.n_springs


def test_observables_match_host_sums():
    m = g.tensile_network(seed=5, fibres=40, beads=20, box=(40.0, 30.0, 8.0), z_range=(1.0, 7.0),
                          clamp_lo=2.0, clamp_hi=38.0, pull=0.2, cell=2.5)
    s = sim(m, list_capacity=64)
    s.step(50)
    o = s.observe(0, reaction_type=2)
    f = s.get("force")
    want = f[m.type == 2].sum(axis=0)
    np.testing.assert_allclose(o["reaction"], want, rtol=1e-12, atol=1e-12)
    assert o["broken"] == int((s.status()[0] == 0).sum())


def test_reset_energy_and_set_state(oracle_built):
    m = g.plain_network(seed=12, fibres=10, beads=10, box=(12.0, 12.0, 6.0), z_range=(1.0, 5.0))
    s = sim(m, list_capacity=64)
    s.step(5)
    s.reset_energy()
    for f in ["vel", "force", "vel_old"]:
        assert not s.get(f).any()
    v = np.random.default_rng(1).normal(size=(m.n_beads, 3)).astype(np.float32).astype(np.float64)
    s.set("vel_old", v)
    np.testing.assert_array_equal(s.get("vel_old"), v)


def test_bad_model_is_rejected():
    from fibrenet_b200.native import NativeError
    m = g.plain_network(seed=1, fibres=4, beads=5, box=(10.0, 10.0, 6.0), z_range=(1.0, 5.0))
    m.s_p2 = m.s_p2.copy()
    m.s_p2[0] = 10_000
    with pytest.raises(NativeError):
        sim(m)


def _crosslinked(seed=6):
    """Fibres plus random cross-links between nearby beads of different
    fibres: not chain form, so the incidence path runs."""
    m = g.plain_network(seed=seed, fibres=30, beads=20, box=(20.0, 20.0, 6.0), z_range=(1.0, 5.0))
    img = m.img
    d2 = ((img[:, None, :] - img[None, :, :]) ** 2).sum(-1)
    close = np.argwhere((d2 < 2.25) & (m.tag[:, None] < m.tag[None, :]))
    extra = [tuple(x) for x in close[::3][:60]]
    assert len(extra) > 10
    e = np.array(extra, np.int32)
    n = len(e)
    m.s_type = np.concatenate([m.s_type, np.full(n, 1, np.int32)])
    m.s_tag = np.concatenate([m.s_tag, np.full(n, -1, np.int32)])
    m.s_p1 = np.concatenate([m.s_p1, e[:, 0]])
    m.s_p2 = np.concatenate([m.s_p2, e[:, 1]])
    d = np.linalg.norm(img[e[:, 0]] - img[e[:, 1]], axis=1)
    m.s_rest = np.concatenate([m.s_rest, d.astype(np.float32).astype(np.float64)])
    m.s_k = np.concatenate([m.s_k, np.full(n, 80.0)])
    m.s_c1 = np.concatenate([m.s_c1, np.full(n, 1000.0)])
    m.s_c2 = np.concatenate([m.s_c2, np.full(n, 2.0)])
    return m


def _reversed(m):
    """Same chains with every spring and angle listed the other way round."""
    m = m.normalised().copy()
    m.s_p1, m.s_p2 = m.s_p2.copy(), m.s_p1.copy()
    m.a_b1, m.a_b3 = m.a_b3.copy(), m.a_b1.copy()
    m.a_s1, m.a_s2 = m.a_s2.copy(), m.a_s1.copy()
    return m


@pytest.mark.parametrize("kind", ["chain", "reversed", "crosslinked"])
def test_bond_paths_bit_exact_vs_mirror(oracle_built, kind):
    if kind == "crosslinked":
        m = _crosslinked()
    else:
        m = g.tensile_network(seed=8, fibres=40, beads=20, box=(40.0, 30.0, 8.0), z_range=(1.0, 7.0),
                              fail_mu=np.log(0.5), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=38.0,
                              pull=0.5, cell=2.5)
        m.a_type[:] = 1  # HR_FL angles: die with their springs
        if kind == "reversed":
            m = _reversed(m)
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=64)
    o.run(150)
    for chain in (True, False):
        s = sim(m, list_capacity=64, chain=chain)
        want_path = 2 if (chain and kind != "crosslinked") else 1
        assert s.stats()["bond_path"] == want_path
        s.step(150)
        for f in FIELDS:
            np.testing.assert_array_equal(s.get(f), o.get(f), err_msg=f"{kind} chain={chain} {f}")
        np.testing.assert_array_equal(s.status()[0], o.status()[0])
        np.testing.assert_array_equal(s.status()[1], o.status()[1])
    assert (o.status()[0] == 0).sum() > 0


@pytest.mark.parametrize("chain", [True, False])
def test_forces_only_paths(oracle_built, chain):
    m = g.plain_network(seed=22, fibres=60, beads=30).fp32_representable()
    rng = np.random.default_rng(3)
    m.img = (m.img + rng.normal(0.0, 0.03, m.img.shape)).astype(np.float32).astype(np.float64)
    m.pos = np.mod(m.img, np.asarray(m.settings.box))
    r = po.OracleSim(m, po.MODE_REF)
    r.rebuild()
    s = sim(m, list_capacity=64, chain=chain)
    s.rebuild()
    for terms in [(1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1)]:
        r.forces_only(*terms)
        s.forces_only(*terms)
        e = rel_norm(s.get("force"), r.get("force"))
        assert e <= FORCE_TOL, (terms, e)


def test_graph_replay_is_bit_identical():
    """Step segments replayed as CUDA graphs give the bits of direct launches,
    over calls of every length modulo grid_update_freq and both ping-pong
    parities."""
    m = g.tensile_network(seed=9, fibres=40, beads=20, box=(40.0, 30.0, 8.0), z_range=(1.0, 7.0),
                          fail_mu=np.log(0.5), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=38.0,
                          pull=0.5, cell=2.5)
    a = sim(m, list_capacity=64, use_graphs=False)
    b = sim(m, list_capacity=64, use_graphs=True)
    for n in [1, 2, 7, 8, 9, 16, 17, 3, 8, 5, 24]:
        a.step(n)
        b.step(n)
    for f in FIELDS:
        np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)
    np.testing.assert_array_equal(a.status()[0], b.status()[0])
    assert b.stats()["graph_launches"] > 0 and a.stats()["graph_launches"] == 0


def test_autotune_leaves_state_unchanged():
    m = g.plain_network(seed=14, fibres=50, beads=20, box=(25.0, 25.0, 6.0), z_range=(1.0, 5.0))
    a = sim(m, list_capacity=64)
    b = sim(m, list_capacity=64, use_graphs=True)
    a.step(13)
    b.step(13)
    bs = b.autotune(10)
    assert bs in (64, 96, 128, 192, 256, 384, 512) and b.stats()["block_size"] == bs
    assert b.stats()["steps"] == 13
    a.step(20)
    b.step(20)
    for f in FIELDS:
        np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)


@pytest.mark.parametrize("shape", [(64, 1), (64, 2), (96, 8), (128, 4), (192, 2), (256, 8), (128, 0)])
def test_staged_kernel_shapes_bit_exact_vs_mirror(oracle_built, shape):
    """The staged chain kernel at several shapes -- including rounds of fewer
    contact items than a tile holds, so a bead's contacts straddle rounds --
    and the unstaged chain kernel give the mirror's bits, statuses included."""
    m = g.tensile_network(seed=17, fibres=90, beads=40, box=(70.0, 50.0, 10.0), z_range=(1.0, 9.0),
                          fail_mu=np.log(0.6), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=68.0,
                          pull=0.5, cell=2.5, placement="host")
    o = po.OracleSim(m, po.MODE_MIRROR, cell_cap=64, list_cap=64)
    s = sim(m, list_capacity=64, use_graphs=True)
    s.set_kernel_shape(*shape)
    st = s.stats()
    assert (st["block_size"], st["items_per_thread"]) == shape
    for n in (1, 9, 30, 60):
        s.step(n)
        o.run(n)
    for f in FIELDS:
        np.testing.assert_array_equal(s.get(f), o.get(f), err_msg=f"{shape} {f}")
    np.testing.assert_array_equal(s.status()[0], o.status()[0])
    np.testing.assert_array_equal(s.status()[1], o.status()[1])
    assert s.stats()["stalls"] == 0
    if shape[1] in (1, 2):
        # rounds of 64 or 128 items: tiles of 60 beads hold more, so a bead's
        # contacts straddle rounds
        cnt, _ = s.lists()
        per_tile = np.add.reduceat(np.minimum(cnt, 64), np.arange(0, m.n_beads, shape[0] - 4))
        assert per_tile.max() > shape[1] * shape[0]


def test_state_save_restore_repeats_steps():
    """fn_state_restore puts back what fn_state_save took: the same steps from
    the restored state give the same bits, and the step count goes back."""
    m = g.tensile_network(seed=19, fibres=40, beads=30, box=(50.0, 40.0, 8.0), z_range=(1.0, 7.0),
                          fail_mu=np.log(0.6), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=48.0, pull=0.5,
                          cell=2.5)
    s = sim(m, list_capacity=64, use_graphs=True)
    s.step(7)
    s.save_state()
    ms = s.step_timed(25)
    assert ms > 0.0
    first = {f: s.get(f) for f in FIELDS}
    st = s.status()
    assert s.stats()["steps"] == 32
    for _ in range(2):
        s.restore_state()
        assert s.stats()["steps"] == 7
        s.step(25)
        for f in FIELDS:
            np.testing.assert_array_equal(s.get(f), first[f], err_msg=f)
        np.testing.assert_array_equal(s.status()[0], st[0])


@pytest.mark.parametrize("kind", ["tensile", "dense_periodic", "small_grid", "full_cells"])
def test_list_builds_equal_bead_lists(kind):
    """The list builds by bricks of cells and by groups of lanes give the
    per-bead build's lists, entry for entry (same order), on finite and
    periodic boxes, a grid of three cells per axis (every halo wraps onto
    itself) and cells fuller than the cell capacity; and the same
    trajectory."""
    cell_cap = 64
    if kind == "tensile":
        m = g.tensile_network(seed=33, fibres=300, beads=40, box=(120.0, 90.0, 12.0), z_range=(1.0, 11.0),
                              clamp_lo=2.0, clamp_hi=118.0, pull=0.5, cell=2.5)
    elif kind == "dense_periodic":
        m = g.dense_mat(seed=8, fibres=400, beads=40, box=(28.0, 28.0, 28.0))
    elif kind == "small_grid":
        m = g.plain_network(seed=34, fibres=12, beads=6, box=(3.0, 3.0, 3.0), z_range=(0.5, 2.5))
    else:
        m = g.plain_network(seed=35, fibres=60, beads=20, box=(6.0, 6.0, 4.0), z_range=(0.5, 3.5))
        cell_cap = 6
    b = sim(m, list_capacity=64, cell_capacity=cell_cap, reorder=True)
    b.set_list_build("beads")
    assert b.stats()["list_build"] == 0
    builds = {mode: sim(m, list_capacity=64, cell_capacity=cell_cap, reorder=True)
              for mode in ("bricks", "groups")}
    for mode, a in builds.items():
        a.set_list_build(mode)
        assert a.stats()["list_build"] == ("beads", "bricks", "groups").index(mode)
    for n in (1, 8, 17):
        b.step(n)
        cb, pb = b.lists()
        for mode, a in builds.items():
            a.step(n)
            ca, pa = a.lists()
            np.testing.assert_array_equal(ca, cb, err_msg=mode)
            np.testing.assert_array_equal(pa, pb, err_msg=mode)
            assert a.stats()["list_overflow"] == b.stats()["list_overflow"], mode
            assert a.stats()["cell_overflow"] == b.stats()["cell_overflow"], mode
    for mode, a in builds.items():
        for f in FIELDS:
            np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f"{mode} {f}")
        a.close()
    if kind == "full_cells":
        assert b.stats()["cell_overflow"] > 0
    b.close()
