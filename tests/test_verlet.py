"""Displacement-triggered contact-list rebuilds (fn_config.verlet_skin > 0,
not a reference mode): cut-off pairs are listed out to cutoff + skin and the
list is rebuilt only when a bead has moved far enough since the last rebuild.
No pair within reach is ever missed, so the run follows a run that rebuilds
before every step, with far fewer rebuilds."""
import numpy as np
import pytest

from fibrenet_b200 import generate as g

pytestmark = pytest.mark.gpu


def hs_net(gu):
    m = g.plain_network(seed=51, fibres=40, beads=20, box=(24.0, 24.0, 7.5), z_range=(1.0, 6.5),
                        cell=1.5)
    m.settings.grid_update_freq = gu
    m.vel = np.random.default_rng(3).normal(0.0, 0.3, m.vel.shape)
    m.vel_old = m.vel.copy()
    return m


def lj_net(gu):
    m = g.tensile_network(seed=52, fibres=40, beads=15, box=(45.0, 30.0, 12.0), z_range=(2.0, 10.0),
                          clamp_lo=2.0, clamp_hi=43.0, pull=0.5, cell=3.0, min_sep=1.0)
    m.settings.grid_update_freq = gu
    m.vel = np.where((np.asarray(m.mass) > 0)[:, None],
                     np.random.default_rng(4).normal(0.0, 0.3, m.vel.shape), m.vel)
    m.vel_old = m.vel.copy()
    return m


def sim(m, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("list_capacity", 96)
    return Simulation(m, **kw)


@pytest.mark.parametrize("make", [hs_net, lj_net])
def test_follows_rebuild_every_step(make):
    """Same acting pairs as a run that rebuilds before every step; only the
    order of each bead's contact sum differs (lists from older positions), so
    the runs agree to rounding early on and statistically later (the dense
    penalty network is chaotic at the 1e-7 level)."""
    steps = 300
    with sim(make(1)) as ref, sim(make(8), verlet_skin=0.4) as v:
        ref.step(37)
        v.step(37)
        np.testing.assert_allclose(v.get("img"), ref.get("img"), rtol=0, atol=1e-6)
        for n in (100, 163):
            ref.step(n)
            v.step(n)
        ev, er = v.energy(), ref.energy()
        assert ev["total"] == pytest.approx(er["total"], rel=1e-3)
        rebuilds = v.stats()["rebuilds"]
        assert 1 <= rebuilds < steps // 4, rebuilds
        assert ref.stats()["rebuilds"] >= steps


@pytest.mark.parametrize("make", [hs_net, lj_net])
def test_no_acting_pair_is_unlisted(make):
    """After every chunk, each pair that exerts a contact force is in the
    device list (brute force over all pairs on the host)."""
    m = make(8)
    with sim(m, verlet_skin=0.4) as v:
        s = m.settings
        box = np.asarray(s.box)
        per = [bool((s.periodic_mask >> a) & 1) if s.periodic_mask >= 0 else s.bc_type == 0
               for a in range(3)]
        tag, loc = np.asarray(m.tag), np.asarray(m.loc_id)
        reach = s.cutoff if int(m.pair_kind[0]) == 1 else 1.0
        for _ in range(6):
            v.step(29)
            pos = v.get("pos")
            cnt, part = v.lists()
            listed = {(i, int(j)) for i in range(len(cnt)) for j in part[i, :cnt[i]]}
            d = pos[:, None, :] - pos[None, :, :]
            for a in range(3):
                if per[a]:
                    d[..., a] -= box[a] * np.round(d[..., a] / box[a])
            r = np.sqrt((d * d).sum(-1))
            excl = (tag[:, None] == tag[None, :]) & (np.abs(loc[:, None] - loc[None, :]) <= 1)
            ii, jj = np.nonzero((r < reach) & ~excl)
            missing = [(i, j) for i, j in zip(ii, jj) if i != j and (i, j) not in listed]
            assert not missing, missing[:5]


def test_rejects_cell_no_wider_than_cutoff():
    from fibrenet_b200.native import NativeError
    m = lj_net(8)
    m.settings.box_unit_cell = 2.5  # = LJ cut-off: no room for a skin
    with pytest.raises(NativeError, match="grid cell wider"):
        sim(m, verlet_skin=0.3)


def test_zero_skin_keeps_reference_cadence():
    m = hs_net(8)
    with sim(m) as a, sim(m, verlet_skin=0.0) as b:
        a.step(40)
        b.step(40)
        np.testing.assert_array_equal(a.get("img"), b.get("img"))
        assert b.stats()["rebuilds"] == a.stats()["rebuilds"]
