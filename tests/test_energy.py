"""Energy / virial observables (fn_energy_eval) and the recorded time series
(fn_step_series).

CPU: the potentials of tests/energy_ref.py are the ones the reference's
forces derive from: minus their finite-difference gradient equals the
oracle's (REF mode, FP64) spring + angle + contact forces for every contact
kind.  GPU: the device reduction equals the FP64 numpy statement on the
device's own state and pair list; total energy is conserved to second order
in dt; the time series equals the step / observe / energy call sequence bit
for bit.
"""
import numpy as np
import pytest

import energy_ref as er
from fibrenet_b200 import generate as g
from fibrenet_b200.model import PAIR_ST

def perturbed(m, sigma, seed=0):
    rng = np.random.default_rng(seed)
    m = m.fp32_representable()
    m.img = (m.img + rng.normal(0.0, sigma, m.img.shape)).astype(np.float32).astype(np.float64)
    box = np.asarray(m.settings.box)
    per = [bool((m.settings.periodic_mask >> a) & 1) if m.settings.periodic_mask >= 0
           else m.settings.bc_type == 0 for a in range(3)]
    m.pos = np.where(per, np.mod(m.img, box), m.img)
    return m


def hs_net():
    return perturbed(g.plain_network(seed=31, fibres=30, beads=10, box=(12.0, 12.0, 6.0),
                                     z_range=(1.0, 5.0)), 0.05)


def lj_net():
    m = g.tensile_network(seed=5, fibres=24, beads=10, box=(24.0, 16.0, 8.0), z_range=(1.0, 7.0),
                          clamp_lo=1.0, clamp_hi=23.0, min_sep=0.95, fail_mu=np.log(50.0))
    return perturbed(m, 0.03, seed=1)


def st_net():
    m = g.plain_network(seed=32, fibres=30, beads=10, box=(12.0, 12.0, 6.0), z_range=(1.0, 5.0),
                        cell=1.25)
    m.settings.cutoff = 1.2
    m.pair_kind = np.array([PAIR_ST], np.int32)
    m.pair_raw = np.array([[200.0, 50.0, 1.0, 1.03]])
    return perturbed(m, 0.05, seed=2)


def hsr_net():
    return perturbed(g.dense_mat(seed=9, fibres=60, beads=10, box=(10.0, 10.0, 10.0)), 0.05, seed=3)


NETS = {"hs": hs_net, "lj": lj_net, "st": st_net, "hsr": hsr_net}


def internal_energy(m, pos, img, pairs, s_status, a_status):
    us, ua, _ = er.bonded_terms(m, img, s_status, a_status)
    uc, _, _ = er.contact_terms(m, pos, pairs, er.force_mask(m))
    return us + ua + uc


@pytest.mark.parametrize("kind", sorted(NETS))
def test_forces_are_minus_energy_gradient(oracle_built, kind):
    po = oracle_built
    m = NETS[kind]()
    r = po.OracleSim(m, po.MODE_REF)
    r.rebuild()
    r.forces_only()
    F = r.get("force")
    head, part, _ = r.lists()
    pairs = sorted(po.pair_set(head, part))
    s_status, a_status = r.status()
    pos, img = m.pos.copy(), m.img.copy()
    assert internal_energy(m, pos, img, pairs, s_status, a_status) != 0.0
    rng = np.random.default_rng(4)
    h = 1e-6
    scale = np.abs(F).max()
    for _ in range(40):
        i, a = int(rng.integers(m.n_beads)), int(rng.integers(3))
        up_p, up_i = pos.copy(), img.copy()
        dn_p, dn_i = pos.copy(), img.copy()
        up_p[i, a] += h
        up_i[i, a] += h
        dn_p[i, a] -= h
        dn_i[i, a] -= h
        grad = (internal_energy(m, up_p, up_i, pairs, s_status, a_status)
                - internal_energy(m, dn_p, dn_i, pairs, s_status, a_status)) / (2 * h)
        assert abs(-grad - F[i, a]) <= 1e-6 * scale + 1e-6 * abs(F[i, a]), (kind, i, a, -grad, F[i, a])


def test_energy_ref_virial_of_one_spring():
    """Two beads joined by one stretched spring: W = r (x) F with F on p1."""
    m = g.plain_network(seed=1, fibres=1, beads=2, box=(10.0, 10.0, 10.0), z_range=(4.0, 6.0))
    m.img = np.array([[4.0, 5.0, 5.0], [5.5, 5.0, 5.0]])
    m.pos = m.img.copy()
    us, ua, W = er.bonded_terms(m, m.img, [1], [])
    assert us == pytest.approx(0.5 * 100.0 * 0.25)
    r = m.img[0] - m.img[1]
    F = 100.0 * (1.0 - 1.5) * r / 1.5
    np.testing.assert_allclose(W, np.outer(r, F))


# ---------------------------------------------------------------- GPU

def sim(m, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("list_capacity", 128)
    return Simulation(m, **kw)


def device_pairs(s):
    cnt, part = s.lists()
    out = []
    for i in range(len(cnt)):
        for k in range(min(int(cnt[i]), part.shape[1])):
            j = int(part[i, k])
            if j > i:
                out.append((i, j))
    return out


def check_against_numpy(s, m):
    e = s.energy()
    ss, sa = s.status()
    ref = er.energy(m, s.get("pos"), s.get("img"), s.get("vel_old"), ss, sa, device_pairs(s))
    for f in ("kinetic", "spring", "angle", "contact", "wall", "gravity", "total"):
        assert e[f] == pytest.approx(ref[f], rel=1e-9, abs=1e-9), f
    np.testing.assert_allclose(e["virial"], ref["virial"], rtol=1e-9, atol=1e-8)
    assert e["contacts"] == ref["contacts"]
    return e


@pytest.mark.gpu
@pytest.mark.parametrize("kind", sorted(NETS))
@pytest.mark.parametrize("chain", [True, False])
def test_energy_matches_numpy(kind, chain):
    m = NETS[kind]()
    m.vel = np.random.default_rng(7).normal(0.0, 0.2, m.vel.shape)
    m.vel_old = m.vel.copy()
    with sim(m, chain=chain) as s:
        s.step(25)
        e = check_against_numpy(s, m)
    assert e["contact"] != 0.0 and e["kinetic"] > 0.0  # lj contact energy is negative


@pytest.mark.gpu
def test_energy_of_each_network_in_a_batch():
    ms = [hs_net(), hsr_net(), lj_net()]
    with sim(ms) as s:
        s.step(10)
        tot = [s.energy(k)["total"] for k in range(3)]
    for k, m in enumerate(ms):
        with sim(m) as s1:
            s1.step(10)
            assert s1.energy()["total"] == tot[k]


@pytest.mark.gpu
def test_energy_conserved_to_second_order():
    """No damping, no walls, bonded terms only: the largest deviation of the
    total energy over a fixed time shrinks fourfold when dt halves (velocity
    Verlet).  Contacts are left out because the penalty and the cut LJ force
    have kinks, which lower the order; their potentials are checked against
    the forces by finite differences above."""
    def drift(dt, steps):
        m = g.plain_network(seed=12, fibres=40, beads=20, box=(20.0, 20.0, 6.0), z_range=(1.0, 5.0),
                            dt=dt, k_contact=0.0)
        m.vel = np.random.default_rng(3).normal(0.0, 0.2, m.vel.shape)
        m.vel_old = m.vel.copy()
        with sim(m) as s:
            s.step(1)
            e0 = s.energy()["total"]
            dev = 0.0
            for _ in range(20):
                s.step(steps // 20)
                dev = max(dev, abs(s.energy()["total"] - e0))
        return dev / abs(e0)
    d1 = drift(0.002, 2000)
    d2 = drift(0.001, 4000)
    assert d1 < 1e-3
    assert d1 / d2 > 3.5, (d1, d2)


@pytest.mark.gpu
def test_step_series_equals_call_sequence():
    from fibrenet_b200.native import SERIES_COLUMNS
    m = lj_net()
    with sim(m) as s:
        rows = s.step_series(95, 20, reaction_type=2, energy=True)
    assert rows.shape == (5, len(SERIES_COLUMNS))
    with sim(m) as s:
        for q, k in enumerate([20, 20, 20, 20, 15]):
            s.step(k)
            o = s.observe(0, reaction_type=2)
            e = s.energy()
            assert rows[q, 0] == 20 * q + k
            np.testing.assert_array_equal(rows[q, 1:4], o["reaction"])
            assert rows[q, 4] == o["broken"] and rows[q, 5] == o["angles_dead"]
            np.testing.assert_array_equal(rows[q, 6:12], [e[f] for f in ("kinetic", "spring", "angle",
                                                                       "contact", "wall", "gravity")])
            np.testing.assert_array_equal(rows[q, 12:21], e["virial"].ravel())
            assert rows[q, 21] == e["contacts"]
    with sim(m) as s:
        short = s.step_series(95, 20, reaction_type=2)
    np.testing.assert_array_equal(short, rows[:, :6])
