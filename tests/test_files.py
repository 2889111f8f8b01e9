"""The native parser of the reference's input / model / restart files
(include/fibrenet_io.h), on the CPU: round trips, the compat-mode quirks of
SimulationManager.cpp and the errors it reports."""
import os

import numpy as np
import pytest

from fibrenet_b200 import files
from fibrenet_b200 import generate as g
from fibrenet_b200.model import SPRING_HR_FL


@pytest.fixture()
def tmp(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    return tmp_path


def net():
    m = g.plain_network(seed=3, fibres=6, beads=8, box=(12.0, 12.0, 6.0), z_range=(1.0, 5.0))
    m.s_type[::3] = SPRING_HR_FL
    m.s_c1[::3] = 1000.0
    m.s_c2[::3] = 5.0
    return m


def write(m, tmp, **kw):
    files.write_model_file(m, str(tmp / "model.txt"))
    kw.setdefault("run", 20)
    kw.setdefault("output_freq", 10)
    files.write_input_file(m, str(tmp / "in.txt"), "model.txt", "out", **kw)
    return str(tmp / "in.txt")


def test_round_trip_strict(tmp):
    m = net()
    m.vel = np.random.default_rng(0).normal(size=m.vel.shape)
    m.vel_old = m.vel.copy()
    r, info, skin = files.read_input(write(m, tmp), strict=True)
    for f in ["type", "tag", "loc_id", "radius", "mass", "pos", "vel", "vel_old", "img", "s_type",
              "s_p1", "s_p2", "s_rest", "s_k", "s_c1", "s_c2", "a_type", "a_b1", "a_b2", "a_b3",
              "a_s1", "a_s2", "a_theta0", "a_k", "pair_kind"]:
        np.testing.assert_array_equal(getattr(r, f), np.asarray(getattr(m.normalised(), f)), err_msg=f)
    np.testing.assert_array_equal(r.pair_raw[:, 0], m.pair_raw[:, 0])
    assert r.settings.box == m.settings.box and r.settings.dt == m.settings.dt
    assert info["run_steps"] == 20 and info["output_freq"] == 10 and info["export_position"] == 1
    assert skin is None


def test_compat_quirks(tmp):
    """velocity_old.{y,z} = velocity.x (SimulationManager.cpp:1405-1407);
    HR_FL c1/c2 through std::stoi (:1528-1529); rest angle through std::stof
    (:1637)."""
    m = net()
    m.vel[:] = [0.5, -1.25, 2.0]
    m.s_c1[::3] = 1000.7
    m.s_c2[::3] = 5.37
    m.a_theta0[:] = np.pi
    path = write(m, tmp)
    c, _, _ = files.read_input(path, strict=False)
    assert np.all(c.vel_old == 0.5)
    fl = c.s_type == SPRING_HR_FL
    assert np.all(c.s_c1[fl] == 1000.0) and np.all(c.s_c2[fl] == 5.0)
    assert np.all(c.a_theta0 == float(np.float32(np.pi)))
    s, _, _ = files.read_input(path, strict=True)
    np.testing.assert_array_equal(s.vel_old, s.vel)
    assert np.all(s.s_c2[fl] == 5.37) and np.all(s.a_theta0 == np.pi)


def test_missing_wall_forces_finite_box_in_compat(tmp):
    m = net()
    path = write(m, tmp)
    text = open(path).read().replace("box_wall_rep", "# box_wall_rep")
    open(path, "w").write(text)
    c, _, _ = files.read_input(path, strict=False)
    assert c.settings.bc_type == 1  # SimulationManager.cpp:2168
    s, _, _ = files.read_input(path, strict=True)
    assert s.settings.bc_type == 0


def test_lambda_required_in_compat(tmp):
    m = net()
    path = write(m, tmp)
    text = "\n".join(ln for ln in open(path).read().splitlines() if not ln.startswith("lambda"))
    open(path, "w").write(text)
    with pytest.raises(files.InputError, match="lambda"):
        files.read_input(path, strict=False)
    s, _, _ = files.read_input(path, strict=True)
    assert s.settings.lam == 0.5


def test_first_occurrence_wins_and_repeats_accumulate(tmp):
    m = net()
    path = write(m, tmp, extra_lines=["step\t0.5", "output_type\tC1", "modif_bead\tid\t3\tmass\t0.0",
                                      "modif_bead\ttag\t1\tvelocity\t1.0\t2.0\t3.0",
                                      "modif_bead\ttype\tC1\tskin_radius\t0.75",
                                      "modif_spring\tid\t2\tstiffness\t7.5"])
    r, info, skin = files.read_input(path, strict=True)
    assert r.settings.dt == m.settings.dt  # the first 'step' line is read
    assert r.mass[3] == 0.0 and r.mass[4] == m.mass[4]
    assert np.all(r.vel[r.tag == 1] == [1.0, 2.0, 3.0]) and np.all(r.vel_old[r.tag == 1] == [1.0, 2.0, 3.0])
    assert info["has_skin_override"] == 1 and np.all(skin == 0.75)
    assert r.s_k[2] == 7.5


@pytest.mark.parametrize("edit,msg", [
    (lambda t: t.replace("run\t20", "run\t-1"), "run"),
    (lambda t: t.replace("output_freq\t10", "output_freq\t50"), "output_freq"),
    (lambda t: "\n".join(ln for ln in t.splitlines() if not ln.startswith("pair")), "pair"),
    (lambda t: t.replace("box_unit_cell\t1.0", "box_unit_cell\t5.0"), "three unit cells"),
    (lambda t: t.replace("model.txt", "missing.txt"), "unable to open model"),
    (lambda t: t + "\npair\tlj\tC1\tC1\t1.0\n", "tokens"),
    (lambda t: t + "\ntype\tC1\n", "redefined"),
])
def test_input_errors(tmp, edit, msg):
    path = write(net(), tmp)
    text = edit(open(path).read())
    open(path, "w").write(text)
    with pytest.raises(files.InputError, match=msg):
        files.read_input(path)


def test_model_errors(tmp):
    m = net()
    path = write(m, tmp)
    lines = open(tmp / "model.txt").read().splitlines()
    bad = lines[:]
    f = bad[0].split("\t")
    f[6] = "99.0"  # outside the 12-wide box
    bad[0] = "\t".join(f)
    open(tmp / "model.txt", "w").write("\n".join(bad))
    with pytest.raises(files.InputError, match="outside"):
        files.read_input(path)
    bad = lines + ["SPRING\tHR\t0\t0\t9999\t1.0\t1.0"]
    open(tmp / "model.txt", "w").write("\n".join(bad))
    with pytest.raises(files.InputError, match="missing bead"):
        files.read_input(path)


def test_restart_file_is_read(tmp):
    m = net()
    rng = np.random.default_rng(1)
    pos = m.pos + rng.uniform(0, 0.1, m.pos.shape)
    vel = rng.normal(size=m.pos.shape)
    with open(tmp / "r.res", "w") as fh:
        fh.write(f"{m.n_beads}\nFRAME\t100\t0.001\t12\t12\t6\n")
        for i in range(m.n_beads):
            vals = list(pos[i]) + list(pos[i] + 1) + list(vel[i]) + [0.0, 0.0, 0.0]
            fh.write("\t" + m.type_names[m.type[i]] + "\t" + "\t".join(repr(float(v)) for v in vals) + "\n")
    path = write(m, tmp, extra_lines=["restart_file\tr.res", "restart_data\tall"])
    r, _, _ = files.read_input(path, strict=True)
    np.testing.assert_array_equal(r.pos, pos)
    np.testing.assert_array_equal(r.img, pos + 1)
    np.testing.assert_array_equal(r.vel_old, vel)


def test_hsr_pair_keyword_round_trip(tmp):
    """The penalty + soft-repulsion kind (an extension, 'pair hsr T1 T2 K k rc')."""
    m = g.dense_mat(fibres=6, beads=8, box=(12.0, 12.0, 12.0))
    r, _, _ = files.read_input(write(m, tmp), strict=True)
    assert r.pair_kind.tolist() == [4]
    np.testing.assert_array_equal(r.pair_raw[0, :3], [100.0, 10.0, 1.2])
