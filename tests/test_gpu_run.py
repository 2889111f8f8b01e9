"""The reference's Initialize/Run/Close flow (fn_run_input) on reference-format
files: minimisation with energy resets, RunSimulationLoop in output_freq
chunks, XYZ frames per chunk, restart files; checked against stepping the
same model directly through the C ABI and against the FP64 reference."""
import os
import subprocess
import sys

import numpy as np
import pytest

import pyoracle as po
from fibrenet_b200 import files
from fibrenet_b200 import generate as g

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def model():
    m = g.plain_network(seed=41, fibres=20, beads=15, box=(16.0, 16.0, 6.0), z_range=(1.0, 5.0))
    m.vel = np.random.default_rng(2).normal(0.0, 0.2, m.vel.shape).astype(np.float32).astype(np.float64)
    m.vel_old = m.vel.copy()
    return m


def read_res(path):
    lines = open(path).read().splitlines()
    rows = [ln.split() for ln in lines[2:]]
    return np.array([[float(x) for x in r[1:]] for r in rows])


@pytest.mark.parametrize("minimize", [None, (20, 10, True)])
def test_run_flow_matches_direct_stepping(tmp_path, monkeypatch, minimize):
    from fibrenet_b200.native import Simulation
    monkeypatch.chdir(tmp_path)
    m = model()
    files.write_model_file(m, "model.txt")
    files.write_input_file(m, "in.txt", "model.txt", "out", run=45, output_freq=10,
                           output_data=("all",), minimize=minimize)
    files.run_input("in.txt", strict=True)
    frames = files.read_xyz("out_coord.xyz")
    assert [f[0] for f in frames] == [0, 10, 20, 30, 40, 45]
    assert len(files.read_xyz("out_vel.xyz")) == 6 and len(files.read_xyz("out_force.xyz")) == 6
    res = read_res("out_restart.res")

    parsed, _, _ = files.read_input("in.txt", strict=True)
    with Simulation(parsed, list_capacity=128) as s:
        if minimize:
            s.reset_energy()
            for _ in range(minimize[0] // minimize[1]):
                s.step(minimize[1])
                s.reset_energy()
        for chunk in [10, 10, 10, 10, 5]:
            s.step(chunk)
        pos, img, vel, frc = s.get("pos"), s.get("img"), s.get("vel"), s.get("force")
    np.testing.assert_array_equal(res[:, 0:3], pos)
    np.testing.assert_array_equal(res[:, 3:6], img)
    np.testing.assert_array_equal(res[:, 6:9], vel)
    np.testing.assert_array_equal(res[:, 9:12], frc)
    np.testing.assert_allclose(frames[-1][2], pos, atol=6e-6)  # 5 decimals

    # the FP64 reference with the same schedule
    r = po.OracleSim(parsed.fp32_representable(), po.MODE_REF)
    if minimize:
        r.reset_energy()
        for _ in range(minimize[0] // minimize[1]):
            r.run(minimize[1])
            r.reset_energy()
    for chunk in [10, 10, 10, 10, 5]:
        r.run(chunk)
    np.testing.assert_allclose(img, r.get("img"), atol=1e-4)


def test_compat_restart_format_and_cli(tmp_path, monkeypatch):
    """Compat restarts are written like the reference's default stream (6
    significant digits) and are read back by the same parser; the command-line
    runner returns 0."""
    monkeypatch.chdir(tmp_path)
    m = model()
    files.write_model_file(m, "model.txt")
    files.write_input_file(m, "in.txt", "model.txt", "out", run=30, output_freq=10)
    exe = os.path.join(ROOT, "fibrenet_b200", "fibrenet_run")
    r = subprocess.run([exe, "in.txt"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    line = open("out_restart.res").read().splitlines()[2].split()
    assert all(len(x.replace("-", "").replace(".", "").lstrip("0")) <= 6 for x in line[1:] if "e" not in x)
    files.write_input_file(m, "in2.txt", "model.txt", "out2", run=10, output_freq=10,
                           extra_lines=["restart_file\tout_restart.res", "restart_data\tall"])
    r2, _, _ = files.read_input("in2.txt")
    assert r2.n_beads == m.n_beads
    r = subprocess.run([sys.executable, "-m", "fibrenet_b200.cli", "in2.txt"], capture_output=True,
                       text=True, cwd=str(tmp_path), env=dict(os.environ, PYTHONPATH=ROOT))
    assert r.returncode == 0, r.stderr
    assert os.path.exists("out2_restart.res")
