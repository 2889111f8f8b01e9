"""Trajectory of the FP32-state GPU path against the FP64 reference (the
oracle's REF mode, bit-identical to the reference's kernels on the golden
cases) over 1,000 steps, reported chunk by chunk: config 0 (200 fibres x 50
beads, penalty contacts) and a small tensile pull with breakable springs in
a box periodic in y only (REF mode wraps the reference's half-shell table
per axis for such boxes)."""
import numpy as np
import pytest

import pyoracle as po
from fibrenet_b200 import generate as g

pytestmark = pytest.mark.gpu


def divergence(m, chunks, chunk_steps):
    from fibrenet_b200.native import Simulation
    m = m.fp32_representable()
    s = Simulation(m, list_capacity=64)
    r = po.OracleSim(m, po.MODE_REF)
    rows = []
    for k in range(chunks):
        s.step(chunk_steps)
        r.run(chunk_steps)
        dimg = np.abs(s.get("img") - r.get("img")).max()
        f_ref = r.get("force")
        frel = np.linalg.norm(s.get("force") - f_ref) / max(np.linalg.norm(f_ref), 1e-300)
        sg, _ = s.status()
        sr, _ = r.status()
        rows.append((chunk_steps * (k + 1), float(dimg), float(frel), int((sg != sr).sum()),
                     int((sr == 0).sum())))
    s.close()
    return rows


def test_config0_follows_fp64_reference():
    m = g.plain_network(seed=0)
    rows = divergence(m, 10, 100)
    for step, dimg, frel, nflip, nbroken in rows:
        print(f"config0 step {step:5d}  max|d img| {dimg:.3e}  force rel {frel:.3e}")
    # positions stay within FP32 storage rounding of the FP64 run; forces after
    # 100 steps of rounding drift stay within a few 1e-5
    assert max(r[1] for r in rows) < 1e-4
    assert max(r[2] for r in rows) < 5e-5


def test_tensile_pull_follows_fp64_reference():
    """Half of the springs fail during the pull; the FP32-state run breaks
    exactly the springs the FP64 run breaks, step for step, and stays within
    rounding of it."""
    m = g.tensile_network(seed=3, fibres=60, beads=30, box=(60.0, 40.0, 10.0), z_range=(1.0, 9.0),
                          fail_mu=np.log(0.8), fail_sigma=0.4, clamp_lo=2.0, clamp_hi=58.0,
                          pull=0.5, cell=2.5, min_sep=1.0)
    rows = divergence(m, 50, 20)
    for step, dimg, frel, nflip, nbroken in rows[4::5]:
        print(f"tensile step {step:5d}  max|d img| {dimg:.3e}  force rel {frel:.3e}  "
              f"status differences {nflip} of {nbroken} broken")
    assert rows[-1][4] > 500  # the pull breaks springs
    assert all(r[3] == 0 for r in rows)
    assert max(r[1] for r in rows) < 1e-4
    assert max(r[2] for r in rows) < 1e-4
