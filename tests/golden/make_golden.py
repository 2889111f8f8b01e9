"""Generates the golden vectors in this folder from the reference itself.

The reference ships no tests or fixtures, so its own kernels are the only
source of truth: FibreNet/kernel.cl, compiled unmodified as C through
oracle/cl_shim.h into oracle/_ref/libfnref.so, run on one thread (ascending
work-item order makes its atomics deterministic).  Each case is a small
model built from explicit records or the seeded generator, a sequence of
RunSimulationLoop calls, and the resulting state, bond statuses, grid buckets
and contact-list pair set.

Run here, where the reference tree exists:
    python tests/golden/make_golden.py
It rewrites tests/golden/*.npz.  The committed files are what the tests read
on any machine.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402
from fibrenet_b200 import generate as g  # noqa: E402
from fibrenet_b200.model import (ANGLE_HR, ANGLE_HR_FL, PAIR_HS, PAIR_LJ, PAIR_ST, SPRING_HR,  # noqa: E402
                                 SPRING_HR_FL, Settings, model_to_arrays)

PI = g.PI_F32


def bead(t, tag, loc, pos, vel=(0.0, 0.0, 0.0), radius=0.5, mass=1.0, img=None):
    return (t, tag, loc, radius, mass, pos, vel, img if img is not None else pos)


def cases():
    out = {}
    pbc10 = Settings(dt=0.001, lam=0.5, box=(10.0, 10.0, 10.0), box_unit_cell=1.0, cutoff=1.0,
                     bc_type=0, wall_k=0.0)
    hs0 = {(0, 0): (PAIR_HS, [0.0])}

    out["spring_pair"] = (g.explicit_model(
        pbc10, ["A"], hs0,
        [bead(0, 0, 0, (4.0, 5.0, 5.0)), bead(0, 0, 1, (5.25, 5.0, 5.0), vel=(0.0, 0.5, 0.0))],
        springs=[(SPRING_HR, 0, 0, 1, 1.0, 100.0, 0.0, 0.0)]), [10])

    out["angle_triple"] = (g.explicit_model(
        pbc10, ["A"], hs0,
        [bead(0, 0, 0, (4.0, 5.0, 5.0)), bead(0, 0, 1, (5.0, 5.0, 5.0)),
         bead(0, 0, 2, (5.0, 6.0, 5.0))],
        springs=[(SPRING_HR, 0, 0, 1, 1.0, 100.0, 0.0, 0.0), (SPRING_HR, 0, 1, 2, 1.0, 100.0, 0.0, 0.0)],
        angles=[(ANGLE_HR, 0, 0, 1, 2, 0, 1, PI, 10.0)]), [10])

    out["hrfl_break"] = (g.explicit_model(
        pbc10, ["A"], hs0,
        [bead(0, 0, 0, (2.0, 5.0, 5.0)), bead(0, 0, 1, (3.0, 5.0, 5.0)),
         bead(0, 0, 2, (4.03125, 5.0, 5.0)), bead(0, 0, 3, (5.03125, 5.0, 5.0)),
         bead(0, 0, 4, (6.03125, 5.0, 5.0))],
        springs=[(SPRING_HR_FL, 0, 0, 1, 1.0, 100.0, 1000.0, 5.0),
                 (SPRING_HR_FL, 0, 1, 2, 1.0, 100.0, 1000.0, 5.0),
                 (SPRING_HR_FL, 0, 2, 3, 1.0, 100.0, 1000.0, 5.0),
                 (SPRING_HR, 0, 3, 4, 1.0, 100.0, 0.0, 0.0)],
        angles=[(ANGLE_HR_FL, 0, 0, 1, 2, 0, 1, PI, 10.0), (ANGLE_HR, 0, 1, 2, 3, 1, 2, PI, 10.0),
                (ANGLE_HR_FL, 0, 2, 3, 4, 2, 3, PI, 10.0)]), [5])

    lj = Settings(dt=0.0005, lam=0.5, box=(10.0, 10.0, 10.0), box_unit_cell=2.5, cutoff=2.5,
                  bc_type=0, wall_k=0.0)
    out["lj_pair"] = (g.explicit_model(
        lj, ["A"], {(0, 0): (PAIR_LJ, [1.0, 1.0, 2.5])},
        [bead(0, 0, 0, (4.0, 5.0, 5.0)), bead(0, 1, 0, (5.0625, 5.0, 5.0))]), [20])

    out["hs_pair"] = (g.explicit_model(
        pbc10, ["A"], {(0, 0): (PAIR_HS, [50.0])},
        [bead(0, 0, 0, (4.5, 5.0, 5.0)), bead(0, 1, 0, (5.25, 5.125, 5.0))]), [20])

    st = Settings(dt=0.0005, lam=0.5, box=(10.0, 10.0, 10.0), box_unit_cell=1.25, cutoff=1.2,
                  bc_type=0, wall_k=0.0)
    out["st_pair"] = (g.explicit_model(
        st, ["A"], {(0, 0): (PAIR_ST, [2000.0, 500.0, 1.0, 1.03])},
        [bead(0, 0, 0, (4.0, 5.0, 5.0)), bead(0, 1, 0, (5.0078125, 5.0, 5.0))]), [20])

    out["pbc_wrap"] = (g.explicit_model(
        pbc10, ["A"], {(0, 0): (PAIR_HS, [50.0])},
        [bead(0, 0, 0, (9.998046875, 5.0, 5.0), vel=(1.0, 0.0, 0.0)),
         bead(0, 1, 0, (0.001953125, 5.5, 5.0), vel=(-1.0, 0.0, 0.0)),
         bead(0, 2, 0, (5.0, 9.9990234375, 0.0009765625), vel=(0.0, 1.0, -1.0)),
         bead(0, 3, 0, (0.5, 0.5, 0.5))]), [2, 3])

    fin = Settings(dt=0.001, lam=0.5, box=(10.0, 10.0, 10.0), box_unit_cell=1.0, cutoff=1.0,
                   bc_type=1, wall_k=100.0)
    out["finite_wall"] = (g.explicit_model(
        fin, ["A"], {(0, 0): (PAIR_HS, [50.0])},
        [bead(0, 0, 0, (0.0009765625, 5.0, 5.0), vel=(-1.0, 0.0, 0.0)),
         bead(0, 1, 0, (5.0, 9.9990234375, 5.0), vel=(0.0, 1.0, 0.0)),
         bead(0, 2, 0, (0.25, 0.25, 0.25)), bead(0, 3, 0, (0.75, 0.25, 0.25))]), [10])

    net = g.plain_network(seed=5, fibres=20, beads=20, box=(20.0, 20.0, 6.0), z_range=(1.0, 5.0))
    out["net_pbc_hs"] = (net, [50])

    tn = g.tensile_network(seed=7, fibres=16, beads=16, box=(30.0, 30.0, 8.0), z_range=(1.0, 7.0),
                           fail_mu=np.log(0.3), fail_sigma=0.5, clamp_lo=2.0, clamp_hi=28.0,
                           pull=1.0, wall_k=100.0, min_sep=1.0)
    tn.settings.periodic_mask = -1
    tn.settings.bc_type = 1
    out["net_finite_lj_hrfl"] = (tn, [30, 30])

    mt = g.plain_network(seed=11, fibres=12, beads=12, box=(15.0, 15.0, 6.0), z_range=(1.0, 5.0))
    mt.type_names = ["C1", "C2"]
    mt.type = (mt.tag % 2).astype(np.int32)
    mt.pair_kind = np.array([PAIR_HS, PAIR_ST, PAIR_LJ], np.int32)
    mt.pair_raw = np.array([[50.0, 0, 0, 0], [2000.0, 500.0, 1.0, 1.03], [1.0, 0.25, 1.2, 0]])
    mt.settings.cutoff = 1.2
    mt.settings.box_unit_cell = 1.25
    mt.settings.dt = 0.0005
    out["net_multitype"] = (mt, [7, 9, 16])

    dg = g.plain_network(seed=13, fibres=10, beads=10, box=(12.0, 12.0, 6.0), z_range=(1.0, 5.0))
    dg.settings.damping = 0.5
    dg.settings.gravity = (0.0, 0.0, -1.0)
    dg.settings.grid_update_freq = 3
    out["damping_gravity"] = (dg, [20])
    return out


def run_case(model, runs):
    m = model.fp32_representable()
    r = po.RefSim(m, threads=1)
    for n in runs:
        if n == "reset":
            r.reset_energy()
        else:
            r.run(int(n))
    res = {f"out_{f}": r.get(f) for f in po.FIELD}
    s, a = r.status()
    res["out_spring_status"] = s
    res["out_angle_status"] = a
    r.rebuild()
    head, tail = r.grid()
    cells = []
    for c in range(head.shape[0]):
        for k in range(min(int(head[c]), 64)):
            cells.append((c, int(tail[c, k])))
    res["out_grid"] = np.array(sorted(cells), np.int32).reshape(-1, 2)
    res["out_grid_head"] = head
    lh, lt, lp = r.lists()
    res["out_list_head"] = lh
    res["out_pairs"] = np.array(sorted(po.pair_set(lh, lt, lp)), np.int32).reshape(-1, 3)
    res["runs"] = np.array([-1 if n == "reset" else int(n) for n in runs], np.int64)
    res.update(model_to_arrays(m))
    return res


def main():
    po.build()
    cs = cases()
    cs["minimize_reset"] = (g.plain_network(seed=17, fibres=10, beads=10, box=(12.0, 12.0, 6.0),
                                            z_range=(1.0, 5.0)), [6, "reset", 6])
    for name, (model, runs) in cs.items():
        res = run_case(model, runs)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **res)
        print(f"{name}: beads={model.n_beads} pairs={len(res['out_pairs'])} "
              f"broken={int((res['out_spring_status'] == 0).sum())} -> {os.path.basename(path)}")


if __name__ == "__main__":
    main()
