"""A fixed, short run of the benchmark networks for a profiler to attach to.

    python -m fibrenet_b200.profile_run [--network tensile|dense|plain] [--block B]
        [--items-per-thread K] [--list-build beads|bricks|groups] [--steps N] [--observe]

Builds the seeded network (the 1,000,000-bead tensile test, the 4M-bead
dense mat or the 10,000-bead plain network of 200 fibres with penalty
contacts), fixes the step kernel's shape and the list build (no autotuning,
so the launch sequence is the same on every run), runs one fn_step(N) call
and, with --observe, the observables and the energy once.  The launches are
an upload, one drift, ceil(N / 8) rebuilds and N step kernels.
"""
from __future__ import annotations

import argparse


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--network", choices=["tensile", "dense", "plain"], default="tensile")
    p.add_argument("--block", type=int, default=128)
    p.add_argument("--items-per-thread", type=int, default=0)
    p.add_argument("--list-build", choices=["beads", "bricks", "groups"], default="beads")
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--observe", action="store_true")
    a = p.parse_args(argv)
    from . import generate as g
    from .native import Simulation
    if a.network == "tensile":
        m = g.tensile_network(seed=1)
    elif a.network == "dense":
        m = g.dense_mat(seed=2)
    else:
        m = g.plain_network(seed=0)
    with Simulation(m, list_capacity=64, cell_capacity=64, reorder=True) as s:
        s.set_kernel_shape(a.block, a.items_per_thread)
        s.set_list_build(a.list_build)
        s.step(a.steps)
        s.sync()
        st = s.stats()
        print(f"{m.n_beads} beads, {a.steps} steps, block {st['block_size']}, items per thread "
              f"{st['items_per_thread']}, list build {a.list_build}")
        if a.observe:
            print(s.observe(0, reaction_type=2 if m.n_types > 2 else -1))
            print(s.energy(0)["total"])


if __name__ == "__main__":
    main()
