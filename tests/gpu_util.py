"""Helpers shared by the GPU tests."""
import numpy as np

FIELDS = ["pos", "img", "vel", "force", "vel_old"]


def run_seq(sim, runs):
    for n in runs:
        n = int(n)
        if n < 0:
            sim.reset_energy()
        else:
            sim.run(n) if hasattr(sim, "run") else sim.step(n)


def rel_norm(a, b):
    d = np.linalg.norm(np.asarray(a) - np.asarray(b))
    n = np.linalg.norm(np.asarray(b))
    return d / n if n > 0 else d
