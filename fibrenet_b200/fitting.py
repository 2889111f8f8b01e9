"""Fitting binding: the reaction-force curve of a tensile pull as a
differentiable function of the bond parameters, for torch optimisers.

Forward and backward both run on the device through the C ABI
(fn_adjoint_forward / fn_adjoint_backward, include/fibrenet.h); torch only
carries the tensors.  No counterpart in the reference.
"""
from __future__ import annotations

import numpy as np
import torch

from .model import Model
from .native import Simulation


class ReactionCurve:
    """A device context holding one or more networks and their starting state.

    ``curve(spring_k, spring_rest, angle_k, pos0=None)`` restores the starting
    state, loads the parameters (per spring / per angle in upload order,
    concatenated over the networks; ``pos0`` per bead [n, 3] or None), runs
    ``nsamples`` calls of ``every`` steps and returns the reaction of every
    network after each call, a float64 tensor [nsamples, n_networks, 3]
    whose backward runs the adjoint.
    """

    def __init__(self, models, nsamples: int, every: int, checkpoint_every: int,
                 reaction_type: int, **sim_kw):
        self.models = [models] if isinstance(models, Model) else list(models)
        sim_kw.setdefault("list_capacity", 64)
        self.sim = Simulation(self.models, **sim_kw)
        self.nsamples, self.every = nsamples, every
        self.checkpoint_every, self.reaction_type = checkpoint_every, reaction_type
        norm = [m.normalised() for m in self.models]
        cat = lambda f: np.concatenate([np.asarray(getattr(m, f), np.float64) for m in norm])  # noqa: E731
        self.start = {f: cat(f) for f in ("pos", "img", "vel", "vel_old", "force")}
        self.spring_status = np.ones(self.sim.ns, np.int32)
        self.angle_status = np.ones(self.sim.na, np.int32)
        self.params = {"spring_k": cat("s_k"), "spring_rest": cat("s_rest"), "angle_k": cat("a_k"),
                       "angle_theta0": cat("a_theta0"), "spring_c1": cat("s_c1"),
                       "spring_c2": cat("s_c2")}

    def close(self):
        self.sim.close()

    def _load(self, spring_k, spring_rest, angle_k, pos0):
        s = self.sim
        for f in ("vel", "vel_old", "force"):
            s.set(f, self.start[f])
        if pos0 is None:
            s.set("pos", self.start["pos"])
            s.set("img", self.start["img"])
        else:
            p0 = np.asarray(pos0, np.float64).reshape(-1, 3)
            s.set("img", p0)
            s.set("pos", self.start["pos"] + (p0 - self.start["img"]))
        s.set_status(self.spring_status, self.angle_status)
        s.set_springs(rest=np.asarray(spring_rest, np.float64), k=np.asarray(spring_k, np.float64),
                      c1=self.params["spring_c1"], c2=self.params["spring_c2"])
        s.set_angles(theta0=self.params["angle_theta0"], k=np.asarray(angle_k, np.float64))

    def run(self, spring_k, spring_rest, angle_k, pos0=None) -> np.ndarray:
        """Forward only (numpy in, numpy out)."""
        self._load(spring_k, spring_rest, angle_k, pos0)
        return self.sim.adjoint_forward(self.nsamples, self.every, self.checkpoint_every,
                                        self.reaction_type)

    def __call__(self, spring_k, spring_rest, angle_k, pos0=None):
        if pos0 is None:
            pos0 = torch.as_tensor(self.start["img"])
        return _Reaction.apply(spring_k, spring_rest, angle_k, pos0, self)


def _np(t):
    return t.detach().cpu().double().numpy()


class _Reaction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, spring_k, spring_rest, angle_k, pos0, curve: ReactionCurve):
        R = curve.run(_np(spring_k), _np(spring_rest), _np(angle_k), _np(pos0))
        ctx.curve = curve
        ctx.dev = spring_k.device
        return torch.from_numpy(R).to(ctx.dev)

    @staticmethod
    def backward(ctx, grad_r):
        g = ctx.curve.sim.adjoint_backward(_np(grad_r))
        t = lambda a: torch.from_numpy(a).to(ctx.dev)  # noqa: E731
        return t(g["spring_k"]), t(g["spring_rest"]), t(g["angle_k"]), t(g["pos0"]), None
