"""Adjoint of the step loop (fn_adjoint_forward / fn_adjoint_backward) and
its torch binding.

CPU: the FP64 torch statement of the loop (tests/adjoint_ref.py), whose
autograd gradient is the reference gradient, follows the oracle's FP64
restatement of the reference kernels step for step.
GPU: the device gradients of a tensile pull's reaction curve with respect to
spring stiffness / rest length, angle stiffness and the starting positions
and velocities match the FP64 reference gradient and central finite
differences to 1e-3 (relative, norm-wise); batched networks give the same
gradients as single ones; the state after the backward sweep is the state
after the forward pass; a torch optimiser drives the loss down through the
binding.
"""
import numpy as np
import pytest
import torch

import adjoint_ref as ar
from fibrenet_b200 import generate as g
from fibrenet_b200.model import SPRING_HR

CL, CR = 1, 2  # clamp types of the tensile generator (C1, CL, CR)


def pull(seed=5, fibres=24, beads=10, vel_sigma=0.05):
    m = g.tensile_network(seed=seed, fibres=fibres, beads=beads, box=(24.0, 16.0, 8.0),
                          z_range=(2.0, 6.0), clamp_lo=2.0, clamp_hi=22.0, min_sep=0.95, pull=0.5,
                          dt=0.001)
    m.s_type[:] = SPRING_HR
    m = m.fp32_representable()
    rng = np.random.default_rng(seed + 100)
    free = np.asarray(m.mass) > 0
    v = np.where(free[:, None], rng.normal(0.0, vel_sigma, m.vel.shape), m.vel)
    m.vel = v.astype(np.float32).astype(np.float64)
    m.vel_old = m.vel.copy()
    return m


def ref_grads(m, nsamples, every, weights):
    r = ar.RefLoop(m)
    k_s = torch.tensor(np.asarray(m.s_k, np.float32).astype(np.float64), requires_grad=True)
    rest = torch.tensor(np.asarray(m.s_rest, np.float32).astype(np.float64), requires_grad=True)
    k_a = torch.tensor(np.asarray(m.a_k, np.float32).astype(np.float64), requires_grad=True)
    x0 = torch.tensor(np.asarray(m.img), dtype=torch.float64, requires_grad=True)
    v0 = torch.tensor(np.asarray(m.vel_old), dtype=torch.float64, requires_grad=True)
    R = r.run(nsamples, every, CR, k_s, rest, k_a, x0, v0)
    (R * torch.tensor(weights)).sum().backward()
    return R.detach().numpy(), {"spring_k": k_s.grad.numpy(), "spring_rest": rest.grad.numpy(),
                                "angle_k": k_a.grad.numpy(), "pos0": x0.grad.numpy(),
                                "vel0": v0.grad.numpy()}


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def test_reference_loop_follows_oracle(oracle_built):
    po = oracle_built
    m = pull()
    r = ar.RefLoop(m)
    f32 = lambda a: torch.tensor(np.asarray(a, np.float32).astype(np.float64))  # noqa: E731
    o = po.OracleSim(m, po.MODE_REF)
    with torch.no_grad():
        R = r.run(3, 20, CR, f32(m.s_k), f32(m.s_rest), f32(m.a_k)).numpy()
    types = np.asarray(m.type)
    for s in range(3):
        o.run(20)
        Ro = o.get("force")[types == CR].sum(0)
        np.testing.assert_allclose(R[s], Ro, rtol=1e-9, atol=1e-9)
    assert np.abs(R).max() > 1.0


def test_reference_gradient_matches_finite_differences():
    """The FP64 reference gradient against central differences, h = 1e-3
    relative, on 32 random parameters of each kind (one at a time)."""
    m = pull(seed=9)
    ns, every = 4, 20
    w = np.random.default_rng(5).normal(size=(ns, 3))
    _, gr = ref_grads(m, ns, every, w)
    r = ar.RefLoop(m)
    base = {"spring_k": np.asarray(m.s_k, np.float32).astype(np.float64),
            "spring_rest": np.asarray(m.s_rest, np.float32).astype(np.float64),
            "angle_k": np.asarray(m.a_k, np.float32).astype(np.float64)}
    rng = np.random.default_rng(6)

    def loss(p):
        with torch.no_grad():
            R = r.run(ns, every, CR, torch.tensor(p["spring_k"]), torch.tensor(p["spring_rest"]),
                      torch.tensor(p["angle_k"]))
        return float((R.numpy() * w).sum())

    for key in base:
        idx = rng.choice(len(base[key]), 32, replace=False)
        fd = np.zeros(32)
        for q, i in enumerate(idx):
            h = 1e-3 * base[key][i]
            up = {k: v.copy() for k, v in base.items()}
            dn = {k: v.copy() for k, v in base.items()}
            up[key][i] += h
            dn[key][i] -= h
            fd[q] = (loss(up) - loss(dn)) / (2 * h)
        assert rel(gr[key][idx], fd) < 1e-3, (key, rel(gr[key][idx], fd))


# ---------------------------------------------------------------- GPU

def gpu_grads(models, nsamples, every, ckpt, weights, **kw):
    from fibrenet_b200.native import Simulation
    kw.setdefault("list_capacity", 64)
    with Simulation(models, **kw) as s:
        R = s.adjoint_forward(nsamples, every, ckpt, CR)
        gr = s.adjoint_backward(weights)
    return R, gr


@pytest.mark.gpu
@pytest.mark.parametrize("chain", [True, False])
def test_gradients_match_fp64_reference(chain):
    m = pull()
    ns, every = 8, 20
    w = np.random.default_rng(1).normal(size=(ns, 1, 3))
    R, gg = gpu_grads(m, ns, every, 40, w, chain=chain)
    Rr, gr = ref_grads(m, ns, every, w[:, 0, :])
    np.testing.assert_allclose(R[:, 0, :], Rr, rtol=1e-4, atol=1e-4 * np.abs(Rr).max())
    for k in ("spring_k", "spring_rest", "angle_k", "pos0", "vel0"):
        assert rel(gg[k], gr[k]) < 1e-3, (k, rel(gg[k], gr[k]))
        assert np.linalg.norm(gr[k]) > 0, k


@pytest.mark.gpu
def test_directional_finite_differences():
    """Device gradient against central differences of the device forward
    along random directions of 32 random parameters of each kind.  The
    forward keeps velocities and forces in FP32, so the step is h = 1e-2
    relative and the bound 5e-3 (the FP64 reference above is checked at
    1e-3 with h = 1e-3)."""
    from fibrenet_b200.fitting import ReactionCurve
    m = pull(seed=7)
    ns, every = 8, 20
    w = np.random.default_rng(2).normal(size=(ns, 1, 3))
    curve = ReactionCurve(m, ns, every, 40, CR)
    p0 = {k: curve.params[k].copy() for k in ("spring_k", "spring_rest", "angle_k")}
    curve.run(p0["spring_k"], p0["spring_rest"], p0["angle_k"])
    grad = curve.sim.adjoint_backward(w)
    rng = np.random.default_rng(3)
    for key in ("spring_k", "spring_rest", "angle_k"):
        idx = rng.choice(len(p0[key]), 32, replace=False)
        d = np.zeros_like(p0[key])
        d[idx] = rng.normal(size=32) * p0[key][idx] * 1e-2

        def loss(sign):
            p = {k: v.copy() for k, v in p0.items()}
            p[key] = p[key] + sign * d
            return float((curve.run(p["spring_k"], p["spring_rest"], p["angle_k"]) * w).sum())

        fd = (loss(1.0) - loss(-1.0)) / 2.0
        an = float(grad[key] @ d)
        assert abs(fd - an) <= 5e-3 * abs(an), (key, fd, an)
    curve.close()


@pytest.mark.gpu
def test_straight_start_stays_bounded():
    """Fibres that start straight at rest (the fitting networks): the angle
    Jacobian is taken in its regular form, so the position gradients stay
    bounded and the stiffness gradient follows central differences."""
    from fibrenet_b200.fitting import ReactionCurve
    m = pull(seed=41, vel_sigma=0.0)
    ns, every = 8, 20
    curve = ReactionCurve(m, ns, every, 40, CR)
    k0, r0, a0 = (curve.params[k].copy() for k in ("spring_k", "spring_rest", "angle_k"))
    R = curve.run(k0, r0, a0)
    w = np.zeros_like(R)
    w[..., 0] = 1.0
    gr = curve.sim.adjoint_backward(w)
    assert np.all(np.isfinite(gr["pos0"])) and np.abs(gr["pos0"]).max() < 1e6
    d = k0 * 1e-2
    fd = float(((curve.run(k0 + d, r0, a0) - curve.run(k0 - d, r0, a0)) * w).sum()) / 2.0
    an = float(gr["spring_k"] @ d)
    assert abs(fd - an) <= 1e-2 * abs(an), (fd, an)
    curve.close()


@pytest.mark.gpu
def test_batched_gradients_equal_single():
    ms = [pull(seed=s) for s in (11, 12, 13)]
    ns, every = 4, 20
    w = np.random.default_rng(4).normal(size=(ns, 3, 3))
    Rb, gb = gpu_grads(ms, ns, every, 40, w)
    s0 = b0 = a0 = 0
    for k, m in enumerate(ms):
        R1, g1 = gpu_grads(m, ns, every, 40, w[:, k:k + 1, :])
        np.testing.assert_array_equal(Rb[:, k, :], R1[:, 0, :])
        np.testing.assert_array_equal(gb["spring_k"][s0:s0 + m.n_springs], g1["spring_k"])
        np.testing.assert_array_equal(gb["angle_k"][a0:a0 + m.n_angles], g1["angle_k"])
        np.testing.assert_array_equal(gb["pos0"][b0:b0 + m.n_beads], g1["pos0"])
        s0 += m.n_springs
        a0 += m.n_angles
        b0 += m.n_beads


@pytest.mark.gpu
def test_state_after_backward_is_forward_end_state():
    from fibrenet_b200.native import NativeError, Simulation
    m = pull(seed=21)
    with Simulation(m, list_capacity=64) as a, Simulation(m, list_capacity=64) as b:
        a.adjoint_forward(4, 20, 40, CR)
        b.adjoint_forward(4, 20, 40, CR)
        a.adjoint_backward(np.ones((4, 1, 3)))
        for f in ("pos", "img", "vel", "vel_old", "force"):
            np.testing.assert_array_equal(a.get(f), b.get(f), err_msg=f)
        a.step(30)
        b.step(30)
        np.testing.assert_array_equal(a.get("img"), b.get("img"))
        with pytest.raises(NativeError, match="no forward pass"):
            a.adjoint_backward(np.ones((4, 1, 3)))


@pytest.mark.gpu
def test_torch_binding_fits_stiffness():
    """Recover a uniform stiffness scale from a target curve with Adam."""
    from fibrenet_b200.fitting import ReactionCurve
    m = pull(seed=31)
    ns, every = 6, 20
    curve = ReactionCurve(m, ns, every, 60, CR)
    k0 = torch.tensor(curve.params["spring_k"])
    rest = torch.tensor(curve.params["spring_rest"])
    ka = torch.tensor(curve.params["angle_k"])
    with torch.no_grad():
        target = curve(k0 * 1.3, rest, ka)
    scale = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([scale], lr=0.05)
    losses = []
    for _ in range(25):
        opt.zero_grad()
        R = curve(k0 * scale, rest, ka)
        loss = ((R - target) ** 2).sum()
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    curve.close()
    assert losses[-1] < 0.05 * losses[0]
    assert abs(float(scale.detach()) - 1.3) < 0.05
