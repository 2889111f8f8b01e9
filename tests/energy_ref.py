"""FP64 numpy statement of the energy / virial definitions of fn_energy_eval
(include/fibrenet.h), used to check the device reduction.  The potentials are
the ones whose negative gradients are the reference's forces (kernel.cl:195-261
walls and gravity, :366-441 springs, :268-363 angles, :792-1011 contacts);
tests/test_energy.py checks that against the oracle's forces by finite
differences."""
import numpy as np

from fibrenet_b200.model import PAIR_HS, PAIR_HSR, PAIR_LJ, PAIR_ST, pair_index


def _min_image(r, box, mask, half_box_sq):
    r = r.copy()
    l2 = (r * r).sum(-1)
    far = l2 > half_box_sq
    for a in range(3):
        if mask >> a & 1:
            sel = far & (r[:, a] ** 2 > half_box_sq)
            r[sel, a] = np.where(r[sel, a] > 0, r[sel, a] - box[a], r[sel, a] + box[a])
    return r


def pair_coeffs(kind, raw):
    """The c1..c6 derivation of SimulationManager.cpp:891-932 (+ hsr)."""
    c = np.zeros(6)
    if kind == PAIR_LJ:
        c[:3] = raw[:3]
        r2 = c[2] * c[2]
        fr2 = c[0] * c[0] / r2
        fr6 = fr2 ** 3
        c[3] = 48.0 * c[1] * fr6 * (fr6 - 0.5) / r2
    elif kind in (PAIR_HS,):
        c[0] = raw[0]
    elif kind == PAIR_HSR:
        c[:3] = raw[:3]
    elif kind == PAIR_ST:
        c[0], c[1] = raw[1], raw[2]
        c[2] = raw[3] - c[1]
        c[3] = raw[3] ** 2
        c[4] = raw[0]
        c[5] = 2 * raw[2] - raw[3]
    return c


def contact_terms(m, pos, pairs, force_mask):
    """Energy, virial and acting-pair count of the contact pairs (i < j)."""
    s = m.settings
    box = np.asarray(s.box, np.float64)
    half_box_sq = (min(s.box) * 0.5) ** 2
    if len(pairs) == 0:
        return 0.0, np.zeros((3, 3)), 0
    pairs = np.asarray(pairs)
    i, j = pairs[:, 0], pairs[:, 1]
    r = _min_image(pos[i] - pos[j], box, force_mask, half_box_sq)
    r2 = (r * r).sum(-1)
    d = np.sqrt(r2)
    nt = m.n_types
    radius = np.asarray(m.radius, np.float32).astype(np.float64)
    rsum = radius[i] + radius[j]
    U = np.zeros(len(i))
    F = np.zeros(len(i))  # radial force on i (along r / |r|)
    act = np.zeros(len(i), bool)
    t = np.asarray(m.type)
    for q in range(len(i)):
        k = pair_index(int(t[i[q]]), int(t[j[q]]), nt)
        kind = int(m.pair_kind[k])
        c = pair_coeffs(kind, np.asarray(m.pair_raw).reshape(-1, 4)[k])
        rq = d[q]
        if kind == PAIR_LJ:
            if r2[q] < s.cutoff ** 2 and rq < c[2]:
                eps, sg, rc = c[1], c[0], c[2]
                U[q] = (48 * eps * sg ** 12 / 13 * (rq ** -13 - rc ** -13)
                        - 24 * eps * sg ** 6 / 7 * (rq ** -7 - rc ** -7) + c[3] * (rq - rc))
                fr6 = (sg * sg / r2[q]) ** 3
                F[q] = 48 * eps * fr6 * (fr6 - 0.5) / r2[q] - c[3]
                act[q] = True
        elif kind == PAIR_HS:
            p = rsum[q] - rq
            if p > 0:
                U[q], F[q], act[q] = 0.5 * c[0] * p * p, c[0] * p, True
        elif kind == PAIR_HSR:
            p = rsum[q] - rq
            if p > 0:
                U[q] += 0.5 * c[0] * p * p
                F[q] += c[0] * p
                act[q] = True
            if rq < c[2]:
                U[q] += 0.5 * c[1] * (c[2] - rq) ** 2
                F[q] += c[1] * (c[2] - rq)
                act[q] = True
        elif kind == PAIR_ST:
            if r2[q] < c[3]:
                rc = np.sqrt(c[3])
                h = 0.5 * (rc * rc - rq * rq)
                U[q] = c[0] * (c[1] * (rc - rq) - h) + c[4] * (c[5] * (rc - rq) - h)
                F[q] = c[0] * (c[1] - rq) + c[4] * (c[5] - rq)
                act[q] = True
    u = np.where(d > 0, 1.0 / np.where(d > 0, d, 1.0), 0.0)
    Fv = (F * u)[:, None] * r
    W = np.einsum("qa,qb->ab", r[act], Fv[act])
    return float(U[act].sum()), W, int(act.sum())


def bonded_terms(m, img, s_status, a_status):
    img = np.asarray(img, np.float64)
    s_ok = (np.asarray(s_status) == 1) & np.isin(m.s_type, [0, 1])
    p1, p2 = np.asarray(m.s_p1)[s_ok], np.asarray(m.s_p2)[s_ok]
    rest = np.asarray(m.s_rest, np.float32).astype(np.float64)[s_ok]
    k = np.asarray(m.s_k, np.float32).astype(np.float64)[s_ok]
    dv = img[p1] - img[p2]
    L = np.sqrt((dv * dv).sum(-1))
    Us = 0.5 * k * (L - rest) ** 2
    f = (k * (rest - L) / np.where(L > 0, L, 1.0))[:, None] * dv
    W = np.einsum("qa,qb->ab", dv, f)

    a_ok = np.asarray(a_status) == 1
    b1, b2, b3 = (np.asarray(x)[a_ok] for x in (m.a_b1, m.a_b2, m.a_b3))
    th0 = np.asarray(m.a_theta0, np.float32).astype(np.float64)[a_ok]
    ka = np.asarray(m.a_k, np.float32).astype(np.float64)[a_ok]
    ba = img[b1] - img[b2]
    bc = img[b3] - img[b2]
    lba = np.sqrt((ba * ba).sum(-1))
    lbc = np.sqrt((bc * bc).sum(-1))
    dot = (ba * bc).sum(-1) / (lba * lbc)
    dot = np.where(dot < -1.0, -0.999999, np.where(dot > 1.0, 0.999999, dot))
    th = np.arccos(dot)
    Ua = ka * (th - th0) ** 2
    M = -2.0 * ka * (th - th0)
    t = np.cross(ba, bc)
    pa = np.cross(ba, t)
    pc = np.cross(-bc, t)
    na = np.linalg.norm(pa, axis=-1)
    nc = np.linalg.norm(pc, axis=-1)
    pa = pa * (np.where(na > 0, 1.0 / np.where(na > 0, na, 1), 0) * M / lba)[:, None]
    pc = pc * (np.where(nc > 0, 1.0 / np.where(nc > 0, nc, 1), 0) * M / lbc)[:, None]
    W = W + np.einsum("qa,qb->ab", ba, pa) + np.einsum("qa,qb->ab", bc, pc)
    return float(Us.sum()), float(Ua.sum()), W


def bead_terms(m, pos, img, vold, walls):
    s = m.settings
    mass = np.asarray(m.mass, np.float64)
    inv = np.where(mass > 0, 1.0 / np.where(mass > 0, mass, 1.0), 0.0)
    vold = np.asarray(vold, np.float32).astype(np.float64)
    ke = float((np.where(inv > 0, 0.5 / np.where(inv > 0, inv, 1.0), 0.0) * (vold * vold).sum(-1)).sum())
    grav = float(-(np.asarray(img) @ np.asarray(s.gravity, np.float64)).sum())
    wall = 0.0
    for a in range(3):
        if walls >> a & 1:
            lo = np.minimum(pos[:, a], 0.0)
            hi = np.maximum(pos[:, a] - s.box[a], 0.0)
            wall += float((0.5 * s.wall_k * (lo * lo + hi * hi)).sum())
    return ke, wall, grav


def walls_mask(m):
    """Wall axes: every axis of a finite box, or the non-periodic axes of a
    mixed box (periodic_mask >= 0)."""
    s = m.settings
    if s.periodic_mask is not None and s.periodic_mask >= 0:
        return 7 & ~s.periodic_mask
    return 7 if s.bc_type == 1 else 0


def force_mask(m):
    """Axes on which contacts use the minimum image: all of them
    (kernel.cl:844-870 ignores the boundary type), or the periodic axes of a
    mixed box."""
    s = m.settings
    if s.periodic_mask is not None and s.periodic_mask >= 0:
        return s.periodic_mask & 7
    return 7


def energy(m, pos, img, vold, s_status, a_status, pairs):
    ke, wall, grav = bead_terms(m, np.asarray(pos), img, vold, walls_mask(m))
    us, ua, wb = bonded_terms(m, img, s_status, a_status)
    uc, wc, nc = contact_terms(m, np.asarray(pos), pairs, force_mask(m))
    out = {"kinetic": ke, "spring": us, "angle": ua, "contact": uc, "wall": wall, "gravity": grav}
    out["total"] = sum(out.values())
    out["virial"] = wb + wc
    out["contacts"] = nc
    return out
