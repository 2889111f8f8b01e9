"""Seeded synthetic fibre networks in the reference's model layout.

The reference ships no models or benchmark inputs, so every workload is
generated here from a recorded seed: straight fibres of ``beads`` beads
(spacing 1.0) joined by springs between consecutive beads and angles over
consecutive triples, as a model file would list them (README.md:106-120).
``tag`` is the fibre id and ``loc_id`` the index along the fibre, which is
what the reference's contact exclusion keys on (kernel.cl:576-586).

Positions inside the box are written wrapped, with the unwrapped position in
the image columns, because ``ReadBeadsData`` rejects beads outside the box
(SimulationManager.cpp:1392-1400).
"""
from __future__ import annotations

import math

import numpy as np

from .model import (ANGLE_HR, PAIR_HS, PAIR_LJ, SPRING_HR, SPRING_HR_FL, Model, Settings,
                    pair_index)

PI_F32 = float(np.float32(np.pi))  # rest angle as std::stof would parse it


def _directions(rng, n, tilt_deg, mode):
    if mode == "sphere":
        v = rng.normal(size=(n, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    tilt = np.deg2rad(rng.uniform(-tilt_deg, tilt_deg, n))
    return np.stack([np.cos(phi) * np.cos(tilt), np.sin(phi) * np.cos(tilt), np.sin(tilt)], axis=1)


def place_fibres(rng, n_fibres, beads, box, periodic, z_range=None, tilt_deg=5.0,
                 orient="xy", spacing=1.0, min_sep=None, max_tries=200, placement="native"):
    """Returns unwrapped bead positions [n_fibres, beads, 3].

    Centres are uniform in the box (z in ``z_range`` if given); on finite axes
    a fibre is redrawn until it lies inside the box.  With ``min_sep`` each
    new fibre must keep that distance from every bead already placed (minimum
    image on periodic axes): for a drawn (x, y, direction) the centre height is
    chosen uniformly among the heights that satisfy it, and the draw is
    repeated when none does.  ``placement`` picks the implementation of the
    separated placement: "native" (fn_place_fibres in the library) or "host"
    (numpy, no native code; a different random stream, so a different but
    equally distributed network).
    """
    box = np.asarray(box, np.float64)
    off = (np.arange(beads) - (beads - 1) / 2.0) * spacing
    out = np.zeros((n_fibres, beads, 3))
    zlo, zhi = (0.0, box[2]) if z_range is None else z_range
    if min_sep is None:
        done = 0
        while done < n_fibres:
            k = n_fibres - done
            c = rng.uniform(0.0, 1.0, (k, 3)) * box
            c[:, 2] = rng.uniform(zlo, zhi, k)
            d = _directions(rng, k, tilt_deg, orient)
            pts = c[:, None, :] + off[None, :, None] * d[:, None, :]
            ok = np.ones(k, bool)
            for a in range(3):
                if not periodic[a]:
                    ok &= (pts[:, :, a].min(axis=1) >= 0.0) & (pts[:, :, a].max(axis=1) <= box[a])
            pts = pts[ok]
            out[done:done + len(pts)] = pts
            done += len(pts)
        return out
    if placement == "host":
        return _place_separated(rng, n_fibres, beads, box, periodic, zlo, zhi, tilt_deg, orient,
                                off, float(min_sep), max_tries)
    return _place_separated_native(rng, n_fibres, beads, box, periodic, zlo, zhi, tilt_deg,
                                   orient, spacing, float(min_sep), max_tries)


def _place_separated_native(rng, n_fibres, beads, box, periodic, zlo, zhi, tilt_deg, orient,
                            spacing, rmin, max_tries):
    """The separated placement in the native library (fn_place_fibres, same
    algorithm as _place_separated, about 100x faster)."""
    import ctypes as C

    from . import native
    lib = native.load()
    out = np.zeros((n_fibres, beads, 3), np.float64)
    b = np.ascontiguousarray(box, np.float64)
    mask = sum(1 << a for a in range(3) if periodic[a])
    seed = int(rng.integers(0, 2**63 - 1))
    rc = lib.fn_place_fibres(seed, n_fibres, beads, b.ctypes.data_as(C.POINTER(C.c_double)), mask,
                             float(zlo), float(zhi), float(tilt_deg), 1 if orient == "sphere" else 0,
                             float(spacing), rmin, int(max_tries),
                             out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(f"fibre placement failed (code {rc}) at separation {rmin}")
    return out


def _place_separated(rng, n_fibres, beads, box, periodic, zlo, zhi, tilt_deg, orient, off, rmin,
                     max_tries):
    """Separated placement in numpy (no native code; the algorithm of
    fn_place_fibres): for a drawn (x, y, direction) the z intervals where some
    placed bead would come closer than rmin are blocked, and the centre height
    is drawn uniformly from what is left of the admissible range."""
    # columns of size >= rmin in x and y; each keeps the (x, y, z) of its beads
    ncx = max(1, int(box[0] // rmin))
    ncy = max(1, int(box[1] // rmin))
    cw = np.array([box[0] / ncx, box[1] / ncy])
    cap = 32
    col = np.zeros((ncx * ncy, cap, 3))
    coln = np.zeros(ncx * ncy, np.int64)
    out = np.zeros((n_fibres, beads, 3))
    r2 = rmin * rmin
    dxy = np.array([(dx, dy) for dx in (-1, 0, 1) for dy in (-1, 0, 1)], np.int64)  # [9, 2]
    slot = np.arange(cap)
    for f in range(n_fibres):
        for _ in range(max_tries):
            c = rng.uniform(0.0, 1.0, 3) * box
            d = _directions(rng, 1, tilt_deg, orient)[0]
            rel = off[:, None] * d[None, :]
            pts = c[None, :] + rel
            bad = False
            for a in range(2):
                if not periodic[a] and (pts[:, a].min() < 0.0 or pts[:, a].max() > box[a]):
                    bad = True
            if bad:
                continue
            # admissible centre heights: z in [zlo, zhi] for every bead
            lo = max(zlo - rel[:, 2].min(), zlo)
            hi = min(zhi - rel[:, 2].max(), zhi)
            if not periodic[2]:
                lo = max(lo, -rel[:, 2].min())
                hi = min(hi, box[2] - rel[:, 2].max())
            if hi <= lo:
                continue
            # the 3 x 3 neighbouring columns of every bead, all at once
            jx = np.floor(pts[:, 0] / cw[0]).astype(np.int64)[None, :] + dxy[:, 0, None]  # [9, B]
            jy = np.floor(pts[:, 1] / cw[1]).astype(np.int64)[None, :] + dxy[:, 1, None]
            ok = np.ones(jx.shape, bool)
            if periodic[0]:
                jx %= ncx
            else:
                ok &= (jx >= 0) & (jx < ncx)
            if periodic[1]:
                jy %= ncy
            else:
                ok &= (jy >= 0) & (jy < ncy)
            kk, bb = np.nonzero(ok)
            cid = jx[kk, bb] * ncy + jy[kk, bb]
            n = coln[cid]
            zc = None
            if n.max(initial=0) > 0:
                sel = n > 0
                cid, bb, n = cid[sel], bb[sel], n[sel]
                cand = col[cid]  # [m, cap, 3]
                valid = slot[None, :] < n[:, None]
                dd = cand[:, :, :2] - pts[bb, None, :2]
                for a in range(2):
                    if periodic[a]:
                        dd[..., a] -= box[a] * np.round(dd[..., a] / box[a])
                q = (dd ** 2).sum(-1)
                hit = valid & (q < r2)
                if hit.any():
                    mm, ss = np.nonzero(hit)
                    h = np.sqrt(r2 - q[mm, ss])
                    z0 = cand[mm, ss, 2] - rel[bb[mm], 2]
                    iv = np.stack([z0 - h, z0 + h], axis=1)
                    if periodic[2]:
                        iv = np.concatenate([iv, iv - box[2], iv + box[2]])
                    iv = iv[np.argsort(iv[:, 0], kind="stable")]
                    free = []
                    cur = lo
                    for a0, a1 in iv.tolist():
                        if a0 > cur:
                            free.append((cur, min(a0, hi)))
                        cur = max(cur, a1)
                        if cur >= hi:
                            break
                    if cur < hi:
                        free.append((cur, hi))
                    free = [(a, b) for a, b in free if b > a]
                    if not free:
                        continue
                    lens = np.array([b - a for a, b in free])
                    k = rng.choice(len(free), p=lens / lens.sum())
                    zc = rng.uniform(*free[k])
            if zc is None:
                zc = rng.uniform(lo, hi)
            pts[:, 2] = zc + rel[:, 2]
            break
        else:
            raise RuntimeError(f"could not place fibre {f} with separation {rmin}")
        out[f] = pts
        wp = pts.copy()
        for a in range(3):
            if periodic[a]:
                wp[:, a] %= box[a]
        cx = np.minimum(np.floor(wp[:, 0] / cw[0]).astype(np.int64), ncx - 1)
        cy = np.minimum(np.floor(wp[:, 1] / cw[1]).astype(np.int64), ncy - 1)
        for b, cb in enumerate((cx * ncy + cy).tolist()):
            n = coln[cb]
            if n >= cap:
                raise RuntimeError("placement column overflow")
            col[cb, n] = wp[b]
            coln[cb] = n + 1
    return out


def wrap(img, box, periodic):
    pos = img.copy()
    for a in range(3):
        if periodic[a]:
            pos[:, a] = np.mod(pos[:, a], box[a])
            pos[pos[:, a] >= box[a], a] = 0.0
    return pos


def chain_model(img_fibres, settings: Settings, type_names, pair_kind, pair_raw,
                bead_type=None, radius=0.5, mass=1.0, spring_type=SPRING_HR, rest=1.0, k_s=100.0,
                s_c1=0.0, s_c2=0.0, angle_type=ANGLE_HR, theta0=PI_F32, k_a=10.0, vel=None,
                tag_offset=0) -> Model:
    """Assembles fibres (unwrapped positions [F, B, 3]) into a Model with one
    spring per consecutive pair and one angle per consecutive triple."""
    F, B, _ = img_fibres.shape
    N = F * B
    img = img_fibres.reshape(N, 3).astype(np.float64)
    periodic = [bool((settings.periodic_mask >> a) & 1) if settings.periodic_mask >= 0
                else settings.bc_type == 0 for a in range(3)]
    pos = wrap(img, np.asarray(settings.box), periodic)
    fib = np.repeat(np.arange(F), B)
    loc = np.tile(np.arange(B), F)
    bt = np.zeros(N, np.int32) if bead_type is None else np.asarray(bead_type, np.int32)
    v = np.zeros((N, 3)) if vel is None else np.asarray(vel, np.float64).reshape(N, 3)
    # springs (b, b+1) and angles (b, b+1, b+2) along each fibre
    sb = (np.arange(F)[:, None] * B + np.arange(B - 1)[None, :]).ravel()
    s_id = (np.arange(F)[:, None] * (B - 1) + np.arange(B - 1)[None, :])
    ab = (np.arange(F)[:, None] * B + np.arange(B - 2)[None, :]).ravel()
    a_s1 = s_id[:, :-1].ravel()
    a_s2 = s_id[:, 1:].ravel()
    ns, na = len(sb), len(ab)

    def per(x, n):
        a = np.asarray(x, np.float64)
        return np.full(n, float(a)) if a.ndim == 0 else a.reshape(n).astype(np.float64)

    return Model(
        settings=settings, type_names=list(type_names),
        pair_kind=np.asarray(pair_kind, np.int32), pair_raw=np.asarray(pair_raw, np.float64).reshape(-1, 4),
        type=bt, tag=(fib + tag_offset).astype(np.int32), loc_id=loc.astype(np.int32),
        radius=per(radius, N), mass=per(mass, N), pos=pos, vel=v.copy(), vel_old=v.copy(),
        force=np.zeros((N, 3)), img=img,
        s_type=np.full(ns, spring_type, np.int32), s_tag=(sb // B + tag_offset).astype(np.int32),
        s_p1=sb.astype(np.int32), s_p2=(sb + 1).astype(np.int32), s_rest=per(rest, ns),
        s_k=per(k_s, ns), s_c1=per(s_c1, ns), s_c2=per(s_c2, ns),
        a_type=np.full(na, angle_type, np.int32), a_tag=(ab // B + tag_offset).astype(np.int32),
        a_b1=ab.astype(np.int32), a_b2=(ab + 1).astype(np.int32), a_b3=(ab + 2).astype(np.int32),
        a_s1=a_s1.astype(np.int32), a_s2=a_s2.astype(np.int32), a_theta0=per(theta0, na),
        a_k=per(k_a, na),
    )


def _uniform_pairs(n_types, kind, raw):
    n = n_types * (n_types + 1) // 2
    return np.full(n, kind, np.int32), np.tile(np.asarray(raw, np.float64), (n, 1))


# ---------------------------------------------------------------------------
# the workloads


def plain_network(seed=0, fibres=200, beads=50, box=(100.0, 100.0, 10.0), z_range=(1.0, 9.0),
                  k_s=100.0, k_a=10.0, k_contact=50.0, dt=0.001, cell=1.0, grid_update_freq=8,
                  tilt_deg=5.0) -> Model:
    """Periodic box of straight fibres with HR springs and angles and a penalty
    contact: config 0 at its default sizes (200 fibres x 50 beads in
    100x100x10, k_s 100, k_a 10, penalty 50, dt 0.001, cell 1.0)."""
    rng = np.random.default_rng(seed)
    pts = place_fibres(rng, fibres, beads, box, (True, True, True), z_range=z_range,
                       tilt_deg=tilt_deg)
    st = Settings(dt=dt, lam=0.5, damping=0.0, cutoff=cell, box_unit_cell=cell, box=tuple(box),
                  wall_k=0.0, bc_type=0, grid_update_freq=grid_update_freq)
    pk, pr = _uniform_pairs(1, PAIR_HS, [k_contact, 0, 0, 0])
    m = chain_model(pts, st, ["C1"], pk, pr, k_s=k_s, k_a=k_a)
    m.meta.update(kind="plain", seed=seed, fibres=fibres, beads=beads)
    return m


def tensile_network(seed=1, fibres=20000, beads=50, box=(1000.0, 1000.0, 20.0),
                    z_range=(1.0, 19.0), k_s=100.0, young=1e3, fail_mu=math.log(5.0),
                    fail_sigma=0.3, k_a=10.0, lj_eps=1.0, lj_sigma=1.0, lj_cut=2.5, dt=0.0005,
                    clamp_lo=2.0, clamp_hi=998.0, pull=0.01, cell=2.5, wall_k=100.0,
                    min_sep=1.0, grid_update_freq=8, placement="native") -> Model:
    """Tensile test (config 1 at its default sizes): finite in x and z,
    periodic in y; HR_FL springs with E = 1e3 and lognormal failure stress;
    LJ contacts (eps 1, sigma 1, cut-off 2.5); beads with x < 2 clamped, beads
    with x > 998 pulled at +0.01 in x.  Fibres are placed at least ``min_sep``
    apart so the LJ core starts bounded.  Bead types: C1 free, CL left clamp,
    CR right clamp (mass 0).  ``placement``: see place_fibres."""
    rng = np.random.default_rng(seed)
    periodic = (False, True, False)
    pts = place_fibres(rng, fibres, beads, box, periodic, z_range=z_range, min_sep=min_sep,
                       placement=placement)
    N = fibres * beads
    img = pts.reshape(N, 3)
    bt = np.zeros(N, np.int32)
    bt[img[:, 0] < clamp_lo] = 1
    bt[img[:, 0] > clamp_hi] = 2
    mass = np.where(bt == 0, 1.0, 0.0)
    vel = np.zeros((N, 3))
    vel[bt == 2, 0] = pull
    st = Settings(dt=dt, lam=0.5, damping=0.0, cutoff=lj_cut * lj_sigma, box_unit_cell=cell,
                  box=tuple(box), wall_k=wall_k, bc_type=1, grid_update_freq=grid_update_freq,
                  periodic_mask=0b010)
    pk, pr = _uniform_pairs(3, PAIR_LJ, [lj_sigma, lj_eps, lj_cut * lj_sigma, 0])
    ns = fibres * (beads - 1)
    fail = rng.lognormal(fail_mu, fail_sigma, ns)
    m = chain_model(pts, st, ["C1", "CL", "CR"], pk, pr, bead_type=bt, mass=mass,
                    spring_type=SPRING_HR_FL, k_s=k_s, s_c1=young, s_c2=fail, k_a=k_a, vel=vel)
    m.meta.update(kind="tensile", seed=seed, fibres=fibres, beads=beads, clamp_right_type=2,
                  clamp_left_type=1)
    return m


def explicit_model(settings: Settings, type_names, pairs, beads, springs=(), angles=()) -> Model:
    """Builds a Model from explicit records, in model-file field order:

    pairs   dict {(t1, t2): (kind, [raw tokens 4..7])}, every type pair present
    beads   (type, tag, loc_id, radius, mass, pos[3], vel[3], img[3])
    springs (type, tag, p1, p2, rest, k, c1, c2)
    angles  (type, tag, b1, b2, b3, s1, s2, theta0, k)
    """
    nt = len(type_names)
    n_pairs = nt * (nt + 1) // 2
    pk = np.zeros(n_pairs, np.int32)
    pr = np.zeros((n_pairs, 4), np.float64)
    for (t1, t2), (kind, raw) in pairs.items():
        i = pair_index(t1, t2, nt)
        pk[i] = kind
        raw = list(raw) + [0.0] * (4 - len(raw))
        pr[i] = raw[:4]
    N = len(beads)
    col = lambda k, dt=np.float64: np.array([b[k] for b in beads], dt)  # noqa: E731
    vel = np.array([b[6] for b in beads], np.float64).reshape(N, 3)
    sp = list(springs)
    an = list(angles)
    scol = lambda k, dt: np.array([s[k] for s in sp], dt)  # noqa: E731
    acol = lambda k, dt: np.array([a[k] for a in an], dt)  # noqa: E731
    return Model(
        settings=settings, type_names=list(type_names), pair_kind=pk, pair_raw=pr,
        type=col(0, np.int32), tag=col(1, np.int32), loc_id=col(2, np.int32), radius=col(3),
        mass=col(4), pos=np.array([b[5] for b in beads], np.float64).reshape(N, 3), vel=vel.copy(),
        vel_old=vel.copy(), force=np.zeros((N, 3)),
        img=np.array([b[7] for b in beads], np.float64).reshape(N, 3),
        s_type=scol(0, np.int32), s_tag=scol(1, np.int32), s_p1=scol(2, np.int32),
        s_p2=scol(3, np.int32), s_rest=scol(4, np.float64), s_k=scol(5, np.float64),
        s_c1=scol(6, np.float64), s_c2=scol(7, np.float64),
        a_type=acol(0, np.int32), a_tag=acol(1, np.int32), a_b1=acol(2, np.int32),
        a_b2=acol(3, np.int32), a_b3=acol(4, np.int32), a_s1=acol(5, np.int32),
        a_s2=acol(6, np.int32), a_theta0=acol(7, np.float64), a_k=acol(8, np.float64),
    )


def ensemble_networks(seed=3, n_networks=256, fibres_lo=50, fibres_hi=2000, beads=50, z=10.0,
                      k_s=(50.0, 200.0), k_a=(2.0, 20.0), k_contact=50.0, dt=0.001, cell=1.0,
                      grid_update_freq=8):
    """Independent config-0-style networks (config 3 at its default sizes):
    fibre counts uniform in [fibres_lo, fibres_hi], each network in its own
    periodic box sqrt(F/200)*100 wide in x and y and z high, spring stiffness
    uniform in k_s and angle stiffness uniform in k_a per network, penalty
    contacts.  Returns a list of Models."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(fibres_lo, fibres_hi + 1, n_networks)
    out = []
    for k, F in enumerate(counts):
        side = float(np.sqrt(F / 200.0) * 100.0)
        ks = float(rng.uniform(*k_s))
        ka = float(rng.uniform(*k_a))
        m = plain_network(seed=int(rng.integers(0, 2**31 - 1)), fibres=int(F), beads=beads,
                          box=(side, side, z), z_range=(1.0, z - 1.0), k_s=ks, k_a=ka,
                          k_contact=k_contact, dt=dt, cell=cell, grid_update_freq=grid_update_freq)
        m.meta.update(kind="ensemble", index=k, k_s=ks, k_a=ka)
        out.append(m)
    return out


def dense_mat(seed=2, fibres=40000, beads=100, box=(200.0, 200.0, 200.0), k_s=200.0, k_a=5.0,
              k_pen=100.0, k_soft=10.0, rc_soft=1.2, vel_sigma=0.1, dt=0.0005, cell=1.0,
              cutoff=1.2, grid_update_freq=8) -> Model:
    """Dense 3D mat (config 2 at its default sizes): periodic 200^3 box, fibres
    of 100 beads with directions uniform on the sphere, HR springs (rest 1,
    k 200) and angles (k 5), contacts = penalty (k 100) + soft harmonic
    repulsion (k 10 below 1.2) on the same type pair (pair kind 4, an
    extension), Gaussian velocities (sigma 0.1)."""
    from .model import PAIR_HSR
    rng = np.random.default_rng(seed)
    pts = place_fibres(rng, fibres, beads, box, (True, True, True), orient="sphere")
    st = Settings(dt=dt, lam=0.5, damping=0.0, cutoff=cutoff, box_unit_cell=cell, box=tuple(box),
                  wall_k=0.0, bc_type=0, grid_update_freq=grid_update_freq)
    pk, pr = _uniform_pairs(1, PAIR_HSR, [k_pen, k_soft, rc_soft, 0])
    vel = rng.normal(0.0, vel_sigma, (fibres * beads, 3))
    m = chain_model(pts, st, ["C1"], pk, pr, k_s=k_s, k_a=k_a, vel=vel)
    m.meta.update(kind="dense", seed=seed, fibres=fibres, beads=beads)
    return m


def fitting_networks(seed=4, n_networks=64, beads_lo=5000, beads_hi=50000, beads=50, z=20.0,
                     pull=0.01, dt=0.001, k_s=100.0, k_a=10.0):
    """Networks of the stiffness-fitting problem (config 4 at its default
    sizes): the tensile geometry of tensile_network scaled down to 5k-50k
    beads per network (bead counts uniform, fibres of 50 beads, box side
    1000 sqrt(F / 20000) so the fibre density matches the 1M-bead test),
    unbreakable HR springs, clamps pulled at 0.01, dt 0.001."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_networks):
        F = int(rng.integers(beads_lo // beads, beads_hi // beads + 1))
        side = float(1000.0 * np.sqrt(F / 20000.0))
        m = tensile_network(seed=int(rng.integers(0, 2**31 - 1)), fibres=F, beads=beads,
                            box=(side, side, z), z_range=(1.0, z - 1.0), k_s=k_s, k_a=k_a, dt=dt,
                            clamp_lo=2.0, clamp_hi=side - 2.0, pull=pull)
        m.s_type[:] = SPRING_HR
        m.meta.update(kind="fitting", index=k)
        out.append(m)
    return out


def perturbed_stiffness(models, seed=5, sigma=0.2):
    """Copies of ``models`` whose spring stiffnesses are multiplied by
    lognormal(0, sigma) factors (the target of the fitting problem)."""
    import copy
    rng = np.random.default_rng(seed)
    out = []
    for m in models:
        t = copy.copy(m)
        t.s_k = np.asarray(m.s_k, np.float64) * rng.lognormal(0.0, sigma, m.n_springs)
        out.append(t)
    return out
