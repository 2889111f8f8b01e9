"""FP64 reference gradient for the adjoint: the step loop written out in
torch (CPU, float64) with the reference's force arithmetic, differentiated by
torch autograd.  Test infrastructure only.

Follows kernel.cl operation by operation where it matters for the map:
AdvancePosition :195-265 (drift, snap wrap, wall penalty), ResolveSprings
:366-441, ResolveAngles :268-363 (cross-product form, the +-0.999999 clamp),
ResolveContacts :792-1011 (lj / hs / st, minimum image), AdvanceVelocity
:444-464, and the call schedule of SimulationManager.cpp:151-181 (a call opens
with a drift; a rebuild opens every grid_update_freq-step run; the last step
of a call does not drift).  Contact lists are rebuilt from positions by brute
force with BuildContactList's acceptance rule (kernel.cl:532-789) and the
bonded-neighbour exclusion; HR_FL breaks are not modelled (the tests use
unbreakable springs).
"""
import numpy as np
import torch

from fibrenet_b200.model import PAIR_HS, PAIR_HSR, PAIR_LJ, PAIR_ST, pair_index

T = torch.float64


def _coeffs(m):
    nt = m.n_types
    raw = np.asarray(m.pair_raw, np.float64).reshape(-1, 4)
    out = {}
    for t1 in range(nt):
        for t2 in range(t1, nt):
            k = pair_index(t1, t2, nt)
            kind = int(m.pair_kind[k])
            c = np.zeros(6)
            r = raw[k]
            if kind == PAIR_LJ:
                c[:3] = r[:3]
                r2 = c[2] * c[2]
                fr2 = c[0] * c[0] / r2
                fr6 = fr2 ** 3
                c[3] = 48.0 * c[1] * fr6 * (fr6 - 0.5) / r2
            elif kind == PAIR_HS:
                c[0] = r[0]
            elif kind == PAIR_HSR:
                c[:3] = r[:3]
            elif kind == PAIR_ST:
                c[0], c[1], c[2], c[3], c[4], c[5] = r[1], r[2], r[3] - r[2], r[3] ** 2, r[0], 2 * r[2] - r[3]
            out[k] = (kind, c)
    return out


class RefLoop:
    def __init__(self, m):
        m = m.normalised()
        self.m = m
        s = m.settings
        self.s = s
        self.n = m.n_beads
        self.box = torch.tensor(s.box, dtype=T)
        pm = s.periodic_mask
        if pm is not None and pm >= 0:
            self.periodic = pm & 7
            self.force_mi = self.periodic
            self.walls = 7 & ~self.periodic
        else:
            self.periodic = 7 if s.bc_type == 0 else 0
            self.force_mi = 7
            self.walls = 7 if s.bc_type == 1 else 0
        self.list_mi = self.periodic
        self.half_box_sq = (min(s.box) * 0.5) ** 2
        mass = np.asarray(m.mass, np.float64)
        self.minv = torch.tensor(np.where(mass > 0, 1.0 / np.where(mass > 0, mass, 1.0), 0.0), dtype=T)
        self.radius = np.asarray(m.radius, np.float32).astype(np.float64)
        skin = (self.radius.astype(np.float32) + np.float32(s.skin_ratio)).astype(np.float32)
        self.skin = np.asarray(skin, np.float64)
        self.type = np.asarray(m.type)
        self.tag = np.asarray(m.tag)
        self.loc = np.asarray(m.loc_id)
        self.coef = _coeffs(m)
        self.p1 = torch.tensor(np.asarray(m.s_p1), dtype=torch.long)
        self.p2 = torch.tensor(np.asarray(m.s_p2), dtype=torch.long)
        self.b1 = torch.tensor(np.asarray(m.a_b1), dtype=torch.long)
        self.b2 = torch.tensor(np.asarray(m.a_b2), dtype=torch.long)
        self.b3 = torch.tensor(np.asarray(m.a_b3), dtype=torch.long)
        self.theta0 = torch.tensor(np.asarray(m.a_theta0, np.float32).astype(np.float64), dtype=T)
        self.g = torch.tensor(s.gravity, dtype=T)

    # -- contact list (no gradient)
    def _mi(self, r, mask):
        r = r.copy()
        far = (r * r).sum(-1) > self.half_box_sq
        box = np.asarray(self.s.box)
        for a in range(3):
            if mask >> a & 1:
                sel = far & (r[:, a] ** 2 > self.half_box_sq)
                r[sel, a] = np.where(r[sel, a] > 0, r[sel, a] - box[a], r[sel, a] + box[a])
        return r

    def pairs(self, pos):
        p = pos.detach().numpy()
        i, j = np.triu_indices(self.n, 1)
        excl = (self.tag[i] == self.tag[j]) & (np.abs(self.loc[i] - self.loc[j]) <= 1)
        i, j = i[~excl], j[~excl]
        r = self._mi(p[i] - p[j], self.list_mi)
        r2 = (r * r).sum(-1)
        nt = self.m.n_types
        kind_of = np.zeros((nt, nt), np.int64)
        for t1 in range(nt):
            for t2 in range(nt):
                kind_of[t1, t2] = self.coef[pair_index(t1, t2, nt)][0]
        kind = kind_of[self.type[i], self.type[j]]
        cut = np.isin(kind, (PAIR_LJ, PAIR_ST, PAIR_HSR)) & (r2 < self.s.cutoff ** 2)
        lim = np.maximum(self.radius[i], self.radius[j]) + np.minimum(self.skin[i], self.skin[j])
        hs = np.isin(kind, (PAIR_HS, PAIR_HSR)) & (r2 < lim * lim)
        keep = cut | hs
        return i[keep], j[keep]

    # -- forces
    def forces(self, x, pos, k_s, rest, k_a, pairs):
        n = self.n
        F = self.g.expand(n, 3).clone()
        for a in range(3):
            if self.walls >> a & 1:
                pa = pos[:, a]
                wk = self.s.wall_k
                F[:, a] = F[:, a] + torch.where(pa < 0.0, pa * wk * -1.0, torch.zeros_like(pa))
                F[:, a] = F[:, a] + torch.where(pa > self.box[a], (pa - self.box[a]) * wk * -1.0,
                                                torch.zeros_like(pa))
        # springs
        d = x[self.p1] - x[self.p2]
        L = torch.sqrt((d * d).sum(-1))
        fs = ((rest - L) * k_s / L)[:, None] * d
        F = F.index_add(0, self.p1, fs).index_add(0, self.p2, -fs)
        # angles
        ba = x[self.b1] - x[self.b2]
        bc = x[self.b3] - x[self.b2]
        lba = torch.sqrt((ba * ba).sum(-1))
        lbc = torch.sqrt((bc * bc).sum(-1))
        dotp = (ba * bc).sum(-1) / (lba * lbc)
        dotp = torch.where(dotp < -1.0, torch.full_like(dotp, -0.999999), dotp)
        dotp = torch.where(dotp > 1.0, torch.full_like(dotp, 0.999999), dotp)
        # exactly straight triples (clamped fibre ends) have no force and, as
        # on the device, no tangent: keep acos and sqrt off their singular
        # points in the backward pass
        inside = dotp.abs() < 1.0
        theta = torch.where(inside, torch.acos(torch.where(inside, dotp, torch.zeros_like(dotp))),
                            torch.acos(dotp).detach())
        mag = -2.0 * k_a * (theta - self.theta0)
        t = torch.cross(ba, bc, dim=-1)
        pa = torch.cross(ba, t, dim=-1)
        pc = torch.cross(-bc, t, dim=-1)

        def safe_norm(v):
            sq = (v * v).sum(-1)
            return torch.where(sq > 0, torch.sqrt(torch.where(sq > 0, sq, torch.ones_like(sq))),
                               torch.zeros_like(sq))
        la = safe_norm(pa)
        lc = safe_norm(pc)
        pa = pa * torch.where(la != 0, mag / lba / torch.where(la != 0, la, torch.ones_like(la)),
                              torch.zeros_like(la))[:, None]
        pc = pc * torch.where(lc != 0, mag / lbc / torch.where(lc != 0, lc, torch.ones_like(lc)),
                              torch.zeros_like(lc))[:, None]
        F = F.index_add(0, self.b1, pa).index_add(0, self.b3, pc).index_add(0, self.b2, -pa - pc)
        # contacts
        ii, jj = pairs
        if len(ii):
            ti = torch.tensor(ii)
            tj = torch.tensor(jj)
            r = pos[ti] - pos[tj]
            r2 = (r * r).sum(-1)
            far = r2 > self.half_box_sq
            cols = []
            for a in range(3):
                ra = r[:, a]
                if self.force_mi >> a & 1:
                    sel = far & (ra * ra > self.half_box_sq)
                    ra = torch.where(sel, torch.where(ra > 0, ra - self.box[a], ra + self.box[a]), ra)
                cols.append(ra)
            r = torch.stack(cols, -1)
            r2 = (r * r).sum(-1)
            rl = torch.sqrt(r2)
            f = torch.zeros_like(rl)
            nt = self.m.n_types
            pid = np.array([[pair_index(t1, t2, nt) for t2 in range(nt)] for t1 in range(nt)])
            kind_tab = np.array([self.coef[k][0] for k in range(nt * (nt + 1) // 2)])
            coef_tab = np.array([self.coef[k][1] for k in range(nt * (nt + 1) // 2)])
            q = pid[self.type[ii], self.type[jj]]
            kinds = kind_tab[q]
            cs = torch.tensor(coef_tab[q], dtype=T)
            rsum = torch.tensor(self.radius[ii] + self.radius[jj], dtype=T)
            kt = torch.tensor(kinds)
            lj = (kt == PAIR_LJ) & (r2 < self.s.cutoff ** 2) & (rl < cs[:, 2])
            fr6 = (cs[:, 0] ** 2 / r2) ** 3
            f = torch.where(lj, 48.0 * cs[:, 1] * fr6 * (fr6 - 0.5) / r2 - cs[:, 3], f)
            pen = rsum - rl
            f = torch.where((kt == PAIR_HS) & (pen > 0), pen * cs[:, 0], f)
            st = (kt == PAIR_ST) & (r2 < cs[:, 3])
            f = torch.where(st, (cs[:, 1] - rl) * cs[:, 0] + (cs[:, 5] - rl) * cs[:, 4], f)
            hsr = kt == PAIR_HSR
            f = torch.where(hsr, torch.where(pen > 0, pen * cs[:, 0], torch.zeros_like(f))
                            + torch.where(rl < cs[:, 2], (cs[:, 2] - rl) * cs[:, 1], torch.zeros_like(f)), f)
            R = (f / rl)[:, None] * r
            F = F.index_add(0, ti, R).index_add(0, tj, -R)
        return F

    def run(self, nsamples, every, reaction_type, k_s, rest, k_a, x0=None, v0=None):
        """Reaction curve [nsamples, 3] as a differentiable function of the
        spring stiffnesses, rest lengths, angle stiffnesses and the starting
        positions and velocities."""
        m, s = self.m, self.s
        dt = s.dt
        x = torch.tensor(np.asarray(m.img), dtype=T) if x0 is None else x0
        pos = torch.tensor(np.asarray(m.pos), dtype=T) + (x - torch.tensor(np.asarray(m.img), dtype=T))
        v = torch.tensor(np.asarray(m.vel_old), dtype=T) if v0 is None else v0
        F = torch.tensor(np.asarray(m.force), dtype=T)
        c = (dt * dt * 0.5 * self.minv)[:, None]
        b = (dt * 0.5 * self.minv)[:, None]
        clamp = torch.tensor(self.type == reaction_type)
        box = self.box
        out = []

        def drift(x, pos):
            dx = v * dt + F * c
            x = x + dx
            pos = pos + dx
            cols = []
            for a in range(3):
                pa = pos[:, a]
                if self.periodic >> a & 1:
                    pa = torch.where(pa < 0.0, box[a].expand_as(pa), pa)
                    pa = torch.where(pa > box[a], torch.zeros_like(pa), pa)
                cols.append(pa)
            return x, torch.stack(cols, -1)

        for _ in range(nsamples):
            x, pos = drift(x, pos)
            done = 0
            while done < every:
                ln = min(s.grid_update_freq, every - done)
                pairs = self.pairs(pos)
                for kq in range(ln):
                    Fn = self.forces(x, pos, k_s, rest, k_a, pairs)
                    v = v + b * (Fn + F)
                    F = Fn
                    if not (done + kq == every - 1):
                        x, pos = drift(x, pos)
                done += ln
            out.append(F[clamp].sum(0))
        return torch.stack(out)
