/*
 * fibre_oracle.c -- CPU restatement of FibreNet's per-timestep particle
 * dynamics (FibreNet/kernel.cl + SimulationManager::RunSimulationLoop).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle: the tests, the
 * smoke check and the CPU-baseline leg of bench.py call it to check the CUDA
 * path; the product never links it.  It is pinned against the reference's
 * own kernels (oracle/_ref, built from kernel.cl) by the committed golden
 * vectors in tests/golden/.
 *
 * Two modes:
 *   FO_MODE_REF     the reference's arithmetic and accumulation order exactly
 *                   as a single OpenCL work-item sweep would produce it
 *                   (atomics become ordered += in work-item order); FP64 state.
 *                   Bit-identical to oracle/_ref run on one thread.
 *   FO_MODE_MIRROR  the same physics with the storage and ordering choices of
 *                   the B200 path: positions FP64, velocities/forces and bond
 *                   parameters stored FP32, forces gathered per bead in a fixed
 *                   order (base, springs, angles, contacts), contact lists
 *                   enumerated over the 27-cell neighbourhood in a fixed order.
 *                   Bit-identical to the CUDA path, which makes trajectories and
 *                   break sets comparable exactly over many steps.
 *
 * Every formula cites the kernel.cl line range it restates.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_host.h"
#include "oracle_model.h"
/* MIRROR mode uses the device path's arc cosine (IEEE ops only), so both
   sides round identically; REF mode keeps libm acos like kernel.cl:314. */
#include "fn_detmath.h"

#define FO_EXPORT __attribute__((visibility("default")))

enum { FO_MODE_REF = 0, FO_MODE_MIRROR = 1 };

/* kernel.cl:10-11 */
#define REF_GRID_TAIL 64
#define REF_NHOOD 256

typedef struct fo_ctx {
    fo_derived d;
    int mode;
    int nb, ns, na, np;
    int cell_cap, list_cap;
    int periodic;  /* axes wrapped by AdvancePosition and the cell stencil */
    int list_mi;   /* axes where BuildContactList applies the minimum image */
    int force_mi;  /* axes where ResolveContacts applies the minimum image */
    int walls;     /* axes with wall penalty */
    /* bead state, 3 doubles per bead */
    double *pos, *img, *vel, *force, *vel_old, *force_old;
    /* bead constants */
    int *type, *tag, *loc_id;
    double *mass_inv, *lam, *hdt, *hdt2, *radius, *skin;
    /* springs */
    int *s_type, *s_status, *s_p1, *s_p2;
    double *s_rest, *s_k, *s_c1, *s_c2;
    /* angles */
    int *a_type, *a_status, *a_b1, *a_b2, *a_b3, *a_s1, *a_s2;
    double *a_theta0, *a_k;
    /* pair table */
    int* p_kind;
    double* p_c; /* 6 per pair */
    /* grid */
    int* cell_nh;    /* 13 per cell (reference half-shell table) */
    int* grid_head;  /* raw counts */
    int* grid_slot;  /* cell_cap per cell */
    int* bead_cell;  /* cell of each bead after the last rebuild, -1 if none */
    /* contact lists */
    int* list_head;  /* raw counts */
    int* list_j;     /* list_cap per bead */
    int* list_pair;  /* list_cap per bead */
    /* bead -> bond incidence (mirror mode gather order) */
    int *sp_off, *sp_idx, *an_off, *an_idx;
    long overflow_cells, overflow_lists;
} fo_ctx;

static void* zal(size_t n) {
    void* p = calloc(n ? n : 1, 1);
    if (!p) {
        fprintf(stderr, "fibre_oracle: out of host memory\n");
        abort();
    }
    return p;
}

static inline double rf(const fo_ctx* c, double x) {
    return c->mode == FO_MODE_MIRROR ? (double)(float)x : x;
}

/* GETADRESS, kernel.cl:9 */
static inline int getadress(int t1, int t2, int size) {
    return (t1 < t2) ? ((size * t1) + t2 - ((t1 * (t1 + 1)) / 2)) : ((size * t2) + t1 - ((t2 * (t2 + 1)) / 2));
}

FO_EXPORT void fo_destroy(fo_ctx* c) {
    if (!c) return;
    void* ptrs[] = {c->pos,      c->img,       c->vel,      c->force,    c->vel_old,   c->force_old,
                    c->type,     c->tag,       c->loc_id,   c->mass_inv, c->lam,       c->hdt,
                    c->hdt2,     c->radius,    c->skin,     c->s_type,   c->s_status,  c->s_p1,
                    c->s_p2,     c->s_rest,    c->s_k,      c->s_c1,     c->s_c2,      c->a_type,
                    c->a_status, c->a_b1,      c->a_b2,     c->a_b3,     c->a_s1,      c->a_s2,
                    c->a_theta0, c->a_k,       c->p_kind,   c->p_c,      c->cell_nh,   c->grid_head,
                    c->grid_slot, c->bead_cell, c->list_head, c->list_j,  c->list_pair, c->sp_off,
                    c->sp_idx,   c->an_off,    c->an_idx};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); ++i) free(ptrs[i]);
    free(c);
}

/* Bead -> incident springs (entry 2*s + role, role 0 = p1, 1 = p2) and
   bead -> incident angles (entry 3*a + role, role 0 = b1, 1 = b2, 2 = b3),
   both in ascending bond order. */
static void build_incidence(fo_ctx* c) {
    c->sp_off = (int*)zal(sizeof(int) * (size_t)(c->nb + 1));
    c->an_off = (int*)zal(sizeof(int) * (size_t)(c->nb + 1));
    c->sp_idx = (int*)zal(sizeof(int) * (size_t)(2 * c->ns));
    c->an_idx = (int*)zal(sizeof(int) * (size_t)(3 * c->na));
    for (int s = 0; s < c->ns; ++s) {
        c->sp_off[c->s_p1[s] + 1]++;
        c->sp_off[c->s_p2[s] + 1]++;
    }
    for (int a = 0; a < c->na; ++a) {
        c->an_off[c->a_b1[a] + 1]++;
        c->an_off[c->a_b2[a] + 1]++;
        c->an_off[c->a_b3[a] + 1]++;
    }
    for (int i = 0; i < c->nb; ++i) {
        c->sp_off[i + 1] += c->sp_off[i];
        c->an_off[i + 1] += c->an_off[i];
    }
    int* fill = (int*)zal(sizeof(int) * (size_t)(c->nb + 1));
    memcpy(fill, c->sp_off, sizeof(int) * (size_t)c->nb);
    for (int s = 0; s < c->ns; ++s) {
        c->sp_idx[fill[c->s_p1[s]]++] = 2 * s + 0;
        c->sp_idx[fill[c->s_p2[s]]++] = 2 * s + 1;
    }
    memcpy(fill, c->an_off, sizeof(int) * (size_t)c->nb);
    for (int a = 0; a < c->na; ++a) {
        c->an_idx[fill[c->a_b1[a]]++] = 3 * a + 0;
        c->an_idx[fill[c->a_b2[a]]++] = 3 * a + 1;
        c->an_idx[fill[c->a_b3[a]]++] = 3 * a + 2;
    }
    free(fill);
}

FO_EXPORT fo_ctx* fo_create(const fo_model* m, int mode, int cell_cap, int list_cap) {
    fo_ctx* c = (fo_ctx*)zal(sizeof(fo_ctx));
    fo_derive_settings(m, &c->d);
    c->mode = mode;
    c->nb = m->n_beads;
    c->ns = m->n_springs;
    c->na = m->n_angles;
    c->np = m->n_types * (m->n_types + 1) / 2;
    c->cell_cap = mode == FO_MODE_REF ? REF_GRID_TAIL : cell_cap;
    c->list_cap = mode == FO_MODE_REF ? REF_NHOOD : list_cap;
    if (m->periodic_mask < 0) {
        c->periodic = c->d.bc_type == 0 ? 7 : 0;
        c->list_mi = c->periodic;
        c->force_mi = 7; /* kernel.cl:844-870 applies it whatever bc_type is */
    } else {
        c->periodic = m->periodic_mask & 7;
        c->list_mi = c->periodic;
        c->force_mi = c->periodic;
    }
    c->walls = (~c->periodic) & 7;
    if (m->periodic_mask < 0 && c->d.bc_type != 0 && c->d.bc_type != 1) c->walls = 0;

    size_t n3 = sizeof(double) * 3 * (size_t)c->nb;
    c->pos = (double*)zal(n3);
    c->img = (double*)zal(n3);
    c->vel = (double*)zal(n3);
    c->force = (double*)zal(n3);
    c->vel_old = (double*)zal(n3);
    c->force_old = (double*)zal(n3);
    for (int k = 0; k < 3 * c->nb; ++k) {
        c->pos[k] = m->pos[k];
        c->img[k] = m->img[k];
        c->vel[k] = rf(c, m->vel[k]);
        c->vel_old[k] = rf(c, m->vel_old[k]);
        c->force[k] = rf(c, m->force[k]);
        c->force_old[k] = c->force[k];
    }
    size_t ni = sizeof(int) * (size_t)c->nb, nd = sizeof(double) * (size_t)c->nb;
    c->type = (int*)zal(ni);
    c->tag = (int*)zal(ni);
    c->loc_id = (int*)zal(ni);
    c->mass_inv = (double*)zal(nd);
    c->lam = (double*)zal(nd);
    c->hdt = (double*)zal(nd);
    c->hdt2 = (double*)zal(nd);
    c->radius = (double*)zal(nd);
    c->skin = (double*)zal(nd);
    for (int i = 0; i < c->nb; ++i) {
        double k[9];
        fo_derive_bead(&c->d, m->mass[i], rf(c, m->radius[i]), m->skin_ratio, k);
        c->type[i] = m->type[i];
        c->tag[i] = m->tag[i];
        c->loc_id[i] = m->loc_id[i];
        c->mass_inv[i] = k[1];
        c->lam[i] = k[2];
        c->hdt[i] = k[3];
        c->hdt2[i] = k[4];
        c->radius[i] = k[5];
        c->skin[i] = rf(c, k[7]);
    }
    size_t si = sizeof(int) * (size_t)c->ns, sd = sizeof(double) * (size_t)c->ns;
    c->s_type = (int*)zal(si);
    c->s_status = (int*)zal(si);
    c->s_p1 = (int*)zal(si);
    c->s_p2 = (int*)zal(si);
    c->s_rest = (double*)zal(sd);
    c->s_k = (double*)zal(sd);
    c->s_c1 = (double*)zal(sd);
    c->s_c2 = (double*)zal(sd);
    for (int s = 0; s < c->ns; ++s) {
        c->s_type[s] = m->s_type[s];
        c->s_status[s] = 1;
        c->s_p1[s] = m->s_p1[s];
        c->s_p2[s] = m->s_p2[s];
        c->s_rest[s] = rf(c, m->s_rest[s]);
        c->s_k[s] = rf(c, m->s_k[s]);
        c->s_c1[s] = rf(c, m->s_c1[s]);
        c->s_c2[s] = rf(c, m->s_c2[s]);
    }
    size_t ai = sizeof(int) * (size_t)c->na, ad = sizeof(double) * (size_t)c->na;
    c->a_type = (int*)zal(ai);
    c->a_status = (int*)zal(ai);
    c->a_b1 = (int*)zal(ai);
    c->a_b2 = (int*)zal(ai);
    c->a_b3 = (int*)zal(ai);
    c->a_s1 = (int*)zal(ai);
    c->a_s2 = (int*)zal(ai);
    c->a_theta0 = (double*)zal(ad);
    c->a_k = (double*)zal(ad);
    for (int a = 0; a < c->na; ++a) {
        c->a_type[a] = m->a_type[a];
        c->a_status[a] = 1;
        c->a_b1[a] = m->a_b1[a];
        c->a_b2[a] = m->a_b2[a];
        c->a_b3[a] = m->a_b3[a];
        c->a_s1[a] = m->a_s1[a];
        c->a_s2[a] = m->a_s2[a];
        c->a_theta0[a] = rf(c, m->a_theta0[a]);
        c->a_k[a] = rf(c, m->a_k[a]);
    }
    c->p_kind = (int*)zal(sizeof(int) * (size_t)(c->np ? c->np : 1));
    c->p_c = (double*)zal(sizeof(double) * 6 * (size_t)(c->np ? c->np : 1));
    for (int p = 0; p < c->np; ++p) {
        c->p_kind[p] = m->pair_kind[p];
        fo_derive_pair(m->pair_kind[p], m->pair_raw + 4 * p, c->p_c + 6 * p);
    }
    c->cell_nh = (int*)zal(sizeof(int) * 13 * (size_t)c->d.ncells);
    fo_cell_neighbours_mask(&c->d, c->periodic, c->cell_nh);
    c->grid_head = (int*)zal(sizeof(int) * (size_t)c->d.ncells);
    c->grid_slot = (int*)zal(sizeof(int) * (size_t)c->d.ncells * (size_t)c->cell_cap);
    c->bead_cell = (int*)zal(ni);
    c->list_head = (int*)zal(ni);
    c->list_j = (int*)zal(sizeof(int) * (size_t)c->nb * (size_t)c->list_cap);
    c->list_pair = (int*)zal(sizeof(int) * (size_t)c->nb * (size_t)c->list_cap);
    build_incidence(c);
    return c;
}

/* ---------------------------------------------------------------------- */
/* AdvancePosition, kernel.cl:195-265, for one bead.                        */
static void advance_position(fo_ctx* c, int i) {
    double* p = c->pos + 3 * i;
    double* im = c->img + 3 * i;
    double* v = c->vel + 3 * i;
    double* f = c->force + 3 * i;
    double* vo = c->vel_old + 3 * i;
    double* fo = c->force_old + 3 * i;
    double lambda_dt = c->lam[i];
    double half_dt2 = c->hdt2[i];
    double inc[3];
    for (int a = 0; a < 3; ++a) {
        inc[a] = vo[a];
        v[a] = rf(c, f[a] * lambda_dt + inc[a]);
    }
    for (int a = 0; a < 3; ++a) inc[a] *= c->d.dt;
    for (int a = 0; a < 3; ++a) inc[a] = f[a] * half_dt2 + inc[a];
    for (int a = 0; a < 3; ++a) {
        p[a] += inc[a];
        im[a] += inc[a];
    }
    for (int a = 0; a < 3; ++a) {
        fo[a] = f[a];
        f[a] = c->d.damping * v[a];
        f[a] += c->d.gravity[a];
    }
    /* kernel.cl:241-250 snap wrap, z then y then x */
    for (int a = 2; a >= 0; --a)
        if ((c->periodic >> a) & 1)
            if (p[a] < 0.0) p[a] = c->d.box[a];
    for (int a = 2; a >= 0; --a)
        if ((c->periodic >> a) & 1)
            if (p[a] > c->d.box[a]) p[a] = 0.0;
    /* kernel.cl:252-261 wall penalty */
    for (int a = 2; a >= 0; --a)
        if ((c->walls >> a) & 1)
            if (p[a] < 0.0) f[a] += p[a] * c->d.wall_k * -1.0;
    for (int a = 2; a >= 0; --a)
        if ((c->walls >> a) & 1)
            if (p[a] > c->d.box[a]) f[a] += (p[a] - c->d.box[a]) * c->d.wall_k * -1.0;
}

/* AdvanceVelocity, kernel.cl:444-464. */
static void advance_velocity(fo_ctx* c, int i) {
    double half_dt = c->hdt[i];
    for (int a = 0; a < 3; ++a) {
        double f = c->force[3 * i + a];
        f += c->force_old[3 * i + a];
        c->vel_old[3 * i + a] = rf(c, f * half_dt + c->vel_old[3 * i + a]);
    }
}

/* ResolveSprings, kernel.cl:366-441, for spring s.  Returns 1 when a force
   acts; f receives the force on p1 (p2 gets its negation).  *broke is set when
   this call breaks an HR_FL spring (kernel.cl:391-397). */
static int spring_force(const fo_ctx* c, int s, double f[3], int* broke) {
    *broke = 0;
    int type = c->s_type[s];
    if (!(type == 0 || type == 1)) return 0;
    if (c->s_status[s] != 1) return 0;
    const double* a = c->img + 3 * c->s_p1[s];
    const double* b = c->img + 3 * c->s_p2[s];
    double ds[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    double l = sqrt(ds[0] * ds[0] + ds[1] * ds[1] + ds[2] * ds[2]);
    double factor = c->s_rest[s] - l;
    if (l != 0.0) l = 1.0 / l;
    ds[0] *= l;
    ds[1] *= l;
    ds[2] *= l;
    if (type == 1) {
        double stress = -c->s_c1[s] * factor * l;
        if (fabs(stress) > c->s_c2[s]) {
            *broke = 1;
            return 0;
        }
    }
    factor *= c->s_k[s];
    f[0] = ds[0] * factor;
    f[1] = ds[1] * factor;
    f[2] = ds[2] * factor;
    return 1;
}

/* Status of spring s after this step's break test, without changing it. */
static int spring_alive_after(const fo_ctx* c, int s) {
    double f[3];
    int broke;
    if (c->s_status[s] != 1) return 0;
    spring_force(c, s, f, &broke);
    return !broke;
}

/* ResolveAngles, kernel.cl:268-363, force part for angle a (status already
   decided).  pa acts on b1, pc on b3, b2 gets (-pa - pc). */
static void angle_force(const fo_ctx* c, int a, double pa[3], double pc[3]) {
    const double* t2 = c->img + 3 * c->a_b2[a];
    const double* t1 = c->img + 3 * c->a_b1[a];
    const double* t3 = c->img + 3 * c->a_b3[a];
    double ba[3] = {t1[0] - t2[0], t1[1] - t2[1], t1[2] - t2[2]};
    double bc[3] = {t3[0] - t2[0], t3[1] - t2[1], t3[2] - t2[2]};
    double cb[3] = {bc[0] * -1.0, bc[1] * -1.0, bc[2] * -1.0};
    double l_ba = sqrt(ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2]);
    double l_bc = sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    double dotp = (ba[0] * bc[0] + ba[1] * bc[1] + ba[2] * bc[2]) / (l_ba * l_bc);
    if (dotp < -1.0) dotp = -0.999999;
    if (dotp > 1.0) dotp = 0.999999;
    double angle = c->mode == FO_MODE_MIRROR ? fn_acos(dotp) : acos(dotp);
    double magnitude = -2.0 * c->a_k[a] * (angle - c->a_theta0[a]);
    double fa = magnitude / l_ba;
    double fc = magnitude / l_bc;
    double t[3] = {ba[1] * bc[2] - ba[2] * bc[1], ba[2] * bc[0] - ba[0] * bc[2],
                   ba[0] * bc[1] - ba[1] * bc[0]};
    pa[0] = (ba[1] * t[2] - ba[2] * t[1]);
    pa[1] = (ba[2] * t[0] - ba[0] * t[2]);
    pa[2] = (ba[0] * t[1] - ba[1] * t[0]);
    double ln = sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
    if (ln != 0.0) ln = 1.0 / ln;
    ln *= fa;
    pa[0] *= ln;
    pa[1] *= ln;
    pa[2] *= ln;
    pc[0] = (cb[1] * t[2] - cb[2] * t[1]);
    pc[1] = (cb[2] * t[0] - cb[0] * t[2]);
    pc[2] = (cb[0] * t[1] - cb[1] * t[0]);
    ln = sqrt(pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
    if (ln != 0.0) ln = 1.0 / ln;
    ln *= fc;
    pc[0] *= ln;
    pc[1] *= ln;
    pc[2] *= ln;
}

/* Angle status for this step, kernel.cl:274-286.  In REF mode the spring
   statuses were already updated by this step's ResolveSprings; in MIRROR mode
   the break test is re-evaluated, which gives the same answer. */
static int angle_alive(const fo_ctx* c, int a, int springs_done) {
    if (c->a_status[a] != 1) return 0;
    if (c->a_type[a] == 1) {
        int s1 = c->a_s1[a], s2 = c->a_s2[a];
        int ok1 = springs_done ? (c->s_status[s1] == 1) : spring_alive_after(c, s1);
        int ok2 = springs_done ? (c->s_status[s2] == 1) : spring_alive_after(c, s2);
        if (!ok1 || !ok2) return 0;
    }
    return 1;
}

/* Minimum image on the axes in mask, as kernel.cl:598-627 / 844-870. */
static inline double min_image(const fo_ctx* c, double r[3], double length, int mask) {
    double maxDim = c->d.half_box_sq;
    if (length > maxDim) {
        for (int a = 0; a < 3; ++a)
            if ((mask >> a) & 1) {
                if (r[a] * r[a] > maxDim) {
                    if (r[a] > 0.0)
                        r[a] -= c->d.box[a];
                    else
                        r[a] += c->d.box[a];
                }
            }
        length = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    }
    return length;
}

/* One ResolveContacts list entry, kernel.cl:835-999: returns 1 and the force
   on bead i (the partner gets its negation) when the pair interacts. */
static int contact_force(const fo_ctx* c, int i, int j, int pair_id, double R[3]) {
    const double* p1 = c->pos + 3 * i;
    const double* p2 = c->pos + 3 * j;
    double rij[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
    double length = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
    length = min_image(c, rij, length, c->force_mi);
    const double* cc = c->p_c + 6 * pair_id;
    int kind = c->p_kind[pair_id];
    if (kind == 1) {
        if (length < c->d.cutoff_sq) {
            double r2 = length;
            length = sqrt(length);
            if (length < cc[2]) {
                double sigma2 = cc[0];
                double epsilon = cc[1];
                sigma2 *= sigma2;
                double fr2 = sigma2 / r2;
                double fr6 = fr2 * fr2 * fr2;
                double fpr = 48.0 * epsilon * fr6 * (fr6 - 0.5) / r2;
                fpr -= cc[3];
                length = (length != 0.0) ? 1.0 / length : 0.0;
                R[0] = fpr * (rij[0] * length);
                R[1] = fpr * (rij[1] * length);
                R[2] = fpr * (rij[2] * length);
                return 1;
            }
        }
        return 0;
    }
    if (kind == 2) {
        length = sqrt(length);
        double K = cc[0];
        double penetration = (c->radius[i] + c->radius[j]) - length;
        if (penetration > 0.0) {
            length = (length != 0.0) ? 1.0 / length : 0.0;
            penetration *= K;
            R[0] = penetration * (rij[0] * length);
            R[1] = penetration * (rij[1] * length);
            R[2] = penetration * (rij[2] * length);
            return 1;
        }
        return 0;
    }
    if (kind == 4) {
        /* extension without reference counterpart (penalty + soft repulsion) */
        length = sqrt(length);
        double penetration = (c->radius[i] + c->radius[j]) - length;
        double mag = 0.0;
        int acts = 0;
        if (penetration > 0.0) {
            mag += penetration * cc[0];
            acts = 1;
        }
        if (length < cc[2]) {
            mag += (cc[2] - length) * cc[1];
            acts = 1;
        }
        if (acts) {
            length = (length != 0.0) ? 1.0 / length : 0.0;
            R[0] = mag * (rij[0] * length);
            R[1] = mag * (rij[1] * length);
            R[2] = mag * (rij[2] * length);
        }
        return acts;
    }
    if (kind == 3) {
        if (length < cc[3]) {
            length = sqrt(length);
            double K = cc[0];
            double l0 = cc[1];
            double factor = (l0 - length);
            factor *= K; /* both arms of kernel.cl:970-973 are identical */
            factor += (cc[5] - length) * cc[4];
            length = (length != 0.0) ? 1.0 / length : 0.0;
            R[0] = factor * (rij[0] * length);
            R[1] = factor * (rij[1] * length);
            R[2] = factor * (rij[2] * length);
            return 1;
        }
        return 0;
    }
    return 0;
}

/* Candidate test of BuildContactList for beads (b1, b2), kernel.cl:574-659:
   exclusion, minimum image (pbc only), list radius by pair kind.  Returns
   the pair-table index when listed, else -1. */
static int list_candidate(const fo_ctx* c, int b1, int b2) {
    int collidable = 0;
    if (c->tag[b1] != c->tag[b2])
        collidable = 1;
    else if (abs(c->loc_id[b1] - c->loc_id[b2]) > 1)
        collidable = 1;
    if (!collidable) return -1;
    const double* p1 = c->pos + 3 * b1;
    const double* p2 = c->pos + 3 * b2;
    double rij[3] = {p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]};
    double length = rij[0] * rij[0] + rij[1] * rij[1] + rij[2] * rij[2];
    if (c->list_mi) length = min_image(c, rij, length, c->list_mi);
    int pair_id = getadress(c->type[b1], c->type[b2], c->d.types_num);
    int kind = c->p_kind[pair_id];
    if (kind == 1 || kind == 3 || kind == 4) {
        if (length < c->d.cutoff_sq) return pair_id;
    }
    if (kind == 2 || kind == 4) {
        double min_skin = (c->skin[b1] > c->skin[b2]) ? c->skin[b2] : c->skin[b1];
        double max_radius = (c->radius[b1] > c->radius[b2]) ? c->radius[b1] : c->radius[b2];
        double lim = max_radius + min_skin;
        if (length < lim * lim) return pair_id; /* pow(x, 2.0), kernel.cl:650 */
    }
    return -1;
}

static void list_push(fo_ctx* c, int b1, int b2, int pair_id) {
    int size = c->list_head[b1]++;
    if (size < c->list_cap) {
        c->list_j[(size_t)b1 * c->list_cap + size] = b2;
        c->list_pair[(size_t)b1 * c->list_cap + size] = pair_id;
    } else {
        c->overflow_lists++;
    }
}

/* ResetGrid + ResetContactList + FillGrid, kernel.cl:487-525, single sweep
   in ascending bead order (so each cell holds its beads in ascending order and
   keeps the first cell_cap of them). */
static void fill_grid(fo_ctx* c) {
    memset(c->grid_head, 0, sizeof(int) * (size_t)c->d.ncells);
    memset(c->list_head, 0, sizeof(int) * (size_t)c->nb);
    for (int i = 0; i < c->nb; ++i) {
        c->bead_cell[i] = -1;
        const double* p = c->pos + 3 * i;
        double qx = floor(p[0] / c->d.step[0]);
        double qy = floor(p[1] / c->d.step[1]);
        double qz = floor(p[2] / c->d.step[2]);
        if (!(qx >= 0.0 && qx < c->d.nx && qy >= 0.0 && qy < c->d.ny && qz >= 0.0 && qz < c->d.nz)) continue;
        int cell = (int)qx + (int)qy * c->d.nx + (int)qz * c->d.nxy;
        int old = c->grid_head[cell]++;
        if (old < c->cell_cap) {
            c->grid_slot[(size_t)cell * c->cell_cap + old] = i;
            c->bead_cell[i] = cell;
        } else {
            c->overflow_cells++;
        }
    }
}

/* BuildContactList, kernel.cl:532-789, in the reference's visiting order. */
static void build_lists_ref(fo_ctx* c) {
    for (int cell = 0; cell < c->d.ncells; ++cell) {
        int n = c->grid_head[cell];
        if (n <= 0) continue;
        if (n > c->cell_cap) n = c->cell_cap;
        const int* ids = c->grid_slot + (size_t)cell * c->cell_cap;
        for (int ii = 0; ii < n - 1; ii++)
            for (int jj = ii + 1; jj < n; jj++) {
                int pid = list_candidate(c, ids[ii], ids[jj]);
                if (pid >= 0) list_push(c, ids[ii], ids[jj], pid);
            }
        for (int k = 0; k < 13; ++k) {
            int nc = c->cell_nh[(size_t)cell * 13 + k];
            if (nc == -1) continue;
            int m = c->grid_head[nc];
            if (m <= 0) continue;
            if (m > c->cell_cap) m = c->cell_cap;
            const int* nids = c->grid_slot + (size_t)nc * c->cell_cap;
            for (int jj = 0; jj < m; jj++)
                for (int kk = 0; kk < n; kk++) {
                    int pid = list_candidate(c, ids[kk], nids[jj]);
                    if (pid >= 0) list_push(c, ids[kk], nids[jj], pid);
                }
        }
    }
}

/* Cell of (cx+dx, cy+dy, cz+dz) under the wrap rules, or -1. */
static int stencil_cell(const fo_ctx* c, int x, int y, int z) {
    int n[3] = {c->d.nx, c->d.ny, c->d.nz};
    int q[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
        if (q[a] < 0 || q[a] >= n[a]) {
            if (!((c->periodic >> a) & 1)) return -1;
            q[a] = q[a] < 0 ? n[a] - 1 : 0;
        }
    }
    return q[0] + q[1] * c->d.nx + q[2] * c->d.nxy;
}

/* Full per-bead lists over the 27-cell neighbourhood (dz, dy, dx ascending;
   beads ascending inside each cell): the same pair set as the reference's
   half-shell sweep, in the order the B200 path gathers it. */
static void build_lists_mirror(fo_ctx* c) {
    for (int i = 0; i < c->nb; ++i) {
        int cell = c->bead_cell[i];
        if (cell < 0) continue;
        int cz = cell / c->d.nxy, cy = (cell % c->d.nxy) / c->d.nx, cx = cell % c->d.nx;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int nc = stencil_cell(c, cx + dx, cy + dy, cz + dz);
                    if (nc < 0) continue;
                    int m = c->grid_head[nc];
                    if (m > c->cell_cap) m = c->cell_cap;
                    const int* ids = c->grid_slot + (size_t)nc * c->cell_cap;
                    for (int k = 0; k < m; ++k) {
                        int j = ids[k];
                        if (j == i) continue;
                        int pid = list_candidate(c, i, j);
                        if (pid >= 0) list_push(c, i, j, pid);
                    }
                }
    }
}

FO_EXPORT void fo_rebuild(fo_ctx* c) {
    fill_grid(c);
    if (c->mode == FO_MODE_REF)
        build_lists_ref(c);
    else
        build_lists_mirror(c);
}

/* Springs, angles and contacts in the reference's order: one work-item sweep
   per kernel, atomics as ordered additions (kernel.cl:366-441, 268-363,
   792-1011). */
static void forces_ref(fo_ctx* c, int springs, int angles, int contacts) {
    if (springs)
        for (int s = 0; s < c->ns; ++s) {
            double f[3];
            int broke;
            int act = spring_force(c, s, f, &broke);
            if (broke) c->s_status[s] = 0;
            if (act) {
                double* f1 = c->force + 3 * c->s_p1[s];
                double* f2 = c->force + 3 * c->s_p2[s];
                for (int a = 0; a < 3; ++a) f1[a] += f[a];
                for (int a = 0; a < 3; ++a) f2[a] += f[a] * -1.0;
            }
        }
    if (angles)
        for (int a = 0; a < c->na; ++a) {
            if (!angle_alive(c, a, 1)) {
                c->a_status[a] = 0;
                continue;
            }
            double pa[3], pc[3];
            angle_force(c, a, pa, pc);
            double* f1 = c->force + 3 * c->a_b1[a];
            double* f3 = c->force + 3 * c->a_b3[a];
            double* f2 = c->force + 3 * c->a_b2[a];
            for (int k = 0; k < 3; ++k) f1[k] += pa[k];
            for (int k = 0; k < 3; ++k) f3[k] += pc[k];
            for (int k = 0; k < 3; ++k) f2[k] += -pa[k] - pc[k];
        }
    if (contacts)
        for (int i = 0; i < c->nb; ++i) {
            int n = c->list_head[i];
            if (n <= 0) continue;
            if (n > c->list_cap) n = c->list_cap;
            double acc[3] = {0.0, 0.0, 0.0};
            int has_contact = 0;
            for (int k = 0; k < n; ++k) {
                int j = c->list_j[(size_t)i * c->list_cap + k];
                int pid = c->list_pair[(size_t)i * c->list_cap + k];
                double R[3];
                if (contact_force(c, i, j, pid, R)) {
                    for (int a = 0; a < 3; ++a) acc[a] += R[a];
                    for (int a = 0; a < 3; ++a) c->force[3 * j + a] += -R[a];
                    has_contact = 1;
                }
            }
            if (has_contact)
                for (int a = 0; a < 3; ++a) c->force[3 * i + a] += acc[a];
        }
}

/* The same forces gathered per bead in the B200 path's order: the current
   force (base) + incident springs + incident angles + contact list. */
static void forces_mirror(fo_ctx* c, int springs, int angles, int contacts) {
    double* out = (double*)zal(sizeof(double) * 3 * (size_t)c->nb);
    int* sbroke = (int*)zal(sizeof(int) * (size_t)(c->ns ? c->ns : 1));
    int* adead = (int*)zal(sizeof(int) * (size_t)(c->na ? c->na : 1));
    for (int i = 0; i < c->nb; ++i) {
        double F[3] = {c->force[3 * i], c->force[3 * i + 1], c->force[3 * i + 2]};
        if (springs)
            for (int e = c->sp_off[i]; e < c->sp_off[i + 1]; ++e) {
                int s = c->sp_idx[e] >> 1, role = c->sp_idx[e] & 1;
                double f[3];
                int broke;
                if (spring_force(c, s, f, &broke)) {
                    for (int a = 0; a < 3; ++a) F[a] += role == 0 ? f[a] : f[a] * -1.0;
                }
                if (broke) sbroke[s] = 1;
            }
        if (angles)
            for (int e = c->an_off[i]; e < c->an_off[i + 1]; ++e) {
                int a = c->an_idx[e] / 3, role = c->an_idx[e] % 3;
                if (!angle_alive(c, a, 0)) {
                    adead[a] = 1;
                    continue;
                }
                double pa[3], pc[3];
                angle_force(c, a, pa, pc);
                for (int k = 0; k < 3; ++k) F[k] += role == 0 ? pa[k] : role == 2 ? pc[k] : -pa[k] - pc[k];
            }
        if (contacts) {
            int n = c->list_head[i];
            if (n > c->list_cap) n = c->list_cap;
            for (int k = 0; k < n; ++k) {
                int j = c->list_j[(size_t)i * c->list_cap + k];
                int pid = c->list_pair[(size_t)i * c->list_cap + k];
                double R[3];
                if (contact_force(c, i, j, pid, R))
                    for (int a = 0; a < 3; ++a) F[a] += R[a];
            }
        }
        for (int a = 0; a < 3; ++a) out[3 * i + a] = rf(c, F[a]);
    }
    memcpy(c->force, out, sizeof(double) * 3 * (size_t)c->nb);
    for (int s = 0; s < c->ns; ++s)
        if (sbroke[s]) c->s_status[s] = 0;
    for (int a = 0; a < c->na; ++a)
        if (adead[a]) c->a_status[a] = 0;
    free(out);
    free(sbroke);
    free(adead);
}

static void forces(fo_ctx* c, int springs, int angles, int contacts) {
    if (c->mode == FO_MODE_REF)
        forces_ref(c, springs, angles, contacts);
    else
        forces_mirror(c, springs, angles, contacts);
}

/* RunSimulationLoop, SimulationManager.cpp:151-181. */
FO_EXPORT int fo_run(fo_ctx* c, int loop_size) {
    int grid_update_cnt = 0;
    if (loop_size <= 0) return -1;
    for (int step = 0; step < loop_size; step++) {
        if (grid_update_cnt == c->d.grid_update_freq) grid_update_cnt = 0;
        for (int i = 0; i < c->nb; ++i) advance_position(c, i);
        if (grid_update_cnt == 0) fo_rebuild(c);
        forces(c, c->ns > 0, c->na > 0, 1);
        for (int i = 0; i < c->nb; ++i) advance_velocity(c, i);
        grid_update_cnt++;
    }
    return 0;
}

/* ResetBeadEnergy, kernel.cl:468-483. */
FO_EXPORT void fo_reset_energy(fo_ctx* c) {
    for (int k = 0; k < 3 * c->nb; ++k) {
        c->force[k] = 0.0;
        c->vel[k] = 0.0;
        c->force_old[k] = 0.0;
        c->vel_old[k] = 0.0;
    }
}

/* Forces alone at the current positions (zeroed first, no base term) with the
   current contact list; for one-step force parity. */
FO_EXPORT void fo_forces_only(fo_ctx* c, int springs, int angles, int contacts) {
    memset(c->force, 0, sizeof(double) * 3 * (size_t)c->nb);
    forces(c, springs, angles, contacts);
}

static double* field_ptr(fo_ctx* c, int field) {
    switch (field) {
        case 0: return c->pos;
        case 1: return c->img;
        case 2: return c->vel;
        case 3: return c->force;
        case 4: return c->vel_old;
        case 5: return c->force_old;
        default: return NULL;
    }
}

/* field: 0 position, 1 image_position, 2 velocity, 3 force, 4 velocity_old,
   5 force_old (3 doubles per bead). */
FO_EXPORT int fo_get_beads(fo_ctx* c, int field, double* out) {
    double* p = field_ptr(c, field);
    if (!p) return -1;
    memcpy(out, p, sizeof(double) * 3 * (size_t)c->nb);
    return 0;
}

FO_EXPORT int fo_set_beads(fo_ctx* c, int field, const double* in) {
    double* p = field_ptr(c, field);
    if (!p) return -1;
    for (int k = 0; k < 3 * c->nb; ++k) p[k] = (field <= 1) ? in[k] : rf(c, in[k]);
    return 0;
}

FO_EXPORT void fo_get_status(const fo_ctx* c, int* springs, int* angles) {
    if (springs) memcpy(springs, c->s_status, sizeof(int) * (size_t)c->ns);
    if (angles) memcpy(angles, c->a_status, sizeof(int) * (size_t)c->na);
}

FO_EXPORT void fo_set_status(fo_ctx* c, const int* springs, const int* angles) {
    if (springs) memcpy(c->s_status, springs, sizeof(int) * (size_t)c->ns);
    if (angles) memcpy(c->a_status, angles, sizeof(int) * (size_t)c->na);
}

FO_EXPORT int fo_n_cells(const fo_ctx* c) { return c->d.ncells; }
FO_EXPORT int fo_list_cap(const fo_ctx* c) { return c->list_cap; }

/* Cell of each bead after the last rebuild (-1 = outside the grid or beyond
   the cell capacity) and the raw per-cell counts. */
FO_EXPORT void fo_get_cells(const fo_ctx* c, int* bead_cell, int* cell_count) {
    if (bead_cell) memcpy(bead_cell, c->bead_cell, sizeof(int) * (size_t)c->nb);
    if (cell_count) memcpy(cell_count, c->grid_head, sizeof(int) * (size_t)c->d.ncells);
}

/* Contact lists: raw counts and list_cap entries per bead. */
FO_EXPORT void fo_get_lists(const fo_ctx* c, int* head, int* partners, int* pairs) {
    memcpy(head, c->list_head, sizeof(int) * (size_t)c->nb);
    if (partners) memcpy(partners, c->list_j, sizeof(int) * (size_t)c->nb * (size_t)c->list_cap);
    if (pairs) memcpy(pairs, c->list_pair, sizeof(int) * (size_t)c->nb * (size_t)c->list_cap);
}

FO_EXPORT double fo_detmath_acos(double x) { return fn_acos(x); }

/* The settings derived from the input (SimulationManager.cpp:647-720,
   804-805, 2178-2190) as 20 doubles: dt, half_dt, half_dt2, lambda_dt,
   damping, cutoff_sq, wall_k, gravity[3], box[3], step[3], half_box_sq, nx,
   ny, nz; and the pair table (SimulationManager.cpp:859-942): 6 coefficients
   and the kind per pair.  For checks of a host precompute against this one. */
FO_EXPORT void fo_get_derived(const fo_ctx* c, double* out20) {
    const fo_derived* d = &c->d;
    const double v[20] = {d->dt, d->half_dt, d->half_dt2, d->lambda_dt, d->damping, d->cutoff_sq, d->wall_k,
                          d->gravity[0], d->gravity[1], d->gravity[2], d->box[0], d->box[1], d->box[2],
                          d->step[0], d->step[1], d->step[2], d->half_box_sq, (double)d->nx, (double)d->ny,
                          (double)d->nz};
    memcpy(out20, v, sizeof v);
}
FO_EXPORT int fo_get_pairs(const fo_ctx* c, double* coeffs6, int* kinds) {
    memcpy(coeffs6, c->p_c, sizeof(double) * 6 * (size_t)c->np);
    memcpy(kinds, c->p_kind, sizeof(int) * (size_t)c->np);
    return c->np;
}

FO_EXPORT void fo_overflow(const fo_ctx* c, long* out2) {
    out2[0] = c->overflow_cells;
    out2[1] = c->overflow_lists;
}
