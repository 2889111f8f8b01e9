/*
 * ref_driver.c -- host driver that runs the reference's own kernels
 * (FibreNet/kernel.cl, compiled unmodified as C through cl_shim.h) on the CPU.
 * TEST INFRASTRUCTURE ONLY: it is the "reference" the parity tests pin the
 * oracle restatement against, and the timed CPU baseline of bench.py.
 *
 * Built by oracle/Makefile into oracle/_ref/libfnref.so from the sources
 * where they lie; the kernel file is pulled in with FN_KERNEL_CL.
 *
 * The step schedule restates SimulationManager::RunSimulationLoop
 * (SimulationManager.cpp:151-181) and the kernel argument binding of
 * ReadKernelData (SimulationManager.cpp:1236-1304).  threads <= 1 runs every
 * work-item in ascending order on one thread, which makes the reference's
 * atomics deterministic; threads > 1 runs work-items with OpenMP.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cl_shim.h"

_Thread_local int fn_cl_global_id;

#ifndef FN_KERNEL_CL
#error "FN_KERNEL_CL must name the reference kernel file"
#endif
#include FN_KERNEL_CL

#undef inline
#include "oracle_host.h"

typedef struct ref_ctx {
    int nb, ns, na, ncells, threads, grid_update_freq;
    _Bead* beads;
    _particle_info* info;
    _spring* springs;
    angle_bond* angles;
    _pair* pairs;
    int* grid_head;
    _GridCell* grid_tail;
    _gridCellNh* grid_nh;
    int* nh_head;
    _particleNh* nh_tail;
    _particleNh* inter_id;
    _settings settings;
} ref_ctx;

#define REF_EXPORT __attribute__((visibility("default")))

/* Runs work-items 0..n-1 of one kernel call. */
#define RUN_ITEMS(ctx, n, call)                                                      \
    do {                                                                             \
        int n_ = (n);                                                                \
        if ((ctx)->threads <= 1) {                                                   \
            for (int g_ = 0; g_ < n_; ++g_) {                                        \
                fn_cl_global_id = g_;                                                \
                call;                                                                \
            }                                                                        \
        } else {                                                                     \
            int nt_ = (ctx)->threads;                                                \
            _Pragma("omp parallel for num_threads(nt_) schedule(static)")      \
            for (int g_ = 0; g_ < n_; ++g_) {                                        \
                fn_cl_global_id = g_;                                                \
                call;                                                                \
            }                                                                        \
        }                                                                            \
    } while (0)

static void* zalloc(size_t n) {
    void* p = calloc(n ? n : 1, 1);
    if (!p) {
        fprintf(stderr, "ref_driver: out of host memory (%zu bytes)\n", n);
        abort();
    }
    return p;
}

REF_EXPORT void ref_destroy(ref_ctx* c) {
    if (!c) return;
    free(c->beads);
    free(c->info);
    free(c->springs);
    free(c->angles);
    free(c->pairs);
    free(c->grid_head);
    free(c->grid_tail);
    free(c->grid_nh);
    free(c->nh_head);
    free(c->nh_tail);
    free(c->inter_id);
    free(c);
}

/* Builds the reference's buffers from the raw model, as ReadInputFile and
   ReadKernelData would (SimulationManager.cpp:1153-1307). */
REF_EXPORT ref_ctx* ref_create(const fo_model* m, int threads) {
    fo_derived d;
    fo_derive_settings(m, &d);
    ref_ctx* c = (ref_ctx*)zalloc(sizeof(ref_ctx));
    c->nb = m->n_beads;
    c->ns = m->n_springs;
    c->na = m->n_angles;
    c->ncells = d.ncells;
    c->threads = threads;
    c->grid_update_freq = d.grid_update_freq;

    _settings* s = &c->settings;
    memset(s, 0, sizeof(*s));
    s->types_num = d.types_num;
    s->bc_type = d.bc_type;
    s->wall_contact_stiffness = d.wall_k;
    s->cutoff = d.cutoff;
    s->cutoff_sq = d.cutoff_sq;
    s->box_unit_cell = d.box_unit_cell;
    s->dt = d.dt;
    s->half_dt = d.half_dt;
    s->half_dt2 = d.half_dt2;
    s->lambda_dt = d.lambda_dt;
    s->damping = d.damping;
    s->gridCellsX = d.nx;
    s->gridCellsY = d.ny;
    s->gridCellsZ = d.nz;
    s->gridCellsXY = d.nxy;
    s->halfBoxSq = d.half_box_sq;
    s->gridStep.x = d.step[0];
    s->gridStep.y = d.step[1];
    s->gridStep.z = d.step[2];
    s->boxSize.x = d.box[0];
    s->boxSize.y = d.box[1];
    s->boxSize.z = d.box[2];
    s->gravity.x = d.gravity[0];
    s->gravity.y = d.gravity[1];
    s->gravity.z = d.gravity[2];

    c->beads = (_Bead*)zalloc(sizeof(_Bead) * (size_t)c->nb);
    c->info = (_particle_info*)zalloc(sizeof(_particle_info) * (size_t)c->nb);
    for (int i = 0; i < c->nb; ++i) {
        _Bead* b = &c->beads[i];
        b->position.x = m->pos[3 * i + 0];
        b->position.y = m->pos[3 * i + 1];
        b->position.z = m->pos[3 * i + 2];
        b->velocity.x = m->vel[3 * i + 0];
        b->velocity.y = m->vel[3 * i + 1];
        b->velocity.z = m->vel[3 * i + 2];
        b->velocity_old.x = m->vel_old[3 * i + 0];
        b->velocity_old.y = m->vel_old[3 * i + 1];
        b->velocity_old.z = m->vel_old[3 * i + 2];
        b->force.x = m->force[3 * i + 0];
        b->force.y = m->force[3 * i + 1];
        b->force.z = m->force[3 * i + 2];
        b->force_old = b->force;
        b->image_position.x = m->img[3 * i + 0];
        b->image_position.y = m->img[3 * i + 1];
        b->image_position.z = m->img[3 * i + 2];
        double k[9];
        fo_derive_bead(&d, m->mass[i], m->radius[i], m->skin_ratio, k);
        _particle_info* p = &c->info[i];
        p->type = m->type[i];
        p->tag = m->tag[i];
        p->loc_id = m->loc_id[i];
        p->mass = k[0];
        p->mass_inv = k[1];
        p->lambda_dt_mass_inv = k[2];
        p->half_dt_mass_inv = k[3];
        p->half_dt2_mass_inv = k[4];
        p->radius = k[5];
        p->radius_sq = k[6];
        p->skin_radius = k[7];
        p->skin_radius_sq = k[8];
    }
    c->springs = (_spring*)zalloc(sizeof(_spring) * (size_t)c->ns);
    for (int i = 0; i < c->ns; ++i) {
        _spring* sp = &c->springs[i];
        sp->type = m->s_type[i];
        sp->tag = m->s_tag[i];
        sp->status = 1;
        sp->p1 = m->s_p1[i];
        sp->p2 = m->s_p2[i];
        sp->restLength = m->s_rest[i];
        sp->stiffness = m->s_k[i];
        sp->damping = 0.0;
        sp->c1 = m->s_c1[i];
        sp->c2 = m->s_c2[i];
    }
    c->angles = (angle_bond*)zalloc(sizeof(angle_bond) * (size_t)c->na);
    for (int i = 0; i < c->na; ++i) {
        angle_bond* a = &c->angles[i];
        a->type = m->a_type[i];
        a->tag = 0;
        a->status = 1;
        a->b1 = m->a_b1[i];
        a->b2 = m->a_b2[i];
        a->b3 = m->a_b3[i];
        a->s1 = m->a_s1[i];
        a->s2 = m->a_s2[i];
        a->angle = m->a_theta0[i];
        a->c1 = m->a_k[i];
    }
    int np = m->n_types * (m->n_types + 1) / 2;
    c->pairs = (_pair*)zalloc(sizeof(_pair) * (size_t)(np ? np : 1));
    for (int i = 0; i < np; ++i) {
        double cc[6];
        fo_derive_pair(m->pair_kind[i], m->pair_raw + 4 * i, cc);
        c->pairs[i].type = m->pair_kind[i];
        c->pairs[i].c1 = cc[0];
        c->pairs[i].c2 = cc[1];
        c->pairs[i].c3 = cc[2];
        c->pairs[i].c4 = cc[3];
        c->pairs[i].c5 = cc[4];
        c->pairs[i].c6 = cc[5];
    }
    c->grid_head = (int*)zalloc(sizeof(int) * (size_t)c->ncells);
    c->grid_tail = (_GridCell*)zalloc(sizeof(_GridCell) * (size_t)c->ncells);
    c->grid_nh = (_gridCellNh*)zalloc(sizeof(_gridCellNh) * (size_t)c->ncells);
    fo_cell_neighbours(&d, (int*)c->grid_nh);
    c->nh_head = (int*)zalloc(sizeof(int) * (size_t)c->nb);
    c->nh_tail = (_particleNh*)zalloc(sizeof(_particleNh) * (size_t)c->nb);
    c->inter_id = (_particleNh*)zalloc(sizeof(_particleNh) * (size_t)c->nb);
    return c;
}

REF_EXPORT void ref_set_threads(ref_ctx* c, int threads) { c->threads = threads; }

/* ResetGrid, ResetContactList, FillGrid, BuildContactList, in the order of
   SimulationManager.cpp:168-173. */
REF_EXPORT void ref_rebuild(ref_ctx* c) {
    RUN_ITEMS(c, c->ncells, ResetGrid(c->grid_head, c->ncells));
    RUN_ITEMS(c, c->nb, ResetContactList(c->nh_head, c->nb));
    RUN_ITEMS(c, c->nb, FillGrid(c->beads, c->grid_head, c->grid_tail, c->settings, c->nb));
    RUN_ITEMS(c, c->ncells,
              BuildContactList(c->grid_head, c->grid_tail, c->grid_nh, c->nh_head, c->nh_tail,
                               c->beads, c->info, c->inter_id, c->pairs, c->settings, c->ncells));
}

/* SimulationManager::RunSimulationLoop, SimulationManager.cpp:151-181: the
   rebuild counter is local, so every call rebuilds at its first step. */
REF_EXPORT int ref_run(ref_ctx* c, int loop_size) {
    int grid_update_cnt = 0;
    if (loop_size <= 0) return -1;
    for (int step = 0; step < loop_size; step++) {
        if (grid_update_cnt == c->grid_update_freq) grid_update_cnt = 0;
        RUN_ITEMS(c, c->nb, AdvancePosition(c->beads, c->info, c->settings, c->nb));
        if (c->ns > 0) RUN_ITEMS(c, c->ns, ResolveSprings(c->beads, c->springs, c->ns));
        if (c->na > 0) RUN_ITEMS(c, c->na, ResolveAngles(c->angles, c->springs, c->beads, c->na));
        if (grid_update_cnt == 0) ref_rebuild(c);
        RUN_ITEMS(c, c->nb,
                  ResolveContacts(c->nh_head, c->nh_tail, c->beads, c->info, c->inter_id, c->pairs,
                                  c->settings, c->nb));
        RUN_ITEMS(c, c->nb, AdvanceVelocity(c->beads, c->info, c->nb, c->nb));
        grid_update_cnt++;
    }
    return 0;
}

/* ResetBeadEnergy (kernel.cl:468-483), as MinimizeSystemEnergy calls it. */
REF_EXPORT void ref_reset_energy(ref_ctx* c) {
    RUN_ITEMS(c, c->nb, ResetBeadEnergy(c->beads, c->nb));
}

/* Copies one bead field out as 3 doubles per bead:
   0 position, 1 image_position, 2 velocity, 3 force, 4 velocity_old,
   5 force_old. */
REF_EXPORT void ref_get_beads(const ref_ctx* c, int field, double* out) {
    for (int i = 0; i < c->nb; ++i) {
        const _Bead* b = &c->beads[i];
        const my_Vector3* v = field == 0   ? &b->position
                              : field == 1 ? &b->image_position
                              : field == 2 ? &b->velocity
                              : field == 3 ? &b->force
                              : field == 4 ? &b->velocity_old
                                           : &b->force_old;
        out[3 * i + 0] = v->x;
        out[3 * i + 1] = v->y;
        out[3 * i + 2] = v->z;
    }
}

REF_EXPORT void ref_get_status(const ref_ctx* c, int* spring_status, int* angle_status) {
    for (int i = 0; i < c->ns; ++i) spring_status[i] = c->springs[i].status;
    for (int i = 0; i < c->na; ++i) angle_status[i] = c->angles[i].status;
}

REF_EXPORT int ref_n_cells(const ref_ctx* c) { return c->ncells; }

/* Grid buckets: head[c] (raw atomic count) and up to 64 ids per cell. */
REF_EXPORT void ref_get_grid(const ref_ctx* c, int* head, int* tail64) {
    memcpy(head, c->grid_head, sizeof(int) * (size_t)c->ncells);
    memcpy(tail64, c->grid_tail, sizeof(_GridCell) * (size_t)c->ncells);
}

/* Contact lists: head[i] (raw atomic count), up to 256 partner ids and the
   pair-table index of each entry. */
REF_EXPORT void ref_get_lists(const ref_ctx* c, int* head, int* tail256, int* pair256) {
    memcpy(head, c->nh_head, sizeof(int) * (size_t)c->nb);
    memcpy(tail256, c->nh_tail, sizeof(_particleNh) * (size_t)c->nb);
    memcpy(pair256, c->inter_id, sizeof(_particleNh) * (size_t)c->nb);
}

/* The per-step force contributions alone: zero the forces, then one
   ResolveSprings / ResolveAngles / ResolveContacts pass at the current
   positions (contact list must have been built).  Used by the one-step force
   parity tests. */
REF_EXPORT void ref_forces_only(ref_ctx* c, int with_springs, int with_angles, int with_contacts) {
    for (int i = 0; i < c->nb; ++i) {
        c->beads[i].force.x = 0.0;
        c->beads[i].force.y = 0.0;
        c->beads[i].force.z = 0.0;
    }
    if (with_springs && c->ns > 0) RUN_ITEMS(c, c->ns, ResolveSprings(c->beads, c->springs, c->ns));
    if (with_angles && c->na > 0)
        RUN_ITEMS(c, c->na, ResolveAngles(c->angles, c->springs, c->beads, c->na));
    if (with_contacts)
        RUN_ITEMS(c, c->nb,
                  ResolveContacts(c->nh_head, c->nh_tail, c->beads, c->info, c->inter_id, c->pairs,
                                  c->settings, c->nb));
}

REF_EXPORT int ref_sizeof(int which) {
    switch (which) {
        case 0: return (int)sizeof(_Bead);
        case 1: return (int)sizeof(_particle_info);
        case 2: return (int)sizeof(_spring);
        case 3: return (int)sizeof(angle_bond);
        case 4: return (int)sizeof(_pair);
        case 5: return (int)sizeof(_settings);
        default: return -1;
    }
}
