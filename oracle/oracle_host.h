/*
 * oracle_host.h -- CPU restatement of the reference's host-side precompute
 * (SimulationManager.cpp), shared by both parity checkers in this folder.
 * TEST INFRASTRUCTURE ONLY; the product has its own implementation.
 *
 * The reference host cannot run here (MSVC/Windows, interactive OpenCL
 * device selection), so these few derivations are restated in C with the
 * reference's arithmetic kept operation for operation (float literals such as
 * 0.5f are exact in double and are written as doubles).
 */
#ifndef FIBRENET_ORACLE_HOST_H
#define FIBRENET_ORACLE_HOST_H

#include <math.h>
#include "oracle_model.h"

typedef struct fo_derived {
    double dt, half_dt, half_dt2, lambda_dt, damping;
    double cutoff, cutoff_sq, box_unit_cell, wall_k;
    double gravity[3], box[3], step[3];
    double half_box_sq;
    int nx, ny, nz, nxy, ncells;
    int bc_type, types_num, grid_update_freq;
} fo_derived;

/* SimulationManager.cpp:647-671 (gravity, damping negated at :664),
   :684-720 (step, half_dt, half_dt2, lambda_dt), :804-805 (cutoff_sq),
   :2178-2190 (grid size, cell step, half_size_squared). */
static inline void fo_derive_settings(const fo_model* m, fo_derived* d) {
    d->dt = m->dt;
    d->half_dt = m->dt * 0.5;
    d->half_dt2 = m->dt * m->dt * 0.5;
    d->lambda_dt = m->lambda;
    d->lambda_dt *= m->dt;
    d->damping = m->damping * -1.0;
    d->cutoff = m->cutoff;
    d->cutoff_sq = m->cutoff * m->cutoff;
    d->box_unit_cell = m->box_unit_cell;
    d->wall_k = m->wall_k;
    for (int a = 0; a < 3; ++a) {
        d->gravity[a] = m->gravity[a];
        d->box[a] = m->box[a];
    }
    d->nx = (int)floor(m->box[0] / m->box_unit_cell);
    d->ny = (int)floor(m->box[1] / m->box_unit_cell);
    d->nz = (int)floor(m->box[2] / m->box_unit_cell);
    d->nxy = d->nx * d->ny;
    d->ncells = d->nx * d->ny * d->nz;
    d->step[0] = m->box[0] / (double)(float)d->nx;
    d->step[1] = m->box[1] / (double)(float)d->ny;
    d->step[2] = m->box[2] / (double)(float)d->nz;
    double mn = fmin(fmin(m->box[0], m->box[1]), m->box[2]) * 0.5;
    d->half_box_sq = mn * mn;
    d->bc_type = m->bc_type;
    d->types_num = m->n_types;
    d->grid_update_freq = m->grid_update_freq;
}

/* Per-bead constants, SimulationManager.cpp:1429-1445.
   out = {mass, mass_inv, lambda_dt_mass_inv, half_dt_mass_inv,
          half_dt2_mass_inv, radius, radius_sq, skin_radius, skin_radius_sq} */
static inline void fo_derive_bead(const fo_derived* d, double mass, double radius,
                                  double skin_ratio, double out[9]) {
    out[0] = mass;
    if (mass > 0.0) {
        out[1] = 1.0 / mass;
        out[2] = d->lambda_dt * out[1];
        out[3] = d->half_dt * out[1];
        out[4] = d->half_dt2 * out[1];
    } else {
        out[1] = out[2] = out[3] = out[4] = 0.0;
    }
    out[5] = radius;
    out[6] = radius * radius;
    out[7] = radius + skin_ratio;
    out[8] = out[7] * out[7];
}

/* Pair coefficients from the raw 'pair' tokens, SimulationManager.cpp:891-932.
   raw[0..3] are tokens[4..7]; c[0..5] are c1..c6. */
static inline void fo_derive_pair(int kind, const double raw[4], double c[6]) {
    for (int i = 0; i < 6; ++i) c[i] = 0.0;
    if (kind == 1) {
        c[0] = raw[0];
        c[1] = raw[1];
        c[2] = raw[2];
        double r2 = c[2] * c[2];
        double sigma2 = c[0];
        double epsilon = c[1];
        sigma2 *= sigma2;
        double fr2 = sigma2 / r2;
        double fr6 = fr2 * fr2 * fr2;
        double fpr = 48.0 * epsilon * fr6 * (fr6 - 0.5) / r2;
        c[3] = fpr;
    } else if (kind == 2) {
        c[0] = raw[0];
    } else if (kind == 4) { /* extension: penalty K, soft k, rc (no reference counterpart) */
        c[0] = raw[0];
        c[1] = raw[1];
        c[2] = raw[2];
    } else if (kind == 3) {
        c[0] = raw[1];
        c[1] = raw[2];
        c[2] = raw[3] - c[1];
        c[3] = raw[3] * raw[3];
        c[4] = raw[0];
        c[5] = 2 * raw[2] - raw[3];
    }
}

/* One wrap or drop decision of the half-shell table; SimulationManager.cpp
   :2221-2240 (pbc wraps each axis once, finite marks -1). */
static inline int fo_nh_cell(const fo_derived* d, int nx, int ny, int nz) {
    if (d->bc_type == 0) {
        if (nx < 0) nx = d->nx - 1;
        if (nx >= d->nx) nx = 0;
        if (ny < 0) ny = d->ny - 1;
        if (ny >= d->ny) ny = 0;
        if (nz < 0) nz = d->nz - 1;
        if (nz >= d->nz) nz = 0;
        return nx + ny * d->nx + nz * d->nx * d->ny;
    }
    if (nx < 0 || nx >= d->nx || ny < 0 || ny >= d->ny || nz < 0 || nz >= d->nz) return -1;
    return nx + ny * d->nx + nz * d->nx * d->ny;
}

/* The same decision per axis for a box periodic on the axes of mask and
   finite on the others (the per-axis boundary extension; mask 7 gives the
   pbc table above, 0 the finite one). */
static inline int fo_nh_cell_mask(const fo_derived* d, int mask, int nx, int ny, int nz) {
    int q[3] = {nx, ny, nz};
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int a = 0; a < 3; ++a) {
        if (q[a] >= 0 && q[a] < n[a]) continue;
        if (!((mask >> a) & 1)) return -1;
        q[a] = q[a] < 0 ? n[a] - 1 : 0;
    }
    return q[0] + q[1] * d->nx + q[2] * d->nx * d->ny;
}

/* The 13-cell half-shell table, SimulationManager.cpp:2210-2301: nine cells
   at z-1 (dx outer, dy inner), three at x+1 (dy = -1..1), one at y-1. */
static inline void fo_cell_neighbours(const fo_derived* d, int* nh) {
    for (int zz = 0; zz < d->nz; zz++)
        for (int yy = 0; yy < d->ny; yy++)
            for (int xx = 0; xx < d->nx; xx++) {
                int target = xx + yy * d->nx + zz * d->nx * d->ny;
                int* row = nh + (long)target * 13;
                int cnt = 0;
                for (int dx = -1; dx < 2; dx++)
                    for (int dy = -1; dy < 2; dy++) row[cnt++] = fo_nh_cell(d, xx + dx, yy + dy, zz - 1);
                for (int dy = -1; dy < 2; dy++) row[cnt++] = fo_nh_cell(d, xx + 1, yy + dy, zz);
                row[cnt++] = fo_nh_cell(d, xx, yy - 1, zz);
            }
}

/* The half-shell table of a box periodic on the axes of mask. */
static inline void fo_cell_neighbours_mask(const fo_derived* d, int mask, int* nh) {
    for (int zz = 0; zz < d->nz; zz++)
        for (int yy = 0; yy < d->ny; yy++)
            for (int xx = 0; xx < d->nx; xx++) {
                int target = xx + yy * d->nx + zz * d->nx * d->ny;
                int* row = nh + (long)target * 13;
                int cnt = 0;
                for (int dx = -1; dx < 2; dx++)
                    for (int dy = -1; dy < 2; dy++) row[cnt++] = fo_nh_cell_mask(d, mask, xx + dx, yy + dy, zz - 1);
                for (int dy = -1; dy < 2; dy++) row[cnt++] = fo_nh_cell_mask(d, mask, xx + 1, yy + dy, zz);
                row[cnt++] = fo_nh_cell_mask(d, mask, xx, yy - 1, zz);
            }
}

#endif
