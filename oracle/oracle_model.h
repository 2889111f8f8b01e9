/*
 * oracle_model.h -- the raw simulation description both CPU checkers take.
 * TEST INFRASTRUCTURE ONLY (the parity oracle); the product never links it.
 *
 * Values are the ones written in the reference's input and model files
 * (README.md:32-606), before any host precompute: the checkers derive the
 * kernel constants themselves, following SimulationManager.cpp line by line
 * (see oracle_host.h).
 */
#ifndef FIBRENET_ORACLE_MODEL_H
#define FIBRENET_ORACLE_MODEL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fo_model {
    /* input-file settings (SimulationManager.cpp:644-819, 2070-2170) */
    double dt;            /* 'step' */
    double lambda;        /* 'lambda' */
    double damping;       /* 'damping' as written (the host negates it, :664) */
    double gravity[3];    /* 'gravity' */
    double cutoff;        /* 'cutoff' */
    double box_unit_cell; /* 'box_unit_cell' */
    double box[3];        /* 'box_size' */
    double wall_k;        /* 'box_wall_rep' */
    int bc_type;          /* 0 pbc, 1 finite, after the :2168 override */
    int grid_update_freq; /* 'grid_update_freq' (default 8, :23) */
    double skin_ratio;    /* skin_radius = radius + skin_ratio (:26, :1431) */
    int n_types;

    /* pair table in GETADRESS order (kernel.cl:9, SimulationManager.cpp:886):
       kind 1 lj, 2 hs, 3 st; four raw coefficient tokens per pair, as written
       after the two type names (unused trailing ones are ignored) */
    const int* pair_kind;
    const double* pair_raw;

    /* beads (SimulationManager.cpp:1372-1445); vectors are 3 doubles each */
    int n_beads;
    const int* type;
    const int* tag;
    const int* loc_id;
    const double* radius;
    const double* mass;
    const double* pos;
    const double* vel;
    const double* vel_old; /* caller applies (or not) the :1405-1407 quirk */
    const double* force;   /* force_old starts equal to force (:1411-1413) */
    const double* img;

    /* springs (SimulationManager.cpp:1501-1583): type 0 HR, 1 HR_FL */
    int n_springs;
    const int* s_type;
    const int* s_tag;
    const int* s_p1;
    const int* s_p2;
    const double* s_rest;
    const double* s_k;
    const double* s_c1;
    const double* s_c2;

    /* angles (SimulationManager.cpp:1591-1661): type 0 HR, 1 HR_FL */
    int n_angles;
    const int* a_type;
    const int* a_b1;
    const int* a_b2;
    const int* a_b3;
    const int* a_s1;
    const int* a_s2;
    const double* a_theta0;
    const double* a_k;

    /* Extension beyond the reference (which has one global bc_type,
       kernel.cl:241-261): bit a set = axis a periodic.  -1 keeps the
       reference behaviour derived from bc_type. */
    int periodic_mask;
} fo_model;

#ifdef __cplusplus
}
#endif
#endif
