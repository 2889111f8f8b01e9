/*
 * fn_types.h -- structures shared by the host engine and the device kernels.
 *
 * Device layout (structure of arrays, one entry per bead in internal order):
 *   pos   double4  wrapped position; .w packs {radius (float bits, low word),
 *                  type (high word)}                      ping-pong pair
 *   img   double4  unwrapped position; .w = 1/mass (0 for mass 0)  ping-pong
 *   vold  float4   velocity_old
 *   force float4   force of the last completed step
 *   vel   float4   predicted velocity (written when damping or export needs it)
 *   binfo int4     {tag, loc_id, type, skin radius (float bits)}
 * Positions are FP64 because the reference's increments (v dt ~ 5e-6 at
 * x ~ 1e3 in the tensile test) are below FP32 resolution there; velocities,
 * forces and bond parameters are FP32; every force is evaluated in FP64.
 */
#ifndef FIBRENET_TYPES_H
#define FIBRENET_TYPES_H

/* Constants of one network, derived from its input-file settings the way
   SimulationManager.cpp derives them (:664, :686-707, :805, :2178-2188). */
struct FnNet {
    double dt, half_dt, half_dt2, lambda_dt, damping;
    double g[3];
    double box[3];
    double step[3];
    double cutoff_sq, half_box_sq, wall_k;
    int nx, ny, nz, nxy;
    int cell_base;   /* first global cell of this network */
    int periodic;    /* axis mask: snap wrap + wrapped cell stencil */
    int list_mi;     /* axis mask: minimum image while listing */
    int force_mi;    /* axis mask: minimum image in contact forces */
    int walls;       /* axis mask: wall penalty */
    int types_num;
    int pair_base;   /* first entry of this network in the pair table */
    int bead_begin, bead_end;
    int pad_;
    double list_r2_max; /* no pair further apart than this (squared) is listed */
    double list_cut_sq; /* listing radius of cut-off pair kinds (squared): the
                           cut-off, plus the Verlet skin in displacement mode */
};

/* Pair coefficients c1..c6 (SimulationManager.cpp:891-932) and kind. */
struct FnPair {
    double c[6];
    int kind;
    int pad_;
};

/* A run of consecutive beads of one network handled by one thread block. */
struct FnTile {
    int net;
    int begin;
    int end;
    int pad_;
};

/* Device counters (unsigned long long). */
enum { FN_CNT_CELL_OVERFLOW = 0, FN_CNT_LIST_OVERFLOW = 1, FN_CNT_NONFINITE = 2, FN_CNT_REBUILDS = 3,
       FN_CNT_STALL = 4, /* a bounded wait on staged data ran out (the tile was skipped) */
       FN_CNT_N = 5 };

#endif
