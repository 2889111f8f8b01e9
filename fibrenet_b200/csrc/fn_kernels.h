/*
 * fn_kernels.h -- kernel argument blocks and launch wrappers (host side of
 * fn_kernels.cu).
 */
#ifndef FIBRENET_KERNELS_H
#define FIBRENET_KERNELS_H

#include <cuda_runtime.h>

#include "fn_types.h"

namespace fn {

struct StepArgs {
    const FnTile* tiles;
    const FnNet* nets;
    const FnPair* pairs;
    const double4* pos_in;
    const double4* img_in;
    double4* pos_out;
    double4* img_out;
    float4* vold;
    float4* force;
    float4* vel;
    /* springs */
    const int2* sp_ends;
    const float4* sp_par; /* rest, k, c1, c2 */
    const signed char* sp_type;
    signed char* sp_status;
    /* angles */
    const int4* an_b;     /* b1, b2, b3, type */
    const int2* an_s;     /* s1, s2 */
    const float2* an_par; /* theta0, k */
    signed char* an_status;
    /* bead -> bond incidence */
    const int* sp_off;
    const int* sp_ent; /* spring << 1 | role (0 p1, 1 p2) */
    const int* an_off;
    const int* an_ent; /* angle << 2 | role (0 b1, 1 b2, 2 b3) */
    /* contacts */
    const int* list_count;
    const int* list; /* column major: list[k * list_stride + bead] */
    int list_stride;
    int list_cap;
    unsigned long long* counters;
    /* per-tile bonded terms (tiled step kernel): each tile evaluates the
       springs / angles incident to its beads once, into shared memory */
    const int* tile_sp_off;    /* ntiles + 1 */
    const int* tile_sp;        /* spring ids of each tile, ascending */
    const int* tile_an_off;    /* ntiles + 1 */
    const int* tile_an;        /* angle ids of each tile, ascending */
    const int2* tile_an_sslot; /* per tile angle: slots of s1, s2 (HR_FL) or -1 */
    const int* sp_slot;        /* per bead entry: tile spring slot << 1 | role */
    const int* an_slot;        /* per bead entry: tile angle slot << 2 | role */
    int max_tile_sp;
    int max_tile_an;
};

/* dynamic shared memory of the tiled step kernel */
inline size_t step_tiled_smem(int max_sp, int max_an) {
    return sizeof(double) * 3 * (size_t)max_sp + sizeof(double) * 6 * (size_t)max_an +
           (size_t)max_sp + (size_t)max_an + 16;
}

struct RebuildArgs {
    const FnTile* tiles;
    const FnNet* nets;
    const FnPair* pairs;
    const double4* pos;
    const int4* binfo; /* tag, loc_id, type, skin bits */
    int* cell_of;
    int* cell_count;
    int* cell_fill;
    int* cell_start; /* ncells + 1 */
    int* cell_beads;
    int* list_count;
    int* list;
    int list_stride;
    int list_cap;
    int cell_cap;
    unsigned long long* counters;
    int n_nets;
};

struct ObserveArgs {
    const double4* pos;
    const float4* force;
    const signed char* sp_status;
    const signed char* an_status;
    int bead_begin, bead_end;
    int spring_begin, spring_end;
    int angle_begin, angle_end;
    int reaction_type;
    double* partial; /* 5 doubles per block */
};

cudaError_t launch_step(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                        bool store_v, cudaStream_t s);
cudaError_t launch_step_tiled(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                              bool store_v, cudaStream_t s);
cudaError_t prepare_step_tiled(size_t smem_bytes);
cudaError_t launch_drift(const StepArgs& A, int ntiles, int block, bool store_v, cudaStream_t s);
cudaError_t launch_forces_only(const StepArgs& A, int ntiles, int block, int terms, cudaStream_t s);
cudaError_t launch_reset_energy(float4* force, float4* vel, float4* vold, int n, cudaStream_t s);
long long scan_block_count(long long n);
cudaError_t launch_rebuild(const RebuildArgs& R, int ntiles, int block, int nb, long long ncells,
                           int* scan_block_sums, cudaStream_t s);
cudaError_t launch_observe(const ObserveArgs& O, int nblocks, double* out, cudaStream_t s);

}  // namespace fn

#endif
