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
    /* chain form (every spring joins beads j, j+1; every angle is centred on
       its middle bead): per-bead records instead of incidence lists */
    const float4* ch_sp;          /* spring (j, j+1): rest, k, c1, c2 */
    const float2* ch_an;          /* angle centred on j: theta0, k */
    const unsigned char* ch_flags; /* FN_CH_* bits */
    unsigned char* ch_status;     /* bit 0 spring (j, j+1) alive, bit 1 angle alive */
    int nb;
    /* tile-compacted contact list (staged step kernel): the entries of tile
       t's beads, bead after bead in list order, from csr + t * csr_region;
       tile_items[t] of them */
    const int* csr;
    long long csr_region;
    const int* tile_items;
    int chunk; /* contact items staged per round (a multiple of the block size) */
};

/* dynamic shared memory of the tiled step kernel */
inline size_t step_tiled_smem(int max_sp, int max_an) {
    return sizeof(double) * 3 * (size_t)max_sp + sizeof(double) * 6 * (size_t)max_an +
           (size_t)max_sp + (size_t)max_an + 16;
}

/* largest block the chain step kernel is built for (its launch bounds) */
constexpr int kChainMaxBlock = 256;

/* chain flag bits */
enum {
    FN_CH_SPRING = 1,      /* bead has a spring to bead j+1 */
    FN_CH_SP_REV = 2,      /* that spring lists j+1 as p1 */
    FN_CH_SP_FL = 4,       /* HR_FL (else HR) */
    FN_CH_SP_INERT = 8,    /* spring type outside HR/HR_FL: never acts */
    FN_CH_ANGLE = 16,      /* bead is the centre of an angle */
    FN_CH_AN_REV = 32,     /* that angle lists j+1 as b1 */
    FN_CH_AN_FL = 64       /* HR_FL angle (dies with its springs) */
};

/* Byte offsets of the chain step kernel's dynamic shared memory for blocks
   of `block` threads (one layout for host sizing and device carving). */
struct ChainSmem {
    size_t img, spf, ang, flag, stat, tsp, tan, pos, wres, wmap, wresf, total;
};

__host__ __device__ inline size_t smem_align(size_t o, size_t a) { return (o + a - 1) / a * a; }

__host__ __device__ inline ChainSmem chain_smem_layout(int block) {
    ChainSmem L;
    const size_t h = (size_t)block + 4;
    size_t o = 0;
    L.img = o;  /* image positions of beads b0-2 .. b0+n+1, 3 doubles each */
    o += 24 * h;
    L.spf = o;  /* spring forces, lower bead b0-2 .. b0+n */
    o += 24 * h;
    L.ang = o;  /* angle pa, pc, centre b0-1 .. b0+n */
    o += 48 * h;
    L.flag = o; /* bead flags */
    o += h;
    L.stat = o; /* bead statuses */
    o += h;
    L.tsp = o;  /* spring term flags */
    o += h;
    L.tan = o;  /* angle term flags */
    o += h;
    o = smem_align(o, 32);
    L.pos = o;  /* own wrapped positions, double4 */
    o += 32 * (size_t)block;
    L.wres = o; /* per warp: contact results of one window of 32 items */
    o += 24 * (size_t)block;
    L.wmap = o; /* per warp: item -> lane map of the window */
    o += (size_t)block;
    L.wresf = o; /* per warp: result flags */
    o += (size_t)block;
    L.total = smem_align(o, 16);
    return L;
}

inline size_t step_chain_smem(int block) { return chain_smem_layout(block).total; }

/* The staged chain step kernel: largest number of contact items one thread
   gathers per round (chunk <= kStagedMaxItemsPerThread * block). */
constexpr int kStagedMaxItemsPerThread = 8;

/* Byte offsets of the staged step kernel's dynamic shared memory for blocks
   of `block` threads (tiles of block - 4 beads) and `chunk` contact items per
   round. */
struct StagedSmem {
    size_t bar, img, pos, frc, vold, chsp, chan, spf, ang, pj, off, ws, owner, flag, stat, tsp, tan,
        total;
};

__host__ __device__ inline StagedSmem staged_smem_layout(int block, int chunk) {
    StagedSmem L;
    const size_t w = (size_t)block - 4, h = w + 4;
    size_t o = 0;
    L.bar = o;   /* mbarrier of the bulk copies */
    o += 16;
    L.img = o;   /* double4 image positions, slot u <-> bead b0 - 2 + u */
    o += 32 * h;
    L.pos = o;   /* double4 own positions */
    o += 32 * w;
    L.frc = o;   /* float4 force of the last step */
    o += 16 * w;
    L.vold = o;  /* float4 velocity_old */
    o += 16 * w;
    L.chsp = o;  /* float4 spring records, slot u <-> lower bead b0 - 2 + u */
    o += 16 * h;
    L.chan = o;  /* float2 angle records, slot u <-> centre b0 - 1 + u */
    o += 8 * h;
    o = smem_align(o, 16);
    L.spf = o;   /* spring forces */
    o += 24 * h;
    L.ang = o;   /* angle pa, pc */
    o += 48 * h;
    L.pj = o;    /* per item: partner position, then (R, acts) */
    o += 32 * (size_t)chunk;
    L.off = o;   /* per bead: first item */
    o += 4 * ((size_t)block + 1);
    L.ws = o;    /* block scan */
    o += 4 * 33;
    L.owner = o; /* per item: local bead */
    o += (size_t)chunk;
    L.flag = o;
    o += h;
    L.stat = o;
    o += h;
    L.tsp = o;
    o += h;
    L.tan = o;
    o += h;
    L.total = smem_align(o, 16);
    return L;
}

inline size_t step_staged_smem(int block, int chunk) { return staged_smem_layout(block, chunk).total; }

/* bricks of the staged list build: cells per brick along x, y, z, and the
   most halo beads a brick stages in shared memory */
constexpr int kBrickX = 8, kBrickY = 4, kBrickZ = 4, kBrickCands = 512;

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
    const int* gate; /* displacement mode: rebuild only when *gate != 0 */
    /* bricks of the staged list build: network, first cell x, y, z (null:
       the per-bead list build) */
    const int4* bricks;
    int nbricks;
    /* lanes per bead of the grouped list build (k_lists_group), 0: one
       thread per bead (k_lists) */
    int list_lanes;
    /* tile-compacted copy of the list for the staged step kernel (null: none) */
    int* csr;
    long long csr_region;
    int* tile_items;
};

struct ObserveArgs {
    const unsigned char* ch_flags; /* chain form: statuses per bead */
    const unsigned char* ch_status;
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

/* energy and virial of one network (not part of the reference): FP64 sums
   over beads, springs, angles and contact pairs i < j */
enum { FN_EN_KINETIC, FN_EN_SPRING, FN_EN_ANGLE, FN_EN_CONTACT, FN_EN_WALL, FN_EN_GRAVITY,
       FN_EN_VIRIAL, FN_EN_CONTACTS = FN_EN_VIRIAL + 9, FN_EN_N };

struct EnergyArgs {
    const FnNet* nets;
    const FnPair* pairs;
    const double4* pos;
    const double4* img;
    const float4* vold;
    const int2* sp_ends;
    const float4* sp_par;
    const signed char* sp_type;
    const signed char* sp_status;
    const int4* an_b;
    const float2* an_par;
    const signed char* an_status;
    const unsigned char* ch_status; /* chain form: statuses per bead, else null */
    const int* list_count;
    const int* list;
    int list_stride, list_cap;
    int net;
    int bead_begin, bead_end;
    int spring_begin, spring_end;
    int angle_begin, angle_end;
    double* partial; /* FN_EN_N doubles per block */
};

/* device-side upload (fn_upload.cu): per network ranges and settings, the
   caller's arrays as staged on the device (networks concatenated, model-file
   order), and the results of the checks */
struct UpNet {
    int bead_begin, bead_end, spring_begin, spring_end, angle_begin, angle_end;
    int n_types, pad_;
    double box[3];
    double skin_ratio;
};

struct UpRaw {
    const int *type, *tag, *loc_id;
    const double *radius, *mass, *pos, *vel, *vel_old, *force, *img;
    const int *s_type, *s_p1, *s_p2;
    const double *s_rest, *s_k, *s_c1, *s_c2;
    const int *a_type, *a_b1, *a_b2, *a_b3, *a_s1, *a_s2;
    const double *a_theta0, *a_k;
};

struct UpCheck {
    int bad_bead, bad_spring, bad_angle; /* first offending index, INT_MAX if none */
    int not_runs;                        /* springs not joining consecutive beads */
    unsigned long long rmax, smax, gmin; /* order-preserving keys of the radius extremes */
};

cudaError_t launch_upload_checks(const UpNet* nets, int n_nets, const UpRaw& R, UpCheck* out, int nb, int ns, int na,
                                 unsigned char* link, cudaStream_t s);
cudaError_t launch_upload_runs(const UpNet* nets, int n_nets, const UpRaw& R, const unsigned char* link, int* flag,
                               int* run_of, int* scan_sums, int* start, unsigned long long* key, int nb,
                               cudaStream_t s);
cudaError_t launch_upload_convert(const UpNet* nets, int n_nets, const UpRaw& R, const int* flag, const int* run_of,
                                  const int* start, const int* run_out, int reorder, int* inv, int* perm,
                                  double4* pos, double4* img, float4* vold, float4* force, float4* vel, int4* binfo,
                                  int2* sp_ends, float4* sp_par, signed char* sp_type, signed char* sp_status,
                                  int4* an_b, int2* an_s, float2* an_par, signed char* an_status, int nb, int ns,
                                  int na, cudaStream_t s);
cudaError_t launch_upload_chain(const int2* sp_ends, const signed char* sp_type, const float4* sp_par,
                                const int4* an_b, const int2* an_s, const float2* an_par, int* next_sp,
                                int* centre_an, unsigned char* fl, unsigned char* fa, float4* chs, float2* cha,
                                unsigned char* flags, unsigned char* status, int* sp_bead, int* an_bead, int* bad,
                                int nb, int ns, int na, cudaStream_t s);
/* exclusive prefix sum of n ints into out[0..n], out[n] the total;
   block_sums holds scan_block_count(n) + 1 ints */
cudaError_t launch_exclusive_scan(const int* in, long long n, int* out, int* block_sums, cudaStream_t s);

cudaError_t launch_energy(const EnergyArgs& E, int nblocks, double* out, cudaStream_t s);
/* one bead field in upload order as x, y, z doubles (inv: upload -> internal) */
cudaError_t launch_export_xyz(const double4* src, const int* inv, int n, double* out, cudaStream_t s);
cudaError_t launch_export_xyz(const float4* src, const int* inv, int n, double* out, cudaStream_t s);

cudaError_t launch_step(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                        bool store_v, cudaStream_t s);
cudaError_t launch_step_tiled(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                              bool store_v, cudaStream_t s);
cudaError_t prepare_step_tiled(size_t smem_bytes);
cudaError_t launch_step_chain(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                              bool store_v, cudaStream_t s);
cudaError_t launch_forces_chain(const StepArgs& A, int ntiles, int block, int terms, cudaStream_t s);
cudaError_t prepare_step_chain(size_t smem_bytes);
cudaError_t launch_step_staged(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                               bool store_v, cudaStream_t s);
cudaError_t prepare_step_staged(size_t smem_bytes);
cudaError_t launch_drift(const StepArgs& A, int ntiles, int block, bool store_v, cudaStream_t s);
cudaError_t launch_forces_only(const StepArgs& A, int ntiles, int block, int terms, cudaStream_t s);
cudaError_t launch_reset_energy(float4* force, float4* vel, float4* vold, int n, cudaStream_t s);
long long scan_block_count(long long n);
cudaError_t launch_rebuild(const RebuildArgs& R, int ntiles, int block, int nb, long long ncells,
                           int* scan_block_sums, cudaStream_t s);
cudaError_t launch_observe(const ObserveArgs& O, int nblocks, double* out, cudaStream_t s);
/* displacement-triggered rebuild: check, gated rebuild, new reference, clear */
cudaError_t launch_verlet_rebuild(const RebuildArgs& R, const FnTile* tiles, const double4* img,
                                  double4* ref, double thresh2, int* gate, int ntiles, int block, int nb,
                                  long long ncells, int* scan_block_sums, cudaStream_t s);

}  // namespace fn

#endif
