/*
 * fn_engine_internal.h -- the context behind the C ABI, shared by the engine
 * (fn_engine.cu) and the adjoint (fn_adjoint.cu).  Not a public header.
 */
#ifndef FIBRENET_ENGINE_INTERNAL_H
#define FIBRENET_ENGINE_INTERNAL_H

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <system_error>
#include <new>
#include <stdexcept>
#include <tuple>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fibrenet.h"
#include "fn_kernels.h"
#include "fn_types.h"

namespace fnh {

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
};

/* Per-network host bookkeeping. */
struct NetHost {
    int bead_begin, bead_end;
    int spring_begin, spring_end;
    int angle_begin, angle_end;
    long long cell_begin, cell_end;
    int grid_update_freq;
    double damping;
    bool any_cut, any_hs; /* pair kinds present (listing radius) */
    double rmax;          /* largest radius, as stored */
    double skin_gap;      /* smallest skin radius - radius over the beads */
};

struct AdjointState; /* fn_adjoint.cu */

}  // namespace fnh

struct fn_ctx {
    using NetHost = fnh::NetHost;
    template <class T>
    using DevBuf = fnh::DevBuf<T>;

    fn_config cfg{};
    cudaStream_t stream = nullptr;
    std::string err;
    bool uploaded = false;

    int n_nets = 0;
    std::vector<FnNet> nets_h;
    std::vector<NetHost> info;
    std::vector<FnPair> pairs_h;
    long long nb = 0, ns = 0, na = 0, ncells = 0;
    std::vector<int> perm;  // internal -> upload
    std::vector<int> inv;   // upload -> internal
    std::vector<float4> sp_par_h;  // upload order (springs are not renumbered)
    std::vector<float2> an_par_h;
    bool damp = false;
    int grid_update_freq = 8;

    DevBuf<double4> pos[2], img[2];
    DevBuf<float4> vold, force, vel;
    DevBuf<int4> binfo;
    DevBuf<int2> sp_ends;
    DevBuf<float4> sp_par;
    DevBuf<signed char> sp_type, sp_status;
    DevBuf<int4> an_b;
    DevBuf<int2> an_s;
    DevBuf<float2> an_par;
    DevBuf<signed char> an_status;
    DevBuf<int> sp_off, sp_ent, an_off, an_ent;
    /* host copies of the incidence (internal numbering) for the tile lists */
    std::vector<int> sp_off_h, sp_ent_h, an_off_h, an_ent_h;
    std::vector<int4> an_b_h;
    std::vector<int2> sp_ends_h;  /* internal bead numbering */
    bool incidence_ready = false; /* sp_off/sp_ent/an_off/an_ent built (on first need) */
    std::vector<int2> an_s_h;
    /* per-tile bonded term lists of the tiled step kernel */
    DevBuf<int> tile_sp_off, tile_sp, tile_an_off, tile_an, sp_slot, an_slot;
    DevBuf<int2> tile_an_sslot;
    int max_tile_sp = 0, max_tile_an = 0;
    bool tiled = false;
    /* chain form */
    bool chain = false;
    std::vector<int> sp_bead, an_bead; /* spring -> lower bead, angle -> centre bead */
    DevBuf<float4> ch_sp;
    DevBuf<float2> ch_an;
    DevBuf<unsigned char> ch_flags, ch_status;
    /* staged chain step kernel: tile-compacted contact list, items per tile,
       contact items staged per round */
    bool staged = false;
    int chunk = 0;
    long long csr_region = 0;
    DevBuf<int> csr, tile_items;
    DevBuf<int> cell_of, cell_count, cell_fill, cell_start, cell_beads, list_count, list;
    DevBuf<int> scan_sums;
    /* the list build: 0 one thread per bead (the default), 1 by bricks of
       cells (network, first cell x, y, z of each) staged in shared memory,
       2 by groups of 8 lanes per bead */
    DevBuf<int4> bricks;
    int nbricks = 0;
    int list_build = 0;
    DevBuf<FnTile> tiles;
    DevBuf<FnNet> nets;
    DevBuf<FnPair> pairs;
    DevBuf<unsigned long long> counters;
    DevBuf<double> obs_partial, obs_out;
    DevBuf<double> en_partial, en_out;
    DevBuf<double> series; /* rows of fn_step_series */
    int list_stride = 0;
    int cur = 0;
    int block = 128;
    int ntiles = 0;
    long long device_bytes = 0;
    long long steps_done = 0, rebuilds_done = 0;

    /* captured step segments: (parity, length, ends the call) -> graph */
    std::map<std::tuple<int, int, int>, cudaGraphExec_t> graphs;
    long long graph_launches = 0;

    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_step, ev_rebuild;
    size_t ev_next = 0;

    /* export: upload -> internal bead index on the device, x/y/z staging */
    DevBuf<int> inv_d;
    /* after the device path of fn_upload: the numbering and the bond arrays
       exist on the device only, and the host copies above (perm, inv,
       sp_ends_h, sp_par_h, an_b_h, an_s_h, an_par_h, sp_bead, an_bead) are
       filled from these on first need (ensure_host) */
    bool host_stale = false;
    bool uploaded_on_device = false;
    DevBuf<int> perm_d, sp_bead_d, an_bead_d;
    DevBuf<double> export_xyz;

    /* displacement-triggered rebuilds (cfg.verlet_skin > 0) */
    bool verlet = false;
    double verlet_thresh2 = 0.0; /* squared bead displacement that forces a rebuild */
    DevBuf<double4> ref_img;     /* image positions at the last rebuild */
    DevBuf<int> gate;            /* 1: rebuild before the next step */

    /* device snapshot of the dynamic state (fn_state_save / fn_state_restore) */
    DevBuf<unsigned char> snap;
    bool snap_valid = false;
    int snap_cur = 0;
    long long snap_steps = 0, snap_rebuilds = 0;

    /* bumped by every call that changes the state or the parameters */
    long long state_version = 0;
    /* differentiation state (fn_adjoint_*), null until first used */
    fnh::AdjointState* adj = nullptr;
};

namespace fnh {

int fail(fn_ctx* c, int code, const std::string& msg);

/* Named NVTX range over a host-side phase (upload, a RunSimulationLoop call,
   a contact rebuild, a download, ...): a profiler groups the kernels launched
   inside it by that name (ncu --clock-control none --nvtx --nvtx-include "fn_rebuild/"); without a
   profiler attached a push/pop costs a few nanoseconds. */
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

/* Entry points of the C ABI wrap their bodies in FN_TRY ... FN_CATCH(ctx) so
   that no C++ exception (host memory or threads running out) crosses the
   boundary: it becomes FN_ERR_OOM or FN_ERR_ARG with the reason in
   fn_last_error. */
#define FN_TRY try {
#define FN_CATCH(ctx)                                                                     \
    }                                                                                     \
    catch (const std::bad_alloc&) {                                                       \
        return fnh::fail(ctx, FN_ERR_OOM, "out of host memory");                          \
    }                                                                                     \
    catch (const std::system_error& e_) {                                                 \
        return fnh::fail(ctx, FN_ERR_OOM, std::string("host resources: ") + e_.what());   \
    }                                                                                     \
    catch (const std::exception& e_) {                                                    \
        return fnh::fail(ctx, FN_ERR_ARG, e_.what());                                     \
    }

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::fnh::fail(c, e_ == cudaErrorMemoryAllocation ? FN_ERR_OOM : FN_ERR_CUDA, \
                               std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

/* The library's stream-ordered memory pool on `device`, created on first
   use.  Every context buffer comes from it and goes back to it: freed memory
   stays with the pool for the next allocation (of this or a later context in
   the process) instead of returning to the driver, so creating and
   uploading contexts one after another does not pay the device's allocation
   cost each time. */
cudaError_t device_pool(int device, cudaMemPool_t* pool);

/* An allocation is ordered on the context's stream: work on other streams
   (or synchronous copies) may touch it only after that stream has been
   synchronised, as every entry point does before returning. */
template <class T>
cudaError_t dalloc(fn_ctx* c, DevBuf<T>& b, size_t n) {
    if (b.p) {
        cudaFreeAsync(b.p, c->stream);
        c->device_bytes -= (long long)(b.n * sizeof(T));
        b.p = nullptr;
        b.n = 0;
    }
    size_t bytes = sizeof(T) * (n ? n : 1);
    cudaMemPool_t pool;
    cudaError_t e = device_pool(c->cfg.device, &pool);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync((void**)&b.p, bytes, pool, c->stream);
    if (e == cudaSuccess) {
        b.n = n ? n : 1;
        c->device_bytes += (long long)bytes;
    } else {
        b.p = nullptr;
    }
    return e;
}

template <class T>
void dfree(fn_ctx* c, DevBuf<T>& b) {
    if (b.p) {
        cudaFreeAsync(b.p, c->stream);
        c->device_bytes -= (long long)(b.n * sizeof(T));
    }
    b.p = nullptr;
    b.n = 0;
}

int check_ready(fn_ctx* c);
/* fills the host copies of the numbering and the bonds when only the device
   holds them (after the device path of fn_upload) */
int ensure_host(fn_ctx* c);
int ensure_incidence(fn_ctx* c);
fn::StepArgs step_args(fn_ctx* c, bool pingpong);
/* one step launch of the kernel the context uses (chain: staged or plain;
   per-tile or per-bead incidence otherwise) */
int launch_step_kernel(fn_ctx* c, const fn::StepArgs& A, bool do_drift, bool store_v);
fn::RebuildArgs rebuild_args(fn_ctx* c);
void drop_graphs(fn_ctx* c);

/* adjoint state teardown (fn_adjoint.cu), called by free_all */
void adjoint_free(fn_ctx* c);

}  // namespace fnh

#endif
