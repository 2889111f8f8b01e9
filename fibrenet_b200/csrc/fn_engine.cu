/*
 * fn_engine.cu -- host side of the C ABI (include/fibrenet.h).
 *
 * One fn_ctx replaces the reference's OpenclManager + BufferIndex pair
 * (OpenclManager.h:20-174, BufferIndex.h:7-22): it owns the device buffers,
 * derives the kernel constants from the input-file settings the way
 * SimulationManager does, renumbers beads for locality, and sequences the
 * step kernels on one stream (RunSimulationLoop, SimulationManager.cpp:151-181).
 */
#include <cuda_runtime.h>
#include <sched.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <memory>
#include <numeric>
#include <thread>
#include <string>
#include <system_error>
#include <vector>

#include "../../include/fibrenet.h"
#include "fn_engine_internal.h"
#include "fn_kernels.h"
#include "fn_types.h"

using fnh::DevBuf;
using fnh::NetHost;

namespace {

/* contact items per thread and round of the staged chain kernel at upload:
   0, the unstaged chain kernel, which measured faster on the tensile and
   dense networks (fn_autotune may pick a staged shape) */
constexpr int kDefaultItemsPerThread = 0;

/* Largest listing radius squared of one network (kernel.cl:632-650): the
   cutoff for lj/st pairs, largest radius + largest skin for hs pairs. */
double list_r2(const NetHost& h, double cutoff_sq, double smax) {
    double r2 = 0.0;
    if (h.any_cut) r2 = cutoff_sq;
    if (h.any_hs) r2 = std::max(r2, (h.rmax + smax) * (h.rmax + smax));
    return r2;
}

uint32_t spread10(uint32_t v) {
    v &= 0x3ff;
    v = (v | (v << 16)) & 0x030000FF;
    v = (v | (v << 8)) & 0x0300F00F;
    v = (v | (v << 4)) & 0x030C30C3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}

}  // namespace


namespace fnh {

cudaError_t device_pool(int device, cudaMemPool_t* pool) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[device]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        unsigned long long keep = ~0ull; /* freed memory stays in the pool */
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
        pools[device] = p;
    }
    *pool = pools[device];
    return cudaSuccess;
}

int fail(fn_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

/* Host staging array left uninitialised (every element is written before
   use): a zero-filled std::vector would touch each page once more, in one
   thread, before the parallel fill does. */
template <class T>
struct HostArray {
    std::unique_ptr<T[]> p;
    size_t n = 0;
    explicit HostArray(size_t count) : p(new T[count ? count : 1]), n(count) {}
    T& operator[](size_t i) { return p[i]; }
    const T& operator[](size_t i) const { return p[i]; }
};

/* Host threads this process may run on: its CPU affinity mask (what a
   container's cpuset allows), else the machine's count. */
long long host_threads() {
    static const long long n = [] {
        cpu_set_t set;
        CPU_ZERO(&set);
        if (sched_getaffinity(0, sizeof set, &set) == 0 && CPU_COUNT(&set) > 0) return (long long)CPU_COUNT(&set);
        return (long long)std::max(1u, std::thread::hardware_concurrency());
    }();
    return n;
}

/* Runs f(begin, end) over [0, n) on up to 32 host threads (the upload's
   conversions are independent per element). */
template <class F>
void parallel_for(long long n, F f) {
    const long long min_chunk = 1 << 15;
    long long nt = std::min<long long>(32, host_threads());
    nt = std::max(1LL, std::min(nt, (n + min_chunk - 1) / min_chunk));
    if (nt <= 1) {
        f(0LL, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve((size_t)nt);
    const long long chunk = (n + nt - 1) / nt;
    for (long long t = 0; t < nt; ++t) {
        const long long b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) continue;
        try {
            th.emplace_back([=] { f(b, e); });
        } catch (const std::system_error&) {
            f(b, e); /* no thread to be had: this chunk on the calling thread */
        }
    }
    for (auto& x : th) x.join();
}

/* Joins a helper thread when the scope ends, on every path out of it: a
   joinable std::thread that is destroyed ends the process. */
struct JoinOnExit {
    std::thread& t;
    ~JoinOnExit() {
        if (t.joinable()) t.join();
    }
};

/* Smallest i in [0, n) with bad(i), or -1: the checks run on host threads,
   the answer is the one a sequential sweep gives. */
template <class P>
long long first_index(long long n, P bad) {
    std::atomic<long long> best{n};
    parallel_for(n, [&](long long b, long long e) {
        for (long long i = b; i < e && i < best.load(std::memory_order_relaxed); ++i)
            if (bad(i)) {
                long long cur = best.load();
                while (i < cur && !best.compare_exchange_weak(cur, i)) {
                }
                break;
            }
    });
    const long long r = best.load();
    return r < n ? r : -1;
}

template <class T>
cudaError_t h2d(fn_ctx* c, DevBuf<T>& b, const HostArray<T>& v) {
    if (v.n == 0) return cudaSuccess;
    return cudaMemcpyAsync(b.p, v.p.get(), sizeof(T) * v.n, cudaMemcpyHostToDevice, c->stream);
}

template <class T>
cudaError_t h2d(fn_ctx* c, DevBuf<T>& b, const std::vector<T>& v) {
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c->stream);
}

void drop_graphs(fn_ctx* c) {
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
}

void free_all(fn_ctx* c) {
    drop_graphs(c);
    for (int k = 0; k < 2; ++k) {
        dfree(c, c->pos[k]);
        dfree(c, c->img[k]);
    }
    dfree(c, c->vold);
    dfree(c, c->force);
    dfree(c, c->vel);
    dfree(c, c->binfo);
    dfree(c, c->sp_ends);
    dfree(c, c->sp_par);
    dfree(c, c->sp_type);
    dfree(c, c->sp_status);
    dfree(c, c->an_b);
    dfree(c, c->an_s);
    dfree(c, c->an_par);
    dfree(c, c->an_status);
    dfree(c, c->ch_sp);
    dfree(c, c->ch_an);
    dfree(c, c->ch_flags);
    dfree(c, c->ch_status);
    dfree(c, c->csr);
    dfree(c, c->tile_items);
    dfree(c, c->tile_sp_off);
    dfree(c, c->tile_sp);
    dfree(c, c->tile_an_off);
    dfree(c, c->tile_an);
    dfree(c, c->sp_slot);
    dfree(c, c->an_slot);
    dfree(c, c->tile_an_sslot);
    dfree(c, c->sp_off);
    dfree(c, c->sp_ent);
    dfree(c, c->an_off);
    dfree(c, c->an_ent);
    dfree(c, c->cell_of);
    dfree(c, c->cell_count);
    dfree(c, c->cell_fill);
    dfree(c, c->cell_start);
    dfree(c, c->cell_beads);
    dfree(c, c->ref_img);
    dfree(c, c->inv_d);
    dfree(c, c->perm_d);
    dfree(c, c->sp_bead_d);
    dfree(c, c->an_bead_d);
    dfree(c, c->export_xyz);
    dfree(c, c->gate);
    dfree(c, c->list_count);
    dfree(c, c->list);
    dfree(c, c->scan_sums);
    dfree(c, c->bricks);
    dfree(c, c->tiles);
    dfree(c, c->nets);
    dfree(c, c->pairs);
    dfree(c, c->counters);
    dfree(c, c->obs_partial);
    dfree(c, c->obs_out);
    dfree(c, c->en_partial);
    dfree(c, c->en_out);
    dfree(c, c->series);
    dfree(c, c->snap);
    adjoint_free(c);
}

/* Kernel constants of one network (SimulationManager.cpp:647-671, 684-720,
   802-817, 2076-2190, 891-932). */
int derive_net(fn_ctx* c, const fn_settings& s, FnNet& N, int net_index) {
    char buf[256];
    if (!(s.dt > 0.0)) {
        snprintf(buf, sizeof buf, "network %d: 'step' must be positive", net_index);
        return fail(c, FN_ERR_ARG, buf);
    }
    if (!(s.box_unit_cell > 0.0) || !(s.box[0] > 0.0) || !(s.box[1] > 0.0) || !(s.box[2] > 0.0)) {
        snprintf(buf, sizeof buf, "network %d: box and unit cell must be positive", net_index);
        return fail(c, FN_ERR_ARG, buf);
    }
    for (int a = 0; a < 3; ++a)
        if (s.box[a] / s.box_unit_cell < 3.0) {
            snprintf(buf, sizeof buf,
                     "network %d: box must be at least three unit cells per axis "
                     "(SimulationManager.cpp:2104-2109)",
                     net_index);
            return fail(c, FN_ERR_ARG, buf);
        }
    if (s.n_types <= 0) return fail(c, FN_ERR_ARG, "n_types must be positive");
    std::memset(&N, 0, sizeof N);
    N.dt = s.dt;
    N.half_dt = s.dt * 0.5;
    N.half_dt2 = s.dt * s.dt * 0.5;
    N.lambda_dt = s.lambda;
    N.lambda_dt *= s.dt;
    N.damping = s.damping * -1.0;
    for (int a = 0; a < 3; ++a) {
        N.g[a] = s.gravity[a];
        N.box[a] = s.box[a];
    }
    N.cutoff_sq = s.cutoff * s.cutoff;
    N.list_cut_sq = N.cutoff_sq;
    if (c->cfg.verlet_skin > 0.0) N.list_cut_sq = (s.cutoff + c->cfg.verlet_skin) * (s.cutoff + c->cfg.verlet_skin);
    N.wall_k = s.wall_k;
    N.nx = (int)std::floor(s.box[0] / s.box_unit_cell);
    N.ny = (int)std::floor(s.box[1] / s.box_unit_cell);
    N.nz = (int)std::floor(s.box[2] / s.box_unit_cell);
    N.nxy = N.nx * N.ny;
    N.step[0] = s.box[0] / (double)(float)N.nx;
    N.step[1] = s.box[1] / (double)(float)N.ny;
    N.step[2] = s.box[2] / (double)(float)N.nz;
    double mn = std::fmin(std::fmin(s.box[0], s.box[1]), s.box[2]) * 0.5;
    N.half_box_sq = mn * mn;
    if (s.periodic_mask < 0) {
        N.periodic = s.bc_type == 0 ? 7 : 0;
        N.list_mi = N.periodic;
        N.force_mi = 7; /* kernel.cl:844-870 ignores bc_type */
        N.walls = s.bc_type == 1 ? 7 : 0;
    } else {
        N.periodic = s.periodic_mask & 7;
        N.list_mi = N.periodic;
        N.force_mi = N.periodic;
        N.walls = (~N.periodic) & 7;
    }
    N.types_num = s.n_types;
    return FN_OK;
}

void pair_coeffs(int kind, const double* raw, FnPair& P) {
    std::memset(&P, 0, sizeof P);
    P.kind = kind;
    if (kind == FN_PAIR_LJ) {
        P.c[0] = raw[0];
        P.c[1] = raw[1];
        P.c[2] = raw[2];
        double r2 = P.c[2] * P.c[2];
        double sigma2 = P.c[0];
        double epsilon = P.c[1];
        sigma2 *= sigma2;
        double fr2 = sigma2 / r2;
        double fr6 = fr2 * fr2 * fr2;
        P.c[3] = 48.0 * epsilon * fr6 * (fr6 - 0.5) / r2;
    } else if (kind == FN_PAIR_HS) {
        P.c[0] = raw[0];
    } else if (kind == FN_PAIR_HSR) {
        P.c[0] = raw[0];
        P.c[1] = raw[1];
        P.c[2] = raw[2];
    } else if (kind == FN_PAIR_ST) {
        P.c[0] = raw[1];
        P.c[1] = raw[2];
        P.c[2] = raw[3] - P.c[1];
        P.c[3] = raw[3] * raw[3];
        P.c[4] = raw[0];
        P.c[5] = 2 * raw[2] - raw[3];
    }
}

double pack_w(float radius, int type) {
    uint32_t lo;
    std::memcpy(&lo, &radius, 4);
    uint64_t bits = ((uint64_t)(uint32_t)type << 32) | lo;
    double w;
    std::memcpy(&w, &bits, 8);
    return w;
}

int float_bits(float f) {
    int b;
    std::memcpy(&b, &f, 4);
    return b;
}

/* Bead order inside one network: fibres (spring-connected components) sorted
   by the Morton code of their first bead, beads of a fibre kept in file
   order, so bonded partners stay adjacent and nearby fibres get nearby
   indices. */
void network_order(const fn_network_desc& d, const FnNet& N, bool reorder, std::vector<int>& order) {
    const int n = d.n_beads;
    order.resize(n);
    if (!reorder || n == 0) {
        std::iota(order.begin(), order.end(), 0);
        return;
    }
    auto morton_key = [&](int i) {
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            double x = d.pos[3 * i + a] / N.box[a] * 1024.0;
            if (!(x >= 0.0)) x = 0.0;
            if (x > 1023.0) x = 1023.0;
            q[a] = (uint32_t)x;
        }
        const uint64_t m = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
        return (m << 32) | (uint32_t)i;
    };
    /* fibres listed bead after bead (every spring joins i and i + 1): each
       component is a run of consecutive beads starting where no spring
       joins i - 1 and i; the runs are ordered by key and copied out on host
       threads */
    const bool runs =
        first_index(d.n_springs, [&](long long s) { return std::abs(d.s_p1[s] - d.s_p2[s]) != 1; }) < 0;
    if (runs) {
        std::vector<unsigned char> link(n, 0); /* spring between i and i + 1 */
        parallel_for(d.n_springs, [&](long long s0, long long s1) {
            for (long long s = s0; s < s1; ++s)
                __atomic_store_n(&link[std::min(d.s_p1[s], d.s_p2[s])], (unsigned char)1, __ATOMIC_RELAXED);
        });
        std::vector<int> starts;
        for (int i = 0; i < n; ++i)
            if (i == 0 || !link[i - 1]) starts.push_back(i);
        const int R = (int)starts.size();
        std::vector<uint64_t> keys(R);
        parallel_for(R, [&](long long r0, long long r1) {
            for (long long r = r0; r < r1; ++r) keys[r] = morton_key(starts[r]);
        });
        std::sort(keys.begin(), keys.end());
        /* run r of the sorted list: first bead b, length up to the next start */
        std::vector<int> first(R), len(R), out(R);
        int acc = 0;
        for (int r = 0; r < R; ++r) {
            const int b = (int)(uint32_t)keys[r];
            const int k = (int)(std::lower_bound(starts.begin(), starts.end(), b) - starts.begin());
            first[r] = b;
            len[r] = (k + 1 < R ? starts[k + 1] : n) - b;
            out[r] = acc;
            acc += len[r];
        }
        parallel_for(R, [&](long long r0, long long r1) {
            for (long long r = r0; r < r1; ++r)
                for (int t = 0; t < len[r]; ++t) order[out[r] + t] = first[r] + t;
        });
        return;
    }
    std::vector<int> root(n);
    {
        std::vector<int> parent(n);
        std::iota(parent.begin(), parent.end(), 0);
        auto find = [&](int x) {
            while (parent[x] != x) {
                parent[x] = parent[parent[x]];
                x = parent[x];
            }
            return x;
        };
        for (int s = 0; s < d.n_springs; ++s) {
            int a = find(d.s_p1[s]), b = find(d.s_p2[s]);
            if (a != b) parent[std::max(a, b)] = std::min(a, b);
        }
        for (int i = 0; i < n; ++i) root[i] = find(i);
    }
    /* components (roots = their lowest bead) sorted by the Morton code of
       their first bead, ties by index; then every component's beads in
       ascending order: a stable sort of the beads by (key of root, index)
       done as a counting sort in O(n + R log R) */
    std::vector<uint64_t> keys;
    for (int i = 0; i < n; ++i)
        if (root[i] == i) keys.push_back(morton_key(i));
    std::sort(keys.begin(), keys.end());
    std::vector<int> start(n, 0); /* per root: first output slot */
    for (int i = 0; i < n; ++i) start[root[i]]++;
    int acc = 0;
    for (uint64_t k : keys) {
        const int r = (int)(uint32_t)k;
        const int cnt = start[r];
        start[r] = acc;
        acc += cnt;
    }
    for (int i = 0; i < n; ++i) order[start[root[i]]++] = i;
}

int build_tiles(fn_ctx* c, int block, std::vector<FnTile>& out) {
    out.clear();
    for (int k = 0; k < c->n_nets; ++k) {
        const NetHost& h = c->info[k];
        for (int b = h.bead_begin; b < h.bead_end; b += block) {
            FnTile t;
            t.net = k;
            t.begin = b;
            t.end = std::min(b + block, h.bead_end);
            t.pad_ = 0;
            out.push_back(t);
        }
    }
    return (int)out.size();
}

/* Bonded terms of each tile (springs and angles incident to its beads, plus
   the two springs of every HR_FL angle, whose break test decides the angle),
   and the per-bead entries rewritten as tile slots. */
int build_tile_terms(fn_ctx* c, const std::vector<FnTile>& tiles) {
    const size_t nt = tiles.size();
    std::vector<int> tsp_off(nt + 1, 0), tan_off(nt + 1, 0), tsp, tan;
    std::vector<int2> sslot;
    std::vector<int> sp_slot(c->sp_ent_h.size()), an_slot(c->an_ent_h.size());
    int max_sp = 0, max_an = 0;
    std::vector<int> ls, la;
    for (size_t t = 0; t < nt; ++t) {
        ls.clear();
        la.clear();
        for (int i = tiles[t].begin; i < tiles[t].end; ++i) {
            for (int e = c->sp_off_h[i]; e < c->sp_off_h[i + 1]; ++e) ls.push_back(c->sp_ent_h[e] >> 1);
            for (int e = c->an_off_h[i]; e < c->an_off_h[i + 1]; ++e) la.push_back(c->an_ent_h[e] >> 2);
        }
        std::sort(la.begin(), la.end());
        la.erase(std::unique(la.begin(), la.end()), la.end());
        for (int a : la)
            if (c->an_b_h[a].w == 1) {
                ls.push_back(c->an_s_h[a].x);
                ls.push_back(c->an_s_h[a].y);
            }
        std::sort(ls.begin(), ls.end());
        ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
        auto slot_of = [](const std::vector<int>& v, int x) {
            return (int)(std::lower_bound(v.begin(), v.end(), x) - v.begin());
        };
        for (int i = tiles[t].begin; i < tiles[t].end; ++i) {
            for (int e = c->sp_off_h[i]; e < c->sp_off_h[i + 1]; ++e) {
                const int ent = c->sp_ent_h[e];
                sp_slot[e] = (slot_of(ls, ent >> 1) << 1) | (ent & 1);
            }
            for (int e = c->an_off_h[i]; e < c->an_off_h[i + 1]; ++e) {
                const int ent = c->an_ent_h[e];
                an_slot[e] = (slot_of(la, ent >> 2) << 2) | (ent & 3);
            }
        }
        for (int a : la) {
            if (c->an_b_h[a].w == 1)
                sslot.push_back(make_int2(slot_of(ls, c->an_s_h[a].x), slot_of(ls, c->an_s_h[a].y)));
            else
                sslot.push_back(make_int2(0, 0));
        }
        tsp.insert(tsp.end(), ls.begin(), ls.end());
        tan.insert(tan.end(), la.begin(), la.end());
        tsp_off[t + 1] = (int)tsp.size();
        tan_off[t + 1] = (int)tan.size();
        max_sp = std::max(max_sp, (int)ls.size());
        max_an = std::max(max_an, (int)la.size());
    }
    const size_t smem = fn::step_tiled_smem(max_sp, max_an);
    c->tiled = smem <= 160 * 1024;
    if (!c->tiled) return FN_OK;
    CK(fn::prepare_step_tiled(smem));
    CK(dalloc(c, c->tile_sp_off, tsp_off.size()));
    CK(dalloc(c, c->tile_an_off, tan_off.size()));
    CK(dalloc(c, c->tile_sp, tsp.size()));
    CK(dalloc(c, c->tile_an, tan.size()));
    CK(dalloc(c, c->tile_an_sslot, sslot.size()));
    CK(dalloc(c, c->sp_slot, sp_slot.size()));
    CK(dalloc(c, c->an_slot, an_slot.size()));
    CK(h2d(c, c->tile_sp_off, tsp_off));
    CK(h2d(c, c->tile_an_off, tan_off));
    CK(h2d(c, c->tile_sp, tsp));
    CK(h2d(c, c->tile_an, tan));
    CK(h2d(c, c->tile_an_sslot, sslot));
    CK(h2d(c, c->sp_slot, sp_slot));
    CK(h2d(c, c->an_slot, an_slot));
    c->max_tile_sp = max_sp;
    c->max_tile_an = max_an;
    return FN_OK;
}

/* Chain form: every spring joins beads j, j+1 (one spring per j), every
   angle is (j-1, j, j+1) or (j+1, j, j-1) (one per centre), HR_FL angles use
   exactly the two springs around their centre, and around every bead the
   incident springs and angles appear in ascending index in the order
   previous, next (springs) and centre j-1, j, j+1 (angles), which is the
   incidence path's order.  Builds the per-bead records when it holds. */
bool build_chain(fn_ctx* c, const std::vector<int2>& sp_ends, const std::vector<signed char>& sp_type,
                 const std::vector<int4>& an_b, const std::vector<int2>& an_s) {
    using namespace fn;
    const long long nb = c->nb;
    std::vector<int> next_sp(nb, -1), centre_an(nb, -1);
    std::vector<unsigned char> fl(nb, 0), fa(nb, 0);
    std::atomic<bool> bad_form{false};
    /* springs, then angles, each on host threads: in chain form every lower
       bead has at most one spring and every centre at most one angle, so the
       writes do not collide; a second sweep catches the models where they
       would (two bonds claiming one slot) */
    parallel_for(c->ns, [&](long long s0, long long s1) {
        for (long long s = s0; s < s1; ++s) {
            const int a = sp_ends[s].x, b = sp_ends[s].y;
            const int lo = std::min(a, b), hi = std::max(a, b);
            if (hi != lo + 1) {
                bad_form = true;
                continue;
            }
            next_sp[lo] = (int)s;
            unsigned char f = FN_CH_SPRING;
            if (a == hi) f |= FN_CH_SP_REV;
            if (sp_type[s] == 1)
                f |= FN_CH_SP_FL;
            else if (sp_type[s] != 0)
                f |= FN_CH_SP_INERT;
            fl[lo] = f;
        }
    });
    if (bad_form) return false;
    parallel_for(c->ns, [&](long long s0, long long s1) {
        for (long long s = s0; s < s1; ++s)
            if (next_sp[std::min(sp_ends[s].x, sp_ends[s].y)] != (int)s) bad_form = true;
    });
    if (bad_form) return false;
    parallel_for(c->na, [&](long long a0, long long a1) {
        for (long long a = a0; a < a1; ++a) {
            const int4 b = an_b[a];
            const bool fwd = b.x == b.y - 1 && b.z == b.y + 1;
            const bool rev = b.x == b.y + 1 && b.z == b.y - 1;
            if (!(fwd || rev)) {
                bad_form = true;
                continue;
            }
            centre_an[b.y] = (int)a;
            unsigned char f = FN_CH_ANGLE;
            if (rev) f |= FN_CH_AN_REV;
            if (b.w == 1) {
                f |= FN_CH_AN_FL;
                const int sp = next_sp[b.y - 1], sn = next_sp[b.y];
                const int2 ss = an_s[a];
                if (sp < 0 || sn < 0 || !((ss.x == sp && ss.y == sn) || (ss.x == sn && ss.y == sp)))
                    bad_form = true;
            }
            fa[b.y] = f;
        }
    });
    if (bad_form) return false;
    parallel_for(c->na, [&](long long a0, long long a1) {
        for (long long a = a0; a < a1; ++a)
            if (centre_an[an_b[a].y] != (int)a) bad_form = true;
    });
    if (bad_form) return false;
    parallel_for(nb, [&](long long i0, long long i1) {
        for (long long i = i0; i < i1; ++i) fl[i] |= fa[i];
    });
    std::atomic<bool> bad{false};
    parallel_for(nb, [&](long long i0, long long i1) {
        for (long long i = i0; i < i1; ++i) {
            if (i > 0 && next_sp[i - 1] >= 0 && next_sp[i] >= 0 && next_sp[i - 1] > next_sp[i]) bad = true;
            int last = -1;
            for (long long q = i - 1; q <= i + 1; ++q) {
                if (q < 0 || q >= nb || centre_an[q] < 0) continue;
                if (centre_an[q] < last) bad = true;
                last = centre_an[q];
            }
        }
    });
    if (bad) return false;
    HostArray<float4> chs(nb);
    HostArray<float2> cha(nb);
    HostArray<unsigned char> st(nb);
    c->sp_bead.resize(c->ns);
    c->an_bead.resize(c->na);
    /* each spring is the next spring of exactly one bead and each angle is
       centred on exactly one: the scattered writes below never collide */
    parallel_for(nb, [&](long long i0, long long i1) {
        for (long long i = i0; i < i1; ++i) {
            chs[i] = make_float4(0, 0, 0, 0);
            cha[i] = make_float2(0, 0);
            unsigned char b = 0;
            if (next_sp[i] >= 0) {
                chs[i] = c->sp_par_h[next_sp[i]];
                c->sp_bead[next_sp[i]] = (int)i;
                b |= 1;
            }
            if (centre_an[i] >= 0) {
                cha[i] = c->an_par_h[centre_an[i]];
                c->an_bead[centre_an[i]] = (int)i;
                b |= 2;
            }
            st[i] = b;
        }
    });
    if (dalloc(c, c->ch_sp, nb) || dalloc(c, c->ch_an, nb) || dalloc(c, c->ch_flags, nb) ||
        dalloc(c, c->ch_status, nb))
        return false;
    if (h2d(c, c->ch_sp, chs) || h2d(c, c->ch_an, cha) || h2d(c, c->ch_flags, fl) ||
        h2d(c, c->ch_status, st))
        return false;
    return true;
}

/* Bead -> bond incidence (CSR, ascending bond index per bead), built on
   first need: the incidence step kernels, the per-tile term lists and the
   adjoint read it; the chain step kernel does not, so chain-form models skip
   it at upload. */
int ensure_incidence(fn_ctx* c) {
    if (c->incidence_ready) return FN_OK;
    int r0 = ensure_host(c);
    if (r0) return r0;
    const long long nb = c->nb, ns = c->ns, na = c->na;
    const std::vector<int2>& sp_ends = c->sp_ends_h;
    const std::vector<int4>& an_b = c->an_b_h;
    std::vector<int> sp_off(nb + 1, 0), an_off(nb + 1, 0);
    for (long long s = 0; s < ns; ++s) {
        sp_off[sp_ends[s].x + 1]++;
        sp_off[sp_ends[s].y + 1]++;
    }
    for (long long a = 0; a < na; ++a) {
        an_off[an_b[a].x + 1]++;
        an_off[an_b[a].y + 1]++;
        an_off[an_b[a].z + 1]++;
    }
    for (long long i = 0; i < nb; ++i) {
        sp_off[i + 1] += sp_off[i];
        an_off[i + 1] += an_off[i];
    }
    std::vector<int> sp_ent(2 * ns), an_ent(3 * na);
    {
        std::vector<int> fill(sp_off.begin(), sp_off.end() - 1);
        for (long long s = 0; s < ns; ++s) {
            sp_ent[fill[sp_ends[s].x]++] = (int)(s << 1);
            sp_ent[fill[sp_ends[s].y]++] = (int)((s << 1) | 1);
        }
        std::vector<int> fa(an_off.begin(), an_off.end() - 1);
        for (long long a = 0; a < na; ++a) {
            an_ent[fa[an_b[a].x]++] = (int)(a << 2);
            an_ent[fa[an_b[a].y]++] = (int)((a << 2) | 1);
            an_ent[fa[an_b[a].z]++] = (int)((a << 2) | 2);
        }
    }
    c->sp_off_h = std::move(sp_off);
    c->sp_ent_h = std::move(sp_ent);
    c->an_off_h = std::move(an_off);
    c->an_ent_h = std::move(an_ent);
    CK(dalloc(c, c->sp_off, nb + 1));
    CK(dalloc(c, c->sp_ent, 2 * ns));
    CK(dalloc(c, c->an_off, nb + 1));
    CK(dalloc(c, c->an_ent, 3 * na));
    CK(h2d(c, c->sp_off, c->sp_off_h));
    CK(h2d(c, c->sp_ent, c->sp_ent_h));
    CK(h2d(c, c->an_off, c->an_off_h));
    CK(h2d(c, c->an_ent, c->an_ent_h));
    CK(cudaStreamSynchronize(c->stream));
    c->incidence_ready = true;
    return FN_OK;
}

/* Bricks of the staged list build: every network's grid cut into bricks of
   kBrickX x kBrickY x kBrickZ cells (clipped at the grid's far sides). */
int build_bricks(fn_ctx* c) {
    std::vector<int4> b;
    for (int k = 0; k < c->n_nets; ++k) {
        const FnNet& N = c->nets_h[k];
        for (int z = 0; z < N.nz; z += fn::kBrickZ)
            for (int y = 0; y < N.ny; y += fn::kBrickY)
                for (int x = 0; x < N.nx; x += fn::kBrickX) b.push_back(make_int4(k, x, y, z));
    }
    CK(dalloc(c, c->bricks, b.size()));
    CK(h2d(c, c->bricks, b));
    c->nbricks = (int)b.size();
    return FN_OK;
}

/* Block size (and, for the staged chain kernel, contact items per thread and
   round) of the step kernel: tiles, per-tile tables and kernel attributes.
   items_per_thread 0 selects the plain chain kernel. */
int set_block(fn_ctx* c, int block, int items_per_thread) {
    if (c->chain && block > fn::kChainMaxBlock)
        return fail(c, FN_ERR_ARG, "block size " + std::to_string(block) + ": the chain step kernel takes at most " +
                                       std::to_string(fn::kChainMaxBlock) + " threads per block");
    if (items_per_thread < 0 || items_per_thread > fn::kStagedMaxItemsPerThread)
        return fail(c, FN_ERR_ARG, "contact items per thread must be 0 .. " +
                                       std::to_string(fn::kStagedMaxItemsPerThread));
    drop_graphs(c);
    std::vector<FnTile> t;
    /* the chain kernel stages its tile plus a two-bead halo on each side:
       tiles of block - 4 beads make that exactly one slot per thread, so no
       warp runs a second round of the spring and angle phases */
    int n = build_tiles(c, c->chain ? block - 4 : block, t);
    CK(cudaStreamSynchronize(c->stream));
    CK(dalloc(c, c->tiles, t.size()));
    CK(h2d(c, c->tiles, t));
    if (c->chain) {
        CK(fn::prepare_step_chain(fn::step_chain_smem(block)));
        c->staged = items_per_thread > 0;
        c->chunk = items_per_thread * block;
        if (c->staged) {
            const size_t smem = fn::step_staged_smem(block, c->chunk);
            int dev = 0, optin = 0;
            CK(cudaGetDevice(&dev));
            CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            if (smem > (size_t)optin)
                return fail(c, FN_ERR_ARG, "staged step kernel: " + std::to_string(smem) +
                                               " bytes of shared memory per block exceed the device's " +
                                               std::to_string(optin));
            CK(fn::prepare_step_staged(smem));
            /* region per tile: every bead's full list, in whole 16-byte units */
            c->csr_region = ((long long)(block - 4) * c->cfg.list_capacity + 3) / 4 * 4;
            CK(dalloc(c, c->csr, (size_t)n * (size_t)c->csr_region + 16));
            CK(dalloc(c, c->tile_items, (size_t)n));
            CK(cudaMemsetAsync(c->tile_items.p, 0, sizeof(int) * (size_t)n, c->stream));
        } else {
            dfree(c, c->csr);
            dfree(c, c->tile_items);
        }
    } else {
        int r = ensure_incidence(c);
        if (r) return r;
        r = build_tile_terms(c, t);
        if (r) return r;
    }
    CK(cudaStreamSynchronize(c->stream));
    c->ntiles = n;
    c->block = block;
    return FN_OK;
}

int launch_step_kernel(fn_ctx* c, const fn::StepArgs& A, bool do_drift, bool store_v) {
    if (c->chain && c->staged)
        CK(fn::launch_step_staged(A, c->ntiles, c->block, c->damp, do_drift, store_v, c->stream));
    else if (c->chain)
        CK(fn::launch_step_chain(A, c->ntiles, c->block, c->damp, do_drift, store_v, c->stream));
    else if (c->tiled)
        CK(fn::launch_step_tiled(A, c->ntiles, c->block, c->damp, do_drift, store_v, c->stream));
    else
        CK(fn::launch_step(A, c->ntiles, c->block, c->damp, do_drift, store_v, c->stream));
    return FN_OK;
}

fn::StepArgs step_args(fn_ctx* c, bool pingpong) {
    fn::StepArgs A{};
    A.tiles = c->tiles.p;
    A.nets = c->nets.p;
    A.pairs = c->pairs.p;
    A.pos_in = c->pos[c->cur].p;
    A.img_in = c->img[c->cur].p;
    A.pos_out = pingpong ? c->pos[1 - c->cur].p : c->pos[c->cur].p;
    A.img_out = pingpong ? c->img[1 - c->cur].p : c->img[c->cur].p;
    A.vold = c->vold.p;
    A.force = c->force.p;
    A.vel = c->vel.p;
    A.sp_ends = c->sp_ends.p;
    A.sp_par = c->sp_par.p;
    A.sp_type = c->sp_type.p;
    A.sp_status = c->sp_status.p;
    A.an_b = c->an_b.p;
    A.an_s = c->an_s.p;
    A.an_par = c->an_par.p;
    A.an_status = c->an_status.p;
    A.sp_off = c->sp_off.p;
    A.sp_ent = c->sp_ent.p;
    A.an_off = c->an_off.p;
    A.an_ent = c->an_ent.p;
    A.list_count = c->list_count.p;
    A.list = c->list.p;
    A.list_stride = c->list_stride;
    A.list_cap = c->cfg.list_capacity;
    A.counters = c->counters.p;
    A.tile_sp_off = c->tile_sp_off.p;
    A.tile_sp = c->tile_sp.p;
    A.tile_an_off = c->tile_an_off.p;
    A.tile_an = c->tile_an.p;
    A.tile_an_sslot = c->tile_an_sslot.p;
    A.sp_slot = c->sp_slot.p;
    A.an_slot = c->an_slot.p;
    A.max_tile_sp = c->max_tile_sp;
    A.max_tile_an = c->max_tile_an;
    A.ch_sp = c->ch_sp.p;
    A.ch_an = c->ch_an.p;
    A.ch_flags = c->ch_flags.p;
    A.ch_status = c->ch_status.p;
    A.nb = (int)c->nb;
    A.csr = c->csr.p;
    A.csr_region = c->csr_region;
    A.tile_items = c->tile_items.p;
    A.chunk = c->chunk;
    return A;
}

fn::RebuildArgs rebuild_args(fn_ctx* c) {
    fn::RebuildArgs R{};
    R.tiles = c->tiles.p;
    R.nets = c->nets.p;
    R.pairs = c->pairs.p;
    R.pos = c->pos[c->cur].p;
    R.binfo = c->binfo.p;
    R.cell_of = c->cell_of.p;
    R.cell_count = c->cell_count.p;
    R.cell_fill = c->cell_fill.p;
    R.cell_start = c->cell_start.p;
    R.cell_beads = c->cell_beads.p;
    R.gate = c->verlet ? c->gate.p : nullptr;
    R.list_count = c->list_count.p;
    R.list = c->list.p;
    R.list_stride = c->list_stride;
    R.list_cap = c->cfg.list_capacity;
    R.cell_cap = c->cfg.cell_capacity;
    R.counters = c->counters.p;
    R.n_nets = c->n_nets;
    R.bricks = c->list_build == 1 ? c->bricks.p : nullptr;
    R.list_lanes = c->list_build == 2 ? 8 : 0;
    R.nbricks = c->nbricks;
    R.csr = c->staged ? c->csr.p : nullptr;
    R.csr_region = c->csr_region;
    R.tile_items = c->tile_items.p;
    return R;
}

cudaEvent_t next_event(fn_ctx* c) {
    if (c->ev_next >= c->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_next++];
}

int do_rebuild(fn_ctx* c) {
    fnh::NvtxRange nvtx_range_("fn_rebuild");
    fn::RebuildArgs R = rebuild_args(c);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing) {
        e0 = next_event(c);
        e1 = next_event(c);
        CK(cudaEventRecord(e0, c->stream));
    }
    if (c->verlet)
        CK(fn::launch_verlet_rebuild(R, c->tiles.p, c->img[c->cur].p, c->ref_img.p, c->verlet_thresh2, c->gate.p,
                                     c->ntiles, c->block, (int)c->nb, c->ncells, c->scan_sums.p, c->stream));
    else
        CK(fn::launch_rebuild(R, c->ntiles, c->block, (int)c->nb, c->ncells, c->scan_sums.p, c->stream));
    if (c->timing) {
        CK(cudaEventRecord(e1, c->stream));
        c->ev_rebuild.emplace_back(e0, e1);
    }
    c->rebuilds_done++;
    return FN_OK;
}

int launch_one_step(fn_ctx* c, bool do_drift, bool store_v) {
    fn::StepArgs A = step_args(c, true);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing) {
        e0 = next_event(c);
        e1 = next_event(c);
        CK(cudaEventRecord(e0, c->stream));
    }
    int r = launch_step_kernel(c, A, do_drift, store_v);
    if (r) return r;
    if (c->timing) {
        CK(cudaEventRecord(e1, c->stream));
        c->ev_step.emplace_back(e0, e1);
    }
    if (do_drift) c->cur = 1 - c->cur;
    return FN_OK;
}

/* One segment of a RunSimulationLoop call: the contact rebuild that opens
   every grid_update_freq steps, then `len` steps; when `tail` the segment
   ends the call, so its last step does not drift and the step before it
   keeps the predicted velocity. */
int launch_segment(fn_ctx* c, int len, bool tail) {
    int r = do_rebuild(c);
    if (r) return r;
    for (int k = 0; k < len; ++k) {
        if (c->verlet && k > 0) {
            r = do_rebuild(c); /* gated: runs only when a bead moved too far */
            if (r) return r;
        }
        const bool last = tail && k == len - 1;
        r = launch_one_step(c, !last, tail && k == len - 2);
        if (r) return r;
    }
    return FN_OK;
}

/* The segment through a CUDA graph captured on first use (kernel arguments
   depend on the ping-pong parity, the length and whether it ends the call). */
int run_segment(fn_ctx* c, int len, bool tail) {
    if (!c->cfg.use_graphs || c->timing) return launch_segment(c, len, tail);
    const auto key = std::make_tuple(c->cur, len, tail ? 1 : 0);
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        const int cur0 = c->cur;
        const long long rb0 = c->rebuilds_done;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int r = launch_segment(c, len, tail);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) return fail(c, FN_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        cudaGraphExec_t x = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&x, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return fail(c, FN_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        it = c->graphs.emplace(key, x).first;
        c->cur = cur0; /* capture recorded the launches without running them */
        c->rebuilds_done = rb0;
    }
    CK(cudaGraphLaunch(it->second, c->stream));
    c->graph_launches++;
    c->rebuilds_done++;
    const int drifts = tail ? len - 1 : len;
    if (drifts & 1) c->cur = 1 - c->cur;
    return FN_OK;
}

/* Displacement-triggered rebuilds: the smallest gap between listing and
   acting radius that the grid guarantees (a pair outside the 27-cell
   stencil is at least one cell step away), and the bead displacement that
   forces a rebuild (0.45 of it: two beads may close in on each other). */
int verlet_setup(fn_ctx* c) {
    c->verlet = false;
    if (!(c->cfg.verlet_skin > 0.0)) return FN_OK;
    double s_eff = 1e300;
    for (int k = 0; k < c->n_nets; ++k) {
        const FnNet& N = c->nets_h[k];
        const NetHost& h = c->info[k];
        const double step = std::min({N.step[0], N.step[1], N.step[2]});
        if (h.any_cut) s_eff = std::min(s_eff, std::min(step - std::sqrt(N.cutoff_sq), c->cfg.verlet_skin));
        if (h.any_hs) s_eff = std::min(s_eff, std::min(step - 2.0 * h.rmax, h.skin_gap));
    }
    if (!(s_eff > 0.0) || s_eff > 1e299)
        return fail(c, FN_ERR_ARG,
                    "displacement-triggered rebuilds need a grid cell wider than the cut-off (than two radii "
                    "for hs pairs) and a positive skin");
    const double thresh = 0.45 * s_eff;
    c->verlet_thresh2 = thresh * thresh;
    if (!c->ref_img.p || c->ref_img.n < (size_t)c->nb) CK(dalloc(c, c->ref_img, (size_t)c->nb));
    if (!c->gate.p) CK(dalloc(c, c->gate, 1));
    static const int one = 1;
    CK(cudaMemcpyAsync(c->gate.p, &one, sizeof one, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->verlet = true;
    return FN_OK;
}

int check_ready(fn_ctx* c) {
    if (!c) return FN_ERR_ARG;
    if (!c->uploaded) return fail(c, FN_ERR_STATE, "no model uploaded");
    return FN_OK;
}

int ensure_host(fn_ctx* c) {
    if (!c->host_stale) return FN_OK;
    const size_t nb = (size_t)c->nb, ns = (size_t)c->ns, na = (size_t)c->na;
    c->perm.resize(nb);
    c->inv.resize(nb);
    c->sp_ends_h.resize(ns);
    c->sp_par_h.resize(ns);
    c->an_b_h.resize(na);
    c->an_s_h.resize(na);
    c->an_par_h.resize(na);
    c->sp_bead.resize(ns);
    c->an_bead.resize(na);
    auto d2h = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream) : cudaSuccess;
    };
    CK(cudaSetDevice(c->cfg.device));
    CK(d2h(c->perm.data(), c->perm_d.p, sizeof(int) * nb));
    CK(d2h(c->inv.data(), c->inv_d.p, sizeof(int) * nb));
    CK(d2h(c->sp_ends_h.data(), c->sp_ends.p, sizeof(int2) * ns));
    CK(d2h(c->sp_par_h.data(), c->sp_par.p, sizeof(float4) * ns));
    CK(d2h(c->an_b_h.data(), c->an_b.p, sizeof(int4) * na));
    CK(d2h(c->an_s_h.data(), c->an_s.p, sizeof(int2) * na));
    CK(d2h(c->an_par_h.data(), c->an_par.p, sizeof(float2) * na));
    CK(d2h(c->sp_bead.data(), c->sp_bead_d.p, sizeof(int) * ns));
    CK(d2h(c->an_bead.data(), c->an_bead_d.p, sizeof(int) * na));
    CK(cudaStreamSynchronize(c->stream));
    c->host_stale = false;
    return FN_OK;
}

}  // namespace fnh

using namespace fnh;

/* ======================================================================== */

extern "C" {

FN_API int fn_create(const fn_config* cfg, fn_ctx** out) {
    FN_TRY
    if (!cfg || !out) return FN_ERR_ARG;
    *out = nullptr;
    fn_ctx* c = new fn_ctx();
    c->cfg = *cfg;
    if (c->cfg.cell_capacity <= 0) c->cfg.cell_capacity = 64;
    if (c->cfg.list_capacity <= 0) c->cfg.list_capacity = 64;
    if (c->cfg.block_size < 0 || c->cfg.block_size > 512 || (c->cfg.block_size % 32) != 0) {
        delete c;
        return FN_ERR_ARG;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        delete c;
        return FN_ERR_CUDA;
    }
    if (cfg->device < 0 || cfg->device >= ndev) {
        delete c;
        return FN_ERR_ARG;
    }
    if (cudaSetDevice(cfg->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return FN_ERR_CUDA;
    }
    *out = c;
    return FN_OK;
    FN_CATCH(nullptr)
}

FN_API void fn_destroy(fn_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->cfg.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    if (c->stream) cudaStreamSynchronize(c->stream); /* the buffers are back in the pool */
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

FN_API const char* fn_last_error(const fn_ctx* c) { return c ? c->err.c_str() : "null context"; }

/* fn_upload's per-network preamble: argument checks, the network's kernel
   constants and pair table entries, its bead / spring / angle / cell ranges
   (appended to nb, ns, na, ncells).  With element_checks the index checks of
   every bead, spring and angle and the radius extremes run here on host
   threads; the device path leaves both to its kernels and fills the extremes
   in afterwards (set_radius_extremes). */
static int net_preamble(fn_ctx* c, int k, const fn_network_desc& d, long long& nb, long long& ns, long long& na,
                        long long& ncells, bool element_checks) {
    if (d.n_beads <= 0 || d.n_springs < 0 || d.n_angles < 0)
        return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": empty or negative sizes");
    if (!d.type || !d.tag || !d.loc_id || !d.radius || !d.mass || !d.pos || !d.vel ||
        !d.vel_old || !d.force || !d.img || !d.pair_kind || !d.pair_raw)
        return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": null bead array");
    if (d.n_springs > 0 && (!d.s_type || !d.s_p1 || !d.s_p2 || !d.s_rest || !d.s_k || !d.s_c1 || !d.s_c2))
        return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": null spring array");
    if (d.n_angles > 0 && (!d.a_type || !d.a_b1 || !d.a_b2 || !d.a_b3 || !d.a_s1 || !d.a_s2 ||
                           !d.a_theta0 || !d.a_k))
        return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": null angle array");
    int r = derive_net(c, d.settings, c->nets_h[k], k);
    if (r) return r;
    FnNet& N = c->nets_h[k];
    const int nt = d.settings.n_types;
    if (element_checks) {
        /* the first offending bead, spring or angle, as a sequential sweep
           would report it */
        const int nbk = d.n_beads, nsk = d.n_springs;
        const long long bad_bead = first_index(nbk, [&](long long i) {
            return d.type[i] < 0 || d.type[i] >= nt || !(d.mass[i] >= 0.0);
        });
        if (bad_bead >= 0) {
            const long long i = bad_bead;
            if (d.type[i] < 0 || d.type[i] >= nt)
                return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": bead " +
                                               std::to_string(i) + " has an undeclared type");
            return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": negative mass");
        }
        const long long bad_spring = first_index(nsk, [&](long long s) {
            return d.s_p1[s] < 0 || d.s_p1[s] >= nbk || d.s_p2[s] < 0 || d.s_p2[s] >= nbk;
        });
        if (bad_spring >= 0)
            return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": spring " +
                                           std::to_string(bad_spring) + " references a missing bead");
        auto angle_beads_bad = [&](long long a) {
            return d.a_b1[a] < 0 || d.a_b1[a] >= nbk || d.a_b2[a] < 0 || d.a_b2[a] >= nbk ||
                   d.a_b3[a] < 0 || d.a_b3[a] >= nbk;
        };
        const long long bad_angle = first_index(d.n_angles, [&](long long a) {
            return angle_beads_bad(a) ||
                   (d.a_type[a] == 1 &&
                    (d.a_s1[a] < 0 || d.a_s1[a] >= nsk || d.a_s2[a] < 0 || d.a_s2[a] >= nsk));
        });
        if (bad_angle >= 0) {
            if (angle_beads_bad(bad_angle))
                return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": angle " +
                                               std::to_string(bad_angle) + " references a missing bead");
            return fail(c, FN_ERR_ARG, "network " + std::to_string(k) + ": HR_FL angle " +
                                           std::to_string(bad_angle) + " references a missing spring");
        }
    }
    const int npairs = nt * (nt + 1) / 2;
    N.pair_base = (int)c->pairs_h.size();
    bool any_cut = false, any_hs = false;
    for (int p = 0; p < npairs; ++p) {
        FnPair P;
        pair_coeffs(d.pair_kind[p], d.pair_raw + 4 * p, P);
        if (P.kind == FN_PAIR_HSR && !(P.c[2] <= d.settings.cutoff))
            return fail(c, FN_ERR_ARG, "network " + std::to_string(k) +
                                           ": hsr soft radius exceeds the cutoff (pairs would go unlisted)");
        c->pairs_h.push_back(P);
        any_cut |= P.kind == FN_PAIR_LJ || P.kind == FN_PAIR_ST || P.kind == FN_PAIR_HSR;
        any_hs |= P.kind == FN_PAIR_HS || P.kind == FN_PAIR_HSR;
    }
    /* largest listing radius (squared): cutoff for lj/st, the largest
       radius + the largest skin for hs (kernel.cl:632-650) */
    double rmax = 0.0, smax = 0.0, gap = 1e300;
    std::mutex red;
    if (element_checks)
        parallel_for(d.n_beads, [&](long long i0, long long i1) {
        double r = 0.0, sm = 0.0, g = 1e300;
        for (long long i = i0; i < i1; ++i) {
            const float rad = (float)d.radius[i];
            const float skin = (float)((double)rad + d.settings.skin_ratio);
            r = std::max(r, (double)rad);
            sm = std::max(sm, (double)skin);
            g = std::min(g, (double)skin - (double)rad);
        }
        std::lock_guard<std::mutex> lk(red);
        rmax = std::max(rmax, r);
        smax = std::max(smax, sm);
        gap = std::min(gap, g);
    });
    c->info[k].skin_gap = gap;
    c->info[k].any_cut = any_cut;
    c->info[k].any_hs = any_hs;
    c->info[k].rmax = rmax;
    N.list_r2_max = list_r2(c->info[k], N.list_cut_sq, smax);
    NetHost& h = c->info[k];
    h.bead_begin = (int)nb;
    h.bead_end = (int)(nb + d.n_beads);
    h.spring_begin = (int)ns;
    h.spring_end = (int)(ns + d.n_springs);
    h.angle_begin = (int)na;
    h.angle_end = (int)(na + d.n_angles);
    h.cell_begin = ncells;
    h.cell_end = ncells + (long long)N.nx * N.ny * N.nz;
    h.grid_update_freq = d.settings.grid_update_freq;
    h.damping = N.damping;
    N.cell_base = (int)ncells;
    N.bead_begin = h.bead_begin;
    N.bead_end = h.bead_end;
    if (N.damping != 0.0) c->damp = true;
    if (h.grid_update_freq <= 0) return fail(c, FN_ERR_ARG, "grid_update_freq must be positive");
    if (k > 0 && h.grid_update_freq != c->info[0].grid_update_freq)
        return fail(c, FN_ERR_UNSUPPORTED, "all networks of a batch must share grid_update_freq");
    nb += d.n_beads;
    ns += d.n_springs;
    na += d.n_angles;
    ncells = h.cell_end;
    if (nb > 0x7fffffffLL || ns > 0x3fffffffLL || na > 0x1fffffffLL || ncells > 0x7fffffffLL)
        return fail(c, FN_ERR_ARG, "model too large for 32-bit indices");
    return FN_OK;
}

/* largest radius, largest skin radius and smallest skin - radius of network
   k: the listing radius of its hs pairs and the displacement threshold */
static void set_radius_extremes(fn_ctx* c, int k, double rmax, double smax, double gap) {
    c->info[k].skin_gap = gap;
    c->info[k].rmax = rmax;
    c->nets_h[k].list_r2_max = list_r2(c->info[k], c->nets_h[k].list_cut_sq, smax);
}

/* The context's device buffers for a model of these sizes, whichever path
   converts the model. */
static cudaError_t alloc_model(fn_ctx* c, long long nb, long long ns, long long na, long long ncells, int n_networks,
                               std::string& what) {
    cudaError_t e = cudaSuccess;
#define AL(call)                   \
    do {                           \
        if ((e = (call)) != cudaSuccess) { \
            what = #call;          \
            return e;              \
        }                          \
    } while (0)
    const size_t list_n = (size_t)c->list_stride * (size_t)c->cfg.list_capacity;
    for (int k = 0; k < 2; ++k) {
        AL(dalloc(c, c->pos[k], nb));
        AL(dalloc(c, c->img[k], nb));
    }
    AL(dalloc(c, c->vold, nb));
    AL(dalloc(c, c->force, nb));
    AL(dalloc(c, c->vel, nb));
    AL(dalloc(c, c->binfo, nb));
    AL(dalloc(c, c->sp_ends, ns));
    AL(dalloc(c, c->sp_par, ns));
    AL(dalloc(c, c->sp_type, ns));
    AL(dalloc(c, c->sp_status, ns));
    AL(dalloc(c, c->an_b, na));
    AL(dalloc(c, c->an_s, na));
    AL(dalloc(c, c->an_par, na));
    AL(dalloc(c, c->an_status, na));
    AL(dalloc(c, c->cell_of, nb));
    AL(dalloc(c, c->cell_count, ncells));
    AL(dalloc(c, c->cell_fill, ncells));
    AL(dalloc(c, c->cell_start, ncells + 1));
    AL(dalloc(c, c->cell_beads, nb));
    AL(dalloc(c, c->list_count, nb));
    AL(dalloc(c, c->list, list_n));
    AL(dalloc(c, c->scan_sums, (size_t)std::max(fn::scan_block_count(ncells), fn::scan_block_count(nb)) + 1));
    AL(dalloc(c, c->nets, n_networks));
    AL(dalloc(c, c->pairs, c->pairs_h.size()));
    AL(dalloc(c, c->counters, FN_CNT_N));
    AL(dalloc(c, c->obs_partial, 5 * 1024));
    AL(dalloc(c, c->obs_out, 8));
    AL(dalloc(c, c->en_partial, (size_t)fn::FN_EN_N * 1024));
    AL(dalloc(c, c->en_out, fn::FN_EN_N));
#undef AL
    return cudaSuccess;
}

/* The context's totals once every network's preamble has run. */
static void set_totals(fn_ctx* c, long long nb, long long ns, long long na, long long ncells) {
    c->nb = nb;
    c->ns = ns;
    c->na = na;
    c->ncells = ncells;
    c->list_stride = (int)((nb + 31) / 32 * 32);
    c->grid_update_freq = c->info[0].grid_update_freq;
}

/* What fn_upload resets before either path runs. */
static int upload_begin(fn_ctx* c, int n_networks) {
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->uploaded = false;
    c->snap_valid = false;
    c->n_nets = n_networks;
    c->nets_h.assign(n_networks, FnNet{});
    c->info.assign(n_networks, NetHost{});
    c->pairs_h.clear();
    c->damp = false;
    c->host_stale = false;
    c->uploaded_on_device = false;
    c->incidence_ready = false;
    /* freed before any helper thread allocates (all update the context's
       device-byte count) */
    dfree(c, c->inv_d);
    dfree(c, c->perm_d);
    dfree(c, c->sp_bead_d);
    dfree(c, c->an_bead_d);
    return FN_OK;
}

/* The host path of fn_upload: checks, bead order and conversion on host
   threads, device allocations and copies overlapped with them.  Runs for
   every model the device path does not take. */
static int upload_host(fn_ctx* c, int n_networks, const fn_network_desc* nets) {
    int r0 = upload_begin(c, n_networks);
    if (r0) return r0;
    long long nb = 0, ns = 0, na = 0, ncells = 0;
    for (int k = 0; k < n_networks; ++k) {
        int r = net_preamble(c, k, nets[k], nb, ns, na, ncells, true);
        if (r) return r;
    }
    set_totals(c, nb, ns, na, ncells);
    /* device allocations on a helper thread while this one orders and
       converts the model (the sizes are known from here on) */
    cudaError_t alloc_err = cudaSuccess;
    std::string alloc_what;
    std::thread allocator([&, nb, ns, na, ncells, n_networks] {
        if ((alloc_err = cudaSetDevice(c->cfg.device)) != cudaSuccess) return;
        alloc_err = alloc_model(c, nb, ns, na, ncells, n_networks, alloc_what);
    });
    JoinOnExit join_allocator{allocator};


    /* bead order */
    c->perm.assign(nb, 0);
    c->inv.assign(nb, 0);
    for (int k = 0; k < n_networks; ++k) {
        std::vector<int> order;
        network_order(nets[k], c->nets_h[k], c->cfg.reorder != 0, order);
        const int base = c->info[k].bead_begin;
        parallel_for((long long)order.size(), [&](long long q0, long long q1) {
            for (long long q = q0; q < q1; ++q) {
                c->perm[base + q] = base + order[q];
                c->inv[base + order[q]] = base + (int)q;
            }
        });
    }

    /* bead arrays in internal order */
    HostArray<double4> pos(nb), img(nb);
    HostArray<float4> vold(nb), force(nb), vel(nb);
    HostArray<int4> binfo(nb);
    for (int k = 0; k < n_networks; ++k) {
        const fn_network_desc& d = nets[k];
        const int base = c->info[k].bead_begin;
        parallel_for(d.n_beads, [&](long long i0, long long i1) {
        for (int i = (int)i0; i < (int)i1; ++i) {
            const int q = c->inv[base + i];
            const float rad = (float)d.radius[i];
            const double mass = d.mass[i];
            const double minv = mass > 0.0 ? 1.0 / mass : 0.0; /* SimulationManager.cpp:1435-1445 */
            pos[q] = make_double4(d.pos[3 * i], d.pos[3 * i + 1], d.pos[3 * i + 2], pack_w(rad, d.type[i]));
            img[q] = make_double4(d.img[3 * i], d.img[3 * i + 1], d.img[3 * i + 2], minv);
            vold[q] = make_float4((float)d.vel_old[3 * i], (float)d.vel_old[3 * i + 1],
                                  (float)d.vel_old[3 * i + 2], 0.f);
            force[q] = make_float4((float)d.force[3 * i], (float)d.force[3 * i + 1],
                                   (float)d.force[3 * i + 2], 0.f);
            vel[q] = make_float4((float)d.vel[3 * i], (float)d.vel[3 * i + 1], (float)d.vel[3 * i + 2], 0.f);
            const float skin = (float)((double)rad + d.settings.skin_ratio);
            binfo[q] = make_int4(d.tag[i], d.loc_id[i], d.type[i], float_bits(skin));
        }
        });
    }

    /* the device arrays exist from here on: the bead arrays go to the device
       on a helper thread while this one converts the bonds */
    allocator.join();
    if (alloc_err != cudaSuccess)
        return fail(c, alloc_err == cudaErrorMemoryAllocation ? FN_ERR_OOM : FN_ERR_CUDA,
                    alloc_what + ": " + cudaGetErrorString(alloc_err));
    c->cur = 0;
    cudaError_t copy_err[2] = {cudaSuccess, cudaSuccess};
    std::string copy_what[2];
#define CP(k, call)                           \
    do {                                      \
        if ((copy_err[k] = (call)) != cudaSuccess) { \
            copy_what[k] = #call;             \
            return;                           \
        }                                     \
    } while (0)
    std::thread bead_copier([&] {
        if ((copy_err[0] = cudaSetDevice(c->cfg.device)) != cudaSuccess) return;
        CP(0, h2d(c, c->pos[0], pos));
        CP(0, h2d(c, c->img[0], img));
        CP(0, cudaMemcpyAsync(c->pos[1].p, c->pos[0].p, sizeof(double4) * nb, cudaMemcpyDeviceToDevice, c->stream));
        CP(0, cudaMemcpyAsync(c->img[1].p, c->img[0].p, sizeof(double4) * nb, cudaMemcpyDeviceToDevice, c->stream));
        CP(0, h2d(c, c->vold, vold));
        CP(0, h2d(c, c->force, force));
        CP(0, h2d(c, c->vel, vel));
        CP(0, h2d(c, c->binfo, binfo));
        CP(0, h2d(c, c->nets, c->nets_h));
        CP(0, h2d(c, c->pairs, c->pairs_h));
        CP(0, cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * FN_CNT_N, c->stream));
        CP(0, cudaMemsetAsync(c->list_count.p, 0, sizeof(int) * (size_t)nb, c->stream));
        CP(0, cudaMemsetAsync(c->cell_of.p, 0xff, sizeof(int) * (size_t)nb, c->stream));
        CP(0, cudaMemsetAsync(c->cell_count.p, 0, sizeof(int) * (size_t)ncells, c->stream));
    });
    JoinOnExit join_bead_copier{bead_copier};

    /* springs and angles keep their (concatenated) file order; the host
       copies the engine keeps are filled in place */
    std::vector<signed char> sp_type(ns), sp_status(ns, 1);
    c->sp_ends_h.resize(ns);
    c->sp_par_h.resize(ns);
    c->an_b_h.resize(na);
    c->an_s_h.resize(na);
    c->an_par_h.resize(na);
    std::vector<signed char> an_status(na, 1);
    std::vector<int2>& sp_ends = c->sp_ends_h;
    std::vector<int4>& an_b = c->an_b_h;
    std::vector<int2>& an_s = c->an_s_h;
    for (int k = 0; k < n_networks; ++k) {
        const fn_network_desc& d = nets[k];
        const NetHost& h = c->info[k];
        parallel_for(d.n_springs, [&](long long s0, long long s1) {
        for (int s = (int)s0; s < (int)s1; ++s) {
            const int g = h.spring_begin + s;
            sp_ends[g] = make_int2(c->inv[h.bead_begin + d.s_p1[s]], c->inv[h.bead_begin + d.s_p2[s]]);
            sp_type[g] = (signed char)d.s_type[s];
            c->sp_par_h[g] = make_float4((float)d.s_rest[s], (float)d.s_k[s], (float)d.s_c1[s], (float)d.s_c2[s]);
        }
        });
        parallel_for(d.n_angles, [&](long long a0, long long a1) {
        for (int a = (int)a0; a < (int)a1; ++a) {
            const int g = h.angle_begin + a;
            an_b[g] = make_int4(c->inv[h.bead_begin + d.a_b1[a]], c->inv[h.bead_begin + d.a_b2[a]],
                                c->inv[h.bead_begin + d.a_b3[a]], d.a_type[a]);
            const int s1 = d.a_type[a] == 1 ? h.spring_begin + d.a_s1[a] : 0;
            const int s2 = d.a_type[a] == 1 ? h.spring_begin + d.a_s2[a] : 0;
            an_s[g] = make_int2(s1, s2);
            c->an_par_h[g] = make_float2((float)d.a_theta0[a], (float)d.a_k[a]);
        }
        });
    }
    c->incidence_ready = false;

    /* the bond arrays go to the device on a second helper thread while this
       one builds the chain records */
    std::thread bond_copier([&] {
        if ((copy_err[1] = cudaSetDevice(c->cfg.device)) != cudaSuccess) return;
        CP(1, h2d(c, c->sp_ends, sp_ends));
        CP(1, h2d(c, c->sp_par, c->sp_par_h));
        CP(1, h2d(c, c->sp_type, sp_type));
        CP(1, h2d(c, c->sp_status, sp_status));
        CP(1, h2d(c, c->an_b, an_b));
        CP(1, h2d(c, c->an_s, an_s));
        CP(1, h2d(c, c->an_par, c->an_par_h));
        CP(1, h2d(c, c->an_status, an_status));
    });
    JoinOnExit join_bond_copier{bond_copier};
#undef CP
    c->chain = c->cfg.chain_mode != 2 && build_chain(c, sp_ends, sp_type, an_b, an_s);
    bead_copier.join();
    bond_copier.join();
    for (int k = 0; k < 2; ++k)
        if (copy_err[k] != cudaSuccess)
            return fail(c, FN_ERR_CUDA, copy_what[k] + ": " + cudaGetErrorString(copy_err[k]));
    int r = build_bricks(c);
    if (r) return r;
    r = set_block(c, c->cfg.block_size > 0 ? c->cfg.block_size : 128,
                  c->cfg.chain_mode == 0 ? kDefaultItemsPerThread : 0);
    if (r) return r;
    r = verlet_setup(c);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    c->steps_done = 0;
    c->rebuilds_done = 0;
    c->uploaded = true;
    return FN_OK;
}

/* fn_upload returns this internally when the device path leaves the model to
   the host path */
constexpr int kUploadFallback = -1;

/* Stream-ordered scratch of the device path, returned to the pool on every
   way out. */
struct StreamScratch {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~StreamScratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

/* The device path of fn_upload: the caller's arrays are copied to the device
   as they are (one copy per array and network) and checked, ordered and
   converted there (fn_upload.cu); the host sorts one key per fibre.  It takes
   models whose every spring joins consecutive beads (fibres stored bead
   after bead) and whose bonds are in chain form, and leaves every other
   model -- and every invalid one, whose error the host path then reports
   exactly as before -- to the host path (kUploadFallback).  The staged
   arrays are the host path's, bit for bit. */
static int upload_device(fn_ctx* c, int n_networks, const fn_network_desc* nets) {
    int r = upload_begin(c, n_networks);
    if (r) return r;
    long long nb = 0, ns = 0, na = 0, ncells = 0;
    for (int k = 0; k < n_networks; ++k)
        if (net_preamble(c, k, nets[k], nb, ns, na, ncells, false)) return kUploadFallback;
    set_totals(c, nb, ns, na, ncells);

    /* one stream-ordered block for the staged caller arrays and the
       temporaries, carved in 256-byte aligned pieces */
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_type = take(4 * nb), o_tag = take(4 * nb), o_loc = take(4 * nb), o_rad = take(8 * nb),
                 o_mass = take(8 * nb), o_pos = take(24 * nb), o_vel = take(24 * nb), o_vold = take(24 * nb),
                 o_frc = take(24 * nb), o_img = take(24 * nb);
    const size_t o_stype = take(4 * ns), o_p1 = take(4 * ns), o_p2 = take(4 * ns), o_rest = take(8 * ns),
                 o_sk = take(8 * ns), o_c1 = take(8 * ns), o_c2 = take(8 * ns);
    const size_t o_atype = take(4 * na), o_b1 = take(4 * na), o_b2 = take(4 * na), o_b3 = take(4 * na),
                 o_s1 = take(4 * na), o_s2 = take(4 * na), o_th = take(8 * na), o_ak = take(8 * na);
    const size_t o_nets = take(sizeof(fn::UpNet) * n_networks), o_chk = take(sizeof(fn::UpCheck) * n_networks);
    const size_t o_link = take(nb), o_flag = take(4 * nb), o_runof = take(4 * (nb + 1)), o_start = take(4 * nb),
                 o_key = take(8 * nb), o_runout = take(4 * nb), o_next = take(4 * nb), o_centre = take(4 * nb),
                 o_fl = take(nb), o_fa = take(nb), o_bad = take(4);
    StreamScratch sc;
    sc.s = c->stream;
    {
        cudaMemPool_t pool;
        CK(device_pool(c->cfg.device, &pool));
        CK(cudaMallocFromPoolAsync(&sc.p, off, pool, c->stream));
    }
    char* base = static_cast<char*>(sc.p);
    auto at = [&](size_t o) { return (void*)(base + o); };

    std::vector<fn::UpNet> un(n_networks);
    std::vector<fn::UpCheck> chk(n_networks);
    for (int k = 0; k < n_networks; ++k) {
        const NetHost& h = c->info[k];
        fn::UpNet& u = un[k];
        u.bead_begin = h.bead_begin;
        u.bead_end = h.bead_end;
        u.spring_begin = h.spring_begin;
        u.spring_end = h.spring_end;
        u.angle_begin = h.angle_begin;
        u.angle_end = h.angle_end;
        u.n_types = nets[k].settings.n_types;
        u.pad_ = 0;
        for (int a = 0; a < 3; ++a) u.box[a] = nets[k].settings.box[a];
        u.skin_ratio = nets[k].settings.skin_ratio;
        chk[k].bad_bead = chk[k].bad_spring = chk[k].bad_angle = 0x7fffffff;
        chk[k].not_runs = 0;
        chk[k].rmax = chk[k].smax = 0ull;
        chk[k].gmin = ~0ull;
    }
    /* the caller's arrays, network by network */
    for (int k = 0; k < n_networks; ++k) {
        const fn_network_desc& d = nets[k];
        const NetHost& h = c->info[k];
        const size_t b = (size_t)h.bead_begin, n = (size_t)d.n_beads;
        const size_t sb = (size_t)h.spring_begin, sn = (size_t)d.n_springs;
        const size_t ab = (size_t)h.angle_begin, an = (size_t)d.n_angles;
        auto cp = [&](size_t o, size_t first, size_t count, size_t elem, const void* src) -> cudaError_t {
            if (!count) return cudaSuccess;
            return cudaMemcpyAsync(base + o + first * elem, src, count * elem, cudaMemcpyHostToDevice, c->stream);
        };
        CK(cp(o_type, b, n, 4, d.type));
        CK(cp(o_tag, b, n, 4, d.tag));
        CK(cp(o_loc, b, n, 4, d.loc_id));
        CK(cp(o_rad, b, n, 8, d.radius));
        CK(cp(o_mass, b, n, 8, d.mass));
        CK(cp(o_pos, b, n, 24, d.pos));
        CK(cp(o_vel, b, n, 24, d.vel));
        CK(cp(o_vold, b, n, 24, d.vel_old));
        CK(cp(o_frc, b, n, 24, d.force));
        CK(cp(o_img, b, n, 24, d.img));
        CK(cp(o_stype, sb, sn, 4, d.s_type));
        CK(cp(o_p1, sb, sn, 4, d.s_p1));
        CK(cp(o_p2, sb, sn, 4, d.s_p2));
        CK(cp(o_rest, sb, sn, 8, d.s_rest));
        CK(cp(o_sk, sb, sn, 8, d.s_k));
        CK(cp(o_c1, sb, sn, 8, d.s_c1));
        CK(cp(o_c2, sb, sn, 8, d.s_c2));
        CK(cp(o_atype, ab, an, 4, d.a_type));
        CK(cp(o_b1, ab, an, 4, d.a_b1));
        CK(cp(o_b2, ab, an, 4, d.a_b2));
        CK(cp(o_b3, ab, an, 4, d.a_b3));
        CK(cp(o_s1, ab, an, 4, d.a_s1));
        CK(cp(o_s2, ab, an, 4, d.a_s2));
        CK(cp(o_th, ab, an, 8, d.a_theta0));
        CK(cp(o_ak, ab, an, 8, d.a_k));
    }
    /* the model's device buffers while those copies run */
    {
        std::string what;
        cudaError_t e = alloc_model(c, nb, ns, na, ncells, n_networks, what);
        if (e != cudaSuccess)
            return fail(c, e == cudaErrorMemoryAllocation ? FN_ERR_OOM : FN_ERR_CUDA,
                        what + ": " + cudaGetErrorString(e));
    }
    CK(dalloc(c, c->inv_d, (size_t)nb));
    CK(dalloc(c, c->export_xyz, (size_t)(3 * nb)));
    CK(dalloc(c, c->perm_d, (size_t)nb));
    CK(dalloc(c, c->sp_bead_d, (size_t)ns));
    CK(dalloc(c, c->an_bead_d, (size_t)na));
    CK(dalloc(c, c->ch_sp, (size_t)nb));
    CK(dalloc(c, c->ch_an, (size_t)nb));
    CK(dalloc(c, c->ch_flags, (size_t)nb));
    CK(dalloc(c, c->ch_status, (size_t)nb));
    CK(cudaMemcpyAsync(at(o_nets), un.data(), sizeof(fn::UpNet) * n_networks, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(at(o_chk), chk.data(), sizeof(fn::UpCheck) * n_networks, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(at(o_link), 0, (size_t)nb, c->stream));
    fn::UpRaw R;
    R.type = (const int*)at(o_type);
    R.tag = (const int*)at(o_tag);
    R.loc_id = (const int*)at(o_loc);
    R.radius = (const double*)at(o_rad);
    R.mass = (const double*)at(o_mass);
    R.pos = (const double*)at(o_pos);
    R.vel = (const double*)at(o_vel);
    R.vel_old = (const double*)at(o_vold);
    R.force = (const double*)at(o_frc);
    R.img = (const double*)at(o_img);
    R.s_type = (const int*)at(o_stype);
    R.s_p1 = (const int*)at(o_p1);
    R.s_p2 = (const int*)at(o_p2);
    R.s_rest = (const double*)at(o_rest);
    R.s_k = (const double*)at(o_sk);
    R.s_c1 = (const double*)at(o_c1);
    R.s_c2 = (const double*)at(o_c2);
    R.a_type = (const int*)at(o_atype);
    R.a_b1 = (const int*)at(o_b1);
    R.a_b2 = (const int*)at(o_b2);
    R.a_b3 = (const int*)at(o_b3);
    R.a_s1 = (const int*)at(o_s1);
    R.a_s2 = (const int*)at(o_s2);
    R.a_theta0 = (const double*)at(o_th);
    R.a_k = (const double*)at(o_ak);
    const fn::UpNet* unets = (const fn::UpNet*)at(o_nets);
    unsigned char* link = (unsigned char*)at(o_link);
    int* flag = (int*)at(o_flag);
    int* run_of = (int*)at(o_runof);
    int* start = (int*)at(o_start);
    unsigned long long* key = (unsigned long long*)at(o_key);
    int* run_out = (int*)at(o_runout);

    /* checks: any offending index, or a spring between non-consecutive
       beads, leaves the model to the host path */
    CK(fn::launch_upload_checks(unets, n_networks, R, (fn::UpCheck*)at(o_chk), (int)nb, (int)ns, (int)na, link,
                                c->stream));
    const bool reorder = c->cfg.reorder != 0;
    if (reorder)
        CK(fn::launch_upload_runs(unets, n_networks, R, link, flag, run_of, c->scan_sums.p, start, key, (int)nb,
                                  c->stream));
    int n_runs = 0;
    CK(cudaMemcpyAsync(chk.data(), at(o_chk), sizeof(fn::UpCheck) * n_networks, cudaMemcpyDeviceToHost, c->stream));
    if (reorder) CK(cudaMemcpyAsync(&n_runs, run_of + nb, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    auto undkey = [](unsigned long long k) {
        const unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double x;
        std::memcpy(&x, &u, 8);
        return x;
    };
    for (int k = 0; k < n_networks; ++k) {
        const fn::UpCheck& q = chk[k];
        if (q.bad_bead != 0x7fffffff || q.bad_spring != 0x7fffffff || q.bad_angle != 0x7fffffff || q.not_runs)
            return kUploadFallback;
        set_radius_extremes(c, k, undkey(q.rmax), undkey(q.smax), undkey(q.gmin));
    }

    /* bead order: the runs (fibres) of each network sorted by key, as the
       host path sorts them, and laid out one after the other */
    if (reorder) {
        std::vector<int> st(n_runs);
        std::vector<unsigned long long> ky(n_runs);
        CK(cudaMemcpyAsync(st.data(), start, sizeof(int) * (size_t)n_runs, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(ky.data(), key, sizeof(unsigned long long) * (size_t)n_runs, cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
        std::vector<int> out(n_runs), ord(n_runs), tmp(n_runs);
        int r0 = 0;
        for (int k = 0; k < n_networks; ++k) {
            const int bb = c->info[k].bead_begin, be = c->info[k].bead_end;
            int r1 = r0;
            while (r1 < n_runs && st[r1] < be) ++r1;
            /* the runs by key: the key's low word is the run's first bead,
               which grows with the run index, so a stable sort of the runs
               (in index order) by the 30-bit Morton code in the high word
               gives the order of a sort of the whole keys -- three passes of
               a 10-bit counting sort */
            for (int q = r0; q < r1; ++q) ord[q] = q;
            for (int pass = 0; pass < 3; ++pass) {
                const int shift = 32 + 10 * pass;
                int count[1025] = {0};
                for (int q = r0; q < r1; ++q) ++count[((ky[ord[q]] >> shift) & 1023) + 1];
                for (int v = 0; v < 1024; ++v) count[v + 1] += count[v];
                for (int q = r0; q < r1; ++q) tmp[r0 + count[(ky[ord[q]] >> shift) & 1023]++] = ord[q];
                std::copy(tmp.begin() + r0, tmp.begin() + r1, ord.begin() + r0);
            }
            int acc = bb;
            for (int q = r0; q < r1; ++q) {
                const int rr = ord[q];
                const int len = (rr + 1 < r1 ? st[rr + 1] : be) - st[rr];
                out[rr] = acc;
                acc += len;
            }
            r0 = r1;
        }
        CK(cudaMemcpyAsync(run_out, out.data(), sizeof(int) * (size_t)n_runs, cudaMemcpyHostToDevice, c->stream));
    }
    c->cur = 0;
    CK(fn::launch_upload_convert(unets, n_networks, R, flag, run_of, start, run_out, reorder ? 1 : 0, c->inv_d.p,
                                 c->perm_d.p, c->pos[0].p, c->img[0].p, c->vold.p, c->force.p, c->vel.p, c->binfo.p,
                                 c->sp_ends.p, c->sp_par.p, c->sp_type.p, c->sp_status.p, c->an_b.p, c->an_s.p,
                                 c->an_par.p, c->an_status.p, (int)nb, (int)ns, (int)na, c->stream));
    /* chain form: per-bead records, or back to the host path */
    CK(cudaMemsetAsync(at(o_next), 0xff, 4 * (size_t)nb, c->stream));
    CK(cudaMemsetAsync(at(o_centre), 0xff, 4 * (size_t)nb, c->stream));
    CK(cudaMemsetAsync(at(o_fl), 0, (size_t)nb, c->stream));
    CK(cudaMemsetAsync(at(o_fa), 0, (size_t)nb, c->stream));
    CK(cudaMemsetAsync(at(o_bad), 0, 4, c->stream));
    CK(fn::launch_upload_chain(c->sp_ends.p, c->sp_type.p, c->sp_par.p, c->an_b.p, c->an_s.p, c->an_par.p,
                               (int*)at(o_next), (int*)at(o_centre), (unsigned char*)at(o_fl),
                               (unsigned char*)at(o_fa), c->ch_sp.p, c->ch_an.p, c->ch_flags.p, c->ch_status.p,
                               c->sp_bead_d.p, c->an_bead_d.p, (int*)at(o_bad), (int)nb, (int)ns, (int)na,
                               c->stream));
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, at(o_bad), sizeof bad, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (bad) return kUploadFallback;

    CK(cudaMemcpyAsync(c->pos[1].p, c->pos[0].p, sizeof(double4) * nb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->img[1].p, c->img[0].p, sizeof(double4) * nb, cudaMemcpyDeviceToDevice, c->stream));
    CK(h2d(c, c->nets, c->nets_h));
    CK(h2d(c, c->pairs, c->pairs_h));
    CK(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * FN_CNT_N, c->stream));
    CK(cudaMemsetAsync(c->list_count.p, 0, sizeof(int) * (size_t)nb, c->stream));
    CK(cudaMemsetAsync(c->cell_of.p, 0xff, sizeof(int) * (size_t)nb, c->stream));
    CK(cudaMemsetAsync(c->cell_count.p, 0, sizeof(int) * (size_t)ncells, c->stream));
    c->chain = true;
    c->host_stale = true; /* host copies of the numbering and the bonds: on first need */
    c->uploaded_on_device = true;
    r = build_bricks(c);
    if (r) return r;
    r = set_block(c, c->cfg.block_size > 0 ? c->cfg.block_size : 128, c->cfg.chain_mode == 0 ? kDefaultItemsPerThread : 0);
    if (r) return r;
    r = verlet_setup(c);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    c->steps_done = 0;
    c->rebuilds_done = 0;
    c->uploaded = true;
    return FN_OK;
}

/* fn_upload: the device path when the model is in its reach, else (and
   for every invalid model, whose error the host path reports) the host path.
   Host exceptions become status codes. */
FN_API int fn_upload(fn_ctx* c, int n_networks, const fn_network_desc* nets) {
    try {
        fnh::NvtxRange nvtx_range_("fn_upload");
        if (c) c->state_version++;
        if (!c || n_networks <= 0 || !nets) return fail(c, FN_ERR_ARG, "fn_upload: bad arguments");
        if (c->cfg.chain_mode != 2 && !c->cfg.host_upload) {
            const int r = upload_device(c, n_networks, nets);
            if (r != kUploadFallback) return r;
        }
        return upload_host(c, n_networks, nets);
    } catch (const std::bad_alloc&) {
        return fail(c, FN_ERR_OOM, "fn_upload: out of host memory");
    } catch (const std::system_error& e) {
        return fail(c, FN_ERR_OOM, std::string("fn_upload: no host thread: ") + e.what());
    } catch (const std::exception& e) {
        return fail(c, FN_ERR_ARG, std::string("fn_upload: ") + e.what());
    }
}

FN_API int fn_step(fn_ctx* c, int nsteps) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_step");
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if (nsteps <= 0) return fail(c, FN_ERR_ARG, "RunSimulationLoop: loop size should be a positive number");
    CK(cudaSetDevice(c->cfg.device));
    /* AdvancePosition of step 0 */
    {
        fn::StepArgs A = step_args(c, false);
        CK(fn::launch_drift(A, c->ntiles, c->block, c->damp || nsteps == 1, c->stream));
    }
    /* the rebuild counter is local to the call (SimulationManager.cpp:152),
       so the call is a sequence of grid_update_freq-step segments, each
       opened by a rebuild */
    for (int done = 0; done < nsteps;) {
        const int len = std::min(c->grid_update_freq, nsteps - done);
        r = run_segment(c, len, done + len == nsteps);
        if (r) return r;
        done += len;
    }
    c->steps_done += nsteps;
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_rebuild_contacts(fn_ctx* c) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    CK(cudaSetDevice(c->cfg.device));
    if (c->verlet) {
        const int one = 1;
        CK(cudaMemcpyAsync(c->gate.p, &one, sizeof one, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return do_rebuild(c);
    FN_CATCH(c)
}

FN_API int fn_reset_energy(fn_ctx* c) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    CK(cudaSetDevice(c->cfg.device));
    CK(fn::launch_reset_energy(c->force.p, c->vel.p, c->vold.p, (int)c->nb, c->stream));
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_sync(fn_ctx* c) {
    FN_TRY
    if (!c) return FN_ERR_ARG;
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    if (!c->uploaded) return FN_OK;
    unsigned long long cnt[FN_CNT_N];
    CK(cudaMemcpy(cnt, c->counters.p, sizeof cnt, cudaMemcpyDeviceToHost));
    if (cnt[FN_CNT_STALL])
        return fail(c, FN_ERR_CUDA, "a step kernel's wait for staged data ran out in " +
                                        std::to_string(cnt[FN_CNT_STALL]) + " tiles (the state is unusable)");
    const unsigned long long bad = cnt[FN_CNT_NONFINITE];
    if (bad) return fail(c, FN_ERR_NONFINITE, "non-finite force detected in " + std::to_string(bad) + " bead-steps");
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_device_view(fn_ctx* c, int field, fn_view* out) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if (!out) return fail(c, FN_ERR_ARG, "fn_device_view: null output");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    out->n = c->nb;
    out->components = 4;
    switch (field) {
    case FN_POSITION: out->ptr = c->pos[c->cur].p; out->elem_bytes = 8; break;
    case FN_IMAGE: out->ptr = c->img[c->cur].p; out->elem_bytes = 8; break;
    case FN_VELOCITY: out->ptr = c->vel.p; out->elem_bytes = 4; break;
    case FN_FORCE: out->ptr = c->force.p; out->elem_bytes = 4; break;
    case FN_VELOCITY_OLD: out->ptr = c->vold.p; out->elem_bytes = 4; break;
    default: return fail(c, FN_ERR_ARG, "fn_device_view: unknown field");
    }
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_download(fn_ctx* c, int field, double* host) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_download");
    int r = check_ready(c);
    if (r) return r;
    if (!host) return fail(c, FN_ERR_ARG, "fn_download: null host pointer");
    CK(cudaSetDevice(c->cfg.device));
    const long long nb = c->nb;
    /* permuted and unpacked on the device, then one copy into the caller's
       x, y, z layout */
    if (!c->inv_d.p || c->export_xyz.n < (size_t)(3 * nb)) {
        CK(dalloc(c, c->inv_d, (size_t)nb));
        CK(dalloc(c, c->export_xyz, (size_t)(3 * nb)));
        CK(h2d(c, c->inv_d, c->inv));
    }
    if (field == FN_POSITION || field == FN_IMAGE) {
        const DevBuf<double4>& b = field == FN_POSITION ? c->pos[c->cur] : c->img[c->cur];
        CK(fn::launch_export_xyz(b.p, c->inv_d.p, (int)nb, c->export_xyz.p, c->stream));
    } else {
        const DevBuf<float4>* b = field == FN_VELOCITY ? &c->vel
                                  : field == FN_FORCE  ? &c->force
                                  : field == FN_VELOCITY_OLD ? &c->vold
                                                             : nullptr;
        if (!b) return fail(c, FN_ERR_ARG, "fn_download: unknown field");
        CK(fn::launch_export_xyz(b->p, c->inv_d.p, (int)nb, c->export_xyz.p, c->stream));
    }
    CK(cudaMemcpyAsync(host, c->export_xyz.p, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_set_beads(fn_ctx* c, int field, const double* host) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    if (!host) return fail(c, FN_ERR_ARG, "fn_set_beads: null host pointer");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    const long long nb = c->nb;
    if (field == FN_POSITION || field == FN_IMAGE) {
        if (c->verlet) {
            const int one = 1;
            CK(cudaMemcpy(c->gate.p, &one, sizeof one, cudaMemcpyHostToDevice));
        }
        DevBuf<double4>& b = field == FN_POSITION ? c->pos[c->cur] : c->img[c->cur];
        std::vector<double4> tmp(nb);
        CK(cudaMemcpy(tmp.data(), b.p, sizeof(double4) * nb, cudaMemcpyDeviceToHost));
        for (long long q = 0; q < nb; ++q) {
            const long long i = c->perm[q];
            tmp[q].x = host[3 * i];
            tmp[q].y = host[3 * i + 1];
            tmp[q].z = host[3 * i + 2];
        }
        CK(cudaMemcpy(b.p, tmp.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice));
        return FN_OK;
    }
    DevBuf<float4>* b = field == FN_VELOCITY ? &c->vel
                        : field == FN_FORCE  ? &c->force
                        : field == FN_VELOCITY_OLD ? &c->vold
                                                   : nullptr;
    if (!b) return fail(c, FN_ERR_ARG, "fn_set_beads: unknown field");
    std::vector<float4> tmp(nb);
    for (long long q = 0; q < nb; ++q) {
        const long long i = c->perm[q];
        tmp[q] = make_float4((float)host[3 * i], (float)host[3 * i + 1], (float)host[3 * i + 2], 0.f);
    }
    CK(cudaMemcpy(b->p, tmp.data(), sizeof(float4) * nb, cudaMemcpyHostToDevice));
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_set_mass(fn_ctx* c, const double* mass) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    if (!mass) return fail(c, FN_ERR_ARG, "fn_set_mass: null pointer");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    const long long nb = c->nb;
    for (long long i = 0; i < nb; ++i)
        if (!(mass[i] >= 0.0)) return fail(c, FN_ERR_ARG, "fn_set_mass: mass must be zero or positive");
    std::vector<double4> tmp(nb);
    CK(cudaMemcpy(tmp.data(), c->img[c->cur].p, sizeof(double4) * nb, cudaMemcpyDeviceToHost));
    for (long long q = 0; q < nb; ++q) {
        const double m = mass[c->perm[q]];
        tmp[q].w = m > 0.0 ? 1.0 / m : 0.0;
    }
    CK(cudaMemcpy(c->img[c->cur].p, tmp.data(), sizeof(double4) * nb, cudaMemcpyHostToDevice));
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_set_skin(fn_ctx* c, const double* skin) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    if (!skin) return fail(c, FN_ERR_ARG, "fn_set_skin: null pointer");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    const long long nb = c->nb;
    std::vector<int4> tmp(nb);
    CK(cudaMemcpy(tmp.data(), c->binfo.p, sizeof(int4) * nb, cudaMemcpyDeviceToHost));
    for (long long q = 0; q < nb; ++q) tmp[q].w = float_bits((float)skin[c->perm[q]]);
    CK(cudaMemcpy(c->binfo.p, tmp.data(), sizeof(int4) * nb, cudaMemcpyHostToDevice));
    /* radii as stored (float, packed in the position's fourth word), upload order */
    std::vector<double4> p4(nb);
    CK(cudaMemcpy(p4.data(), c->pos[c->cur].p, sizeof(double4) * nb, cudaMemcpyDeviceToHost));
    std::vector<float> radius(nb);
    for (long long q = 0; q < nb; ++q) {
        uint64_t bits;
        std::memcpy(&bits, &p4[q].w, 8);
        const uint32_t lo = (uint32_t)bits;
        std::memcpy(&radius[c->perm[q]], &lo, 4);
    }
    for (int k = 0; k < c->n_nets; ++k) {
        double smax = 0.0;
        double gap = 1e300;
        for (int i = c->info[k].bead_begin; i < c->info[k].bead_end; ++i) {
            smax = std::max(smax, (double)(float)skin[i]);
            gap = std::min(gap, (double)(float)skin[i] - (double)radius[i]);
        }
        c->info[k].skin_gap = gap;
        c->nets_h[k].list_r2_max = list_r2(c->info[k], c->nets_h[k].list_cut_sq, smax);
    }
    CK(cudaMemcpy(c->nets.p, c->nets_h.data(), sizeof(FnNet) * c->n_nets, cudaMemcpyHostToDevice));
    r = verlet_setup(c);
    if (r) return r;
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_set_springs(fn_ctx* c, const double* rest, const double* k, const double* c1,
                          const double* c2) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    for (long long s = 0; s < c->ns; ++s) {
        float4& p = c->sp_par_h[s];
        if (rest) p.x = (float)rest[s];
        if (k) p.y = (float)k[s];
        if (c1) p.z = (float)c1[s];
        if (c2) p.w = (float)c2[s];
    }
    if (c->ns > 0)
        CK(cudaMemcpy(c->sp_par.p, c->sp_par_h.data(), sizeof(float4) * c->ns, cudaMemcpyHostToDevice));
    if (c->chain && c->ns > 0) {
        std::vector<float4> chs(c->nb, make_float4(0, 0, 0, 0));
        for (long long q = 0; q < c->ns; ++q) chs[c->sp_bead[q]] = c->sp_par_h[q];
        CK(cudaMemcpy(c->ch_sp.p, chs.data(), sizeof(float4) * c->nb, cudaMemcpyHostToDevice));
    }
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_set_angles(fn_ctx* c, const double* theta0, const double* k) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    for (long long a = 0; a < c->na; ++a) {
        if (theta0) c->an_par_h[a].x = (float)theta0[a];
        if (k) c->an_par_h[a].y = (float)k[a];
    }
    if (c->na > 0)
        CK(cudaMemcpy(c->an_par.p, c->an_par_h.data(), sizeof(float2) * c->na, cudaMemcpyHostToDevice));
    if (c->chain && c->na > 0) {
        std::vector<float2> cha(c->nb, make_float2(0, 0));
        for (long long q = 0; q < c->na; ++q) cha[c->an_bead[q]] = c->an_par_h[q];
        CK(cudaMemcpy(c->ch_an.p, cha.data(), sizeof(float2) * c->nb, cudaMemcpyHostToDevice));
    }
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_download_status(fn_ctx* c, int* spring_status, int* angle_status) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    CK(cudaSetDevice(c->cfg.device));
    if (c->chain) {
        std::vector<unsigned char> st(c->nb);
        CK(cudaMemcpyAsync(st.data(), c->ch_status.p, c->nb, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (spring_status)
            for (long long q = 0; q < c->ns; ++q) spring_status[q] = st[c->sp_bead[q]] & 1;
        if (angle_status)
            for (long long q = 0; q < c->na; ++q) angle_status[q] = (st[c->an_bead[q]] >> 1) & 1;
        return FN_OK;
    }
    std::vector<signed char> s(c->ns), a(c->na);
    if (c->ns > 0 && spring_status)
        CK(cudaMemcpyAsync(s.data(), c->sp_status.p, c->ns, cudaMemcpyDeviceToHost, c->stream));
    if (c->na > 0 && angle_status)
        CK(cudaMemcpyAsync(a.data(), c->an_status.p, c->na, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (spring_status)
        for (long long q = 0; q < c->ns; ++q) spring_status[q] = s[q];
    if (angle_status)
        for (long long q = 0; q < c->na; ++q) angle_status[q] = a[q];
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_set_status(fn_ctx* c, const int* spring_status, const int* angle_status) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    if (c->chain) {
        std::vector<unsigned char> st(c->nb);
        CK(cudaMemcpy(st.data(), c->ch_status.p, c->nb, cudaMemcpyDeviceToHost));
        if (spring_status)
            for (long long q = 0; q < c->ns; ++q)
                st[c->sp_bead[q]] = (unsigned char)((st[c->sp_bead[q]] & ~1u) | (spring_status[q] == 1 ? 1u : 0u));
        if (angle_status)
            for (long long q = 0; q < c->na; ++q)
                st[c->an_bead[q]] = (unsigned char)((st[c->an_bead[q]] & ~2u) | (angle_status[q] == 1 ? 2u : 0u));
        CK(cudaMemcpy(c->ch_status.p, st.data(), c->nb, cudaMemcpyHostToDevice));
        return FN_OK;
    }
    if (spring_status && c->ns > 0) {
        std::vector<signed char> s(c->ns);
        for (long long q = 0; q < c->ns; ++q) s[q] = (signed char)spring_status[q];
        CK(cudaMemcpy(c->sp_status.p, s.data(), c->ns, cudaMemcpyHostToDevice));
    }
    if (angle_status && c->na > 0) {
        std::vector<signed char> a(c->na);
        for (long long q = 0; q < c->na; ++q) a[q] = (signed char)angle_status[q];
        CK(cudaMemcpy(c->an_status.p, a.data(), c->na, cudaMemcpyHostToDevice));
    }
    return FN_OK;
    FN_CATCH(c)
}

namespace {

/* Blocks of 256 threads of the observables reduction of network `net`: one
   per 256 beads, springs or angles, at most 1024 (each block then loops), so
   the partial sums and their order depend on the network alone. */
int observe_blocks(const fn_ctx* c, int net) {
    const NetHost& h = c->info[net];
    const long long span = std::max({(long long)(h.bead_end - h.bead_begin), (long long)(h.spring_end - h.spring_begin),
                                     (long long)(h.angle_end - h.angle_begin), 1LL});
    return (int)std::min<long long>(1024, (span + 255) / 256);
}

/* Observables of network `net` into out[0..4] on the context's stream, with
   the partial sums in `partial` (5 doubles per block). */
int observe_into(fn_ctx* c, int net, int reaction_type, double* partial, double* out) {
    const NetHost& h = c->info[net];
    fn::ObserveArgs O{};
    O.ch_flags = c->chain ? c->ch_flags.p : nullptr;
    O.ch_status = c->chain ? c->ch_status.p : nullptr;
    O.pos = c->pos[c->cur].p;
    O.force = c->force.p;
    O.sp_status = c->sp_status.p;
    O.an_status = c->an_status.p;
    O.bead_begin = h.bead_begin;
    O.bead_end = h.bead_end;
    O.spring_begin = h.spring_begin;
    O.spring_end = h.spring_end;
    O.angle_begin = h.angle_begin;
    O.angle_end = h.angle_end;
    O.reaction_type = reaction_type;
    O.partial = partial;
    CK(fn::launch_observe(O, observe_blocks(c, net), out, c->stream));
    return FN_OK;
}

int observe_async(fn_ctx* c, int net, int reaction_type, double* out) {
    return observe_into(c, net, reaction_type, c->obs_partial.p, out);
}

/* Energy and virial of network `net` into out[0..FN_EN_N) on the stream. */
int energy_async(fn_ctx* c, int net, double* out) {
    const NetHost& h = c->info[net];
    fn::EnergyArgs E{};
    E.nets = c->nets.p;
    E.pairs = c->pairs.p;
    E.pos = c->pos[c->cur].p;
    E.img = c->img[c->cur].p;
    E.vold = c->vold.p;
    E.sp_ends = c->sp_ends.p;
    E.sp_par = c->sp_par.p;
    E.sp_type = c->sp_type.p;
    E.sp_status = c->sp_status.p;
    E.an_b = c->an_b.p;
    E.an_par = c->an_par.p;
    E.an_status = c->an_status.p;
    E.ch_status = c->chain ? c->ch_status.p : nullptr;
    E.list_count = c->list_count.p;
    E.list = c->list.p;
    E.list_stride = c->list_stride;
    E.list_cap = c->cfg.list_capacity;
    E.net = net;
    E.bead_begin = h.bead_begin;
    E.bead_end = h.bead_end;
    E.spring_begin = h.spring_begin;
    E.spring_end = h.spring_end;
    E.angle_begin = h.angle_begin;
    E.angle_end = h.angle_end;
    E.partial = c->en_partial.p;
    long long span = std::max({(long long)(h.bead_end - h.bead_begin), (long long)(h.spring_end - h.spring_begin),
                               (long long)(h.angle_end - h.angle_begin), 1LL});
    int nblocks = (int)std::min<long long>(1024, (span + 255) / 256);
    CK(fn::launch_energy(E, nblocks, out, c->stream));
    return FN_OK;
}

}  // namespace

FN_API int fn_observe(fn_ctx* c, int net, int reaction_type, fn_observables* out) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_observe");
    int r = check_ready(c);
    if (r) return r;
    if (!out || net < 0 || net >= c->n_nets) return fail(c, FN_ERR_ARG, "fn_observe: bad arguments");
    CK(cudaSetDevice(c->cfg.device));
    r = observe_async(c, net, reaction_type, c->obs_out.p);
    if (r) return r;
    double res[5];
    CK(cudaMemcpyAsync(res, c->obs_out.p, sizeof res, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int a = 0; a < 3; ++a) out->reaction[a] = res[a];
    out->broken = (long long)res[3];
    out->angles_dead = (long long)res[4];
    return FN_OK;
    FN_CATCH(c)
}


FN_API int fn_energy_eval(fn_ctx* c, int net, fn_energy* out) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_energy_eval");
    int r = check_ready(c);
    if (r) return r;
    if (!out || net < 0 || net >= c->n_nets) return fail(c, FN_ERR_ARG, "fn_energy_eval: bad arguments");
    CK(cudaSetDevice(c->cfg.device));
    r = energy_async(c, net, c->en_out.p);
    if (r) return r;
    double res[fn::FN_EN_N];
    CK(cudaMemcpyAsync(res, c->en_out.p, sizeof res, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out->kinetic = res[fn::FN_EN_KINETIC];
    out->spring = res[fn::FN_EN_SPRING];
    out->angle = res[fn::FN_EN_ANGLE];
    out->contact = res[fn::FN_EN_CONTACT];
    out->wall = res[fn::FN_EN_WALL];
    out->gravity = res[fn::FN_EN_GRAVITY];
    for (int k = 0; k < 9; ++k) out->virial[k] = res[fn::FN_EN_VIRIAL + k];
    out->contacts = (long long)res[fn::FN_EN_CONTACTS];
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_step_series(fn_ctx* c, int nsteps, int every, int net, int reaction_type,
                          int with_energy, double* host_rows) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_step_series");
    int r = check_ready(c);
    if (r) return r;
    if (nsteps <= 0 || every <= 0 || net < 0 || net >= c->n_nets || !host_rows)
        return fail(c, FN_ERR_ARG, "fn_step_series: bad arguments");
    CK(cudaSetDevice(c->cfg.device));
    const int width = with_energy ? 6 + fn::FN_EN_N : 6;
    const long long rows = (nsteps + (long long)every - 1) / every;
    const size_t need = (size_t)rows * width;
    if (c->series.n < need) {
        dfree(c, c->series);
        CK(dalloc(c, c->series, need));
    }
    std::vector<double> steps_done(rows);
    int done = 0;
    for (long long q = 0; q < rows; ++q) {
        const int k = std::min(every, nsteps - done);
        r = fn_step(c, k);
        if (r) return r;
        done += k;
        double* row = c->series.p + (size_t)q * width;
        r = observe_async(c, net, reaction_type, row + 1);
        if (r) return r;
        if (with_energy) {
            r = energy_async(c, net, row + 6);
            if (r) return r;
        }
        steps_done[q] = (double)done;
    }
    CK(cudaMemcpyAsync(host_rows, c->series.p, sizeof(double) * need, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (long long q = 0; q < rows; ++q) host_rows[(size_t)q * width] = steps_done[q];
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_get_stats(fn_ctx* c, fn_stats* out) {
    FN_TRY
    if (!c || !out) return FN_ERR_ARG;
    std::memset(out, 0, sizeof *out);
    out->block_size = c->block;
    out->items_per_thread = c->staged ? c->chunk / c->block : 0;
    out->upload_on_device = c->uploaded_on_device ? 1 : 0;
    out->list_by_bricks = c->list_build == 1 ? 1 : 0;
    out->list_build = c->list_build;
    out->bond_path = c->chain ? 2 : (c->tiled ? 1 : 0);
    out->graph_launches = c->graph_launches;
    out->n_networks = c->n_nets;
    out->n_beads = c->nb;
    out->device_bytes = c->device_bytes;
    out->steps = c->steps_done;
    out->rebuilds = c->rebuilds_done;
    if (!c->uploaded) return FN_OK;
    CK(cudaSetDevice(c->cfg.device));
    unsigned long long cnt[FN_CNT_N];
    CK(cudaMemcpyAsync(cnt, c->counters.p, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->verlet) out->rebuilds = (long long)cnt[FN_CNT_REBUILDS];
    out->nonfinite = (long long)cnt[FN_CNT_NONFINITE];
    out->stalls = (long long)cnt[FN_CNT_STALL];
    out->cell_overflow = (long long)cnt[FN_CNT_CELL_OVERFLOW];
    out->list_overflow = (long long)cnt[FN_CNT_LIST_OVERFLOW];
    if (cnt[FN_CNT_NONFINITE]) c->err = "non-finite force detected";
    return FN_OK;
    FN_CATCH(c)
}

FN_API long long fn_n_cells(fn_ctx* c) { return c ? c->ncells : -1; }

FN_API int fn_get_cells(fn_ctx* c, int* bead_cell, int* cell_count, long long n_cells) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    CK(cudaSetDevice(c->cfg.device));
    if (bead_cell) {
        std::vector<int> tmp(c->nb);
        CK(cudaMemcpyAsync(tmp.data(), c->cell_of.p, sizeof(int) * c->nb, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (long long q = 0; q < c->nb; ++q) bead_cell[c->perm[q]] = tmp[q];
    }
    if (cell_count) {
        if (n_cells != c->ncells) return fail(c, FN_ERR_ARG, "fn_get_cells: wrong cell count");
        CK(cudaMemcpyAsync(cell_count, c->cell_count.p, sizeof(int) * c->ncells, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_get_lists(fn_ctx* c, int* count, int* partners, int cap) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    CK(cudaSetDevice(c->cfg.device));
    const long long nb = c->nb;
    std::vector<int> cnt(nb);
    CK(cudaMemcpyAsync(cnt.data(), c->list_count.p, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->stream));
    std::vector<int> lst;
    if (partners) {
        lst.resize((size_t)c->list_stride * c->cfg.list_capacity);
        CK(cudaMemcpyAsync(lst.data(), c->list.p, sizeof(int) * lst.size(), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    for (long long q = 0; q < nb; ++q) {
        const long long i = c->perm[q];
        if (count) count[i] = cnt[q];
        if (partners) {
            const int n = std::min(std::min(cnt[q], c->cfg.list_capacity), cap);
            for (int k = 0; k < n; ++k)
                partners[(size_t)i * cap + k] = c->perm[lst[(size_t)k * c->list_stride + q]];
        }
    }
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_get_permutation(fn_ctx* c, int* perm) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    if (!perm) return FN_ERR_ARG;
    std::memcpy(perm, c->perm.data(), sizeof(int) * c->nb);
    return FN_OK;
    FN_CATCH(c)
}

/* Starts (on != 0) or stops a timing window: while on, every step-kernel
   launch and every rebuild is bracketed by CUDA events on the context's
   stream; fn_kernel_time averages the window. */
FN_API int fn_enable_timing(fn_ctx* c, int on) {
    FN_TRY
    if (!c) return FN_ERR_ARG;
    if (on) {
        CK(cudaSetDevice(c->cfg.device));
        CK(cudaStreamSynchronize(c->stream));
        c->ev_next = 0;
        c->ev_step.clear();
        c->ev_rebuild.clear();
    }
    c->timing = on != 0;
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_kernel_time(fn_ctx* c, double* step_ms, long long* launches, double* rebuild_ms,
                          long long* rebuilds) {
    FN_TRY
    if (!c) return FN_ERR_ARG;
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    double ts = 0.0, tr = 0.0;
    for (auto& p : c->ev_step) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p.first, p.second));
        ts += ms;
    }
    for (auto& p : c->ev_rebuild) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, p.first, p.second));
        tr += ms;
    }
    if (step_ms) *step_ms = c->ev_step.empty() ? 0.0 : ts / (double)c->ev_step.size();
    if (launches) *launches = (long long)c->ev_step.size();
    if (rebuild_ms) *rebuild_ms = c->ev_rebuild.empty() ? 0.0 : tr / (double)c->ev_rebuild.size();
    if (rebuilds) *rebuilds = (long long)c->ev_rebuild.size();
    return FN_OK;
    FN_CATCH(c)
}

/* Step-kernel tuner: for each candidate shape -- block size and, for the
   staged chain kernel, contact items per thread and round (0: the plain chain
   kernel) -- the same `steps_per_trial` steps run from one snapshot of the
   state (restored after every trial, so the simulation does not advance),
   timed with CUDA events; the fastest shape is kept, then the faster list
   build (by bricks or bead by bead) at that shape. */
FN_API int fn_autotune(fn_ctx* c, int steps_per_trial) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_autotune");
    int r = check_ready(c);
    if (r) return r;
    if (steps_per_trial <= 0) return fail(c, FN_ERR_ARG, "fn_autotune: steps_per_trial must be positive");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    const size_t nb = (size_t)c->nb;
    struct Snap {
        void* p;
        const void* src;
        size_t bytes;
    };
    std::vector<Snap> snaps;
    auto add = [&](const void* src, size_t bytes) {
        if (src && bytes) snaps.push_back({nullptr, src, bytes});
    };
    add(c->pos[c->cur].p, sizeof(double4) * nb);
    add(c->img[c->cur].p, sizeof(double4) * nb);
    add(c->vold.p, sizeof(float4) * nb);
    add(c->force.p, sizeof(float4) * nb);
    add(c->vel.p, sizeof(float4) * nb);
    add(c->sp_status.p, (size_t)c->ns);
    add(c->an_status.p, (size_t)c->na);
    if (c->chain) add(c->ch_status.p, nb);
    add(c->counters.p, sizeof(unsigned long long) * FN_CNT_N);
    for (auto& sn : snaps) {
        CK(cudaMalloc(&sn.p, sn.bytes));
        CK(cudaMemcpyAsync(sn.p, sn.src, sn.bytes, cudaMemcpyDeviceToDevice, c->stream));
    }
    const int cur0 = c->cur;
    const long long steps0 = c->steps_done, rb0 = c->rebuilds_done;
    const bool timing0 = c->timing;
    c->timing = false;
    std::vector<std::pair<int, int>> shapes;
    for (int b : {64, 96, 128, 192, 256, 384, 512}) {
        if (c->chain && b > fn::kChainMaxBlock) continue;
        if (c->chain && c->cfg.chain_mode == 0)
            for (int k : {2, 4, 8}) shapes.emplace_back(b, k);
        shapes.emplace_back(b, 0);
    }
    int dev = 0, optin = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    std::pair<int, int> best{c->block, c->staged ? c->chunk / c->block : 0};
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (const auto& sh : shapes) {
        if (sh.second > 0 && fn::step_staged_smem(sh.first, sh.first * sh.second) > (size_t)optin) continue;
        if ((r = set_block(c, sh.first, sh.second))) break;
        for (int rep = 0; rep < 2 && !r; ++rep) { /* first run warms up */
            c->cur = cur0;
            for (auto& sn : snaps)
                CK(cudaMemcpyAsync(const_cast<void*>(sn.src), sn.p, sn.bytes, cudaMemcpyDeviceToDevice, c->stream));
            CK(cudaEventRecord(e0, c->stream));
            r = fn_step(c, steps_per_trial);
            CK(cudaEventRecord(e1, c->stream));
        }
        if (r) break;
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
            best_ms = ms;
            best = sh;
        }
    }
    /* then the list build (bead by bead, by bricks, by groups of lanes) at
       that shape */
    int best_build = c->list_build;
    if (!r && (r = set_block(c, best.first, best.second)) == 0) {
        float ms_build[3] = {1e30f, 1e30f, 1e30f};
        for (int mode = 0; mode < 3 && !r; ++mode) {
            c->list_build = mode;
            drop_graphs(c);
            for (int rep = 0; rep < 2 && !r; ++rep) {
                c->cur = cur0;
                for (auto& sn : snaps)
                    CK(cudaMemcpyAsync(const_cast<void*>(sn.src), sn.p, sn.bytes, cudaMemcpyDeviceToDevice, c->stream));
                CK(cudaEventRecord(e0, c->stream));
                r = fn_step(c, steps_per_trial);
                CK(cudaEventRecord(e1, c->stream));
            }
            if (r) break;
            CK(cudaEventSynchronize(e1));
            CK(cudaEventElapsedTime(&ms_build[mode], e0, e1));
        }
        best_build = 0;
        for (int mode = 1; mode < 3; ++mode)
            if (ms_build[mode] < ms_build[best_build]) best_build = mode;
    }
    c->list_build = best_build;
    drop_graphs(c);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->cur = cur0;
    for (auto& sn : snaps) {
        cudaMemcpyAsync(const_cast<void*>(sn.src), sn.p, sn.bytes, cudaMemcpyDeviceToDevice, c->stream);
    }
    cudaStreamSynchronize(c->stream);
    for (auto& sn : snaps) cudaFree(sn.p);
    c->steps_done = steps0;
    c->rebuilds_done = rb0;
    c->timing = timing0;
    if (r) return r;
    return set_block(c, best.first, best.second);
    FN_CATCH(c)
}

/* Chooses how contact lists are built: 0 bead by bead from global memory, 1
   by bricks of cells staged in shared memory, 2 by groups of 8 lanes per
   bead.  Same lists, entry for entry, every way. */
FN_API int fn_set_list_build(fn_ctx* c, int bricks) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if (bricks < 0 || bricks > 2) return fail(c, FN_ERR_ARG, "fn_set_list_build: 0, 1 or 2");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->list_build = bricks;
    return FN_OK;
    FN_CATCH(c)
}

/* Sets the step kernel's shape directly (what fn_autotune picks). */
FN_API int fn_set_kernel_shape(fn_ctx* c, int block, int items_per_thread) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if (block < 32 || block > 512 || block % 32 != 0)
        return fail(c, FN_ERR_ARG, "fn_set_kernel_shape: block must be a multiple of 32 in 32 .. 512");
    if (items_per_thread != 0 && !(c->chain && c->cfg.chain_mode == 0))
        return fail(c, FN_ERR_UNSUPPORTED, "fn_set_kernel_shape: contact staging needs the chain path (chain_mode 0)");
    if (c->chain && block < 64) return fail(c, FN_ERR_ARG, "fn_set_kernel_shape: chain tiles need blocks of 64 or more");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    return set_block(c, block, items_per_thread);
    FN_CATCH(c)
}

/* The dynamic state a step changes, as (device pointer, bytes) pairs in a
   fixed order: positions and images of the current ping-pong half,
   velocity_old, force, velocity, spring/angle statuses (both layouts), the
   device counters and, in displacement mode, the reference images and the
   rebuild gate.  Contact lists are not state: every fn_step call rebuilds
   them at its step 0. */
static std::vector<std::pair<void*, size_t>> state_arrays(fn_ctx* c) {
    const size_t nb = (size_t)c->nb;
    std::vector<std::pair<void*, size_t>> v;
    v.emplace_back(c->pos[c->cur].p, sizeof(double4) * nb);
    v.emplace_back(c->img[c->cur].p, sizeof(double4) * nb);
    v.emplace_back(c->vold.p, sizeof(float4) * nb);
    v.emplace_back(c->force.p, sizeof(float4) * nb);
    v.emplace_back(c->vel.p, sizeof(float4) * nb);
    v.emplace_back(c->sp_status.p, (size_t)c->ns);
    v.emplace_back(c->an_status.p, (size_t)c->na);
    if (c->chain) v.emplace_back(c->ch_status.p, nb);
    v.emplace_back(c->counters.p, sizeof(unsigned long long) * FN_CNT_N);
    if (c->verlet) {
        v.emplace_back(c->ref_img.p, sizeof(double4) * nb);
        v.emplace_back(c->gate.p, sizeof(int));
    }
    return v;
}

/* Device-side snapshot of the dynamic state (no counterpart in the reference,
   whose restart files go through the host): one device buffer held by the
   context, copied on its stream. */
FN_API int fn_state_save(fn_ctx* c) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    CK(cudaSetDevice(c->cfg.device));
    const auto arrs = state_arrays(c);
    size_t total = 0;
    for (const auto& a : arrs) total += (a.second + 255) / 256 * 256;
    if (c->snap.n < total) CK(dalloc(c, c->snap, total));
    size_t off = 0;
    for (const auto& a : arrs) {
        if (a.first && a.second)
            CK(cudaMemcpyAsync(c->snap.p + off, a.first, a.second, cudaMemcpyDeviceToDevice, c->stream));
        off += (a.second + 255) / 256 * 256;
    }
    c->snap_valid = true;
    c->snap_cur = c->cur;
    c->snap_steps = c->steps_done;
    c->snap_rebuilds = c->rebuilds_done;
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_state_restore(fn_ctx* c) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    if (!c->snap_valid) return fail(c, FN_ERR_STATE, "fn_state_restore: no snapshot (call fn_state_save first)");
    CK(cudaSetDevice(c->cfg.device));
    c->cur = c->snap_cur;
    const auto arrs = state_arrays(c);
    size_t off = 0;
    for (const auto& a : arrs) {
        if (a.first && a.second)
            CK(cudaMemcpyAsync(a.first, c->snap.p + off, a.second, cudaMemcpyDeviceToDevice, c->stream));
        off += (a.second + 255) / 256 * 256;
    }
    c->steps_done = c->snap_steps;
    c->rebuilds_done = c->snap_rebuilds;
    return FN_OK;
    FN_CATCH(c)
}

/* fn_step bracketed by CUDA events on the context's stream; waits for the
   second event and returns the device time between them. */
FN_API int fn_step_timed(fn_ctx* c, int nsteps, double* ms) {
    FN_TRY
    int r = check_ready(c);
    if (r) return r;
    if (!ms) return fail(c, FN_ERR_ARG, "fn_step_timed: null output");
    CK(cudaSetDevice(c->cfg.device));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(c, FN_ERR_CUDA, "fn_step_timed: cudaEventCreate");
    }
    cudaError_t e = cudaEventRecord(e0, c->stream);
    if (e == cudaSuccess) {
        r = fn_step(c, nsteps);
        if (r == FN_OK) {
            e = cudaEventRecord(e1, c->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float f = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
            *ms = f;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r) return r;
    if (e != cudaSuccess) return fail(c, FN_ERR_CUDA, std::string("fn_step_timed: ") + cudaGetErrorString(e));
    return FN_OK;
    FN_CATCH(c)
}

/* Forces alone at the current positions (zeroed, no base term), for the
   one-step parity checks: terms bit 0 springs, 1 angles, 2 contacts. */
FN_API int fn_forces_only(fn_ctx* c, int terms) {
    FN_TRY
    if (c) c->state_version++;
    int r = check_ready(c);
    if (r) return r;
    CK(cudaSetDevice(c->cfg.device));
    fn::StepArgs A = step_args(c, false);
    if (c->chain)
        CK(fn::launch_forces_chain(A, c->ntiles, c->block, terms, c->stream));
    else
        CK(fn::launch_forces_only(A, c->ntiles, c->block, terms, c->stream));
    return FN_OK;
    FN_CATCH(c)
}

}  // extern "C"

/* ======================================================================== */
/* Observables without any device allocation.                               */

/* Partial sums of the observables reduction: one slot of 5 doubles per block,
   for the FN_OBSERVE_NOALLOC_MAX_BLOCKS blocks that fn_observe's reduction
   uses at most (larger networks loop inside each block), so any network fits
   and the sums are fn_observe's, bit for bit.  It lives in the library image:
   every GPU that loads the library holds these 40 KB until the process exits,
   and every call shares them. */
#define FN_OBSERVE_NOALLOC_MAX_BLOCKS 1024
static __device__ __align__(256) double fn_observe_scratch[5 * FN_OBSERVE_NOALLOC_MAX_BLOCKS];

namespace {

/* Device address of fn_observe_scratch on each device, looked up once per
   device.  In host code the array's name only stands in for the symbol; its
   address on a device comes from cudaGetSymbolAddress with that device
   current.  The cached address belongs to the device's primary context: a
   cudaDeviceReset (or any other teardown of that context) makes it stale, so
   a process that resets a device must not call fn_observe_noalloc on it
   afterwards. */
constexpr int FN_NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_scratch[FN_NOALLOC_MAX_DEVICES] = {};

int noalloc_scratch(fn_ctx* c, double** out) {
    const int dev = c->cfg.device;
    if (dev < 0 || dev >= FN_NOALLOC_MAX_DEVICES)
        return fail(c, FN_ERR_UNSUPPORTED, "fn_observe_noalloc: device ordinal beyond 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_scratch[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, fn_observe_scratch);
        if (e != cudaSuccess || !p)
            return fail(c, FN_ERR_CUDA, std::string("fn_observe_noalloc: cudaGetSymbolAddress: ") +
                                            cudaGetErrorString(e));
        g_noalloc_scratch[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_scratch[dev];
    return FN_OK;
}

}  // namespace

extern "C" FN_API int fn_observe_noalloc(fn_ctx* c, int net, int reaction_type, double* out_device) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_observe_noalloc");
    int r = check_ready(c);
    if (r) return r;
    if (!out_device || net < 0 || net >= c->n_nets)
        return fail(c, FN_ERR_ARG, "fn_observe_noalloc: bad arguments");
    const int nblocks = observe_blocks(c, net);
    if (nblocks > FN_OBSERVE_NOALLOC_MAX_BLOCKS) /* guards the scratch should the block rule change */
        return fail(c, FN_ERR_CAPACITY,
                    "fn_observe_noalloc: the reduction needs " + std::to_string(nblocks) +
                        " partial sums; the static scratch holds " +
                        std::to_string(FN_OBSERVE_NOALLOC_MAX_BLOCKS) + " (use fn_observe)");
    CK(cudaSetDevice(c->cfg.device));
    double* scratch = nullptr;
    r = noalloc_scratch(c, &scratch);
    if (r) return r;
    return observe_into(c, net, reaction_type, scratch, out_device);
    FN_CATCH(c)
}
