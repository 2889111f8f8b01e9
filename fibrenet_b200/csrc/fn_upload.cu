/*
 * fn_upload.cu -- kernels of the device-side model upload (fn_upload's fast
 * path, orchestrated in fn_engine.cu).
 *
 * The caller's arrays (model-file order, networks concatenated) are copied to
 * the device as they are; these kernels then do what ReadBeadsData /
 * ReadSpringData / ReadAngleData and the argument binding do on the
 * reference's host (SimulationManager.cpp:1372-1661, 1236-1304), plus the
 * renumbering of this implementation:
 *   - the index checks of the model file (bead types, masses, spring and
 *     angle ends, HR_FL angle springs) and the radius / skin extremes of each
 *     network;
 *   - the bead order: runs of consecutive beads joined by springs (fibres
 *     stored bead after bead) with a Morton key each, sorted on the host (one
 *     key per fibre), then the permutation;
 *   - the conversion into the device layout (double4 positions with packed
 *     radius/type and inverse mass, float4 velocities and forces, int4 bead
 *     info, bond arrays in the internal numbering);
 *   - the chain-form records of fibres (per-bead spring and angle records).
 * Each step produces what the host path of fn_upload produces, bit for bit
 * (same conversions, same rounding); anything outside this fast path (an
 * invalid model, springs joining non-consecutive beads, bonds not in chain
 * form) is reported back and the host path runs instead.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "fn_kernels.h"
#include "fn_types.h"

namespace fn {

/* network of global item x, given per-network first items (ascending) */
__device__ __forceinline__ int up_net(const UpNet* __restrict__ nets, int n_nets, int x, int which) {
    int lo = 0, hi = n_nets - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int b = which == 0 ? nets[mid].bead_begin : which == 1 ? nets[mid].spring_begin : nets[mid].angle_begin;
        if (b <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

/* order-preserving 64-bit keys of doubles (max of keys = max of values) */
__device__ __forceinline__ unsigned long long dkey(double x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

/* Index checks and radius extremes of every bead: first bad bead per network
   (undeclared type or a mass that is not >= 0), max radius, max skin radius,
   min (skin - radius), all as the host path computes them in double from
   the float-rounded radius. */
__global__ void __launch_bounds__(256) k_up_beads_check(const UpNet* __restrict__ nets, int n_nets, UpRaw R,
                                                        UpCheck* out, int nb) {
    __shared__ unsigned long long s_max_r[8], s_max_s[8], s_min_g[8];
    __shared__ int s_net0, s_net1;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int first = blockIdx.x * blockDim.x;
    const int last = min(first + (int)blockDim.x, nb) - 1;
    if (threadIdx.x == 0) {
        s_net0 = up_net(nets, n_nets, first, 0);
        s_net1 = up_net(nets, n_nets, last, 0);
    }
    __syncthreads();
    unsigned long long kr = 0, ks = 0, kg = ~0ull;
    int k = s_net0;
    if (u < nb) {
        k = s_net0 == s_net1 ? s_net0 : up_net(nets, n_nets, u, 0);
        const UpNet& N = nets[k];
        const int i = u - N.bead_begin;
        const int t = R.type[u];
        const double mass = R.mass[u];
        if (t < 0 || t >= N.n_types || !(mass >= 0.0)) atomicMin(&out[k].bad_bead, i);
        const float rad = (float)R.radius[u];
        const float skin = (float)((double)rad + N.skin_ratio);
        kr = dkey((double)rad);
        ks = dkey((double)skin);
        kg = dkey((double)skin - (double)rad);
    }
    if (s_net0 != s_net1) {
        /* the block spans two or more networks: one atomic per bead */
        if (u < nb) {
            atomicMax(&out[k].rmax, kr);
            atomicMax(&out[k].smax, ks);
            atomicMin(&out[k].gmin, kg);
        }
        return;
    }
    /* one network: reduce over the block, one atomic each */
    for (int o = 16; o > 0; o >>= 1) {
        kr = max(kr, __shfl_xor_sync(0xffffffffu, kr, o));
        ks = max(ks, __shfl_xor_sync(0xffffffffu, ks, o));
        kg = min(kg, __shfl_xor_sync(0xffffffffu, kg, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_max_r[w] = kr;
        s_max_s[w] = ks;
        s_min_g[w] = kg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int q = 1; q < nw; ++q) {
            kr = max(kr, s_max_r[q]);
            ks = max(ks, s_max_s[q]);
            kg = min(kg, s_min_g[q]);
        }
        atomicMax(&out[k].rmax, kr);
        atomicMax(&out[k].smax, ks);
        atomicMin(&out[k].gmin, kg);
    }
}

/* Spring index checks; springs that do not join consecutive beads are
   counted (the fast path needs none); link[lower bead] marks a spring to the
   next bead. */
__global__ void k_up_springs_check(const UpNet* __restrict__ nets, int n_nets, UpRaw R, UpCheck* out, int ns,
                                   unsigned char* link) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int k = up_net(nets, n_nets, s, 1);
    const UpNet& N = nets[k];
    const int nbk = N.bead_end - N.bead_begin;
    const int p1 = R.s_p1[s], p2 = R.s_p2[s];
    if (p1 < 0 || p1 >= nbk || p2 < 0 || p2 >= nbk) {
        atomicMin(&out[k].bad_spring, s - N.spring_begin);
        return;
    }
    if (abs(p1 - p2) != 1) {
        atomicAdd(&out[k].not_runs, 1);
        return;
    }
    link[N.bead_begin + min(p1, p2)] = 1;
}

__global__ void k_up_angles_check(const UpNet* __restrict__ nets, int n_nets, UpRaw R, UpCheck* out, int na) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    const int k = up_net(nets, n_nets, a, 2);
    const UpNet& N = nets[k];
    const int nbk = N.bead_end - N.bead_begin, nsk = N.spring_end - N.spring_begin;
    const int b1 = R.a_b1[a], b2 = R.a_b2[a], b3 = R.a_b3[a];
    bool bad = b1 < 0 || b1 >= nbk || b2 < 0 || b2 >= nbk || b3 < 0 || b3 >= nbk;
    if (!bad && R.a_type[a] == 1) {
        const int s1 = R.a_s1[a], s2 = R.a_s2[a];
        bad = s1 < 0 || s1 >= nsk || s2 < 0 || s2 >= nsk;
    }
    if (bad) atomicMin(&out[k].bad_angle, a - N.angle_begin);
}

/* 1 where a run of spring-joined consecutive beads starts */
__global__ void k_up_run_starts(const UpNet* __restrict__ nets, int n_nets, const unsigned char* link, int* flag,
                                int nb) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nb) return;
    const int k = up_net(nets, n_nets, u, 0);
    flag[u] = (u == nets[k].bead_begin || !link[u - 1]) ? 1 : 0;
}

__device__ __forceinline__ uint32_t up_spread10(uint32_t v) {
    v &= 0x3ff;
    v = (v | (v << 16)) & 0x030000FF;
    v = (v | (v << 8)) & 0x0300F00F;
    v = (v | (v << 4)) & 0x030C30C3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}

/* Runs compacted in bead order: first bead and the key the host path sorts
   by -- the Morton code of the first bead's position (1024 steps per axis of
   the network's box) above its network-local index. */
__global__ void k_up_run_keys(const UpNet* __restrict__ nets, int n_nets, UpRaw R, const int* flag,
                              const int* run_of, int* start, unsigned long long* key, int nb) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nb || !flag[u]) return;
    const int k = up_net(nets, n_nets, u, 0);
    const UpNet& N = nets[k];
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        double x = R.pos[3 * (size_t)u + a] / N.box[a] * 1024.0;
        if (!(x >= 0.0)) x = 0.0;
        if (x > 1023.0) x = 1023.0;
        q[a] = (uint32_t)x;
    }
    const unsigned long long m = up_spread10(q[0]) | (up_spread10(q[1]) << 1) | (up_spread10(q[2]) << 2);
    const int r = run_of[u];
    start[r] = u;
    key[r] = (m << 32) | (uint32_t)(u - N.bead_begin);
}

/* internal index of every bead: its run's first slot (run_out, ordered on
   the host) plus its place in the run; identity without reordering */
__global__ void k_up_perm(const int* flag, const int* run_of, const int* start, const int* run_out, int* inv,
                          int* perm, int nb, int reorder) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nb) return;
    int q = u;
    if (reorder) {
        const int r = run_of[u] + flag[u] - 1;
        q = run_out[r] + (u - start[r]);
    }
    inv[u] = q;
    perm[q] = u;
}

/* Bead arrays in the device layout at their internal index
   (SimulationManager.cpp:1435-1445 for the inverse mass; skin radius =
   radius + skin ratio, :1431). */
__global__ void k_up_beads(const UpNet* __restrict__ nets, int n_nets, UpRaw R, const int* inv, double4* pos,
                           double4* img, float4* vold, float4* force, float4* vel, int4* binfo, int nb) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nb) return;
    const int k = up_net(nets, n_nets, u, 0);
    const int q = inv[u];
    const size_t v = 3 * (size_t)u;
    const int t = R.type[u];
    const float rad = (float)R.radius[u];
    const double mass = R.mass[u];
    const double minv = mass > 0.0 ? 1.0 / mass : 0.0;
    pos[q] = make_double4(R.pos[v], R.pos[v + 1], R.pos[v + 2], __hiloint2double(t, __float_as_int(rad)));
    img[q] = make_double4(R.img[v], R.img[v + 1], R.img[v + 2], minv);
    vold[q] = make_float4((float)R.vel_old[v], (float)R.vel_old[v + 1], (float)R.vel_old[v + 2], 0.f);
    force[q] = make_float4((float)R.force[v], (float)R.force[v + 1], (float)R.force[v + 2], 0.f);
    vel[q] = make_float4((float)R.vel[v], (float)R.vel[v + 1], (float)R.vel[v + 2], 0.f);
    const float skin = (float)((double)rad + nets[k].skin_ratio);
    binfo[q] = make_int4(R.tag[u], R.loc_id[u], t, __float_as_int(skin));
}

/* Springs and angles keep their (concatenated) file order; their bead ends
   move to the internal numbering. */
__global__ void k_up_springs(const UpNet* __restrict__ nets, int n_nets, UpRaw R, const int* inv, int2* ends,
                             float4* par, signed char* type, signed char* status, int ns) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int k = up_net(nets, n_nets, s, 1);
    const int bb = nets[k].bead_begin;
    ends[s] = make_int2(inv[bb + R.s_p1[s]], inv[bb + R.s_p2[s]]);
    type[s] = (signed char)R.s_type[s];
    status[s] = 1;
    par[s] = make_float4((float)R.s_rest[s], (float)R.s_k[s], (float)R.s_c1[s], (float)R.s_c2[s]);
}

__global__ void k_up_angles(const UpNet* __restrict__ nets, int n_nets, UpRaw R, const int* inv, int4* b,
                            int2* sp, float2* par, signed char* status, int na) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    const int k = up_net(nets, n_nets, a, 2);
    const int bb = nets[k].bead_begin, sb = nets[k].spring_begin;
    const int t = R.a_type[a];
    b[a] = make_int4(inv[bb + R.a_b1[a]], inv[bb + R.a_b2[a]], inv[bb + R.a_b3[a]], t);
    sp[a] = t == 1 ? make_int2(sb + R.a_s1[a], sb + R.a_s2[a]) : make_int2(0, 0);
    status[a] = 1;
    par[a] = make_float2((float)R.a_theta0[a], (float)R.a_k[a]);
}

/* Chain form (the conditions of the host path's build_chain): every spring
   joins beads j, j + 1 of the internal numbering, one spring per lower bead
   (claimed with a compare-and-swap: a second claim breaks the form). */
__global__ void k_up_chain_springs(const int2* ends, const signed char* type, int* next_sp, unsigned char* fl,
                                   int* bad, int ns) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int a = ends[s].x, b = ends[s].y;
    const int lo = min(a, b), hi = max(a, b);
    if (hi != lo + 1) {
        atomicOr(bad, 1);
        return;
    }
    if (atomicCAS(next_sp + lo, -1, s) != -1) {
        atomicOr(bad, 2);
        return;
    }
    unsigned char f = FN_CH_SPRING;
    if (a == hi) f |= FN_CH_SP_REV;
    if (type[s] == 1)
        f |= FN_CH_SP_FL;
    else if (type[s] != 0)
        f |= FN_CH_SP_INERT;
    fl[lo] = f;
}

/* every angle is (j-1, j, j+1) or (j+1, j, j-1), one per centre; an HR_FL
   angle's springs are exactly the two around its centre */
__global__ void k_up_chain_angles(const int4* ab, const int2* as, const int* next_sp, int* centre_an,
                                  unsigned char* fa, int* bad, int na) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    const int4 b = ab[a];
    const bool fwd = b.x == b.y - 1 && b.z == b.y + 1;
    const bool rev = b.x == b.y + 1 && b.z == b.y - 1;
    if (!(fwd || rev)) {
        atomicOr(bad, 4);
        return;
    }
    if (atomicCAS(centre_an + b.y, -1, a) != -1) {
        atomicOr(bad, 8);
        return;
    }
    unsigned char f = FN_CH_ANGLE;
    if (rev) f |= FN_CH_AN_REV;
    if (b.w == 1) {
        f |= FN_CH_AN_FL;
        const int sp = next_sp[b.y - 1], sn = next_sp[b.y];
        const int2 ss = as[a];
        if (sp < 0 || sn < 0 || !((ss.x == sp && ss.y == sn) || (ss.x == sn && ss.y == sp))) atomicOr(bad, 16);
    }
    fa[b.y] = f;
}

/* around every bead the incident bonds come in ascending index order
   (previous, next spring; angles centred on j-1, j, j+1), then the per-bead
   records */
__global__ void k_up_chain_records(const int* next_sp, const int* centre_an, const unsigned char* fl,
                                   const unsigned char* fa, const float4* sp_par, const float2* an_par,
                                   float4* chs, float2* cha, unsigned char* flags, unsigned char* status,
                                   int* sp_bead, int* an_bead, int* bad, int nb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    if (i > 0 && next_sp[i - 1] >= 0 && next_sp[i] >= 0 && next_sp[i - 1] > next_sp[i]) atomicOr(bad, 32);
    int last = -1;
    for (int q = i - 1; q <= i + 1; ++q) {
        if (q < 0 || q >= nb || centre_an[q] < 0) continue;
        if (centre_an[q] < last) atomicOr(bad, 64);
        last = centre_an[q];
    }
    float4 s4 = make_float4(0, 0, 0, 0);
    float2 a2 = make_float2(0, 0);
    unsigned char st = 0;
    if (next_sp[i] >= 0) {
        s4 = sp_par[next_sp[i]];
        sp_bead[next_sp[i]] = i;
        st |= 1;
    }
    if (centre_an[i] >= 0) {
        a2 = an_par[centre_an[i]];
        an_bead[centre_an[i]] = i;
        st |= 2;
    }
    chs[i] = s4;
    cha[i] = a2;
    flags[i] = (unsigned char)(fl[i] | fa[i]);
    status[i] = st;
}

static inline unsigned grid(long long n, int block) { return (unsigned)((n + block - 1) / block); }

cudaError_t launch_upload_checks(const UpNet* nets, int n_nets, const UpRaw& R, UpCheck* out, int nb, int ns, int na,
                                 unsigned char* link, cudaStream_t s) {
    if (nb > 0) k_up_beads_check<<<grid(nb, 256), 256, 0, s>>>(nets, n_nets, R, out, nb);
    if (ns > 0) k_up_springs_check<<<grid(ns, 256), 256, 0, s>>>(nets, n_nets, R, out, ns, link);
    if (na > 0) k_up_angles_check<<<grid(na, 256), 256, 0, s>>>(nets, n_nets, R, out, na);
    return cudaGetLastError();
}

cudaError_t launch_upload_runs(const UpNet* nets, int n_nets, const UpRaw& R, const unsigned char* link, int* flag,
                               int* run_of, int* scan_sums, int* start, unsigned long long* key, int nb,
                               cudaStream_t s) {
    if (nb <= 0) return cudaSuccess;
    k_up_run_starts<<<grid(nb, 256), 256, 0, s>>>(nets, n_nets, link, flag, nb);
    cudaError_t e = launch_exclusive_scan(flag, nb, run_of, scan_sums, s);
    if (e) return e;
    k_up_run_keys<<<grid(nb, 256), 256, 0, s>>>(nets, n_nets, R, flag, run_of, start, key, nb);
    return cudaGetLastError();
}

cudaError_t launch_upload_convert(const UpNet* nets, int n_nets, const UpRaw& R, const int* flag, const int* run_of,
                                  const int* start, const int* run_out, int reorder, int* inv, int* perm,
                                  double4* pos, double4* img, float4* vold, float4* force, float4* vel, int4* binfo,
                                  int2* sp_ends, float4* sp_par, signed char* sp_type, signed char* sp_status,
                                  int4* an_b, int2* an_s, float2* an_par, signed char* an_status, int nb, int ns,
                                  int na, cudaStream_t s) {
    if (nb > 0) {
        k_up_perm<<<grid(nb, 256), 256, 0, s>>>(flag, run_of, start, run_out, inv, perm, nb, reorder);
        k_up_beads<<<grid(nb, 256), 256, 0, s>>>(nets, n_nets, R, inv, pos, img, vold, force, vel, binfo, nb);
    }
    if (ns > 0) k_up_springs<<<grid(ns, 256), 256, 0, s>>>(nets, n_nets, R, inv, sp_ends, sp_par, sp_type, sp_status, ns);
    if (na > 0) k_up_angles<<<grid(na, 256), 256, 0, s>>>(nets, n_nets, R, inv, an_b, an_s, an_par, an_status, na);
    return cudaGetLastError();
}

cudaError_t launch_upload_chain(const int2* sp_ends, const signed char* sp_type, const float4* sp_par,
                                const int4* an_b, const int2* an_s, const float2* an_par, int* next_sp,
                                int* centre_an, unsigned char* fl, unsigned char* fa, float4* chs, float2* cha,
                                unsigned char* flags, unsigned char* status, int* sp_bead, int* an_bead, int* bad,
                                int nb, int ns, int na, cudaStream_t s) {
    if (ns > 0) k_up_chain_springs<<<grid(ns, 256), 256, 0, s>>>(sp_ends, sp_type, next_sp, fl, bad, ns);
    if (na > 0) k_up_chain_angles<<<grid(na, 256), 256, 0, s>>>(an_b, an_s, next_sp, centre_an, fa, bad, na);
    if (nb > 0)
        k_up_chain_records<<<grid(nb, 256), 256, 0, s>>>(next_sp, centre_an, fl, fa, sp_par, an_par, chs, cha, flags,
                                                         status, sp_bead, an_bead, bad, nb);
    return cudaGetLastError();
}

}  // namespace fn
