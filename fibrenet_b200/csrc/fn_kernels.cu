/*
 * fn_kernels.cu -- sm_100a kernels of the FibreNet step loop.
 *
 * One time step is one launch of k_step: every thread owns one bead and
 *   1. rebuilds the base force the reference writes in AdvancePosition
 *      (damping * v + gravity + wall penalty, kernel.cl:231-261),
 *   2. gathers its incident springs (kernel.cl:366-441), angles
 *      (kernel.cl:268-363) and contacts (kernel.cl:792-1011) in a fixed order
 *      instead of the reference's FP64 atomics,
 *   3. applies AdvanceVelocity (kernel.cl:444-464), and
 *   4. applies the next step's AdvancePosition (kernel.cl:195-265), writing the
 *      drifted position into the other half of a ping-pong pair so neighbours
 *      still read this step's positions.
 * A standalone k_drift opens each fn_step call.  The contact list is rebuilt
 * between steps (k_cells -> scan -> k_scatter -> k_cell_sort -> k_lists),
 * giving the same pair set as FillGrid + BuildContactList (kernel.cl:487-789)
 * with deterministic order.
 *
 * All force arithmetic is FP64 with the reference's operation order; the
 * library is built with -fmad=false so nothing is contracted into FMAs, which
 * keeps results bit-identical to the host mirror checker.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <climits>

#include "fn_detmath.h"
#include "fn_device.cuh"
#include "fn_kernels.h"
#include "fn_types.h"

namespace fn {


__device__ __forceinline__ int spring_pts(double ax, double ay, double az, double bx, double by,
                                          double bz, float4 par, int type, double& fx, double& fy,
                                          double& fz, int& broke);

/* Spring s (kernel.cl:371-437): returns 1 when a force acts, f = force on p1
   (p2 takes f * -1.0); broke = 1 when this evaluation breaks an HR_FL
   spring (kernel.cl:391-397). */
__device__ __forceinline__ int spring_eval(const StepArgs& A, int s, double& fx, double& fy,
                                           double& fz, int& broke) {
    broke = 0;
    const int type = A.sp_type[s];
    if (!(type == 0 || type == 1)) return 0;
    if (A.sp_status[s] != 1) return 0;
    const int2 e = A.sp_ends[s];
    const double4 a = A.img_in[e.x];
    const double4 b = A.img_in[e.y];
    return spring_pts(a.x, a.y, a.z, b.x, b.y, b.z, A.sp_par[s], type, fx, fy, fz, broke);
}

/* The spring force of kernel.cl:377-424 from the image positions of p1 (a)
   and p2 (b); shared by the incidence and chain kernels. */
__device__ __forceinline__ int spring_pts(double ax, double ay, double az, double bx, double by,
                                          double bz, float4 par, int type, double& fx, double& fy,
                                          double& fz, int& broke) {
    broke = 0;
    double dx = ax - bx, dy = ay - by, dz = az - bz;
    double l = sqrt(dx * dx + dy * dy + dz * dz);
    double factor = (double)par.x - l;
    if (l != 0.0) l = 1.0 / l;
    dx *= l;
    dy *= l;
    dz *= l;
    if (type == 1) {
        double stress = -(double)par.z * factor * l;
        if (fabs(stress) > (double)par.w) {
            broke = 1;
            return 0;
        }
    }
    factor *= (double)par.y;
    fx = dx * factor;
    fy = dy * factor;
    fz = dz * factor;
    return 1;
}

__device__ __forceinline__ int spring_alive_after(const StepArgs& A, int s) {
    if (A.sp_status[s] != 1) return 0;
    double fx, fy, fz;
    int broke;
    spring_eval(A, s, fx, fy, fz, broke);
    return !broke;
}

/* Angle force (kernel.cl:291-348) from the image positions of b1 (t1),
   b2 (t2), b3 (t3): pa acts on b1, pc on b3. */
__device__ __forceinline__ void angle_pts(double t1x, double t1y, double t1z, double t2x,
                                          double t2y, double t2z, double t3x, double t3y,
                                          double t3z, float2 par, double& pax, double& pay,
                                          double& paz, double& pcx, double& pcy, double& pcz) {
    const double bax = t1x - t2x, bay = t1y - t2y, baz = t1z - t2z;
    const double bcx = t3x - t2x, bcy = t3y - t2y, bcz = t3z - t2z;
    const double cbx = bcx * -1.0, cby = bcy * -1.0, cbz = bcz * -1.0;
    const double l_ba = sqrt(bax * bax + bay * bay + baz * baz);
    const double l_bc = sqrt(bcx * bcx + bcy * bcy + bcz * bcz);
    double dotp = (bax * bcx + bay * bcy + baz * bcz) / (l_ba * l_bc);
    if (dotp < -1.0) dotp = -0.999999;
    if (dotp > 1.0) dotp = 0.999999;
    const double angle = fn_acos(dotp);
    const double magnitude = -2.0 * (double)par.y * (angle - (double)par.x);
    const double fa = magnitude / l_ba;
    const double fc = magnitude / l_bc;
    const double tx = bay * bcz - baz * bcy;
    const double ty = baz * bcx - bax * bcz;
    const double tz = bax * bcy - bay * bcx;
    pax = (bay * tz - baz * ty);
    pay = (baz * tx - bax * tz);
    paz = (bax * ty - bay * tx);
    double ln = sqrt(pax * pax + pay * pay + paz * paz);
    if (ln != 0.0) ln = 1.0 / ln;
    ln *= fa;
    pax *= ln;
    pay *= ln;
    paz *= ln;
    pcx = (cby * tz - cbz * ty);
    pcy = (cbz * tx - cbx * tz);
    pcz = (cbx * ty - cby * tx);
    ln = sqrt(pcx * pcx + pcy * pcy + pcz * pcz);
    if (ln != 0.0) ln = 1.0 / ln;
    ln *= fc;
    pcx *= ln;
    pcy *= ln;
    pcz *= ln;
}

__device__ __forceinline__ void angle_eval(const StepArgs& A, int4 b, float2 par, double& pax,
                                           double& pay, double& paz, double& pcx, double& pcy,
                                           double& pcz) {
    const double4 t2 = A.img_in[b.y];
    const double4 t1 = A.img_in[b.x];
    const double4 t3 = A.img_in[b.z];
    angle_pts(t1.x, t1.y, t1.z, t2.x, t2.y, t2.z, t3.x, t3.y, t3.z, par, pax, pay, paz, pcx, pcy,
              pcz);
}

/* One contact-list entry (kernel.cl:835-999): force on bead i. */
__device__ __forceinline__ int contact_eval(const FnNet& N, const FnPair* __restrict__ pairs,
                                            double4 pi, double4 pj, double& Rx, double& Ry,
                                            double& Rz) {
    double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
    double length = rx * rx + ry * ry + rz * rz;
    length = min_image(N, rx, ry, rz, length, N.force_mi);
    const int pid = N.pair_base + getadress(w_type(pi.w), w_type(pj.w), N.types_num);
    const FnPair* P = pairs + pid;
    const int kind = P->kind;
    if (kind == 1) {
        if (length < N.cutoff_sq) {
            const double r2 = length;
            length = sqrt(length);
            if (length < P->c[2]) {
                double sigma2 = P->c[0];
                const double epsilon = P->c[1];
                sigma2 *= sigma2;
                const double fr2 = sigma2 / r2;
                const double fr6 = fr2 * fr2 * fr2;
                double fpr = 48.0 * epsilon * fr6 * (fr6 - 0.5) / r2;
                fpr -= P->c[3];
                length = (length != 0.0) ? 1.0 / length : 0.0;
                Rx = fpr * (rx * length);
                Ry = fpr * (ry * length);
                Rz = fpr * (rz * length);
                return 1;
            }
        }
        return 0;
    }
    if (kind == 2) {
        length = sqrt(length);
        const double K = P->c[0];
        double penetration = ((double)w_radius(pi.w) + (double)w_radius(pj.w)) - length;
        if (penetration > 0.0) {
            length = (length != 0.0) ? 1.0 / length : 0.0;
            penetration *= K;
            Rx = penetration * (rx * length);
            Ry = penetration * (ry * length);
            Rz = penetration * (rz * length);
            return 1;
        }
        return 0;
    }
    if (kind == 4) {
        /* extension, no counterpart in the reference: penalty spring K (c1)
           on the overlap plus a soft harmonic repulsion k (c2) below rc (c3) */
        length = sqrt(length);
        const double penetration = ((double)w_radius(pi.w) + (double)w_radius(pj.w)) - length;
        double mag = 0.0;
        int acts = 0;
        if (penetration > 0.0) {
            mag += penetration * P->c[0];
            acts = 1;
        }
        if (length < P->c[2]) {
            mag += (P->c[2] - length) * P->c[1];
            acts = 1;
        }
        if (acts) {
            length = (length != 0.0) ? 1.0 / length : 0.0;
            Rx = mag * (rx * length);
            Ry = mag * (ry * length);
            Rz = mag * (rz * length);
        }
        return acts;
    }
    if (kind == 3) {
        if (length < P->c[3]) {
            length = sqrt(length);
            double factor = (P->c[1] - length);
            factor *= P->c[0]; /* both arms of kernel.cl:970-973 multiply by K */
            factor += (P->c[5] - length) * P->c[4];
            length = (length != 0.0) ? 1.0 / length : 0.0;
            Rx = factor * (rx * length);
            Ry = factor * (ry * length);
            Rz = factor * (rz * length);
            return 1;
        }
        return 0;
    }
    return 0;
}

/* AdvancePosition (kernel.cl:200-250) on registers: returns the drifted
   position/image, the predicted velocity. */
__device__ __forceinline__ void drift(const FnNet& N, double minv, float fx, float fy, float fz,
                                      float vox, float voy, float voz, double4& p, double4& im,
                                      float4& v) {
    const double lambda_dt = N.lambda_dt * minv;
    const double half_dt2 = N.half_dt2 * minv;
    v.x = (float)((double)fx * lambda_dt + (double)vox);
    v.y = (float)((double)fy * lambda_dt + (double)voy);
    v.z = (float)((double)fz * lambda_dt + (double)voz);
    v.w = 0.0f;
    double ix = (double)vox, iy = (double)voy, iz = (double)voz;
    ix *= N.dt;
    iy *= N.dt;
    iz *= N.dt;
    ix = (double)fx * half_dt2 + ix;
    iy = (double)fy * half_dt2 + iy;
    iz = (double)fz * half_dt2 + iz;
    p.x += ix;
    p.y += iy;
    p.z += iz;
    im.x += ix;
    im.y += iy;
    im.z += iz;
    /* snap wrap, kernel.cl:241-250 */
    if (N.periodic & 4)
        if (p.z < 0.0) p.z = N.box[2];
    if (N.periodic & 2)
        if (p.y < 0.0) p.y = N.box[1];
    if (N.periodic & 1)
        if (p.x < 0.0) p.x = N.box[0];
    if (N.periodic & 4)
        if (p.z > N.box[2]) p.z = 0.0;
    if (N.periodic & 2)
        if (p.y > N.box[1]) p.y = 0.0;
    if (N.periodic & 1)
        if (p.x > N.box[0]) p.x = 0.0;
}

/* Base force of AdvancePosition: damping * v + gravity, then the wall
   penalty at the drifted position (kernel.cl:231-261). */
template <bool DAMP>
__device__ __forceinline__ void base_force(const StepArgs& A, const FnNet& N, int i, double4 p,
                                           double& Fx, double& Fy, double& Fz) {
    if (DAMP) {
        const float4 v = A.vel[i];
        Fx = N.damping * (double)v.x;
        Fy = N.damping * (double)v.y;
        Fz = N.damping * (double)v.z;
    } else {
        Fx = 0.0;
        Fy = 0.0;
        Fz = 0.0;
    }
    Fx += N.g[0];
    Fy += N.g[1];
    Fz += N.g[2];
    if (N.walls) {
        if ((N.walls & 4) && p.z < 0.0) Fz += p.z * N.wall_k * -1.0;
        if ((N.walls & 2) && p.y < 0.0) Fy += p.y * N.wall_k * -1.0;
        if ((N.walls & 1) && p.x < 0.0) Fx += p.x * N.wall_k * -1.0;
        if ((N.walls & 4) && p.z > N.box[2]) Fz += (p.z - N.box[2]) * N.wall_k * -1.0;
        if ((N.walls & 2) && p.y > N.box[1]) Fy += (p.y - N.box[1]) * N.wall_k * -1.0;
        if ((N.walls & 1) && p.x > N.box[0]) Fx += (p.x - N.box[0]) * N.wall_k * -1.0;
    }
}

/* Contacts, AdvanceVelocity and the next step's AdvancePosition for bead i,
   given its base + bonded force (Fx, Fy, Fz) in FP64. */
template <bool DAMP, bool DRIFT, bool STORE_V>
__device__ __forceinline__ void kick_drift_store(const StepArgs& A, const FnNet& N, int i,
                                                 double4 p, double Fx, double Fy, double Fz);

template <bool DAMP, bool DRIFT, bool STORE_V>
__device__ __forceinline__ void finish_bead(const StepArgs& A, const FnNet& N, int i, double4 p,
                                            double Fx, double Fy, double Fz) {
    /* contacts */
    int n = A.list_count[i];
    if (n > A.list_cap) n = A.list_cap;
    const int* __restrict__ lst = A.list + i;
    for (int k = 0; k < n; ++k) {
        const int j = lst[(size_t)k * A.list_stride];
        double Rx, Ry, Rz;
        if (contact_eval(N, A.pairs, p, A.pos_in[j], Rx, Ry, Rz)) {
            Fx += Rx;
            Fy += Ry;
            Fz += Rz;
        }
    }
    kick_drift_store<DAMP, DRIFT, STORE_V>(A, N, i, p, Fx, Fy, Fz);
}

/* AdvanceVelocity and the next AdvancePosition for bead i with its complete
   force (Fx, Fy, Fz), then the stores. */
template <bool DAMP, bool DRIFT, bool STORE_V>
__device__ __forceinline__ void kick_drift_store(const StepArgs& A, const FnNet& N, int i,
                                                 double4 p, double Fx, double Fy, double Fz) {
    const float fx = (float)Fx, fy = (float)Fy, fz = (float)Fz;
    if (!(isfinite(fx) && isfinite(fy) && isfinite(fz)))
        atomicAdd(A.counters + FN_CNT_NONFINITE, 1ull);

    /* AdvanceVelocity, kernel.cl:451-462 */
    double4 im = A.img_in[i];
    const double minv = im.w;
    const double half_dt = N.half_dt * minv;
    const float4 fo = A.force[i];
    const float4 vo = A.vold[i];
    double tx = (double)fx, ty = (double)fy, tz = (double)fz;
    tx += (double)fo.x;
    ty += (double)fo.y;
    tz += (double)fo.z;
    const float vox = (float)(tx * half_dt + (double)vo.x);
    const float voy = (float)(ty * half_dt + (double)vo.y);
    const float voz = (float)(tz * half_dt + (double)vo.z);
    A.force[i] = make_float4(fx, fy, fz, 0.0f);
    A.vold[i] = make_float4(vox, voy, voz, 0.0f);

    if (DRIFT) {
        float4 v;
        drift(N, minv, fx, fy, fz, vox, voy, voz, p, im, v);
        A.pos_out[i] = p;
        A.img_out[i] = im;
        if (DAMP || STORE_V) A.vel[i] = v;
    }
}

template <bool DAMP, bool DRIFT, bool STORE_V>
__global__ void __launch_bounds__(512) k_step(const StepArgs A) {
    const FnTile t = A.tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    if (i >= t.end) return;
    const FnNet& N = A.nets[t.net];

    const double4 p = A.pos_in[i];
    double Fx, Fy, Fz;
    base_force<DAMP>(A, N, i, p, Fx, Fy, Fz);

    /* springs */
    const int se = A.sp_off[i + 1];
    for (int e = A.sp_off[i]; e < se; ++e) {
        const int ent = A.sp_ent[e];
        const int s = ent >> 1;
        double fx, fy, fz;
        int broke;
        if (spring_eval(A, s, fx, fy, fz, broke)) {
            if ((ent & 1) == 0) {
                Fx += fx;
                Fy += fy;
                Fz += fz;
            } else {
                Fx += fx * -1.0;
                Fy += fy * -1.0;
                Fz += fz * -1.0;
            }
        }
        if (broke && (ent & 1) == 0) A.sp_status[s] = 0;
    }

    /* angles */
    const int ae = A.an_off[i + 1];
    for (int e = A.an_off[i]; e < ae; ++e) {
        const int ent = A.an_ent[e];
        const int a = ent >> 2;
        const int role = ent & 3;
        if (A.an_status[a] != 1) continue;
        const int4 b = A.an_b[a];
        if (b.w == 1) {
            const int2 ss = A.an_s[a];
            if (!spring_alive_after(A, ss.x) || !spring_alive_after(A, ss.y)) {
                if (role == 1) A.an_status[a] = 0;
                continue;
            }
        }
        double pax, pay, paz, pcx, pcy, pcz;
        angle_eval(A, b, A.an_par[a], pax, pay, paz, pcx, pcy, pcz);
        if (role == 0) {
            Fx += pax;
            Fy += pay;
            Fz += paz;
        } else if (role == 2) {
            Fx += pcx;
            Fy += pcy;
            Fz += pcz;
        } else {
            Fx += -pax - pcx;
            Fy += -pay - pcy;
            Fz += -paz - pcz;
        }
    }

    finish_bead<DAMP, DRIFT, STORE_V>(A, N, i, p, Fx, Fy, Fz);
}

/* The same step with the bonded terms evaluated once per tile: the block
   first evaluates every spring, then every angle incident to its beads into
   shared memory (flag bits: 1 force acts, 2 broke this step, 4 alive at step
   start), then each thread gathers its bead's terms from the shared slots in
   the same order as k_step, so the result is bit-identical to k_step. */
template <bool DAMP, bool DRIFT, bool STORE_V>
__global__ void __launch_bounds__(512) k_step_tiled(const StepArgs A) {
    extern __shared__ double smem[];
    const int t = blockIdx.x;
    const FnTile tile = A.tiles[t];
    double* sp_f = smem;
    double* an_f = sp_f + 3 * A.max_tile_sp;
    unsigned char* sp_flag = reinterpret_cast<unsigned char*>(an_f + 6 * A.max_tile_an);
    unsigned char* an_flag = sp_flag + A.max_tile_sp;

    const int sp0 = A.tile_sp_off[t], nsp = A.tile_sp_off[t + 1] - sp0;
    for (int q = threadIdx.x; q < nsp; q += blockDim.x) {
        const int s = A.tile_sp[sp0 + q];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        int broke;
        const int alive0 = A.sp_status[s] == 1;
        const int acts = spring_eval(A, s, fx, fy, fz, broke);
        sp_f[3 * q] = fx;
        sp_f[3 * q + 1] = fy;
        sp_f[3 * q + 2] = fz;
        sp_flag[q] = (unsigned char)(acts | (broke << 1) | (alive0 << 2));
        if (broke) A.sp_status[s] = 0;
    }
    __syncthreads();
    const int an0 = A.tile_an_off[t], nan = A.tile_an_off[t + 1] - an0;
    for (int q = threadIdx.x; q < nan; q += blockDim.x) {
        const int a = A.tile_an[an0 + q];
        int alive = A.an_status[a] == 1;
        const int4 b = A.an_b[a];
        if (alive && b.w == 1) {
            const int2 ss = A.tile_an_sslot[an0 + q];
            const unsigned f1 = sp_flag[ss.x], f2 = sp_flag[ss.y];
            const int ok1 = (f1 & 4) && !(f1 & 2);
            const int ok2 = (f2 & 4) && !(f2 & 2);
            if (!ok1 || !ok2) {
                alive = 0;
                A.an_status[a] = 0;
            }
        }
        an_flag[q] = (unsigned char)alive;
        if (alive) {
            double* o = an_f + 6 * q;
            angle_eval(A, b, A.an_par[a], o[0], o[1], o[2], o[3], o[4], o[5]);
        }
    }
    __syncthreads();

    const int i = tile.begin + (int)threadIdx.x;
    if (i >= tile.end) return;
    const FnNet& N = A.nets[tile.net];
    const double4 p = A.pos_in[i];
    double Fx, Fy, Fz;
    base_force<DAMP>(A, N, i, p, Fx, Fy, Fz);
    const int se = A.sp_off[i + 1];
    for (int e = A.sp_off[i]; e < se; ++e) {
        const int ent = A.sp_slot[e];
        const int q = ent >> 1;
        if (sp_flag[q] & 1) {
            const double* f = sp_f + 3 * q;
            if ((ent & 1) == 0) {
                Fx += f[0];
                Fy += f[1];
                Fz += f[2];
            } else {
                Fx += f[0] * -1.0;
                Fy += f[1] * -1.0;
                Fz += f[2] * -1.0;
            }
        }
    }
    const int ae = A.an_off[i + 1];
    for (int e = A.an_off[i]; e < ae; ++e) {
        const int ent = A.an_slot[e];
        const int q = ent >> 2;
        const int role = ent & 3;
        if (!an_flag[q]) continue;
        const double* o = an_f + 6 * q;
        if (role == 0) {
            Fx += o[0];
            Fy += o[1];
            Fz += o[2];
        } else if (role == 2) {
            Fx += o[3];
            Fy += o[4];
            Fz += o[5];
        } else {
            Fx += -o[0] - o[3];
            Fy += -o[1] - o[4];
            Fz += -o[2] - o[5];
        }
    }
    finish_bead<DAMP, DRIFT, STORE_V>(A, N, i, p, Fx, Fy, Fz);
}

/* Exclusive prefix sum of v over the block (any size up to 1024); total
   receives the block sum.  warp_sums needs 33 ints. */
__device__ __forceinline__ int block_scan_any(int v, int* warp_sums, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < nwarps ? warp_sums[lane] : 0;
        int sacc = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, sacc, o);
            if (lane >= o) sacc += y;
        }
        warp_sums[lane] = sacc - w;
        if (lane == 31) warp_sums[32] = sacc;
    }
    __syncthreads();
    total = warp_sums[32];
    const int r = x - v + warp_sums[warp];
    __syncthreads();
    return r;
}

/* Step kernel for networks in chain form (every spring joins consecutive
   beads j, j+1 and every angle is centred on its middle bead, as fibres
   are).  The block stages the image positions of its beads plus two halo
   beads on each side in shared memory, evaluates every spring and angle
   touching its beads once (springs first: an HR_FL angle dies with either of
   its springs in the same step, kernel.cl:274-286), then each thread adds its
   bead's terms in ascending bond order -- previous spring, next spring,
   angles centred on j-1, j, j+1 -- which is the order of the incidence path,
   so both produce identical bits.  Statuses are written back by the owning
   thread.  FORCES_ONLY evaluates the selected terms alone (no base force, no
   kick or drift, no status change). */
template <bool DAMP, bool DRIFT, bool STORE_V, bool FORCES_ONLY>
/* At most 256 threads per block and 4 such blocks per SM, i.e. at most 64
   registers: the kernel waits on dependent loads of contact partners, and
   both resident warps and the registers that keep the next list index in
   flight hide that latency (measured on the 1M-bead tensile network: 0.135 ms
   per step at 64 registers, 0.144 ms at 48 registers, 0.154 ms at 76). */
__global__ void __launch_bounds__(kChainMaxBlock, 4) k_step_chain(const StepArgs A, int terms) {
    extern __shared__ __align__(32) unsigned char smem_raw[];
    const FnTile tile = A.tiles[blockIdx.x];
    const int b0 = tile.begin, n = tile.end - tile.begin;
    const ChainSmem L = chain_smem_layout(blockDim.x);
    double* s_img = reinterpret_cast<double*>(smem_raw + L.img);  /* slot u <-> bead b0 - 2 + u */
    double* s_spf = reinterpret_cast<double*>(smem_raw + L.spf);  /* lower bead b0 - 2 + u */
    double* s_ang = reinterpret_cast<double*>(smem_raw + L.ang);  /* centre bead b0 - 1 + u */
    unsigned char* s_flag = smem_raw + L.flag;
    unsigned char* s_stat = smem_raw + L.stat;
    unsigned char* s_tsp = smem_raw + L.tsp; /* spring term: 1 acts, 2 broke, 4 alive at start */
    unsigned char* s_tan = smem_raw + L.tan; /* angle term alive */
    const int tid = threadIdx.x;

    for (int u = tid; u < n + 4; u += blockDim.x) {
        const int j = b0 - 2 + u;
        unsigned char fl = 0, st = 0;
        if (j >= 0 && j < A.nb) {
            const double4 q = A.img_in[j];
            s_img[3 * u] = q.x;
            s_img[3 * u + 1] = q.y;
            s_img[3 * u + 2] = q.z;
            fl = A.ch_flags[j];
            st = A.ch_status[j];
        }
        s_flag[u] = fl;
        s_stat[u] = st;
    }
    __syncthreads();

    const bool want_sp = !FORCES_ONLY || (terms & 1);
    const bool want_an = !FORCES_ONLY || (terms & 2);
    for (int u = tid; u < n + 3; u += blockDim.x) {
        const unsigned fl = s_flag[u];
        unsigned char tf = 0;
        if (fl & FN_CH_SPRING) {
            const int alive0 = s_stat[u] & 1;
            tf = (unsigned char)(alive0 << 2);
            if (alive0 && !(fl & FN_CH_SP_INERT)) {
                const int j = b0 - 2 + u;
                const float4 par = A.ch_sp[j];
                const double* a = s_img + 3 * ((fl & FN_CH_SP_REV) ? u + 1 : u);
                const double* b = s_img + 3 * ((fl & FN_CH_SP_REV) ? u : u + 1);
                double fx = 0.0, fy = 0.0, fz = 0.0;
                int broke;
                const int acts = spring_pts(a[0], a[1], a[2], b[0], b[1], b[2], par,
                                            (fl & FN_CH_SP_FL) ? 1 : 0, fx, fy, fz, broke);
                s_spf[3 * u] = fx;
                s_spf[3 * u + 1] = fy;
                s_spf[3 * u + 2] = fz;
                tf |= (unsigned char)(acts | (broke << 1));
            }
        }
        s_tsp[u] = tf;
    }
    __syncthreads();

    for (int u = tid; u < n + 2; u += blockDim.x) {
        const unsigned fl = s_flag[u + 1];
        int alive = (fl & FN_CH_ANGLE) && (s_stat[u + 1] & 2);
        if (alive && (fl & FN_CH_AN_FL)) {
            const unsigned f1 = s_tsp[u], f2 = s_tsp[u + 1];
            if (!((f1 & 4) && !(f1 & 2)) || !((f2 & 4) && !(f2 & 2))) alive = 0;
        }
        s_tan[u] = (unsigned char)alive;
        if (alive && want_an) {
            const int j = b0 - 1 + u;
            const double* t1 = s_img + 3 * ((fl & FN_CH_AN_REV) ? u + 2 : u);
            const double* t2 = s_img + 3 * (u + 1);
            const double* t3 = s_img + 3 * ((fl & FN_CH_AN_REV) ? u : u + 2);
            double* o = s_ang + 6 * u;
            angle_pts(t1[0], t1[1], t1[2], t2[0], t2[1], t2[2], t3[0], t3[1], t3[2], A.ch_an[j],
                      o[0], o[1], o[2], o[3], o[4], o[5]);
        }
    }
    __syncthreads();

    const bool active = tid < n;
    const int i = b0 + tid;
    const FnNet& N = A.nets[tile.net];
    double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    int nc = 0;
    if (active) {
        p = A.pos_in[i];
        if (!FORCES_ONLY) base_force<DAMP>(A, N, i, p, Fx, Fy, Fz);
        if (want_sp) {
            /* spring (i-1, i): bead i is p1 when the spring is reversed */
            const unsigned fp = s_flag[tid + 1];
            if ((fp & FN_CH_SPRING) && (s_tsp[tid + 1] & 1)) {
                const double* f = s_spf + 3 * (tid + 1);
                if (fp & FN_CH_SP_REV) {
                    Fx += f[0];
                    Fy += f[1];
                    Fz += f[2];
                } else {
                    Fx += f[0] * -1.0;
                    Fy += f[1] * -1.0;
                    Fz += f[2] * -1.0;
                }
            }
            /* spring (i, i+1): bead i is p1 unless reversed */
            const unsigned fn = s_flag[tid + 2];
            if ((fn & FN_CH_SPRING) && (s_tsp[tid + 2] & 1)) {
                const double* f = s_spf + 3 * (tid + 2);
                if (fn & FN_CH_SP_REV) {
                    Fx += f[0] * -1.0;
                    Fy += f[1] * -1.0;
                    Fz += f[2] * -1.0;
                } else {
                    Fx += f[0];
                    Fy += f[1];
                    Fz += f[2];
                }
            }
        }
        if (want_an) {
            /* centred on i-1: bead i is b3, or b1 when reversed */
            if (s_tan[tid]) {
                const double* o = s_ang + 6 * tid;
                const int k = (s_flag[tid + 1] & FN_CH_AN_REV) ? 0 : 3;
                Fx += o[k];
                Fy += o[k + 1];
                Fz += o[k + 2];
            }
            /* centred on i: bead i is b2 */
            if (s_tan[tid + 1]) {
                const double* o = s_ang + 6 * (tid + 1);
                Fx += -o[0] - o[3];
                Fy += -o[1] - o[4];
                Fz += -o[2] - o[5];
            }
            /* centred on i+1: bead i is b1, or b3 when reversed */
            if (s_tan[tid + 2]) {
                const double* o = s_ang + 6 * (tid + 2);
                const int k = (s_flag[tid + 3] & FN_CH_AN_REV) ? 3 : 0;
                Fx += o[k];
                Fy += o[k + 1];
                Fz += o[k + 2];
            }
        }
        if (!FORCES_ONLY || (terms & 4)) {
            nc = A.list_count[i];
            if (nc > A.list_cap) nc = A.list_cap;
        }
    }

    /* contacts, load-balanced inside each warp: after a direct phase over the
       leading items of every list, the remaining items are taken 32 at a
       time, lane l evaluating item (window base + l); a 32-byte map tells each
       lane whose item it holds, results go to shared memory and every bead
       then adds its own items in list order (the order of a sequential loop
       over its list, so the sums are identical).  Only warp barriers are
       involved. */
    {
        const int lane = tid & 31, wid = tid >> 5;
        unsigned char* s_map = smem_raw + L.wmap + 32 * (size_t)wid;
        double* s_R = reinterpret_cast<double*>(smem_raw + L.wres) + 3 * 32 * (size_t)wid;
        unsigned char* s_Rf = smem_raw + L.wresf + 32 * (size_t)wid;
        const double4* s_pos = reinterpret_cast<const double4*>(smem_raw + L.pos);
        double4* s_pos_w = reinterpret_cast<double4*>(smem_raw + L.pos);
        if (active) s_pos_w[tid] = p;
        /* direct phase: every lane first evaluates the leading KD items of its
           own list, one list row per iteration (coalesced loads, no window
           bookkeeping); the longer lists' tails then go through the windows.
           KD is picked per warp among mean - 1 .. mean + 2 (mean rounded
           down) to minimise 2 x KD + 3 x windows, a window costing about 1.5
           direct iterations. */
        int kd;
        {
            const int m = __reduce_add_sync(0xffffffffu, nc) >> 5;
            kd = m;
            int best = 2 * m + 3 * ((__reduce_add_sync(0xffffffffu, max(nc - m, 0)) + 31) >> 5);
            for (int k = max(m - 1, 0); k <= m + 2; ++k) {
                if (k == m) continue;
                const int c = 2 * k + 3 * ((__reduce_add_sync(0xffffffffu, max(nc - k, 0)) + 31) >> 5);
                if (c < best) {
                    best = c;
                    kd = k;
                }
            }
        }
        const int nd = min(nc, kd);
        const int nr = nc - nd; /* items left for the windows */
        int off = nr;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += y;
        }
        const int total = __shfl_sync(0xffffffffu, off, 31);
        off -= nr; /* exclusive */
        /* owner lane and list index of the first window's items, loaded
           before the direct phase so their latency overlaps it */
        int b_first = 0, j_first = 0;
        if (total > 0) {
            const int lim = min(32, total);
            for (int w = off; w < min(off + nr, lim); ++w) s_map[w] = (unsigned char)lane;
            __syncwarp();
            b_first = lane < lim ? s_map[lane] : 0;
            const int ob = __shfl_sync(0xffffffffu, off - nd, b_first);
            if (lane < lim)
                j_first = A.list[(size_t)(lane - ob) * A.list_stride + (b0 + (tid & ~31) + b_first)];
        }
        int jn = nd > 0 ? A.list[i] : 0; /* next list index, loaded one item ahead */
        for (int k = 0; k < kd; ++k) {
            if (k < nd) {
                const int j = jn;
                if (k + 1 < nd) jn = A.list[(size_t)(k + 1) * A.list_stride + i];
                double Rx = 0.0, Ry = 0.0, Rz = 0.0;
                if (contact_eval(N, A.pairs, p, A.pos_in[j], Rx, Ry, Rz)) {
                    Fx += Rx;
                    Fy += Ry;
                    Fz += Rz;
                }
            }
        }
        for (int base = 0; base < total; base += 32) {
            const int lim = min(base + 32, total);
            const int w = base + lane;
            int b = b_first, j = j_first;
            if (base > 0) {
                for (int q = max(off, base); q < min(off + nr, lim); ++q) s_map[q - base] = (unsigned char)lane;
                __syncwarp();
                b = w < lim ? s_map[lane] : 0;
                const int ob = __shfl_sync(0xffffffffu, off - nd, b); /* list row = w - ob */
                if (w < lim) j = A.list[(size_t)(w - ob) * A.list_stride + (b0 + (tid & ~31) + b)];
            }
            if (w < lim) {
                const int ib = (tid & ~31) + b; /* block-local bead of the item */
                double Rx = 0.0, Ry = 0.0, Rz = 0.0;
                const int acts = contact_eval(N, A.pairs, s_pos[ib], A.pos_in[j], Rx, Ry, Rz);
                s_R[3 * lane] = Rx;
                s_R[3 * lane + 1] = Ry;
                s_R[3 * lane + 2] = Rz;
                s_Rf[lane] = (unsigned char)acts;
            }
            __syncwarp();
            for (int q = max(off, base); q < min(off + nr, lim); ++q) {
                if (s_Rf[q - base]) {
                    Fx += s_R[3 * (q - base)];
                    Fy += s_R[3 * (q - base) + 1];
                    Fz += s_R[3 * (q - base) + 2];
                }
            }
            __syncwarp();
        }
    }
    if (!active) return;
    if (FORCES_ONLY) {
        A.force[i] = make_float4((float)Fx, (float)Fy, (float)Fz, 0.0f);
        return;
    }
    /* statuses after this step (kernel.cl:396-397, 278-284) */
    const unsigned st0 = s_stat[tid + 2];
    unsigned st = st0;
    if ((s_tsp[tid + 2] & 2)) st &= ~1u;
    if ((st0 & 2) && (s_flag[tid + 2] & FN_CH_ANGLE) && !s_tan[tid + 1]) st &= ~2u;
    if (st != st0) A.ch_status[i] = (unsigned char)st;
    kick_drift_store<DAMP, DRIFT, STORE_V>(A, N, i, p, Fx, Fy, Fz);
}

/* ------------------------------------------------------------------------ */
/* Staged chain step kernel                                                  */

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* mbarrier + bulk-copy (TMA, non-tensor) primitives for one CTA */
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
/* Waits for phase `parity` of the barrier for at most ~2 s of SM clock;
   false when the wait ran out. */
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > 4000000000LL) return false;
    return true;
}
/* bytes (a multiple of 16) from global src to shared dst, both 16-byte
   aligned, completing on the barrier */
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
/* 16 bytes global -> shared through L2 (LDGSTS) */
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_all;" ::: "memory");
}

/* Issues the partner-position copies of contact items [c0, c0 + nch) of the
   tile: item q's partner j (tile-compacted list) -> pj slot q - c0.  The
   entries are loaded first, all at once, so their latency is paid once. */
__device__ __forceinline__ void gather_partners(const StepArgs& A, const int* __restrict__ ent, int c0,
                                                int nch, unsigned char* s_pj) {
    int j[kStagedMaxItemsPerThread];
#pragma unroll
    for (int k = 0; k < kStagedMaxItemsPerThread; ++k) {
        const int q = (int)threadIdx.x + k * (int)blockDim.x;
        j[k] = q < nch ? ent[c0 + q] : -1;
    }
#pragma unroll
    for (int k = 0; k < kStagedMaxItemsPerThread; ++k) {
        const int q = (int)threadIdx.x + k * (int)blockDim.x;
        if ((unsigned)j[k] < (unsigned)A.nb) {
            const double4* src = A.pos_in + j[k];
            const uint32_t dst = smem_addr(s_pj + 32 * (size_t)q);
            cp_async16(dst, src);
            cp_async16(dst + 16, reinterpret_cast<const char*>(src) + 16);
        }
    }
}

/* The chain step (same arithmetic and summation order as k_step_chain, so
   the same bits) with the tile's data staged in shared memory before any of
   it is used, instead of a chain of dependent loads:
     - one thread issues bulk copies (cp.async.bulk, completing on an
       mbarrier) of the image positions (with a two-bead halo each side),
       positions, forces, velocities_old and spring records of the tile;
     - meanwhile every thread loads the tile's contact entries (a contiguous
       run of the tile-compacted list) and copies each partner's position
       into shared memory (cp.async), and the byte-sized flags, statuses,
       angle records and list lengths with plain loads;
     - then springs and angles are evaluated once per tile, every contact
       item is evaluated by some thread of the block (items spread evenly over
       the threads, results kept per item), and each thread sums its bead's
       terms in the fixed order: base, previous and next spring, angles
       centred on j-1, j, j+1, contacts in list order.
   Tiles with more contact items than `chunk` take them in rounds. */
template <bool DAMP, bool DRIFT, bool STORE_V>
__global__ void __launch_bounds__(kChainMaxBlock) k_step_staged(const StepArgs A) {
    extern __shared__ __align__(128) unsigned char sm[];
    const StagedSmem L = staged_smem_layout(blockDim.x, A.chunk);
    const FnTile tile = A.tiles[blockIdx.x];
    const int items = A.tile_items[blockIdx.x];
    const int b0 = tile.begin, n = tile.end - tile.begin;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int* __restrict__ ent = A.csr + (size_t)blockIdx.x * (size_t)A.csr_region;
    const uint32_t bar = smem_addr(sm + L.bar);
    const int j0 = max(b0 - 2, 0), j1 = min(b0 + n + 2, A.nb), js1 = min(b0 + n + 1, A.nb);
    double* s_spf = reinterpret_cast<double*>(sm + L.spf);
    double* s_ang = reinterpret_cast<double*>(sm + L.ang);
    const double4* s_img = reinterpret_cast<const double4*>(sm + L.img);
    const double4* s_pos = reinterpret_cast<const double4*>(sm + L.pos);
    const float4* s_frc = reinterpret_cast<const float4*>(sm + L.frc);
    const float4* s_vold = reinterpret_cast<const float4*>(sm + L.vold);
    const float4* s_chsp = reinterpret_cast<const float4*>(sm + L.chsp);
    float2* s_chan = reinterpret_cast<float2*>(sm + L.chan);
    unsigned char* s_pj = sm + L.pj;
    int* s_off = reinterpret_cast<int*>(sm + L.off);
    int* s_ws = reinterpret_cast<int*>(sm + L.ws);
    unsigned char* s_owner = sm + L.owner;
    unsigned char* s_flag = sm + L.flag;
    unsigned char* s_stat = sm + L.stat;
    unsigned char* s_tsp = sm + L.tsp;
    unsigned char* s_tan = sm + L.tan;

    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = 32u * (uint32_t)(j1 - j0) + 32u * (uint32_t)n + 32u * (uint32_t)n +
                               16u * (uint32_t)(js1 - j0);
        mbar_expect_tx(bar, bytes);
        bulk_g2s(smem_addr(sm + L.img) + 32u * (uint32_t)(j0 - (b0 - 2)), A.img_in + j0, 32u * (j1 - j0), bar);
        bulk_g2s(smem_addr(sm + L.pos), A.pos_in + b0, 32u * n, bar);
        bulk_g2s(smem_addr(sm + L.frc), A.force + b0, 16u * n, bar);
        bulk_g2s(smem_addr(sm + L.vold), A.vold + b0, 16u * n, bar);
        bulk_g2s(smem_addr(sm + L.chsp) + 16u * (uint32_t)(j0 - (b0 - 2)), A.ch_sp + j0, 16u * (js1 - j0), bar);
    }
    /* the first round's contact partners, while the bulk copies run */
    const int nch0 = min(items, A.chunk);
    gather_partners(A, ent, 0, nch0, s_pj);
    /* byte-sized and 8-byte arrays, list length */
    const bool active = tid < n;
    const int i = b0 + tid;
    int nc = 0;
    if (active) {
        nc = A.list_count[i];
        if (nc > A.list_cap) nc = A.list_cap;
    }
    for (int u = tid; u < n + 4; u += nt) {
        const int j = b0 - 2 + u;
        unsigned char fl = 0, st = 0;
        if (j >= 0 && j < A.nb) {
            fl = A.ch_flags[j];
            st = A.ch_status[j];
        }
        s_flag[u] = fl;
        s_stat[u] = st;
        if (u < n + 2) {
            const int ja = b0 - 1 + u;
            s_chan[u] = (ja >= 0 && ja < A.nb) ? A.ch_an[ja] : make_float2(0.f, 0.f);
        }
    }
    /* each bead's first contact item and the item -> bead map of round 0 */
    int total;
    const int off = block_scan_any(nc, s_ws, total);
    if (tid < n) s_off[tid] = off;
    for (int q = off; q < min(off + nc, nch0); ++q) s_owner[q] = (unsigned char)tid;

    cp_async_wait_all();
    bool ok = mbar_wait_bounded(bar, 0);
    ok = __syncthreads_and(ok);
    if (!ok) {
        /* the staged data never arrived: skip the tile, counted for fn_sync */
        if (tid == 0) {
            atomicAdd(A.counters + FN_CNT_STALL, 1ull);
            mbar_wait_bounded(bar, 0);
        }
        __syncthreads();
        return;
    }

    /* springs: lower bead b0 - 2 + u, u < n + 3 */
    for (int u = tid; u < n + 3; u += nt) {
        const unsigned fl = s_flag[u];
        unsigned char tf = 0;
        if (fl & FN_CH_SPRING) {
            const int alive0 = s_stat[u] & 1;
            tf = (unsigned char)(alive0 << 2);
            if (alive0 && !(fl & FN_CH_SP_INERT)) {
                const double4 a = s_img[(fl & FN_CH_SP_REV) ? u + 1 : u];
                const double4 b = s_img[(fl & FN_CH_SP_REV) ? u : u + 1];
                double fx = 0.0, fy = 0.0, fz = 0.0;
                int broke;
                const int acts = spring_pts(a.x, a.y, a.z, b.x, b.y, b.z, s_chsp[u], (fl & FN_CH_SP_FL) ? 1 : 0,
                                            fx, fy, fz, broke);
                s_spf[3 * u] = fx;
                s_spf[3 * u + 1] = fy;
                s_spf[3 * u + 2] = fz;
                tf |= (unsigned char)(acts | (broke << 1));
            }
        }
        s_tsp[u] = tf;
    }
    __syncthreads();
    /* angles: centre b0 - 1 + u, u < n + 2 */
    for (int u = tid; u < n + 2; u += nt) {
        const unsigned fl = s_flag[u + 1];
        int alive = (fl & FN_CH_ANGLE) && (s_stat[u + 1] & 2);
        if (alive && (fl & FN_CH_AN_FL)) {
            const unsigned f1 = s_tsp[u], f2 = s_tsp[u + 1];
            if (!((f1 & 4) && !(f1 & 2)) || !((f2 & 4) && !(f2 & 2))) alive = 0;
        }
        s_tan[u] = (unsigned char)alive;
        if (alive) {
            const double4 t1 = s_img[(fl & FN_CH_AN_REV) ? u + 2 : u];
            const double4 t2 = s_img[u + 1];
            const double4 t3 = s_img[(fl & FN_CH_AN_REV) ? u : u + 2];
            double* o = s_ang + 6 * u;
            angle_pts(t1.x, t1.y, t1.z, t2.x, t2.y, t2.z, t3.x, t3.y, t3.z, s_chan[u], o[0], o[1], o[2], o[3],
                      o[4], o[5]);
        }
    }
    __syncthreads();

    const FnNet& N = A.nets[tile.net];
    double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    if (active) {
        p = s_pos[tid];
        base_force<DAMP>(A, N, i, p, Fx, Fy, Fz);
        const unsigned fp = s_flag[tid + 1];
        if ((fp & FN_CH_SPRING) && (s_tsp[tid + 1] & 1)) {
            const double* f = s_spf + 3 * (tid + 1);
            if (fp & FN_CH_SP_REV) {
                Fx += f[0];
                Fy += f[1];
                Fz += f[2];
            } else {
                Fx += f[0] * -1.0;
                Fy += f[1] * -1.0;
                Fz += f[2] * -1.0;
            }
        }
        const unsigned fn = s_flag[tid + 2];
        if ((fn & FN_CH_SPRING) && (s_tsp[tid + 2] & 1)) {
            const double* f = s_spf + 3 * (tid + 2);
            if (fn & FN_CH_SP_REV) {
                Fx += f[0] * -1.0;
                Fy += f[1] * -1.0;
                Fz += f[2] * -1.0;
            } else {
                Fx += f[0];
                Fy += f[1];
                Fz += f[2];
            }
        }
        if (s_tan[tid]) {
            const double* o = s_ang + 6 * tid;
            const int k = (s_flag[tid + 1] & FN_CH_AN_REV) ? 0 : 3;
            Fx += o[k];
            Fy += o[k + 1];
            Fz += o[k + 2];
        }
        if (s_tan[tid + 1]) {
            const double* o = s_ang + 6 * (tid + 1);
            Fx += -o[0] - o[3];
            Fy += -o[1] - o[4];
            Fz += -o[2] - o[5];
        }
        if (s_tan[tid + 2]) {
            const double* o = s_ang + 6 * (tid + 2);
            const int k = (s_flag[tid + 3] & FN_CH_AN_REV) ? 3 : 0;
            Fx += o[k];
            Fy += o[k + 1];
            Fz += o[k + 2];
        }
    }

    /* contacts, in rounds of at most `chunk` items */
    for (int c0 = 0; c0 < items; c0 += A.chunk) {
        const int nch = min(items - c0, A.chunk);
        if (c0 > 0) {
            __syncthreads(); /* the previous round's results are summed */
            gather_partners(A, ent, c0, nch, s_pj);
            for (int q = max(off, c0); q < min(off + nc, c0 + nch); ++q) s_owner[q - c0] = (unsigned char)tid;
            cp_async_wait_all();
            __syncthreads();
        }
        for (int q = tid; q < nch; q += nt) {
            const int t = min((int)s_owner[q], n - 1);
            double4* slot = reinterpret_cast<double4*>(s_pj + 32 * (size_t)q);
            const double4 pj = *slot;
            double Rx = 0.0, Ry = 0.0, Rz = 0.0;
            const int acts = contact_eval(N, A.pairs, s_pos[t], pj, Rx, Ry, Rz);
            *slot = make_double4(Rx, Ry, Rz, acts ? 1.0 : 0.0);
        }
        __syncthreads();
        if (active) {
            for (int q = max(off, c0); q < min(off + nc, c0 + nch); ++q) {
                const double4 r = *reinterpret_cast<const double4*>(s_pj + 32 * (size_t)(q - c0));
                if (r.w != 0.0) {
                    Fx += r.x;
                    Fy += r.y;
                    Fz += r.z;
                }
            }
        }
    }
    if (!active) return;

    /* statuses after this step (kernel.cl:396-397, 278-284) */
    const unsigned st0 = s_stat[tid + 2];
    unsigned st = st0;
    if ((s_tsp[tid + 2] & 2)) st &= ~1u;
    if ((st0 & 2) && (s_flag[tid + 2] & FN_CH_ANGLE) && !s_tan[tid + 1]) st &= ~2u;
    if (st != st0) A.ch_status[i] = (unsigned char)st;

    /* AdvanceVelocity (kernel.cl:451-462) and the next AdvancePosition */
    const float fx = (float)Fx, fy = (float)Fy, fz = (float)Fz;
    if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicAdd(A.counters + FN_CNT_NONFINITE, 1ull);
    double4 im = s_img[tid + 2];
    const double minv = im.w;
    const double half_dt = N.half_dt * minv;
    const float4 fo = s_frc[tid];
    const float4 vo = s_vold[tid];
    double tx = (double)fx, ty = (double)fy, tz = (double)fz;
    tx += (double)fo.x;
    ty += (double)fo.y;
    tz += (double)fo.z;
    const float vox = (float)(tx * half_dt + (double)vo.x);
    const float voy = (float)(ty * half_dt + (double)vo.y);
    const float voz = (float)(tz * half_dt + (double)vo.z);
    A.force[i] = make_float4(fx, fy, fz, 0.0f);
    A.vold[i] = make_float4(vox, voy, voz, 0.0f);
    if (DRIFT) {
        float4 v;
        drift(N, minv, fx, fy, fz, vox, voy, voz, p, im, v);
        A.pos_out[i] = p;
        A.img_out[i] = im;
        if (DAMP || STORE_V) A.vel[i] = v;
    }
}

template <bool STORE_V>
__global__ void __launch_bounds__(512) k_drift(const StepArgs A) {
    const FnTile t = A.tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    if (i >= t.end) return;
    const FnNet& N = A.nets[t.net];
    double4 p = A.pos_in[i];
    double4 im = A.img_in[i];
    const float4 f = A.force[i];
    const float4 vo = A.vold[i];
    float4 v;
    drift(N, im.w, f.x, f.y, f.z, vo.x, vo.y, vo.z, p, im, v);
    A.pos_out[i] = p;
    A.img_out[i] = im;
    if (STORE_V) A.vel[i] = v;
}

/* Forces alone (no base, no kick, no drift), selected terms; for the
   one-step force parity checks.  Writes force and the bond statuses. */
__global__ void k_forces_only(const StepArgs A, int terms) {
    const FnTile t = A.tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    if (i >= t.end) return;
    const FnNet& N = A.nets[t.net];
    const double4 p = A.pos_in[i];
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    if (terms & 1) {
        for (int e = A.sp_off[i]; e < A.sp_off[i + 1]; ++e) {
            const int ent = A.sp_ent[e];
            double fx, fy, fz;
            int broke;
            if (spring_eval(A, ent >> 1, fx, fy, fz, broke)) {
                const double sg = (ent & 1) ? -1.0 : 1.0;
                Fx += fx * sg;
                Fy += fy * sg;
                Fz += fz * sg;
            }
        }
    }
    if (terms & 2) {
        for (int e = A.an_off[i]; e < A.an_off[i + 1]; ++e) {
            const int ent = A.an_ent[e];
            const int a = ent >> 2, role = ent & 3;
            if (A.an_status[a] != 1) continue;
            const int4 b = A.an_b[a];
            if (b.w == 1) {
                const int2 ss = A.an_s[a];
                if (!spring_alive_after(A, ss.x) || !spring_alive_after(A, ss.y)) continue;
            }
            double pax, pay, paz, pcx, pcy, pcz;
            angle_eval(A, b, A.an_par[a], pax, pay, paz, pcx, pcy, pcz);
            if (role == 0) {
                Fx += pax; Fy += pay; Fz += paz;
            } else if (role == 2) {
                Fx += pcx; Fy += pcy; Fz += pcz;
            } else {
                Fx += -pax - pcx; Fy += -pay - pcy; Fz += -paz - pcz;
            }
        }
    }
    if (terms & 4) {
        int n = A.list_count[i];
        if (n > A.list_cap) n = A.list_cap;
        for (int k = 0; k < n; ++k) {
            const int j = A.list[(size_t)k * A.list_stride + i];
            double Rx, Ry, Rz;
            if (contact_eval(N, A.pairs, p, A.pos_in[j], Rx, Ry, Rz)) {
                Fx += Rx; Fy += Ry; Fz += Rz;
            }
        }
    }
    A.force[i] = make_float4((float)Fx, (float)Fy, (float)Fz, 0.0f);
}

/* ResetBeadEnergy, kernel.cl:468-483. */
__global__ void k_reset_energy(float4* force, float4* vel, float4* vold, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    force[i] = z;
    vel[i] = z;
    vold[i] = z;
}

/* ------------------------------------------------------------------------ */
/* Contact-list rebuild                                                      */

/* FillGrid's cell computation (kernel.cl:492-501) + per-cell counting. */
/* Displacement-triggered mode: every rebuild kernel returns at once unless
   the device gate says a rebuild is due (a null gate always rebuilds). */
#define FN_GATED(g)                   \
    if ((g) != nullptr && *(g) == 0) \
    return

__global__ void k_fill_int(int* p, long long n, int v, const int* gate) {
    FN_GATED(gate);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void k_cells(const RebuildArgs R) {
    FN_GATED(R.gate);
    const FnTile t = R.tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    if (i >= t.end) return;
    const FnNet& N = R.nets[t.net];
    const double4 p = R.pos[i];
    const double qx = floor(p.x / N.step[0]);
    const double qy = floor(p.y / N.step[1]);
    const double qz = floor(p.z / N.step[2]);
    int cell = -1;
    if (qx >= 0.0 && qx < (double)N.nx && qy >= 0.0 && qy < (double)N.ny && qz >= 0.0 &&
        qz < (double)N.nz) {
        cell = N.cell_base + (int)qx + (int)qy * N.nx + (int)qz * N.nxy;
        atomicAdd(R.cell_count + cell, 1);
    }
    R.cell_of[i] = cell;
    R.list_count[i] = 0; /* k_lists counts only the beads it lists */
}

__global__ void k_scatter(const RebuildArgs R, int nb) {
    FN_GATED(R.gate);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int c = R.cell_of[i];
    if (c < 0) return;
    const int slot = atomicAdd(R.cell_fill + c, 1);
    R.cell_beads[R.cell_start[c] + slot] = i;
}

/* Orders each cell's beads by index (the order a one-thread FillGrid sweep
   would store them in) and drops the ones beyond the cell capacity, like the
   `old < GRID_TAIL_SIZE` test of kernel.cl:503. */
__global__ void k_cell_sort(const RebuildArgs R, int ncells) {
    FN_GATED(R.gate);
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const int n = R.cell_count[c];
    if (n <= 1) return;
    int* b = R.cell_beads + R.cell_start[c];
    if (n <= 8 && n <= R.cell_cap) {
        /* the common case (about one bead per cell): sorted in registers by
           Batcher's 8-input network, absent slots holding INT_MAX */
        int v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = k < n ? b[k] : INT_MAX;
        constexpr int net[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6},
                                    {5, 7}, {1, 2}, {5, 6}, {0, 4}, {1, 5}, {2, 6}, {3, 7},
                                    {2, 4}, {3, 5}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int lo = min(v[net[q][0]], v[net[q][1]]);
            const int hi = max(v[net[q][0]], v[net[q][1]]);
            v[net[q][0]] = lo;
            v[net[q][1]] = hi;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (k < n) b[k] = v[k];
        return;
    }
    /* selection of the first min(n, cap) positions: ascending order there,
       O(cap * n) even for an overfull cell */
    const int keep = n < R.cell_cap ? n : R.cell_cap;
    for (int k = 0; k < keep; ++k) {
        int best = k;
        for (int m = k + 1; m < n; ++m)
            if (b[m] < b[best]) best = m;
        const int v = b[best];
        b[best] = b[k];
        b[k] = v;
    }
    if (n > R.cell_cap) {
        for (int k = R.cell_cap; k < n; ++k) R.cell_of[b[k]] = -1;
        atomicAdd(R.counters + FN_CNT_CELL_OVERFLOW, (unsigned long long)(n - R.cell_cap));
    }
}

/* BuildContactList's test (kernel.cl:574-586, 630-659) once the (minimum-
   image) squared distance is known: exclusion of bonded neighbours, then the
   listing radius of the pair kind (the cut-off, widened by the Verlet skin in
   displacement-triggered mode; radius + skin radius for hs pairs). */
__device__ __forceinline__ bool list_accept(const FnNet& N, const FnPair* __restrict__ pairs,
                                            double length, double4 pi, int4 bi, double4 pj,
                                            int4 bj) {
    if (bi.x == bj.x && abs(bi.y - bj.y) <= 1) return false;
    const int kind = pairs[N.pair_base + getadress(bi.z, bj.z, N.types_num)].kind;
    if (kind == 1 || kind == 3) return length < N.list_cut_sq;
    if (kind == 2 || kind == 4) {
        if (kind == 4 && length < N.list_cut_sq) return true;
        const double si = (double)__int_as_float(bi.w), sj = (double)__int_as_float(bj.w);
        const double ri = (double)w_radius(pi.w), rj = (double)w_radius(pj.w);
        const double min_skin = (si > sj) ? sj : si;
        const double max_radius = (ri > rj) ? ri : rj;
        const double lim = max_radius + min_skin;
        return length < lim * lim;
    }
    return false;
}

/* Network owning bead i (networks hold consecutive bead ranges). */
__device__ __forceinline__ int net_of_bead(const FnNet* __restrict__ nets, int n_nets, int i) {
    int lo = 0, hi = n_nets - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (nets[mid].bead_begin <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

/* Candidates j of one run of consecutive beads in cell order. */
__device__ __forceinline__ void scan_run(const RebuildArgs& R, const FnNet& N, int i, double4 pi,
                                         int4 bi, const int* ids, int m, int* __restrict__ out,
                                         int& n) {
    for (int k = 0; k < m; ++k) {
        const int j = ids[k];
        if (j == i) continue;
        const double4 pj = R.pos[j];
        double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
        double length = rx * rx + ry * ry + rz * rz;
        if (N.list_mi) length = min_image(N, rx, ry, rz, length, N.list_mi);
        if (!(length < N.list_r2_max)) continue; /* listed by no pair kind */
        if (list_accept(N, R.pairs, length, pi, bi, pj, R.binfo[j])) {
            if (n < R.list_cap) out[(size_t)n * R.list_stride] = j;
            ++n;
        }
    }
}

/* Full per-bead lists over the 27-cell neighbourhood (dz, dy, dx ascending,
   beads ascending within a cell): the symmetric closure of the reference's
   half-shell pair set, in a fixed order.  Threads walk the beads in cell
   order, so neighbouring threads share their candidate cells; the three
   cells of one (dz, dy) row are one contiguous run of the sorted bead array
   unless the row wraps or a cell overflows. */
/* 12 blocks of 128 per SM (at most 40 registers, a few spilled): the scan
   waits on dependent loads, and the extra resident warps hide more of that
   latency than the spills cost (measured: 0.355 vs 0.373 ms per 1M-bead
   rebuild at the 54 registers the compiler picks unbounded; with the single
   candidate loop, 0.319 vs 0.327 ms at 10 blocks and 48 registers). */
__device__ __forceinline__ void list_one_bead(const RebuildArgs& R, const FnNet& N, int i, int c);

/* Runs of consecutive candidates a thread of k_lists keeps in shared memory
   (a row of three cells is one run unless it wraps or a cell is full). */
constexpr int kListRuns = 12;

/* Bead i's candidates (cell c) as runs of the sorted bead array, in list
   order (dz, dy, dx ascending, beads ascending within a cell); false when
   they take more than kListRuns runs. */
__device__ __forceinline__ bool list_runs(const RebuildArgs& R, const FnNet& N, int c, int cz, int cy, int cx,
                                          int2* runs, int& nr) {
    for (int dz = -1; dz <= 1; ++dz) {
        int z = cz + dz;
        if (z < 0 || z >= N.nz) {
            if (!(N.periodic & 4)) continue;
            z = z < 0 ? N.nz - 1 : 0;
        }
        for (int dy = -1; dy <= 1; ++dy) {
            int y = cy + dy;
            if (y < 0 || y >= N.ny) {
                if (!(N.periodic & 2)) continue;
                y = y < 0 ? N.ny - 1 : 0;
            }
            const int row = N.cell_base + y * N.nx + z * N.nxy;
            if (cx >= 1 && cx + 1 < N.nx) {
                const int c0 = row + cx - 1;
                const int s0 = R.cell_start[c0];
                const int s3 = R.cell_start[c0 + 3];
                if (s3 - s0 <= R.cell_cap ||
                    (R.cell_count[c0] <= R.cell_cap && R.cell_count[c0 + 1] <= R.cell_cap &&
                     R.cell_count[c0 + 2] <= R.cell_cap)) {
                    if (s3 > s0) {
                        if (nr == kListRuns) return false;
                        runs[nr++] = make_int2(s0, s3 - s0);
                    }
                    continue;
                }
            }
            for (int dx = -1; dx <= 1; ++dx) {
                int x = cx + dx;
                if (x < 0 || x >= N.nx) {
                    if (!(N.periodic & 1)) continue;
                    x = x < 0 ? N.nx - 1 : 0;
                }
                const int nc = row + x;
                int m = R.cell_count[nc];
                if (m > R.cell_cap) m = R.cell_cap;
                if (m > 0) {
                    if (nr == kListRuns) return false;
                    runs[nr++] = make_int2(R.cell_start[nc], m);
                }
            }
        }
    }
    return true;
}

__global__ void __launch_bounds__(128, 12) k_lists(const RebuildArgs R, long long ncells) {
    FN_GATED(R.gate);
    __shared__ int2 s_runs[128 * kListRuns];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= R.cell_start[ncells]) return; /* beads placed in the grid */
    const int i = R.cell_beads[t];
    const int c = R.cell_of[i];
    if (c < 0) return; /* beyond its cell's capacity: listed nowhere */
    const FnNet& N = R.nets[net_of_bead(R.nets, R.n_nets, i)];
    /* the bead's candidates as runs of the sorted bead array, in list order
       (dz, dy, dx ascending, beads ascending within a cell) */
    int2* runs = s_runs + threadIdx.x * kListRuns;
    int nr = 0;
    bool spill = false;
    const int lc = c - N.cell_base;
    const int cz = lc / N.nxy;
    const int cy = (lc - cz * N.nxy) / N.nx;
    const int cx = lc - cz * N.nxy - cy * N.nx;
    for (int dz = -1; dz <= 1 && !spill; ++dz) {
        int z = cz + dz;
        if (z < 0 || z >= N.nz) {
            if (!(N.periodic & 4)) continue;
            z = z < 0 ? N.nz - 1 : 0;
        }
        for (int dy = -1; dy <= 1 && !spill; ++dy) {
            int y = cy + dy;
            if (y < 0 || y >= N.ny) {
                if (!(N.periodic & 2)) continue;
                y = y < 0 ? N.ny - 1 : 0;
            }
            const int row = N.cell_base + y * N.nx + z * N.nxy;
            if (cx >= 1 && cx + 1 < N.nx) {
                const int c0 = row + cx - 1;
                const int s0 = R.cell_start[c0];
                const int s3 = R.cell_start[c0 + 3];
                if (s3 - s0 <= R.cell_cap ||
                    (R.cell_count[c0] <= R.cell_cap && R.cell_count[c0 + 1] <= R.cell_cap &&
                     R.cell_count[c0 + 2] <= R.cell_cap)) {
                    if (s3 > s0) {
                        if (nr == kListRuns) {
                            spill = true;
                            break;
                        }
                        runs[nr++] = make_int2(s0, s3 - s0);
                    }
                    continue;
                }
            }
            for (int dx = -1; dx <= 1; ++dx) {
                int x = cx + dx;
                if (x < 0 || x >= N.nx) {
                    if (!(N.periodic & 1)) continue;
                    x = x < 0 ? N.nx - 1 : 0;
                }
                const int nc = row + x;
                int m = R.cell_count[nc];
                if (m > R.cell_cap) m = R.cell_cap;
                if (m > 0) {
                    if (nr == kListRuns) {
                        spill = true;
                        break;
                    }
                    runs[nr++] = make_int2(R.cell_start[nc], m);
                }
            }
        }
    }
    if (spill) { /* more runs than the table holds: the row-by-row scan */
        list_one_bead(R, N, i, c);
        return;
    }
    /* one loop over all runs, so a warp iterates as often as its busiest lane
       has candidates, not as often as the sum of each row's busiest lane */
    const double4 pi = R.pos[i];
    const int4 bi = R.binfo[i];
    int* __restrict__ out = R.list + i;
    int n = 0;
    int r = 0, q = 0, qe = 0;
    if (nr > 0) {
        q = runs[0].x;
        qe = q + runs[0].y;
    }
    while (r < nr) {
        const int j = R.cell_beads[q];
        if (j != i) {
            const double4 pj = R.pos[j];
            double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
            double length = rx * rx + ry * ry + rz * rz;
            if (N.list_mi) length = min_image(N, rx, ry, rz, length, N.list_mi);
            if (length < N.list_r2_max && list_accept(N, R.pairs, length, pi, bi, pj, R.binfo[j])) {
                if (n < R.list_cap) out[(size_t)n * R.list_stride] = j;
                ++n;
            }
        }
        if (++q == qe && ++r < nr) {
            q = runs[r].x;
            qe = q + runs[r].y;
        }
    }
    if (n > R.list_cap)
        atomicAdd(R.counters + FN_CNT_LIST_OVERFLOW, (unsigned long long)(n - R.list_cap));
    R.list_count[i] = n;
}

/* BuildContactList with G lanes per bead (the same lists as k_lists, entry
   for entry), for networks too small to hide k_lists' chain of dependent
   loads with one thread per bead: a bead's candidates are taken G at a time,
   lane l of its group testing candidate (round x G + l), and the accepted
   ones are written in candidate order by a ballot over the group.  Blocks
   of 128 threads, 128 / G beads in cell order. */
template <int G>
__global__ void __launch_bounds__(128) k_lists_group(const RebuildArgs R, long long ncells) {
    FN_GATED(R.gate);
    constexpr int PER = 128 / G;
    __shared__ int2 s_runs[PER * kListRuns];
    __shared__ int s_nr[PER];
    const int lane = threadIdx.x & 31, gl = threadIdx.x % G, grp = threadIdx.x / G;
    const int t = blockIdx.x * PER + grp;
    int i = -1, c = -1;
    if (t < R.cell_start[ncells]) { /* beads placed in the grid */
        i = R.cell_beads[t];
        c = R.cell_of[i];
        if (c < 0) i = -1; /* beyond its cell's capacity: listed nowhere */
    }
    const FnNet& N = R.nets[i >= 0 ? net_of_bead(R.nets, R.n_nets, i) : 0];
    int2* runs = s_runs + grp * kListRuns;
    if (gl == 0) {
        int nr = 0;
        if (i >= 0) {
            const int lc = c - N.cell_base;
            const int cz = lc / N.nxy;
            const int cy = (lc - cz * N.nxy) / N.nx;
            const int cx = lc - cz * N.nxy - cy * N.nx;
            if (!list_runs(R, N, c, cz, cy, cx, runs, nr)) nr = -1; /* row by row, below */
        }
        s_nr[grp] = nr;
    }
    __syncwarp(); /* a group's lanes share a warp */
    const int nr = s_nr[grp];
    int total = 0;
    for (int r = 0; r < nr; ++r) total += runs[r].y;
    const int rounds = __reduce_max_sync(0xffffffffu, (total + G - 1) / G);
    double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
    int4 bi = make_int4(0, 0, 0, 0);
    if (nr > 0) {
        pi = R.pos[i];
        bi = R.binfo[i];
    }
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
    const unsigned below = (1u << lane) - 1u;
    int* __restrict__ out = R.list + (i >= 0 ? i : 0);
    int n = 0;
    int r = 0, off = gl; /* this lane's candidate: offset off in run r */
    while (r < nr && off >= runs[r].y) off -= runs[r++].y;
    for (int k = 0; k < rounds; ++k) {
        bool acc = false;
        int j = -1;
        if (r < nr) {
            j = R.cell_beads[runs[r].x + off];
            if (j != i) {
                const double4 pj = R.pos[j];
                double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
                double length = rx * rx + ry * ry + rz * rz;
                if (N.list_mi) length = min_image(N, rx, ry, rz, length, N.list_mi);
                acc = length < N.list_r2_max && list_accept(N, R.pairs, length, pi, bi, pj, R.binfo[j]);
            }
        }
        const unsigned mine = __ballot_sync(0xffffffffu, acc) & gmask;
        if (acc) {
            const int pos = n + __popc(mine & below);
            if (pos < R.list_cap) out[(size_t)pos * R.list_stride] = j;
        }
        n += __popc(mine);
        off += G;
        while (r < nr && off >= runs[r].y) off -= runs[r++].y;
    }
    if (gl == 0 && i >= 0) {
        if (nr < 0) {
            list_one_bead(R, N, i, c);
        } else {
            if (n > R.list_cap)
                atomicAdd(R.counters + FN_CNT_LIST_OVERFLOW, (unsigned long long)(n - R.list_cap));
            R.list_count[i] = n;
        }
    }
}

/* Bead i's full list, reading its candidates from global memory (k_lists,
   and bricks with more candidates than their shared memory holds). */
__device__ __forceinline__ void list_one_bead(const RebuildArgs& R, const FnNet& N, int i, int c) {
    const double4 pi = R.pos[i];
    const int4 bi = R.binfo[i];
    const int lc = c - N.cell_base;
    const int cz = lc / N.nxy;
    const int cy = (lc - cz * N.nxy) / N.nx;
    const int cx = lc - cz * N.nxy - cy * N.nx;
    int* __restrict__ out = R.list + i;
    int n = 0;
    for (int dz = -1; dz <= 1; ++dz) {
        int z = cz + dz;
        if (z < 0 || z >= N.nz) {
            if (!(N.periodic & 4)) continue;
            z = z < 0 ? N.nz - 1 : 0;
        }
        for (int dy = -1; dy <= 1; ++dy) {
            int y = cy + dy;
            if (y < 0 || y >= N.ny) {
                if (!(N.periodic & 2)) continue;
                y = y < 0 ? N.ny - 1 : 0;
            }
            const int row = N.cell_base + y * N.nx + z * N.nxy;
            if (cx >= 1 && cx + 1 < N.nx) {
                const int c0 = row + cx - 1;
                const int s0 = R.cell_start[c0];
                const int s3 = R.cell_start[c0 + 3];
                if (s3 - s0 <= R.cell_cap ||
                    (R.cell_count[c0] <= R.cell_cap && R.cell_count[c0 + 1] <= R.cell_cap &&
                     R.cell_count[c0 + 2] <= R.cell_cap)) {
                    scan_run(R, N, i, pi, bi, R.cell_beads + s0, s3 - s0, out, n);
                    continue;
                }
            }
            for (int dx = -1; dx <= 1; ++dx) {
                int x = cx + dx;
                if (x < 0 || x >= N.nx) {
                    if (!(N.periodic & 1)) continue;
                    x = x < 0 ? N.nx - 1 : 0;
                }
                const int nc = row + x;
                int m = R.cell_count[nc];
                if (m > R.cell_cap) m = R.cell_cap;
                scan_run(R, N, i, pi, bi, R.cell_beads + R.cell_start[nc], m, out, n);
            }
        }
    }
    if (n > R.list_cap)
        atomicAdd(R.counters + FN_CNT_LIST_OVERFLOW, (unsigned long long)(n - R.list_cap));
    R.list_count[i] = n;
}

/* BuildContactList by bricks of cells (the same lists as k_lists, entry for
   entry): one block per brick of kBrickX x kBrickY x kBrickZ cells of one
   network.  The block stages, once, every listable bead of the brick's cells
   and of the cells around them (ids, positions and bead info, in cell order:
   halo rows z-major, then y, then x, beads ascending within a cell, the first
   cell_cap of a full cell), in three wide rounds of loads -- cell counts and
   starts, bead ids, then positions and bead info by cp.async -- instead of a
   chain of dependent loads per candidate.  Each bead of the brick then scans
   its 27 cells from shared memory in k_lists' order (dz, dy, dx ascending),
   so the lists are k_lists' lists.  A brick whose halo holds more than
   kBrickCands beads lists its beads from global memory (list_one_bead). */
constexpr int kBrickHalo = (kBrickX + 2) * (kBrickY + 2) * (kBrickZ + 2);
constexpr int kBrickCells = kBrickX * kBrickY * kBrickZ;
constexpr int kBrickThreads = 128;

/* last index h of a[0..n] with a[h] <= q (a non-decreasing, a[0] <= q) */
__device__ __forceinline__ int last_le(const int* a, int n, int q) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (a[mid] <= q)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

/* exclusive scan of v[0..n) into out[0..n] (out[n] the total) by one block */
__device__ __forceinline__ void block_scan_array(const int* v, int n, int* out, int* ws) {
    const int per = (n + (int)blockDim.x - 1) / (int)blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, n);
    int sum = 0;
    for (int k = b; k < e; ++k) sum += v[k];
    int total;
    int acc = block_scan_any(sum, ws, total);
    for (int k = b; k < e; ++k) {
        out[k] = acc;
        acc += v[k];
    }
    if (threadIdx.x == 0) out[n] = total;
    __syncthreads();
}

__global__ void __launch_bounds__(kBrickThreads) k_lists_brick(const RebuildArgs R, const int4* __restrict__ bricks) {
    FN_GATED(R.gate);
    __shared__ int s_cnt[kBrickHalo], s_start[kBrickHalo], s_coff[kBrickHalo + 1];
    __shared__ int s_icnt[kBrickCells], s_ioff[kBrickCells + 1];
    __shared__ int s_ws[33];
    __shared__ int s_id[kBrickCands];
    __shared__ double4 s_pos[kBrickCands];
    __shared__ int4 s_bin[kBrickCands];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int4 B = bricks[blockIdx.x]; /* network, first cell x, y, z */
    const FnNet& N = R.nets[B.x];
    const int ex = min(kBrickX, N.nx - B.y), ey = min(kBrickY, N.ny - B.z), ez = min(kBrickZ, N.nz - B.w);
    const int HX = ex + 2, HY = ey + 2, H = HX * HY * (ez + 2), NIC = ex * ey * ez;
    /* round 1: count (first cell_cap of a full cell) and start of every halo
       cell; a cell off a non-periodic side holds nothing */
    for (int hc = tid; hc < H; hc += nt) {
        const int hx = hc % HX, hy = (hc / HX) % HY, hz = hc / (HX * HY);
        int gx = B.y - 1 + hx, gy = B.z - 1 + hy, gz = B.w - 1 + hz;
        bool ok = true;
        if (gx < 0 || gx >= N.nx) {
            if (N.periodic & 1)
                gx = gx < 0 ? N.nx - 1 : 0;
            else
                ok = false;
        }
        if (gy < 0 || gy >= N.ny) {
            if (N.periodic & 2)
                gy = gy < 0 ? N.ny - 1 : 0;
            else
                ok = false;
        }
        if (gz < 0 || gz >= N.nz) {
            if (N.periodic & 4)
                gz = gz < 0 ? N.nz - 1 : 0;
            else
                ok = false;
        }
        int cnt = 0, st = 0;
        if (ok) {
            const int cell = N.cell_base + gx + gy * N.nx + gz * N.nxy;
            cnt = min(R.cell_count[cell], R.cell_cap);
            st = R.cell_start[cell];
        }
        s_cnt[hc] = cnt;
        s_start[hc] = st;
    }
    __syncthreads();
    for (int ic = tid; ic < NIC; ic += nt) {
        const int ix = ic % ex, iy = (ic / ex) % ey, iz = ic / (ex * ey);
        s_icnt[ic] = s_cnt[((iz + 1) * HY + (iy + 1)) * HX + (ix + 1)];
    }
    __syncthreads();
    block_scan_array(s_cnt, H, s_coff, s_ws);
    block_scan_array(s_icnt, NIC, s_ioff, s_ws);
    const int C = s_coff[H], NI = s_ioff[NIC];
    if (C > kBrickCands) {
        /* too many to stage: each bead from global memory */
        for (int u = tid; u < NI; u += nt) {
            const int ic = last_le(s_ioff, NIC, u);
            const int ix = ic % ex, iy = (ic / ex) % ey, iz = ic / (ex * ey);
            const int hc = ((iz + 1) * HY + (iy + 1)) * HX + (ix + 1);
            const int i = R.cell_beads[s_start[hc] + (u - s_ioff[ic])];
            list_one_bead(R, N, i, R.cell_of[i]);
        }
        return;
    }
    /* round 2: bead ids; round 3: their positions and bead info */
    constexpr int kPer = (kBrickCands + kBrickThreads - 1) / kBrickThreads;
    int ids[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int q = tid + k * nt;
        ids[k] = -1;
        if (q < C) {
            const int hc = last_le(s_coff, H, q);
            ids[k] = R.cell_beads[s_start[hc] + (q - s_coff[hc])];
        }
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int q = tid + k * nt;
        if (q < C && ids[k] >= 0) {
            s_id[q] = ids[k];
            const uint32_t dp = smem_addr(s_pos + q), db = smem_addr(s_bin + q);
            cp_async16(dp, R.pos + ids[k]);
            cp_async16(dp + 16, reinterpret_cast<const char*>(R.pos + ids[k]) + 16);
            cp_async16(db, R.binfo + ids[k]);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    for (int u = tid; u < NI; u += nt) {
        const int ic = last_le(s_ioff, NIC, u);
        const int ix = ic % ex, iy = (ic / ex) % ey, iz = ic / (ex * ey);
        const int q = s_coff[((iz + 1) * HY + (iy + 1)) * HX + (ix + 1)] + (u - s_ioff[ic]);
        const int i = s_id[q];
        const double4 pi = s_pos[q];
        const int4 bi = s_bin[q];
        int* __restrict__ out = R.list + i;
        int n = 0;
        for (int dz = 0; dz < 3; ++dz)
            for (int dy = 0; dy < 3; ++dy) {
                const int row = ((iz + dz) * HY + (iy + dy)) * HX + ix; /* halo cell of dx = -1 */
                const int q1 = s_coff[row + 3];
                for (int qq = s_coff[row]; qq < q1; ++qq) {
                    const int j = s_id[qq];
                    if (j == i) continue;
                    const double4 pj = s_pos[qq];
                    double rx = pi.x - pj.x, ry = pi.y - pj.y, rz = pi.z - pj.z;
                    double length = rx * rx + ry * ry + rz * rz;
                    if (N.list_mi) length = min_image(N, rx, ry, rz, length, N.list_mi);
                    if (!(length < N.list_r2_max)) continue; /* listed by no pair kind */
                    if (list_accept(N, R.pairs, length, pi, bi, pj, s_bin[qq])) {
                        if (n < R.list_cap) out[(size_t)n * R.list_stride] = j;
                        ++n;
                    }
                }
            }
        if (n > R.list_cap)
            atomicAdd(R.counters + FN_CNT_LIST_OVERFLOW, (unsigned long long)(n - R.list_cap));
        R.list_count[i] = n;
    }
}

/* Tile-compacted copy of the contact list for the staged step kernel: tile
   t's entries, bead after bead and in list order within a bead, from
   csr + t * region (region >= beads per tile x list capacity), and their
   number in tile_items[t].  One block of at least the tile's bead count. */
__global__ void k_list_tiles(const RebuildArgs R) {
    FN_GATED(R.gate);
    __shared__ int ws[33];
    const FnTile t = R.tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    int c = 0;
    if (i < t.end) {
        c = R.list_count[i];
        if (c > R.list_cap) c = R.list_cap;
    }
    int total;
    const int off = block_scan_any(c, ws, total);
    int* out = R.csr + (size_t)blockIdx.x * (size_t)R.csr_region + off;
    for (int k = 0; k < c; ++k) out[k] = R.list[(size_t)k * R.list_stride + i];
    if (threadIdx.x == 0) R.tile_items[blockIdx.x] = total;
}

/* ------------------------------------------------------------------------ */
/* Exclusive scan of int counts (1024 threads x 2 items per block).          */

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 2;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = warp_sums[lane];
        int s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s - w;
        if (lane == 31) warp_sums[32] = s;
    }
    __syncthreads();
    total = warp_sums[32];
    const int r = x - v + warp_sums[warp];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_partials(const int* in, long long n,
                                                                 int* block_sums, const int* gate) {
    FN_GATED(gate);
    __shared__ int ws[33];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) s += in[base + k];
    int total;
    block_exclusive_scan(s, ws, total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

/* One block scans the block sums in chunks, carrying the running total. */
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(int* block_sums, int nblocks,
                                                             int* grand_total, const int* gate) {
    FN_GATED(gate);
    __shared__ int ws[33];
    int carry = 0;
    for (int base = 0; base < nblocks; base += SCAN_THREADS) {
        const int idx = base + (int)threadIdx.x;
        const int v = idx < nblocks ? block_sums[idx] : 0;
        int total;
        const int ex = block_exclusive_scan(v, ws, total);
        if (idx < nblocks) block_sums[idx] = ex + carry;
        carry += total;
    }
    if (threadIdx.x == 0) *grand_total = carry;
}

/* Exclusive scan, last pass: each block's offset added, written to out;
   zero (if given) is cleared alongside, sparing a launch. */
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const int* in, long long n,
                                                              const int* block_sums, int* out,
                                                              const int* gate, int* zero) {
    FN_GATED(gate);
    __shared__ int ws[33];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int ex = block_exclusive_scan(s, ws, total) + block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) {
            out[base + k] = ex;
            if (zero) zero[base + k] = 0;
        }
        ex += v[k];
    }
}

/* Exclusive scan, last pass, without a pass of its own over the block sums:
   each block adds up the raw sums of the blocks before it (a few thousand at
   most, read from L2), the last block writes the grand total; zero (if
   given) is cleared alongside. */
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply_direct(const int* in, long long n,
                                                                     const int* block_sums, int nblocks,
                                                                     int* out, int* grand_total,
                                                                     const int* gate, int* zero) {
    FN_GATED(gate);
    __shared__ int ws[33];
    int before = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += SCAN_THREADS) before += block_sums[b];
    int offset;
    block_exclusive_scan(before, ws, offset); /* offset: the block sums' total */
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int ex = block_exclusive_scan(s, ws, total) + offset;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) {
            out[base + k] = ex;
            if (zero) zero[base + k] = 0;
        }
        ex += v[k];
    }
    if (blockIdx.x == nblocks - 1 && threadIdx.x == 0) *grand_total = offset + total;
}

/* ------------------------------------------------------------------------ */
/* Observables: deterministic two-pass FP64 reduction per network.           */

__global__ void k_observe_partial(const ObserveArgs O) {
    __shared__ double sx[256], sy[256], sz[256];
    __shared__ long long sb[256], sa[256];
    const int tid = threadIdx.x;
    double x = 0.0, y = 0.0, z = 0.0;
    long long nb = 0, na = 0;
    for (int i = O.bead_begin + blockIdx.x * blockDim.x + tid; i < O.bead_end;
         i += gridDim.x * blockDim.x) {
        if (w_type(O.pos[i].w) == O.reaction_type) {
            const float4 f = O.force[i];
            x += (double)f.x;
            y += (double)f.y;
            z += (double)f.z;
        }
    }
    if (O.ch_flags) {
        for (int i = O.bead_begin + blockIdx.x * blockDim.x + tid; i < O.bead_end;
             i += gridDim.x * blockDim.x) {
            const unsigned f = O.ch_flags[i], st = O.ch_status[i];
            nb += (f & FN_CH_SPRING) && !(st & 1);
            na += (f & FN_CH_ANGLE) && !(st & 2);
        }
    } else {
        for (int s = O.spring_begin + blockIdx.x * blockDim.x + tid; s < O.spring_end;
             s += gridDim.x * blockDim.x)
            nb += O.sp_status[s] == 0;
        for (int a = O.angle_begin + blockIdx.x * blockDim.x + tid; a < O.angle_end;
             a += gridDim.x * blockDim.x)
            na += O.an_status[a] == 0;
    }
    sx[tid] = x;
    sy[tid] = y;
    sz[tid] = z;
    sb[tid] = nb;
    sa[tid] = na;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (tid < o) {
            sx[tid] += sx[tid + o];
            sy[tid] += sy[tid + o];
            sz[tid] += sz[tid + o];
            sb[tid] += sb[tid + o];
            sa[tid] += sa[tid + o];
        }
        __syncthreads();
    }
    if (tid == 0) {
        double* o = O.partial + 5 * (size_t)blockIdx.x;
        o[0] = sx[0];
        o[1] = sy[0];
        o[2] = sz[0];
        o[3] = (double)sb[0];
        o[4] = (double)sa[0];
    }
}

__global__ void k_observe_final(const double* partial, int nblocks, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nblocks; ++b)
        for (int k = 0; k < 5; ++k) a[k] += partial[5 * (size_t)b + k];
    for (int k = 0; k < 5; ++k) out[k] = a[k];
}

/* ------------------------------------------------------------------------ */
/* launch wrappers                                                           */

cudaError_t launch_step(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                        bool store_v, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    if (damp) {
        if (do_drift)
            k_step<true, true, true><<<ntiles, block, 0, s>>>(A);
        else
            k_step<true, false, false><<<ntiles, block, 0, s>>>(A);
    } else {
        if (do_drift) {
            if (store_v)
                k_step<false, true, true><<<ntiles, block, 0, s>>>(A);
            else
                k_step<false, true, false><<<ntiles, block, 0, s>>>(A);
        } else {
            k_step<false, false, false><<<ntiles, block, 0, s>>>(A);
        }
    }
    return cudaGetLastError();
}

template <bool DAMP, bool DRIFT, bool STORE_V>
static cudaError_t set_tiled_smem(size_t bytes) {
    return cudaFuncSetAttribute(k_step_tiled<DAMP, DRIFT, STORE_V>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

/* The dynamic shared-memory limit is an attribute of the kernel on a
   device, shared by every context of the process: it is only ever raised
   (a context with smaller tiles must not lower it under another's launch). */
static bool raise_limit(size_t* table, size_t& bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
    if (bytes <= table[dev]) return false;
    table[dev] = bytes;
    return true;
}

cudaError_t prepare_step_tiled(size_t bytes) {
    static size_t done[64] = {};
    if (!raise_limit(done, bytes)) return cudaSuccess;
    cudaError_t e;
    if ((e = set_tiled_smem<true, true, true>(bytes))) return e;
    if ((e = set_tiled_smem<true, false, false>(bytes))) return e;
    if ((e = set_tiled_smem<false, true, true>(bytes))) return e;
    if ((e = set_tiled_smem<false, true, false>(bytes))) return e;
    return set_tiled_smem<false, false, false>(bytes);
}

cudaError_t launch_step_tiled(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                              bool store_v, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    const size_t sm = step_tiled_smem(A.max_tile_sp, A.max_tile_an);
    if (damp) {
        if (do_drift)
            k_step_tiled<true, true, true><<<ntiles, block, sm, s>>>(A);
        else
            k_step_tiled<true, false, false><<<ntiles, block, sm, s>>>(A);
    } else {
        if (do_drift) {
            if (store_v)
                k_step_tiled<false, true, true><<<ntiles, block, sm, s>>>(A);
            else
                k_step_tiled<false, true, false><<<ntiles, block, sm, s>>>(A);
        } else {
            k_step_tiled<false, false, false><<<ntiles, block, sm, s>>>(A);
        }
    }
    return cudaGetLastError();
}

template <bool DAMP, bool DRIFT, bool STORE_V, bool FO>
static cudaError_t set_chain_smem(size_t bytes) {
    return cudaFuncSetAttribute(k_step_chain<DAMP, DRIFT, STORE_V, FO>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t prepare_step_chain(size_t bytes) {
    static size_t done[64] = {};
    if (!raise_limit(done, bytes)) return cudaSuccess;
    cudaError_t e;
    if ((e = set_chain_smem<true, true, true, false>(bytes))) return e;
    if ((e = set_chain_smem<true, false, false, false>(bytes))) return e;
    if ((e = set_chain_smem<false, true, true, false>(bytes))) return e;
    if ((e = set_chain_smem<false, true, false, false>(bytes))) return e;
    if ((e = set_chain_smem<false, false, false, false>(bytes))) return e;
    return set_chain_smem<false, false, false, true>(bytes);
}

cudaError_t launch_step_chain(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                              bool store_v, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    const size_t sm = step_chain_smem(block);
    if (damp) {
        if (do_drift)
            k_step_chain<true, true, true, false><<<ntiles, block, sm, s>>>(A, 0);
        else
            k_step_chain<true, false, false, false><<<ntiles, block, sm, s>>>(A, 0);
    } else {
        if (do_drift) {
            if (store_v)
                k_step_chain<false, true, true, false><<<ntiles, block, sm, s>>>(A, 0);
            else
                k_step_chain<false, true, false, false><<<ntiles, block, sm, s>>>(A, 0);
        } else {
            k_step_chain<false, false, false, false><<<ntiles, block, sm, s>>>(A, 0);
        }
    }
    return cudaGetLastError();
}

template <bool DAMP, bool DRIFT, bool STORE_V>
static cudaError_t set_staged_smem(size_t bytes) {
    return cudaFuncSetAttribute(k_step_staged<DAMP, DRIFT, STORE_V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bytes);
}

cudaError_t prepare_step_staged(size_t bytes) {
    static size_t done[64] = {};
    if (!raise_limit(done, bytes)) return cudaSuccess;
    cudaError_t e;
    if ((e = set_staged_smem<true, true, true>(bytes))) return e;
    if ((e = set_staged_smem<true, false, false>(bytes))) return e;
    if ((e = set_staged_smem<false, true, true>(bytes))) return e;
    if ((e = set_staged_smem<false, true, false>(bytes))) return e;
    return set_staged_smem<false, false, false>(bytes);
}

cudaError_t launch_step_staged(const StepArgs& A, int ntiles, int block, bool damp, bool do_drift,
                               bool store_v, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    const size_t sm = step_staged_smem(block, A.chunk);
    if (damp) {
        if (do_drift)
            k_step_staged<true, true, true><<<ntiles, block, sm, s>>>(A);
        else
            k_step_staged<true, false, false><<<ntiles, block, sm, s>>>(A);
    } else {
        if (do_drift) {
            if (store_v)
                k_step_staged<false, true, true><<<ntiles, block, sm, s>>>(A);
            else
                k_step_staged<false, true, false><<<ntiles, block, sm, s>>>(A);
        } else {
            k_step_staged<false, false, false><<<ntiles, block, sm, s>>>(A);
        }
    }
    return cudaGetLastError();
}


cudaError_t launch_forces_chain(const StepArgs& A, int ntiles, int block, int terms, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    k_step_chain<false, false, false, true><<<ntiles, block, step_chain_smem(block), s>>>(A, terms);
    return cudaGetLastError();
}

cudaError_t launch_drift(const StepArgs& A, int ntiles, int block, bool store_v, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    if (store_v)
        k_drift<true><<<ntiles, block, 0, s>>>(A);
    else
        k_drift<false><<<ntiles, block, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_forces_only(const StepArgs& A, int ntiles, int block, int terms,
                               cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    k_forces_only<<<ntiles, block, 0, s>>>(A, terms);
    return cudaGetLastError();
}

cudaError_t launch_reset_energy(float4* force, float4* vel, float4* vold, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_reset_energy<<<(n + 255) / 256, 256, 0, s>>>(force, vel, vold, n);
    return cudaGetLastError();
}

long long scan_block_count(long long n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

cudaError_t launch_exclusive_scan(const int* in, long long n, int* out, int* block_sums, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const long long nblk = scan_block_count(n);
    k_scan_partials<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(in, n, block_sums, nullptr);
    k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(block_sums, (int)nblk, out + n, nullptr);
    k_scan_apply<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(in, n, block_sums, out, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_rebuild(const RebuildArgs& R, int ntiles, int block, int nb, long long ncells,
                           int* scan_block_sums, cudaStream_t s) {
    cudaError_t e;
    const unsigned fill_blocks = (unsigned)std::min<long long>(4096, (ncells + 255) / 256 + 1);
    /* cell fills are cleared by the scan's last pass and list counts by
       k_cells, so only the cell counts need a pass of their own */
    if (R.gate)
        k_fill_int<<<fill_blocks, 256, 0, s>>>(R.cell_count, ncells, 0, R.gate);
    else if ((e = cudaMemsetAsync(R.cell_count, 0, sizeof(int) * (size_t)ncells, s)))
        return e;
    if (ntiles > 0) k_cells<<<ntiles, block, 0, s>>>(R);
    const long long nblk = scan_block_count(ncells);
    k_scan_partials<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(R.cell_count, ncells, scan_block_sums, R.gate);
    k_scan_apply_direct<<<(unsigned)nblk, SCAN_THREADS, 0, s>>>(R.cell_count, ncells, scan_block_sums, (int)nblk,
                                                                 R.cell_start, R.cell_start + ncells, R.gate,
                                                                 R.cell_fill);
    if (nb > 0) k_scatter<<<(nb + 255) / 256, 256, 0, s>>>(R, nb);
    k_cell_sort<<<(unsigned)((ncells + 255) / 256), 256, 0, s>>>(R, (int)ncells);
    if (R.bricks) {
        if (R.nbricks > 0) k_lists_brick<<<R.nbricks, kBrickThreads, 0, s>>>(R, R.bricks);
    } else if (nb > 0 && R.list_lanes == 8) {
        k_lists_group<8><<<(nb + 15) / 16, 128, 0, s>>>(R, ncells);
    } else if (nb > 0) {
        /* every bead may sit in the grid; threads past the grid total return */
        k_lists<<<(nb + 127) / 128, 128, 0, s>>>(R, ncells);
    }
    /* the staged step kernel's copy, one block per tile (tiles are at most
       block - 4 beads wide) */
    if (R.csr && ntiles > 0) k_list_tiles<<<ntiles, block, 0, s>>>(R);
    return cudaGetLastError();
}

/* Displacement mode: raises the gate when a bead has moved more than the
   threshold since the last rebuild (image positions, so wraps do not count). */
__global__ void k_disp_check(const FnTile* tiles, const double4* img, const double4* ref, double thresh2,
                             int* gate) {
    const FnTile t = tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    if (i >= t.end) return;
    const double4 a = img[i], b = ref[i];
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    if (!(dx * dx + dy * dy + dz * dz <= thresh2)) *gate = 1;
}

/* After a gated rebuild: the new reference positions. */
__global__ void k_ref_update(const FnTile* tiles, const double4* img, double4* ref, const int* gate) {
    FN_GATED(gate);
    const FnTile t = tiles[blockIdx.x];
    const int i = t.begin + (int)threadIdx.x;
    if (i >= t.end) return;
    ref[i] = img[i];
}

__global__ void k_gate_clear(int* gate, unsigned long long* counters) {
    if (*gate) {
        counters[FN_CNT_REBUILDS] += 1ull;
        *gate = 0;
    }
}

cudaError_t launch_verlet_rebuild(const RebuildArgs& R, const FnTile* tiles, const double4* img,
                                  double4* ref, double thresh2, int* gate, int ntiles, int block, int nb,
                                  long long ncells, int* scan_block_sums, cudaStream_t s) {
    if (ntiles > 0) k_disp_check<<<ntiles, block, 0, s>>>(tiles, img, ref, thresh2, gate);
    cudaError_t e = launch_rebuild(R, ntiles, block, nb, ncells, scan_block_sums, s);
    if (e) return e;
    if (ntiles > 0) k_ref_update<<<ntiles, block, 0, s>>>(tiles, img, ref, gate);
    k_gate_clear<<<1, 1, 0, s>>>(gate, R.counters);
    return cudaGetLastError();
}

/* Export of one bead field in upload order as x, y, z doubles (the host
   buffer layout of fn_download): out[3 u + a] = src[inv[u]].a. */
template <class T>
__global__ void k_export_xyz(const T* __restrict__ src, const int* __restrict__ inv, int n,
                             double* __restrict__ out) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const T v = src[inv[u]];
    out[3 * (size_t)u] = (double)v.x;
    out[3 * (size_t)u + 1] = (double)v.y;
    out[3 * (size_t)u + 2] = (double)v.z;
}

cudaError_t launch_export_xyz(const double4* src, const int* inv, int n, double* out, cudaStream_t s) {
    if (n > 0) k_export_xyz<double4><<<(n + 255) / 256, 256, 0, s>>>(src, inv, n, out);
    return cudaGetLastError();
}

cudaError_t launch_export_xyz(const float4* src, const int* inv, int n, double* out, cudaStream_t s) {
    if (n > 0) k_export_xyz<float4><<<(n + 255) / 256, 256, 0, s>>>(src, inv, n, out);
    return cudaGetLastError();
}

/* ---------------------------------------------------------------------------
   Energy and virial (an addition: the reference computes neither).  Each term
   is the potential whose negative gradient is the force the step applies:
     spring   k/2 (L - L0)^2                      (F = k (L0 - L) u)
     angle    k (theta - theta0)^2                (M = -2 k (theta - theta0))
     hs       K/2 p^2, p = r_i + r_j - r > 0
     hsr      K/2 p^2 + k/2 (rc - r)^2 for r < rc
     lj       48 eps s^12/13 (r^-13 - rc^-13) - 24 eps s^6/7 (r^-7 - rc^-7)
              + c4 (r - rc), the integral of the shifted force to rc = c3
     st       K (c2 (rc - r) - (rc^2 - r^2)/2) + K0 (c6 (rc - r) - (rc^2 - r^2)/2)
     wall     wall_k/2 d^2 for a penetration d past a wall
     gravity  -g . x (image position; g is a force per bead)
   Kinetic energy is m/2 |v|^2 of the step-end velocity (velocity_old) over
   beads of non-zero mass.  The virial is sum r_ij (x) F_ij over springs,
   angles (r_ba (x) F_a + r_bc (x) F_c) and contact pairs, each pair once. */
__device__ __forceinline__ double contact_energy(const FnNet& N, const FnPair* __restrict__ pairs,
                                                 double4 pi, double4 pj, double& Rx, double& Ry,
                                                 double& Rz, double& rx, double& ry, double& rz,
                                                 int& acts) {
    rx = pi.x - pj.x;
    ry = pi.y - pj.y;
    rz = pi.z - pj.z;
    double r2 = rx * rx + ry * ry + rz * rz;
    r2 = min_image(N, rx, ry, rz, r2, N.force_mi);
    acts = contact_eval(N, pairs, pi, pj, Rx, Ry, Rz);
    if (!acts) return 0.0;
    const FnPair* P = pairs + N.pair_base + getadress(w_type(pi.w), w_type(pj.w), N.types_num);
    const double r = sqrt(r2);
    const double rsum = (double)w_radius(pi.w) + (double)w_radius(pj.w);
    switch (P->kind) {
    case 1: {
        const double rc = P->c[2], s2 = P->c[0] * P->c[0], eps = P->c[1];
        const double s6 = s2 * s2 * s2, s12 = s6 * s6;
        const double ir = 1.0 / r, irc = 1.0 / rc;
        /* r^-7 and r^-13 by products (within a few ulp of pow, far cheaper) */
        const double ir2 = ir * ir, ir6 = ir2 * ir2 * ir2, ir7 = ir6 * ir, ir13 = ir6 * ir7;
        const double irc2 = irc * irc, irc6 = irc2 * irc2 * irc2, irc7 = irc6 * irc, irc13 = irc6 * irc7;
        return 48.0 * eps * s12 / 13.0 * (ir13 - irc13) - 24.0 * eps * s6 / 7.0 * (ir7 - irc7) +
               P->c[3] * (r - rc);
    }
    case 2: {
        const double p = rsum - r;
        return 0.5 * P->c[0] * p * p;
    }
    case 3: {
        const double rc = sqrt(P->c[3]);
        const double q = 0.5 * (rc * rc - r * r);
        return P->c[0] * (P->c[1] * (rc - r) - q) + P->c[4] * (P->c[5] * (rc - r) - q);
    }
    case 4: {
        const double p = rsum - r;
        double u = p > 0.0 ? 0.5 * P->c[0] * p * p : 0.0;
        if (r < P->c[2]) u += 0.5 * P->c[1] * (P->c[2] - r) * (P->c[2] - r);
        return u;
    }
    }
    return 0.0;
}

__device__ __forceinline__ void add_outer(double* w, double ax, double ay, double az, double bx,
                                          double by, double bz) {
    w[0] += ax * bx;
    w[1] += ax * by;
    w[2] += ax * bz;
    w[3] += ay * bx;
    w[4] += ay * by;
    w[5] += ay * bz;
    w[6] += az * bx;
    w[7] += az * by;
    w[8] += az * bz;
}

/* At most 85 registers (3 blocks of 256 per SM, a few accumulators spilled):
   the per-bead contact walk waits on partner loads, which more resident warps
   hide (measured on the 1M-bead tensile network: 0.37 ms per evaluation
   against 0.45 ms at the 102 registers the compiler picks unbounded). */
__global__ void __launch_bounds__(256, 3) k_energy_partial(const EnergyArgs E) {
    __shared__ double red[256];
    const FnNet& N = E.nets[E.net];
    double acc[FN_EN_N];
#pragma unroll
    for (int k = 0; k < FN_EN_N; ++k) acc[k] = 0.0;
    double* W = acc + FN_EN_VIRIAL;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;

    for (int i = E.bead_begin + t0; i < E.bead_end; i += stride) {
        const double4 p = E.pos[i];
        const double4 im = E.img[i];
        if (im.w > 0.0) {
            const float4 v = E.vold[i];
            const double vx = v.x, vy = v.y, vz = v.z;
            acc[FN_EN_KINETIC] += 0.5 / im.w * (vx * vx + vy * vy + vz * vz);
        }
        acc[FN_EN_GRAVITY] -= N.g[0] * im.x + N.g[1] * im.y + N.g[2] * im.z;
        if (N.walls) {
            const double pc[3] = {p.x, p.y, p.z};
            for (int a = 0; a < 3; ++a) {
                if (!(N.walls & (1 << a))) continue;
                double d = 0.0;
                if (pc[a] < 0.0) d = pc[a];
                if (pc[a] > N.box[a]) d = pc[a] - N.box[a];
                acc[FN_EN_WALL] += 0.5 * N.wall_k * d * d;
            }
        }
        int n = E.list_count[i];
        if (n > E.list_cap) n = E.list_cap;
        for (int k = 0; k < n; ++k) {
            const int j = E.list[(size_t)k * E.list_stride + i];
            if (j <= i) continue;
            double Rx, Ry, Rz, rx, ry, rz;
            int acts;
            const double u = contact_energy(N, E.pairs, p, E.pos[j], Rx, Ry, Rz, rx, ry, rz, acts);
            if (acts) {
                acc[FN_EN_CONTACT] += u;
                acc[FN_EN_CONTACTS] += 1.0;
                add_outer(W, rx, ry, rz, Rx, Ry, Rz);
            }
        }
    }
    for (int s = E.spring_begin + t0; s < E.spring_end; s += stride) {
        const int type = E.sp_type[s];
        if (!(type == 0 || type == 1)) continue;
        const int2 e = E.sp_ends[s];
        const int alive = E.ch_status ? (E.ch_status[min(e.x, e.y)] & 1) : (E.sp_status[s] == 1);
        if (!alive) continue;
        const double4 a = E.img[e.x], b = E.img[e.y];
        const float4 par = E.sp_par[s];
        double fx, fy, fz;
        int broke;
        spring_pts(a.x, a.y, a.z, b.x, b.y, b.z, par, 0, fx, fy, fz, broke);
        const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
        const double L = sqrt(dx * dx + dy * dy + dz * dz) - (double)par.x;
        acc[FN_EN_SPRING] += 0.5 * (double)par.y * L * L;
        add_outer(W, dx, dy, dz, fx, fy, fz);
    }
    for (int q = E.angle_begin + t0; q < E.angle_end; q += stride) {
        const int4 b = E.an_b[q];
        const int alive = E.ch_status ? ((E.ch_status[b.y] >> 1) & 1) : (E.an_status[q] == 1);
        if (!alive) continue;
        const double4 t1 = E.img[b.x], t2 = E.img[b.y], t3 = E.img[b.z];
        const float2 par = E.an_par[q];
        double pax, pay, paz, pcx, pcy, pcz;
        angle_pts(t1.x, t1.y, t1.z, t2.x, t2.y, t2.z, t3.x, t3.y, t3.z, par, pax, pay, paz, pcx,
                  pcy, pcz);
        const double bax = t1.x - t2.x, bay = t1.y - t2.y, baz = t1.z - t2.z;
        const double bcx = t3.x - t2.x, bcy = t3.y - t2.y, bcz = t3.z - t2.z;
        double dotp = (bax * bcx + bay * bcy + baz * bcz) /
                      (sqrt(bax * bax + bay * bay + baz * baz) * sqrt(bcx * bcx + bcy * bcy + bcz * bcz));
        if (dotp < -1.0) dotp = -0.999999;
        if (dotp > 1.0) dotp = 0.999999;
        const double d = fn_acos(dotp) - (double)par.x;
        acc[FN_EN_ANGLE] += (double)par.y * d * d;
        add_outer(W, bax, bay, baz, pax, pay, paz);
        add_outer(W, bcx, bcy, bcz, pcx, pcy, pcz);
    }
    /* fixed-order block reduction, one quantity at a time */
    for (int k = 0; k < FN_EN_N; ++k) {
        red[threadIdx.x] = acc[k];
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) E.partial[(size_t)FN_EN_N * blockIdx.x + k] = red[0];
        __syncthreads();
    }
}

__global__ void k_energy_final(const double* partial, int nblocks, double* out) {
    const int k = threadIdx.x;
    if (blockIdx.x != 0 || k >= FN_EN_N) return;
    double a = 0.0;
    for (int b = 0; b < nblocks; ++b) a += partial[(size_t)FN_EN_N * b + k];
    out[k] = a;
}

cudaError_t launch_energy(const EnergyArgs& E, int nblocks, double* out, cudaStream_t s) {
    k_energy_partial<<<nblocks, 256, 0, s>>>(E);
    k_energy_final<<<1, 32, 0, s>>>(E.partial, nblocks, out);
    return cudaGetLastError();
}

cudaError_t launch_observe(const ObserveArgs& O, int nblocks, double* out, cudaStream_t s) {
    k_observe_partial<<<nblocks, 256, 0, s>>>(O);
    k_observe_final<<<1, 32, 0, s>>>(O.partial, nblocks, out);
    return cudaGetLastError();
}

}  // namespace fn
