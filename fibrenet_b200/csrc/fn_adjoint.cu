/*
 * fn_adjoint.cu -- discrete adjoint of the step loop (no counterpart in the
 * reference): gradients of a loss on the recorded clamp reaction force with
 * respect to every spring stiffness and rest length, every angle stiffness
 * and the initial positions and velocities.
 *
 * The forward map of one step, as the step kernels apply it (FP32 storage
 * aside), with b = dt/(2m) and c = dt^2/(2m) (both 0 for mass-0 beads):
 *     F_j     = f(x_j)                       springs, angles, contacts, walls
 *     v_j     = v_{j-1} + b (F_{j-1} + F_j)  AdvanceVelocity
 *     x_{j+1} = x_j + dt v_j + c F_j         AdvancePosition
 * Its adjoint, with X = dL/dx_{j+1}, V = dL/dv_j and L_j = dL/dF_j from the
 * loss (the reaction sampled at evaluation j), reduces to
 *     V    <- V + dt X
 *     Fbar  = (dt/m) V + L_j
 *     X    <- X + J_j^T Fbar,   J_j = df/dx at x_j
 *     g    += (df/dtheta)^T Fbar
 * Every force here is minus the gradient of a potential, so J_j is symmetric
 * and J^T Fbar is the directional derivative of f along Fbar: central
 * springs and contacts use their closed-form Jacobian, angles are
 * differentiated with dual numbers.  Contact sets, HR_FL break events and the
 * list of each rebuild interval are those of the forward pass (the recorded
 * statuses; lists rebuilt from the recorded positions by the same kernels).
 *
 * Storage: the forward saves a checkpoint every K steps; the reverse sweep
 * replays each K-step segment from its checkpoint into per-step position
 * buffers (bit-identical to the forward, checked against the next
 * checkpoint) and walks it backwards.  Adjoint state X, V, Fbar is FP32;
 * parameter gradients accumulate in FP64.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "fn_detmath.h"
#include "fn_device.cuh"
#include "fn_engine_internal.h"

namespace fn {

/* ---------------------------------------------------------------- duals */

struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual dl(double v) { return {v, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double s) { return {a.v * s, a.d * s}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double r = sqrt(a.v);
    return {r, r > 0.0 ? a.d / (2.0 * r) : 0.0};
}

/* The angle force of kernel.cl:291-348 at unit stiffness, with tangents:
   t1..t3 positions of b1..b3 with tangent directions w1..w3.  Returns pa (on
   b1) and pc (on b3) as duals; the force scales linearly with the stiffness.
   The clamp of the cosine to +-0.999999 outside [-1, 1] has zero tangent. */
__device__ void angle_dual(const double* t1, const double* t2, const double* t3, const float* w1,
                           const float* w2, const float* w3, double theta0, Dual pa[3], Dual pc[3]) {
    Dual ba[3], bc[3], cb[3];
    for (int a = 0; a < 3; ++a) {
        ba[a] = {t1[a] - t2[a], (double)w1[a] - (double)w2[a]};
        bc[a] = {t3[a] - t2[a], (double)w3[a] - (double)w2[a]};
        cb[a] = bc[a] * -1.0;
    }
    const Dual l_ba = dsqrt(ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2]);
    const Dual l_bc = dsqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    Dual dotp = (ba[0] * bc[0] + ba[1] * bc[1] + ba[2] * bc[2]) / (l_ba * l_bc);
    if (dotp.v < -1.0) dotp = dl(-0.999999);
    if (dotp.v > 1.0) dotp = dl(0.999999);
    const double s = 1.0 - dotp.v * dotp.v;
    const Dual angle = {fn_acos(dotp.v), s > 0.0 ? -dotp.d / sqrt(s) : 0.0};
    const Dual magnitude = (angle - dl(theta0)) * -2.0;
    const Dual fa = magnitude / l_ba;
    const Dual fc = magnitude / l_bc;
    const Dual tx = ba[1] * bc[2] - ba[2] * bc[1];
    const Dual ty = ba[2] * bc[0] - ba[0] * bc[2];
    const Dual tz = ba[0] * bc[1] - ba[1] * bc[0];
    pa[0] = ba[1] * tz - ba[2] * ty;
    pa[1] = ba[2] * tx - ba[0] * tz;
    pa[2] = ba[0] * ty - ba[1] * tx;
    Dual ln = dsqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
    Dual sc = ln.v != 0.0 ? fa / ln : dl(0.0);
    for (int a = 0; a < 3; ++a) pa[a] = pa[a] * sc;
    pc[0] = cb[1] * tz - cb[2] * ty;
    pc[1] = cb[2] * tx - cb[0] * tz;
    pc[2] = cb[0] * ty - cb[1] * tx;
    ln = dsqrt(pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
    sc = ln.v != 0.0 ? fc / ln : dl(0.0);
    for (int a = 0; a < 3; ++a) pc[a] = pc[a] * sc;
}

__device__ __forceinline__ Dual dsin(Dual a) { return {sin(a.v), cos(a.v) * a.d}; }

/* The same angle force for a rest angle of pi in its regular form
     pa = 2k G (w - cos(theta) u) / |ba|,  pc = 2k G (u - cos(theta) w) / |bc|,
     G = (theta - pi) / sin(theta) = -phi / sin(phi),  phi = pi - theta,
   with u, w the unit arms (at unit stiffness).  It equals kernel.cl's cross-
   product form for theta0 = pi.  A rest angle stored as the FP32 rounding
   of pi adds a term of constant size 2k (theta0 - pi) / |ba| whose direction
   turns with the bend, so its Jacobian grows like (theta0 - pi) / phi and is
   unbounded for the straight fibres the tensile networks start from; the
   adjoint differentiates the regular form (the dropped term is below 1.8e-6
   k / |ba| in force).  phi^2 comes from |u + w|^2 = 4 sin^2(phi / 2), which
   keeps full precision near straight.  Exactly straight triples (zero cross
   product, where the step applies no force) get no tangent. */
__device__ void angle_dual_straight(const double* t1, const double* t2, const double* t3,
                                    const float* w1, const float* w2, const float* w3, Dual pa[3],
                                    Dual pc[3]) {
    Dual ba[3], bc[3];
    for (int a = 0; a < 3; ++a) {
        ba[a] = {t1[a] - t2[a], (double)w1[a] - (double)w2[a]};
        bc[a] = {t3[a] - t2[a], (double)w3[a] - (double)w2[a]};
    }
    const double cx = ba[1].v * bc[2].v - ba[2].v * bc[1].v;
    const double cy = ba[2].v * bc[0].v - ba[0].v * bc[2].v;
    const double cz = ba[0].v * bc[1].v - ba[1].v * bc[0].v;
    if (cx == 0.0 && cy == 0.0 && cz == 0.0) {
        for (int a = 0; a < 3; ++a) pa[a] = pc[a] = dl(0.0);
        return;
    }
    const Dual l_ba = dsqrt(ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2]);
    const Dual l_bc = dsqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    Dual u[3], w[3];
    for (int a = 0; a < 3; ++a) {
        u[a] = ba[a] / l_ba;
        w[a] = bc[a] / l_bc;
    }
    const Dual c = u[0] * w[0] + u[1] * w[1] + u[2] * w[2];
    const Dual q = (u[0] + w[0]) * (u[0] + w[0]) + (u[1] + w[1]) * (u[1] + w[1]) +
                   (u[2] + w[2]) * (u[2] + w[2]);
    Dual G;
    if (q.v < 1e-2) {
        /* phi^2 = q + q^2/12 + q^3/90;  -G = 1 + p/6 + 7p^2/360 + 31p^3/15120 */
        const Dual p = q + q * q * (1.0 / 12.0) + q * q * q * (1.0 / 90.0);
        G = (dl(1.0) + p * (1.0 / 6.0) + p * p * (7.0 / 360.0) + p * p * p * (31.0 / 15120.0)) * -1.0;
    } else {
        const Dual sq = dsqrt(q);
        const double h = sq.v * 0.5;
        const Dual phi = {2.0 * asin(h), h < 1.0 ? sq.d / sqrt(1.0 - h * h) : 0.0};
        G = (phi / dsin(phi)) * -1.0;
    }
    const Dual sa = G * 2.0 / l_ba, sc = G * 2.0 / l_bc;
    for (int a = 0; a < 3; ++a) {
        pa[a] = (w[a] - c * u[a]) * sa;
        pc[a] = (u[a] - c * w[a]) * sc;
    }
}

/* Tangent of a central pair force f(r) r_hat along dr: (f/r)(dr - r_hat
   (r_hat.dr)) + f'(r) r_hat (r_hat.dr). */
__device__ __forceinline__ void central_tangent(double rx, double ry, double rz, double r, double f,
                                                double fp, double dx, double dy, double dz, double& tx,
                                                double& ty, double& tz) {
    const double ir = r > 0.0 ? 1.0 / r : 0.0;
    const double ux = rx * ir, uy = ry * ir, uz = rz * ir;
    const double ud = ux * dx + uy * dy + uz * dz;
    const double fr = f * ir;
    tx = fr * (dx - ux * ud) + fp * ux * ud;
    ty = fr * (dy - uy * ud) + fp * uy * ud;
    tz = fr * (dz - uz * ud) + fp * uz * ud;
}

/* Radial contact force f(r) and its derivative for one listed pair, under
   the same acting conditions as the step's contact term. */
__device__ __forceinline__ int contact_f(const FnNet& N, const FnPair* __restrict__ pairs, double4 pi,
                                         double4 pj, double r2, double& f, double& fp) {
    const FnPair* P = pairs + N.pair_base + getadress(w_type(pi.w), w_type(pj.w), N.types_num);
    const int kind = P->kind;
    const double r = sqrt(r2);
    if (kind == 1) {
        if (!(r2 < N.cutoff_sq) || !(r < P->c[2])) return 0;
        const double s2 = P->c[0] * P->c[0], eps = P->c[1];
        const double s6 = s2 * s2 * s2, s12 = s6 * s6;
        const double ir = 1.0 / r;
        const double ir2 = ir * ir, ir4 = ir2 * ir2, ir8 = ir4 * ir4;
        const double ir14 = ir8 * ir4 * ir2;
        f = 48.0 * eps * s12 * ir14 - 24.0 * eps * s6 * ir8 - P->c[3];
        fp = -672.0 * eps * s12 * ir14 * ir + 192.0 * eps * s6 * ir8 * ir;
        return 1;
    }
    const double rsum = (double)w_radius(pi.w) + (double)w_radius(pj.w);
    if (kind == 2) {
        if (!(rsum - r > 0.0)) return 0;
        f = P->c[0] * (rsum - r);
        fp = -P->c[0];
        return 1;
    }
    if (kind == 3) {
        if (!(r2 < P->c[3])) return 0;
        f = P->c[0] * (P->c[1] - r) + P->c[4] * (P->c[5] - r);
        fp = -(P->c[0] + P->c[4]);
        return 1;
    }
    if (kind == 4) {
        int acts = 0;
        f = 0.0;
        fp = 0.0;
        if (rsum - r > 0.0) {
            f += P->c[0] * (rsum - r);
            fp -= P->c[0];
            acts = 1;
        }
        if (r < P->c[2]) {
            f += P->c[1] * (P->c[2] - r);
            fp -= P->c[1];
            acts = 1;
        }
        return acts;
    }
    return 0;
}

struct AdjArgs {
    const FnTile* tiles;
    const FnNet* nets;
    const FnPair* pairs;
    const double4* pos;  /* positions of evaluation j */
    const double4* img;
    /* statuses after evaluation j: chain form per bead, else per bond */
    const unsigned char* ch_status;
    const signed char* sp_status;
    const signed char* an_status;
    const int2* sp_ends;
    const float4* sp_par;
    const signed char* sp_type;
    const int4* an_b;
    const float2* an_par;
    const int* sp_off;
    const int* sp_ent;
    const int* an_off;
    const int* an_ent;
    const int* list_count;
    const int* list;
    int list_stride, list_cap;
    int ns, na, nb;
    /* adjoint state */
    const double* minv; /* 1/mass per bead (0 for mass 0), the image positions' w */
    float4* X;
    float4* V;
    const float4* fbar;    /* Fbar of evaluation j */
    float4* fbar_next;     /* Fbar of evaluation j - 1 */
    float4* sp_tan;        /* per spring: tangent force on p1 */
    float4* an_tan;        /* per angle: tangent on b1, then on b3 (2 entries) */
    /* chain form: the same tangents by bead, so a bead reads its neighbours'
       slots instead of incidence lists: spring (j, j+1) at j as the tangent
       on bead j; angle centred on j at 2j (on bead j-1) and 2j+1 (on j+1);
       slots without a bond stay zero */
    float4* sp_tan_b;
    float4* an_tan_b;
    double2* g_spring;     /* d loss / d (k, rest) */
    double* g_angle;       /* d loss / d k */
    /* loss injection at evaluation j - 1: per network 3 doubles, or null */
    const double* lam_next;
    int reaction_type;
};

__device__ __forceinline__ bool spring_acts(const AdjArgs& A, int s, int2 e) {
    const int type = A.sp_type[s];
    if (!(type == 0 || type == 1)) return false;
    return A.ch_status ? (A.ch_status[min(e.x, e.y)] & 1) : (A.sp_status[s] == 1);
}

/* Per spring and per angle: tangent forces along Fbar and the parameter
   gradients (one thread per bond: no atomics, FP64 accumulators). */
__global__ void __launch_bounds__(256) k_adj_bonds(const AdjArgs A) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < A.ns) {
        const int s = t;
        const int2 e = A.sp_ends[s];
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (spring_acts(A, s, e)) {
            const double4 a = A.img[e.x], b = A.img[e.y];
            const float4 par = A.sp_par[s];
            const float4 w1 = A.fbar[e.x], w2 = A.fbar[e.y];
            const double rx = a.x - b.x, ry = a.y - b.y, rz = a.z - b.z;
            const double L = sqrt(rx * rx + ry * ry + rz * rz);
            const double dx = (double)w1.x - (double)w2.x, dy = (double)w1.y - (double)w2.y,
                         dz = (double)w1.z - (double)w2.z;
            const double k = par.y, rest = par.x;
            double tx, ty, tz;
            central_tangent(rx, ry, rz, L, k * (rest - L), -k, dx, dy, dz, tx, ty, tz);
            out = make_float4((float)tx, (float)ty, (float)tz, 0.f);
            const double ud = L > 0.0 ? (rx * dx + ry * dy + rz * dz) / L : 0.0;
            double2 g = A.g_spring[s];
            g.x += (rest - L) * ud;
            g.y += k * ud;
            A.g_spring[s] = g;
        }
        if (A.sp_tan_b) {
            if (e.x < e.y)
                A.sp_tan_b[e.x] = out;
            else
                A.sp_tan_b[e.y] = make_float4(-out.x, -out.y, -out.z, 0.f);
        } else {
            A.sp_tan[s] = out;
        }
        return;
    }
    const int q = t - A.ns;
    if (q >= A.na) return;
    const int4 b = A.an_b[q];
    const int alive = A.ch_status ? ((A.ch_status[b.y] >> 1) & 1) : (A.an_status[q] == 1);
    float4 o1 = make_float4(0.f, 0.f, 0.f, 0.f), o3 = o1;
    if (alive) {
        const double4 p1 = A.img[b.x], p2 = A.img[b.y], p3 = A.img[b.z];
        const float4 w1 = A.fbar[b.x], w2 = A.fbar[b.y], w3 = A.fbar[b.z];
        const double t1[3] = {p1.x, p1.y, p1.z}, t2[3] = {p2.x, p2.y, p2.z}, t3[3] = {p3.x, p3.y, p3.z};
        const float f1[3] = {w1.x, w1.y, w1.z}, f2[3] = {w2.x, w2.y, w2.z}, f3[3] = {w3.x, w3.y, w3.z};
        const float2 par = A.an_par[q];
        Dual pa[3], pc[3];
        if (fabs((double)par.x - 3.14159265358979323846) < 1e-6)
            angle_dual_straight(t1, t2, t3, f1, f2, f3, pa, pc);
        else
            angle_dual(t1, t2, t3, f1, f2, f3, (double)par.x, pa, pc);
        const double k = par.y;
        o1 = make_float4((float)(k * pa[0].d), (float)(k * pa[1].d), (float)(k * pa[2].d), 0.f);
        o3 = make_float4((float)(k * pc[0].d), (float)(k * pc[1].d), (float)(k * pc[2].d), 0.f);
        double g = 0.0;
        const double F1[3] = {f1[0], f1[1], f1[2]}, F2[3] = {f2[0], f2[1], f2[2]},
                     F3[3] = {f3[0], f3[1], f3[2]};
        for (int a = 0; a < 3; ++a) g += pa[a].v * (F1[a] - F2[a]) + pc[a].v * (F3[a] - F2[a]);
        A.g_angle[q] += g;
    }
    if (A.an_tan_b) {
        const bool fwd = b.x < b.y;
        A.an_tan_b[2 * (size_t)b.y] = fwd ? o1 : o3;
        A.an_tan_b[2 * (size_t)b.y + 1] = fwd ? o3 : o1;
    } else {
        A.an_tan[2 * (size_t)q] = o1;
        A.an_tan[2 * (size_t)q + 1] = o3;
    }
}

/* Per bead: X += (J Fbar)_i from the bond tangents, the contacts of its
   list and the walls; then the prologue of evaluation j - 1:
   V += dt X, Fbar_{j-1} = (dt/m) V + loss injection. */
template <bool CHAIN>
__global__ void __launch_bounds__(512) k_adj_beads(const AdjArgs A) {
    const FnTile tl = A.tiles[blockIdx.x];
    const int i = tl.begin + (int)threadIdx.x;
    if (i >= tl.end) return;
    const FnNet& N = A.nets[tl.net];
    const double4 p = A.pos[i];
    const float4 wi = A.fbar[i];
    double jx = 0.0, jy = 0.0, jz = 0.0;
    if (CHAIN) {
        /* spring (i-1, i), spring (i, i+1); angles centred on i-1, i, i+1 */
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 sp = i > 0 ? A.sp_tan_b[i - 1] : zero;
        const float4 sn = A.sp_tan_b[i];
        const float4 ap = i > 0 ? A.an_tan_b[2 * (size_t)(i - 1) + 1] : zero;
        const float4 c0 = A.an_tan_b[2 * (size_t)i], c1 = A.an_tan_b[2 * (size_t)i + 1];
        const float4 an = i + 1 < A.nb ? A.an_tan_b[2 * (size_t)(i + 1)] : zero;
        jx += -(double)sp.x + (double)sn.x + (double)ap.x - ((double)c0.x + (double)c1.x) + (double)an.x;
        jy += -(double)sp.y + (double)sn.y + (double)ap.y - ((double)c0.y + (double)c1.y) + (double)an.y;
        jz += -(double)sp.z + (double)sn.z + (double)ap.z - ((double)c0.z + (double)c1.z) + (double)an.z;
    }
    for (int e = CHAIN ? 0 : A.sp_off[i]; e < (CHAIN ? 0 : A.sp_off[i + 1]); ++e) {
        const int ent = A.sp_ent[e];
        const float4 t = A.sp_tan[ent >> 1];
        const double sg = (ent & 1) ? -1.0 : 1.0;
        jx += sg * (double)t.x;
        jy += sg * (double)t.y;
        jz += sg * (double)t.z;
    }
    for (int e = CHAIN ? 0 : A.an_off[i]; e < (CHAIN ? 0 : A.an_off[i + 1]); ++e) {
        const int ent = A.an_ent[e];
        const int q = ent >> 2, role = ent & 3;
        if (role == 0) {
            const float4 t1 = A.an_tan[2 * (size_t)q];
            jx += t1.x;
            jy += t1.y;
            jz += t1.z;
        } else if (role == 2) {
            const float4 t3 = A.an_tan[2 * (size_t)q + 1];
            jx += t3.x;
            jy += t3.y;
            jz += t3.z;
        } else {
            const float4 t1 = A.an_tan[2 * (size_t)q], t3 = A.an_tan[2 * (size_t)q + 1];
            jx -= (double)t1.x + (double)t3.x;
            jy -= (double)t1.y + (double)t3.y;
            jz -= (double)t1.z + (double)t3.z;
        }
    }
    int n = A.list_count[i];
    if (n > A.list_cap) n = A.list_cap;
    for (int k = 0; k < n; ++k) {
        const int j = A.list[(size_t)k * A.list_stride + i];
        const double4 pj = A.pos[j];
        double rx = p.x - pj.x, ry = p.y - pj.y, rz = p.z - pj.z;
        double r2 = rx * rx + ry * ry + rz * rz;
        r2 = min_image(N, rx, ry, rz, r2, N.force_mi);
        double f, fp;
        if (!contact_f(N, A.pairs, p, pj, r2, f, fp)) continue;
        const float4 wj = A.fbar[j];
        double tx, ty, tz;
        central_tangent(rx, ry, rz, sqrt(r2), f, fp, (double)wi.x - (double)wj.x,
                        (double)wi.y - (double)wj.y, (double)wi.z - (double)wj.z, tx, ty, tz);
        jx += tx;
        jy += ty;
        jz += tz;
    }
    if (N.walls) {
        if ((N.walls & 1) && (p.x < 0.0 || p.x > N.box[0])) jx -= N.wall_k * (double)wi.x;
        if ((N.walls & 2) && (p.y < 0.0 || p.y > N.box[1])) jy -= N.wall_k * (double)wi.y;
        if ((N.walls & 4) && (p.z < 0.0 || p.z > N.box[2])) jz -= N.wall_k * (double)wi.z;
    }
    float4 X = A.X[i];
    X.x = (float)((double)X.x + jx);
    X.y = (float)((double)X.y + jy);
    X.z = (float)((double)X.z + jz);
    A.X[i] = X;
    /* prologue of evaluation j - 1 */
    const double minv = A.minv[i];
    float4 V = A.V[i];
    V.x = (float)((double)V.x + N.dt * (double)X.x);
    V.y = (float)((double)V.y + N.dt * (double)X.y);
    V.z = (float)((double)V.z + N.dt * (double)X.z);
    A.V[i] = V;
    double fx = N.dt * minv * (double)V.x, fy = N.dt * minv * (double)V.y, fz = N.dt * minv * (double)V.z;
    if (A.lam_next && w_type(p.w) == A.reaction_type) {
        fx += A.lam_next[3 * tl.net];
        fy += A.lam_next[3 * tl.net + 1];
        fz += A.lam_next[3 * tl.net + 2];
    }
    A.fbar_next[i] = make_float4((float)fx, (float)fy, (float)fz, 0.f);
}

/* Fbar of the last evaluation: the loss injection alone (X = V = 0). */
__global__ void k_adj_start(const AdjArgs A) {
    const FnTile tl = A.tiles[blockIdx.x];
    const int i = tl.begin + (int)threadIdx.x;
    if (i >= tl.end) return;
    float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
    if (A.lam_next && w_type(A.pos[i].w) == A.reaction_type)
        f = make_float4((float)A.lam_next[3 * tl.net], (float)A.lam_next[3 * tl.net + 1],
                        (float)A.lam_next[3 * tl.net + 2], 0.f);
    A.fbar_next[i] = f;
    A.X[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    A.V[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

/* Reaction of every network at once: blocks (chunk, network) sum the force
   on beads of the reaction type over 2048-bead chunks, then one thread per
   network adds its chunks in order (fixed-order FP64 reduction). */
constexpr int kReactionChunk = 2048;

__global__ void __launch_bounds__(256) k_reaction_partial(const FnNet* nets, const double4* pos,
                                                          const float4* force, int reaction_type,
                                                          double* partial) {
    __shared__ double sx[256], sy[256], sz[256];
    const FnNet& N = nets[blockIdx.y];
    const int begin = N.bead_begin + blockIdx.x * kReactionChunk;
    const int end = min(N.bead_end, begin + kReactionChunk);
    double x = 0.0, y = 0.0, z = 0.0;
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
        if (w_type(pos[i].w) == reaction_type) {
            const float4 f = force[i];
            x += (double)f.x;
            y += (double)f.y;
            z += (double)f.z;
        }
    }
    sx[threadIdx.x] = x;
    sy[threadIdx.x] = y;
    sz[threadIdx.x] = z;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sx[threadIdx.x] += sx[threadIdx.x + o];
            sy[threadIdx.x] += sy[threadIdx.x + o];
            sz[threadIdx.x] += sz[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* o = partial + 3 * ((size_t)blockIdx.y * gridDim.x + blockIdx.x);
        o[0] = sx[0];
        o[1] = sy[0];
        o[2] = sz[0];
    }
}

__global__ void k_reaction_final(const double* partial, int nchunks, int n_nets, double* out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nets) return;
    double x = 0.0, y = 0.0, z = 0.0;
    for (int k = 0; k < nchunks; ++k) {
        const double* p = partial + 3 * ((size_t)n * nchunks + k);
        x += p[0];
        y += p[1];
        z += p[2];
    }
    out[3 * n] = x;
    out[3 * n + 1] = y;
    out[3 * n + 2] = z;
}

/* Copies the first max(count) columns of a column-major contact list. */
__global__ void k_list_max(const int* count, int n, int cap, int* kmax) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) atomicMax(kmax, min(count[i], cap));
}

__global__ void k_list_copy(const int* count, const int* list, int n, int stride, const int* kmax,
                            int* count_out, int* list_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    count_out[i] = count[i];
    const int km = *kmax;
    for (int k = 0; k < km; ++k) list_out[(size_t)k * stride + i] = list[(size_t)k * stride + i];
}

/* 1/mass of every bead, read once from the image positions' w. */
__global__ void k_take_minv(const double4* img, int n, double* minv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) minv[i] = img[i].w;
}

/* Counts beads whose positions differ bit-wise between two buffers. */
__global__ void k_count_diff(const double4* a, const double4* b, int n, unsigned long long* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 x = a[i], y = b[i];
    if (__double_as_longlong(x.x) != __double_as_longlong(y.x) ||
        __double_as_longlong(x.y) != __double_as_longlong(y.y) ||
        __double_as_longlong(x.z) != __double_as_longlong(y.z))
        atomicAdd(out, 1ull);
}

}  // namespace fn

/* ======================================================================== */

namespace fnh {

struct AdjointState {
    int every = 0, nsamples = 0, ckpt_every = 0, reaction_type = -1;
    int nckpt = 0;          /* checkpoints 0..nckpt-1, slot nckpt = final state */
    long long version = -1; /* context state version right after the forward */
    size_t st_bytes = 0;    /* status bytes per step record */
    DevBuf<double4> ck_pos, ck_img;
    DevBuf<float4> ck_vold, ck_force, ck_vel;
    DevBuf<unsigned char> ck_st;
    DevBuf<int> saved_count, saved_list;
    DevBuf<double> reaction; /* nsamples x n_nets x 3 */
    /* replay */
    DevBuf<double4> rec_pos, rec_img;
    DevBuf<unsigned char> rec_st;
    DevBuf<int> rec_count, rec_list, kmax; /* the contact list of each rebuild in the segment */
    DevBuf<double> react_partial;
    int nchunks = 1;
    /* adjoint */
    DevBuf<float4> X, V, fbar[2], sp_tan, an_tan, sp_tan_b, an_tan_b;
    DevBuf<double> minv;
    DevBuf<double2> g_spring;
    DevBuf<double> g_angle, lam;
    DevBuf<unsigned long long> diff;
};

void adjoint_free(fn_ctx* c) {
    AdjointState* S = c->adj;
    if (!S) return;
    dfree(c, S->ck_pos);
    dfree(c, S->ck_img);
    dfree(c, S->ck_vold);
    dfree(c, S->ck_force);
    dfree(c, S->ck_vel);
    dfree(c, S->ck_st);
    dfree(c, S->saved_count);
    dfree(c, S->saved_list);
    dfree(c, S->reaction);
    dfree(c, S->rec_pos);
    dfree(c, S->rec_img);
    dfree(c, S->rec_st);
    dfree(c, S->rec_count);
    dfree(c, S->rec_list);
    dfree(c, S->kmax);
    dfree(c, S->react_partial);
    dfree(c, S->X);
    dfree(c, S->minv);
    dfree(c, S->V);
    dfree(c, S->fbar[0]);
    dfree(c, S->fbar[1]);
    dfree(c, S->sp_tan);
    dfree(c, S->an_tan);
    dfree(c, S->sp_tan_b);
    dfree(c, S->an_tan_b);
    dfree(c, S->g_spring);
    dfree(c, S->g_angle);
    dfree(c, S->lam);
    dfree(c, S->diff);
    delete S;
    c->adj = nullptr;
}

namespace {

/* Grows a buffer to at least n elements (buffers are kept between calls so
   a fitting loop allocates once). */
template <class T>
cudaError_t ensure(fn_ctx* c, DevBuf<T>& b, size_t n) {
    if (b.p && b.n >= n) return cudaSuccess;
    return dalloc(c, b, n);
}

size_t status_bytes(fn_ctx* c) { return c->chain ? (size_t)c->nb : (size_t)(c->ns + c->na); }

/* status arrays of the context <-> one record */
int save_status(fn_ctx* c, unsigned char* dst) {
    if (c->chain) {
        CK(cudaMemcpyAsync(dst, c->ch_status.p, c->nb, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        if (c->ns) CK(cudaMemcpyAsync(dst, c->sp_status.p, c->ns, cudaMemcpyDeviceToDevice, c->stream));
        if (c->na) CK(cudaMemcpyAsync(dst + c->ns, c->an_status.p, c->na, cudaMemcpyDeviceToDevice, c->stream));
    }
    return FN_OK;
}

int load_status(fn_ctx* c, const unsigned char* src) {
    if (c->chain) {
        CK(cudaMemcpyAsync(c->ch_status.p, src, c->nb, cudaMemcpyDeviceToDevice, c->stream));
    } else {
        if (c->ns) CK(cudaMemcpyAsync(c->sp_status.p, src, c->ns, cudaMemcpyDeviceToDevice, c->stream));
        if (c->na) CK(cudaMemcpyAsync(c->an_status.p, src + c->ns, c->na, cudaMemcpyDeviceToDevice, c->stream));
    }
    return FN_OK;
}

int save_checkpoint(fn_ctx* c, int slot) {
    AdjointState* S = c->adj;
    const size_t nb = (size_t)c->nb, o = (size_t)slot * nb;
    CK(cudaMemcpyAsync(S->ck_pos.p + o, c->pos[c->cur].p, nb * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(S->ck_img.p + o, c->img[c->cur].p, nb * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(S->ck_vold.p + o, c->vold.p, nb * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(S->ck_force.p + o, c->force.p, nb * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(S->ck_vel.p + o, c->vel.p, nb * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    return save_status(c, S->ck_st.p + (size_t)slot * S->st_bytes);
}

int load_checkpoint(fn_ctx* c, int slot) {
    AdjointState* S = c->adj;
    const size_t nb = (size_t)c->nb, o = (size_t)slot * nb;
    c->cur = 0;
    CK(cudaMemcpyAsync(c->pos[0].p, S->ck_pos.p + o, nb * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->img[0].p, S->ck_img.p + o, nb * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->vold.p, S->ck_vold.p + o, nb * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->force.p, S->ck_force.p + o, nb * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->vel.p, S->ck_vel.p + o, nb * sizeof(float4), cudaMemcpyDeviceToDevice, c->stream));
    return load_status(c, S->ck_st.p + (size_t)slot * S->st_bytes);
}

int launch_step_args(fn_ctx* c, const fn::StepArgs& A, bool do_drift, bool store_v) {
    return launch_step_kernel(c, A, do_drift, store_v);
}

int rebuild_from(fn_ctx* c, const double4* pos) {
    fn::RebuildArgs R = rebuild_args(c);
    R.pos = pos;
    CK(fn::launch_rebuild(R, c->ntiles, c->block, (int)c->nb, c->ncells, c->scan_sums.p, c->stream));
    return FN_OK;
}

/* Records the current contact list (its used columns only) in slot. */
int save_list(fn_ctx* c, int slot) {
    AdjointState* S = c->adj;
    const size_t nb = (size_t)c->nb, stride = (size_t)c->list_stride;
    CK(cudaMemsetAsync(S->kmax.p, 0, sizeof(int), c->stream));
    const int nblk = (int)((nb + 255) / 256);
    fn::k_list_max<<<nblk, 256, 0, c->stream>>>(c->list_count.p, (int)nb, c->cfg.list_capacity, S->kmax.p);
    fn::k_list_copy<<<nblk, 256, 0, c->stream>>>(c->list_count.p, c->list.p, (int)nb, (int)stride, S->kmax.p,
                                                  S->rec_count.p + (size_t)slot * nb,
                                                  S->rec_list.p + (size_t)slot * stride * c->cfg.list_capacity);
    CK(cudaGetLastError());
    return FN_OK;
}

/* Evaluation index (within a segment) where the contact list used by each
   evaluation was built: the schedule of fn_step (a call opens with a drift,
   then rebuild-led runs of grid_update_freq steps). */
std::vector<int> rebuild_points(int every, int gu, int K) {
    std::vector<int> at(K);
    for (int call0 = 0; call0 < K; call0 += every)
        for (int done = 0; done < every;) {
            const int len = std::min(gu, every - done);
            for (int k = 0; k < len; ++k) at[call0 + done + k] = call0 + done;
            done += len;
        }
    return at;
}

/* Replays segment q from its checkpoint: evaluation positions into
   rec_pos/rec_img[0..K), statuses after each evaluation into rec_st. */
int replay_segment(fn_ctx* c, int q) {
    AdjointState* S = c->adj;
    const int K = S->ckpt_every, every = S->every, gu = c->grid_update_freq;
    const size_t nb = (size_t)c->nb;
    int r = load_checkpoint(c, q);
    if (r) return r;
    int slot = 0;
    auto P = [&](int j) { return S->rec_pos.p + (size_t)j * nb; };
    auto I = [&](int j) { return S->rec_img.p + (size_t)j * nb; };
    for (int call0 = 0; call0 < K; call0 += every) {
        fn::StepArgs A = step_args(c, false);
        if (call0 > 0) {
            A.pos_in = P(call0 - 1);
            A.img_in = I(call0 - 1);
        }
        A.pos_out = P(call0);
        A.img_out = I(call0);
        CK(fn::launch_drift(A, c->ntiles, c->block, c->damp || every == 1, c->stream));
        for (int done = 0; done < every;) {
            const int len = std::min(gu, every - done);
            const bool tail = done + len == every;
            r = rebuild_from(c, P(call0 + done));
            if (r) return r;
            r = save_list(c, slot++);
            if (r) return r;
            for (int k = 0; k < len; ++k) {
                const int j = call0 + done + k;
                const bool last = tail && k == len - 1;
                fn::StepArgs B = step_args(c, true);
                B.pos_in = P(j);
                B.img_in = I(j);
                B.pos_out = last ? P(j) : P(j + 1);
                B.img_out = last ? I(j) : I(j + 1);
                r = launch_step_args(c, B, !last, tail && k == len - 2);
                if (r) return r;
                r = save_status(c, S->rec_st.p + (size_t)j * S->st_bytes);
                if (r) return r;
            }
            done += len;
        }
    }
    /* the replay must land on the next checkpoint bit for bit */
    CK(cudaMemsetAsync(S->diff.p, 0, sizeof(unsigned long long), c->stream));
    const int nblk = (int)((nb + 255) / 256);
    fn::k_count_diff<<<nblk, 256, 0, c->stream>>>(P(K - 1), S->ck_pos.p + (size_t)(q + 1) * nb, (int)nb,
                                                     S->diff.p);
    fn::k_count_diff<<<nblk, 256, 0, c->stream>>>(I(K - 1), S->ck_img.p + (size_t)(q + 1) * nb, (int)nb,
                                                     S->diff.p);
    CK(cudaGetLastError());
    unsigned long long bad = 0;
    CK(cudaMemcpyAsync(&bad, S->diff.p, sizeof bad, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (bad) return fail(c, FN_ERR_STATE, "adjoint: replay of segment " + std::to_string(q) +
                                              " diverged from the forward pass");
    return FN_OK;
}

fn::AdjArgs adj_args(fn_ctx* c, int j_local, int parity) {
    AdjointState* S = c->adj;
    const size_t nb = (size_t)c->nb;
    fn::AdjArgs A{};
    A.tiles = c->tiles.p;
    A.nets = c->nets.p;
    A.pairs = c->pairs.p;
    A.pos = S->rec_pos.p + (size_t)j_local * nb;
    A.img = S->rec_img.p + (size_t)j_local * nb;
    const unsigned char* st = S->rec_st.p + (size_t)j_local * S->st_bytes;
    if (c->chain) {
        A.ch_status = st;
    } else {
        A.sp_status = (const signed char*)st;
        A.an_status = (const signed char*)(st + c->ns);
    }
    A.sp_ends = c->sp_ends.p;
    A.sp_par = c->sp_par.p;
    A.sp_type = c->sp_type.p;
    A.an_b = c->an_b.p;
    A.an_par = c->an_par.p;
    A.sp_off = c->sp_off.p;
    A.sp_ent = c->sp_ent.p;
    A.an_off = c->an_off.p;
    A.an_ent = c->an_ent.p;
    A.list_count = c->list_count.p;
    A.list = c->list.p;
    A.list_stride = c->list_stride;
    A.list_cap = c->cfg.list_capacity;
    A.ns = (int)c->ns;
    A.na = (int)c->na;
    A.nb = (int)c->nb;
    if (c->chain) {
        A.sp_tan_b = S->sp_tan_b.p;
        A.an_tan_b = S->an_tan_b.p;
    }
    A.minv = S->minv.p;
    A.X = S->X.p;
    A.V = S->V.p;
    A.fbar = S->fbar[parity].p;
    A.fbar_next = S->fbar[1 - parity].p;
    A.sp_tan = S->sp_tan.p;
    A.an_tan = S->an_tan.p;
    A.g_spring = S->g_spring.p;
    A.g_angle = S->g_angle.p;
    A.reaction_type = S->reaction_type;
    return A;
}

}  // namespace
}  // namespace fnh

using namespace fnh;

extern "C" {

FN_API int fn_adjoint_forward(fn_ctx* c, int nsamples, int every, int checkpoint_every, int reaction_type,
                              double* reaction) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_adjoint_forward");
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    if (nsamples <= 0 || every <= 0 || checkpoint_every <= 0 || checkpoint_every % every != 0)
        return fail(c, FN_ERR_ARG, "fn_adjoint_forward: checkpoint_every must be a positive multiple of every");
    if (c->damp) return fail(c, FN_ERR_ARG, "fn_adjoint_forward: damping must be 0 (velocity-dependent forces are not differentiated)");
    if (c->verlet) return fail(c, FN_ERR_ARG, "fn_adjoint_forward: needs the fixed rebuild cadence (verlet_skin 0)");
    CK(cudaSetDevice(c->cfg.device));
    const long long total = (long long)nsamples * every;
    if (total % checkpoint_every != 0)
        return fail(c, FN_ERR_ARG, "fn_adjoint_forward: nsamples * every must be a multiple of checkpoint_every");
    if (!c->adj) c->adj = new AdjointState();
    AdjointState* S = c->adj;
    S->version = -1;
    S->every = every;
    S->nsamples = nsamples;
    S->ckpt_every = checkpoint_every;
    S->reaction_type = reaction_type;
    S->nckpt = (int)(total / checkpoint_every);
    S->st_bytes = status_bytes(c);
    const size_t nb = (size_t)c->nb, slots = (size_t)S->nckpt + 1;
    CK(ensure(c, S->ck_pos, slots * nb));
    CK(ensure(c, S->ck_img, slots * nb));
    CK(ensure(c, S->ck_vold, slots * nb));
    CK(ensure(c, S->ck_force, slots * nb));
    CK(ensure(c, S->ck_vel, slots * nb));
    CK(ensure(c, S->ck_st, slots * S->st_bytes));
    CK(ensure(c, S->saved_count, nb));
    CK(ensure(c, S->saved_list, (size_t)c->list_stride * c->cfg.list_capacity));
    CK(ensure(c, S->reaction, (size_t)nsamples * c->n_nets * 3));
    int maxb = 1;
    for (int k = 0; k < c->n_nets; ++k) maxb = std::max(maxb, c->info[k].bead_end - c->info[k].bead_begin);
    S->nchunks = (maxb + fn::kReactionChunk - 1) / fn::kReactionChunk;
    CK(ensure(c, S->react_partial, (size_t)3 * S->nchunks * c->n_nets));
    for (int s = 0; s < nsamples; ++s) {
        if (((long long)s * every) % checkpoint_every == 0) {
            r = save_checkpoint(c, (int)(((long long)s * every) / checkpoint_every));
            if (r) return r;
        }
        r = fn_step(c, every);
        if (r) return r;
        fn::k_reaction_partial<<<dim3(S->nchunks, c->n_nets), 256, 0, c->stream>>>(
            c->nets.p, c->pos[c->cur].p, c->force.p, reaction_type, S->react_partial.p);
        fn::k_reaction_final<<<(c->n_nets + 127) / 128, 128, 0, c->stream>>>(
            S->react_partial.p, S->nchunks, c->n_nets, S->reaction.p + (size_t)s * c->n_nets * 3);
        CK(cudaGetLastError());
    }
    r = save_checkpoint(c, S->nckpt);
    if (r) return r;
    CK(cudaMemcpyAsync(S->saved_count.p, c->list_count.p, nb * sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(S->saved_list.p, c->list.p, (size_t)c->list_stride * c->cfg.list_capacity * sizeof(int),
                       cudaMemcpyDeviceToDevice, c->stream));
    if (reaction)
        CK(cudaMemcpyAsync(reaction, S->reaction.p, sizeof(double) * (size_t)nsamples * c->n_nets * 3,
                           cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    S->version = c->state_version;
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_adjoint_backward(fn_ctx* c, const double* dloss_dreaction, double* grad_spring_k,
                               double* grad_spring_rest, double* grad_angle_k, double* grad_pos0,
                               double* grad_vel0) {
    FN_TRY
    fnh::NvtxRange nvtx_range_("fn_adjoint_backward");
    int r = check_ready(c);
    if (r) return r;
    if ((r = ensure_host(c))) return r;
    AdjointState* S = c->adj;
    if (!S || S->version != c->state_version)
        return fail(c, FN_ERR_STATE, "fn_adjoint_backward: no forward pass matches the current state");
    if (!dloss_dreaction) return fail(c, FN_ERR_ARG, "fn_adjoint_backward: null loss gradient");
    CK(cudaSetDevice(c->cfg.device));
    if (!c->chain) { /* the chain form gathers bond tangents by bead */
        r = ensure_incidence(c);
        if (r) return r;
    }
    const size_t nb = (size_t)c->nb;
    const int K = S->ckpt_every;
    CK(ensure(c, S->rec_pos, (size_t)K * nb));
    CK(ensure(c, S->rec_img, (size_t)K * nb));
    CK(ensure(c, S->rec_st, (size_t)K * S->st_bytes));
    const std::vector<int> rb = rebuild_points(S->every, c->grid_update_freq, K);
    std::vector<int> rb_slot(K);
    int nrb = 0;
    for (int j = 0; j < K; ++j) {
        if (j == 0 || rb[j] != rb[j - 1]) ++nrb;
        rb_slot[j] = nrb - 1;
    }
    CK(ensure(c, S->rec_count, (size_t)nrb * nb));
    CK(ensure(c, S->rec_list, (size_t)nrb * c->list_stride * c->cfg.list_capacity));
    CK(ensure(c, S->kmax, 1));
    CK(ensure(c, S->X, nb));
    CK(ensure(c, S->minv, nb));
    fn::k_take_minv<<<(int)((nb + 255) / 256), 256, 0, c->stream>>>(S->ck_img.p, (int)nb, S->minv.p);
    CK(cudaGetLastError());
    CK(ensure(c, S->V, nb));
    CK(ensure(c, S->fbar[0], nb));
    CK(ensure(c, S->fbar[1], nb));
    CK(ensure(c, S->sp_tan, (size_t)c->ns));
    CK(ensure(c, S->an_tan, 2 * (size_t)c->na));
    if (c->chain) {
        CK(ensure(c, S->sp_tan_b, nb));
        CK(ensure(c, S->an_tan_b, 2 * nb));
        CK(cudaMemsetAsync(S->sp_tan_b.p, 0, sizeof(float4) * nb, c->stream));
        CK(cudaMemsetAsync(S->an_tan_b.p, 0, sizeof(float4) * 2 * nb, c->stream));
    }
    CK(ensure(c, S->g_spring, (size_t)c->ns));
    CK(ensure(c, S->g_angle, (size_t)c->na));
    CK(ensure(c, S->diff, 1));
    const size_t nlam = (size_t)S->nsamples * c->n_nets * 3;
    CK(ensure(c, S->lam, nlam));
    CK(cudaMemcpyAsync(S->lam.p, dloss_dreaction, nlam * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(S->g_spring.p, 0, sizeof(double2) * S->g_spring.n, c->stream));
    CK(cudaMemsetAsync(S->g_angle.p, 0, sizeof(double) * S->g_angle.n, c->stream));

    const int every = S->every;
    const long long total = (long long)S->nsamples * every;
    /* loss injection of global evaluation j, or null */
    auto lam_at = [&](long long j) -> const double* {
        if (j < 0 || (j + 1) % every != 0) return nullptr;
        return S->lam.p + (size_t)((j + 1) / every - 1) * c->n_nets * 3;
    };
    const int nbond = (int)(c->ns + c->na);
    int parity = 0;
    {
        fn::AdjArgs A = adj_args(c, 0, 1);
        A.pos = S->ck_pos.p + (size_t)S->nckpt * nb;  /* types only */
        A.lam_next = lam_at(total - 1);
        fn::k_adj_start<<<c->ntiles, c->block, 0, c->stream>>>(A);
        CK(cudaGetLastError());
    }
    for (int q = S->nckpt - 1; q >= 0; --q) {
        r = replay_segment(c, q);
        if (r) return r;
        for (int jl = K - 1; jl >= 0; --jl) {
            const long long j = (long long)q * K + jl;
            fn::AdjArgs A = adj_args(c, jl, parity);
            A.list_count = S->rec_count.p + (size_t)rb_slot[jl] * nb;
            A.list = S->rec_list.p + (size_t)rb_slot[jl] * c->list_stride * c->cfg.list_capacity;
            A.lam_next = lam_at(j - 1);
            if (nbond > 0) {
                fn::k_adj_bonds<<<(nbond + 255) / 256, 256, 0, c->stream>>>(A);
                CK(cudaGetLastError());
            }
            if (c->chain)
                fn::k_adj_beads<true><<<c->ntiles, c->block, 0, c->stream>>>(A);
            else
                fn::k_adj_beads<false><<<c->ntiles, c->block, 0, c->stream>>>(A);
            CK(cudaGetLastError());
            parity = 1 - parity;
        }
    }
    /* back to the state the forward pass ended in */
    r = load_checkpoint(c, S->nckpt);
    if (r) return r;
    CK(cudaMemcpyAsync(c->list_count.p, S->saved_count.p, nb * sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->list.p, S->saved_list.p, (size_t)c->list_stride * c->cfg.list_capacity * sizeof(int),
                       cudaMemcpyDeviceToDevice, c->stream));

    std::vector<double2> gs(c->ns);
    std::vector<double> ga(c->na);
    std::vector<float4> X(nb), V(nb);
    if (c->ns) CK(cudaMemcpyAsync(gs.data(), S->g_spring.p, sizeof(double2) * c->ns, cudaMemcpyDeviceToHost, c->stream));
    if (c->na) CK(cudaMemcpyAsync(ga.data(), S->g_angle.p, sizeof(double) * c->na, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(X.data(), S->X.p, sizeof(float4) * nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(V.data(), S->V.p, sizeof(float4) * nb, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (long long s = 0; s < c->ns; ++s) {
        if (grad_spring_k) grad_spring_k[s] = gs[s].x;
        if (grad_spring_rest) grad_spring_rest[s] = gs[s].y;
    }
    if (grad_angle_k)
        for (long long a = 0; a < c->na; ++a) grad_angle_k[a] = ga[a];
    for (size_t q = 0; q < nb; ++q) {
        const size_t i = (size_t)c->perm[q];
        if (grad_pos0) {
            grad_pos0[3 * i] = X[q].x;
            grad_pos0[3 * i + 1] = X[q].y;
            grad_pos0[3 * i + 2] = X[q].z;
        }
        if (grad_vel0) {
            grad_vel0[3 * i] = V[q].x;
            grad_vel0[3 * i + 1] = V[q].y;
            grad_vel0[3 * i + 2] = V[q].z;
        }
    }
    return FN_OK;
    FN_CATCH(c)
}

FN_API int fn_adjoint_release(fn_ctx* c) {
    FN_TRY
    if (!c) return FN_ERR_ARG;
    cudaSetDevice(c->cfg.device);
    cudaStreamSynchronize(c->stream);
    adjoint_free(c);
    return FN_OK;
    FN_CATCH(c)
}

}  // extern "C"
