/*
 * harness.cu -- TEST INFRASTRUCTURE ONLY.
 *
 * The library's host engine (fn_engine.cu) built against the host stand-ins
 * of fake_cuda.h, with the kernel launchers stubbed, so that fn_create +
 * fn_upload run to completion on a machine without a GPU.  The hu_* entry
 * points expose what the upload staged (bead order, packed bead arrays,
 * spring ends, the bond path chosen) to tests/test_upload_host.py.
 */
#include "../../fibrenet_b200/csrc/fn_engine.cu"

namespace fn {
/* no kernel runs here: every launcher reports success and does nothing */
cudaError_t launch_energy(const EnergyArgs&, int, double*, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_export_xyz(const double4*, const int*, int, double*, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_export_xyz(const float4*, const int*, int, double*, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_step(const StepArgs&, int, int, bool, bool, bool, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_step_tiled(const StepArgs&, int, int, bool, bool, bool, cudaStream_t) { return cudaSuccess; }
cudaError_t prepare_step_tiled(size_t) { return cudaSuccess; }
cudaError_t launch_step_chain(const StepArgs&, int, int, bool, bool, bool, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_forces_chain(const StepArgs&, int, int, int, cudaStream_t) { return cudaSuccess; }
cudaError_t prepare_step_chain(size_t) { return cudaSuccess; }
cudaError_t launch_step_staged(const StepArgs&, int, int, bool, bool, bool, cudaStream_t) { return cudaSuccess; }
cudaError_t prepare_step_staged(size_t) { return cudaSuccess; }
cudaError_t launch_drift(const StepArgs&, int, int, bool, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_forces_only(const StepArgs&, int, int, int, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_reset_energy(float4*, float4*, float4*, int, cudaStream_t) { return cudaSuccess; }
long long scan_block_count(long long n) { return (n + 2047) / 2048; }
cudaError_t launch_rebuild(const RebuildArgs&, int, int, int, long long, int*, cudaStream_t) { return cudaSuccess; }
cudaError_t launch_observe(const ObserveArgs&, int, double*, cudaStream_t) { return cudaSuccess; }
/* the device path of fn_upload is never taken here (host_upload = 1) */
cudaError_t launch_upload_checks(const UpNet*, int, const UpRaw&, UpCheck*, int, int, int, unsigned char*,
                                 cudaStream_t) {
    return cudaErrorNotSupported;
}
cudaError_t launch_upload_runs(const UpNet*, int, const UpRaw&, const unsigned char*, int*, int*, int*, int*,
                               unsigned long long*, int, cudaStream_t) {
    return cudaErrorNotSupported;
}
cudaError_t launch_upload_convert(const UpNet*, int, const UpRaw&, const int*, const int*, const int*, const int*,
                                  int, int*, int*, double4*, double4*, float4*, float4*, float4*, int4*, int2*,
                                  float4*, signed char*, signed char*, int4*, int2*, float2*, signed char*, int, int,
                                  int, cudaStream_t) {
    return cudaErrorNotSupported;
}
cudaError_t launch_upload_chain(const int2*, const signed char*, const float4*, const int4*, const int2*,
                                const float2*, int*, int*, unsigned char*, unsigned char*, float4*, float2*,
                                unsigned char*, unsigned char*, int*, int*, int*, int, int, int, cudaStream_t) {
    return cudaErrorNotSupported;
}
cudaError_t launch_exclusive_scan(const int*, long long, int*, int*, cudaStream_t) { return cudaErrorNotSupported; }
cudaError_t launch_verlet_rebuild(const RebuildArgs&, const FnTile*, const double4*, double4*, double, int*, int,
                                  int, int, long long, int*, cudaStream_t) {
    return cudaSuccess;
}
}  // namespace fn

namespace fnh {
/* the adjoint state is never created here */
void adjoint_free(fn_ctx*) {}
}  // namespace fnh

#define HU_API extern "C" __attribute__((visibility("default")))

HU_API int hu_create(int reorder, int chain_mode, fn_ctx** out) {
    fn_config cfg = {0, 64, 64, reorder, 0, 128, chain_mode, 0.0, 1}; /* the host path under test */
    return fn_create(&cfg, out);
}
HU_API int hu_upload(fn_ctx* c, int n, const fn_network_desc* d) { return fn_upload(c, n, d); }
HU_API const char* hu_error(fn_ctx* c) { return fn_last_error(c); }
HU_API int hu_permutation(fn_ctx* c, int* perm) { return fn_get_permutation(c, perm); }
HU_API int hu_chain(fn_ctx* c) { return c->chain ? 1 : 0; }
/* packed bead arrays in internal order: position (.w radius/type) and image (.w 1/mass) */
HU_API void hu_beads(fn_ctx* c, double* pos4, double* img4) {
    std::memcpy(pos4, c->pos[0].p, sizeof(double4) * c->nb);
    std::memcpy(img4, c->img[0].p, sizeof(double4) * c->nb);
}
/* spring ends in internal numbering, as the device holds them */
HU_API void hu_springs(fn_ctx* c, int* ends) { std::memcpy(ends, c->sp_ends.p, sizeof(int2) * c->ns); }
/* the tile table every launch reads: (network, first bead, end bead) */
HU_API int hu_tiles(fn_ctx* c, int* out3, int cap) {
    for (int t = 0; t < c->ntiles && t < cap; ++t) {
        const FnTile& x = c->tiles.p[t];
        out3[3 * t] = x.net;
        out3[3 * t + 1] = x.begin;
        out3[3 * t + 2] = x.end;
    }
    return c->ntiles;
}
HU_API int hu_block(fn_ctx* c) { return c->block; }
/* bead -> spring incidence (CSR, internal numbering; entry = spring << 1 | end) */
HU_API void hu_spring_incidence(fn_ctx* c, int* off, int* ent) {
    std::memcpy(off, c->sp_off_h.data(), sizeof(int) * c->sp_off_h.size());
    std::memcpy(ent, c->sp_ent_h.data(), sizeof(int) * c->sp_ent_h.size());
}
/* network k's derived settings in the oracle's fo_get_derived layout */
HU_API void hu_net(fn_ctx* c, int k, double* out20) {
    const FnNet& N = c->nets_h[k];
    const double v[20] = {N.dt, N.half_dt, N.half_dt2, N.lambda_dt, N.damping, N.cutoff_sq, N.wall_k,
                          N.g[0], N.g[1], N.g[2], N.box[0], N.box[1], N.box[2],
                          N.step[0], N.step[1], N.step[2], N.half_box_sq, (double)N.nx, (double)N.ny,
                          (double)N.nz};
    std::memcpy(out20, v, sizeof v);
}
/* network k's pair table: 6 coefficients and the kind per pair */
HU_API int hu_pairs(fn_ctx* c, int k, double* coeffs6, int* kinds) {
    const int base = c->nets_h[k].pair_base, nt = c->nets_h[k].types_num, np = nt * (nt + 1) / 2;
    for (int p = 0; p < np; ++p) {
        std::memcpy(coeffs6 + 6 * p, c->pairs_h[base + p].c, sizeof(double) * 6);
        kinds[p] = c->pairs_h[base + p].kind;
    }
    return np;
}
/* chain-form records per bead (internal order): next spring rest, k, c1, c2
   and centred angle theta0, k */
HU_API void hu_chain_records(fn_ctx* c, float* sp4, float* an2) {
    std::memcpy(sp4, c->ch_sp.p, sizeof(float4) * c->nb);
    std::memcpy(an2, c->ch_an.p, sizeof(float2) * c->nb);
}
HU_API void hu_destroy(fn_ctx* c) { fn_destroy(c); }
