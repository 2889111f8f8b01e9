/*
 * fibrenet_generate.h -- seeded synthetic fibre placement (host only).
 *
 * No counterpart in the reference, which reads every model from a model file
 * (SimulationManager.cpp:1315-1364); the benchmark workloads are generated
 * because the reference ships none.
 */
#ifndef FIBRENET_GENERATE_H
#define FIBRENET_GENERATE_H

#ifdef __cplusplus
extern "C" {
#endif

#define FN_GEN_API __attribute__((visibility("default")))

/* Places n_fibres straight fibres of `beads` beads, writing their unwrapped
   bead positions to out[(f * beads + b) * 3 + axis].  periodic_mask: bit a =
   axis a periodic.  orient 0: direction uniform in xy with a z tilt uniform in
   +-tilt_deg; 1: uniform on the sphere.  min_sep > 0 keeps every bead at least
   that far from the beads placed before it.  Returns 0, 1 on bad arguments,
   2 when a fibre found no place in max_tries draws, 3 when host memory runs
   out. */
FN_GEN_API int fn_place_fibres(unsigned long long seed, int n_fibres, int beads, const double box[3],
                               int periodic_mask, double zlo, double zhi, double tilt_deg,
                               int orient, double spacing, double min_sep, int max_tries,
                               double* out);

#ifdef __cplusplus
}
#endif
#endif
