/*
 * fibrenet_io.h -- the reference's input, model and restart files, its XYZ
 * and .res outputs, and its Initialize/Run/Close flow, without the
 * interactive prompts (host code; the simulation runs through fibrenet.h).
 *
 * Formats: README.md:32-659.  Two parse modes:
 *   compat (strict = 0) reproduces SimulationManager's quirks:
 *     velocity_old.{y,z} = velocity.x (SimulationManager.cpp:1405-1407);
 *     HR_FL c1, c2 read with std::stoi (:1528-1529, "5.37" -> 5);
 *     rest angles read with std::stof (:1637);
 *     a missing 'lambda' is an error (:716-719);
 *     a missing 'box_wall_rep' forces a finite box (:2168);
 *     restart files written with 6 significant digits (:1906-1924).
 *   strict (strict = 1) reads every number as a double, sets velocity_old =
 *     velocity, defaults lambda to 0.5, keeps box_type when box_wall_rep is
 *     absent (walls then have stiffness 0) and writes restarts exactly (%.17g).
 * Both modes reject what the reference accepts with undefined behaviour
 * (pair lines with the wrong token count, bond indices out of range).
 */
#ifndef FIBRENET_IO_H
#define FIBRENET_IO_H

#include "fibrenet.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FN_IO_API __attribute__((visibility("default")))

typedef struct fn_input fn_input;

/* Run settings of an input file (SimulationManager.cpp:681-819, 979-1091). */
typedef struct fn_run_info {
    int run_steps;            /* 'run' */
    int output_freq;          /* 'output_freq' */
    int minimize_steps;       /* 'minimize_steps' */
    int minimize_substeps;    /* 'minimize_substeps' */
    int minimize_reset;       /* 'minimize_reset yes' */
    int export_position;      /* 'output_data position|all' */
    int export_velocity;
    int export_force;
    int has_skin_override;    /* 'modif_bead ... skin_radius' was used */
    int strict;
} fn_run_info;

/* Reads an input file and everything it names (model file, restart file)
   and applies modif_bead / modif_spring, in ReadInputFile's order
   (SimulationManager.cpp:1153-1171).  Relative model/restart paths are taken
   relative to the current directory, as the reference does.  Returns FN_OK
   or FN_ERR_ARG with the reason in err (may be null). */
FN_IO_API int fn_input_read(const char* input_path, int strict, fn_input** out, char* err,
                            int err_len);
FN_IO_API void fn_input_free(fn_input* in);

/* The parsed network as an upload descriptor (arrays owned by `in`). */
FN_IO_API int fn_input_desc(const fn_input* in, fn_network_desc* out);
FN_IO_API int fn_input_info(const fn_input* in, fn_run_info* out);
/* Per-bead skin radius (only meaningful when has_skin_override). */
FN_IO_API const double* fn_input_skin(const fn_input* in);
/* Name of bead type t ('type' lines, in order), or null. */
FN_IO_API const char* fn_input_type_name(const fn_input* in, int t);
/* Output file stem ('output_file'). */
FN_IO_API const char* fn_input_output_stem(const fn_input* in);

/* Initialize + Run + Close of SimulationManager (SimulationManager.cpp:8-103):
   optional minimisation, RunSimulationLoop in output_freq chunks, an XYZ
   frame per chunk for each exported quantity, restart files at 25/50/75% and
   at the end.  Output names: <stem>_coord.xyz, _vel.xyz, _force.xyz,
   _restart.res (:991-994), next to the current directory.  log may be null
   (then stderr). */
FN_IO_API int fn_run_input(const char* input_path, int device, int strict, char* err, int err_len);

#ifdef __cplusplus
}
#endif
#endif
