/*
 * fibrenet.h -- C ABI of the B200 FibreNet step loop.
 *
 * Replaces the reference's device layer (OpenclManager + BufferIndex, used
 * only by SimulationManager) with one opaque context per simulation: the
 * context owns every device buffer, host pointers are borrowed for the
 * duration of a call, and every entry point returns an int status
 * (FN_OK = 0) instead of the reference's bool / negative int.  Calls on one
 * context are not thread-safe; separate contexts are independent.
 *
 * Units, field meanings and file semantics are the reference's
 * (README.md:32-659).  Bead, spring and angle indices are the model-file
 * order; the context may renumber beads internally but every call here uses
 * the caller's numbering.
 */
#ifndef FIBRENET_H
#define FIBRENET_H

#ifdef __cplusplus
extern "C" {
#endif

#define FN_API __attribute__((visibility("default")))

/* status codes */
enum {
    FN_OK = 0,
    FN_ERR_ARG = 1,        /* bad argument (null, size, index out of range) */
    FN_ERR_CUDA = 2,       /* CUDA runtime error (text in fn_last_error) */
    FN_ERR_OOM = 3,        /* device allocation failed */
    FN_ERR_CAPACITY = 4,   /* a cell or contact list exceeded its capacity */
    FN_ERR_STATE = 5,      /* call out of order (e.g. step before upload) */
    FN_ERR_NONFINITE = 6,  /* NaN/inf detected in the state */
    FN_ERR_UNSUPPORTED = 7 /* request outside what this build implements */
};

/* bead fields for fn_download / fn_set_beads (3 doubles per bead) */
enum {
    FN_POSITION = 0,      /* wrapped position, Bead.position */
    FN_IMAGE = 1,         /* unwrapped position, Bead.image_position */
    FN_VELOCITY = 2,      /* predicted velocity, Bead.velocity */
    FN_FORCE = 3,         /* Bead.force */
    FN_VELOCITY_OLD = 4   /* Bead.velocity_old */
};

/* pair kinds (SimulationManager.cpp:891-932); FN_PAIR_HSR is an extension
   without reference counterpart: penalty K plus a soft harmonic repulsion k
   below rc on one type pair (raw tokens K, k, rc; listed within the hs
   radius or the cutoff) */
enum { FN_PAIR_LJ = 1, FN_PAIR_HS = 2, FN_PAIR_ST = 3, FN_PAIR_HSR = 4 };

typedef struct fn_ctx fn_ctx;

/* Input-file settings of one network, as written in the input file
   (SimulationManager.cpp:644-819, 2070-2170). */
typedef struct fn_settings {
    double dt;            /* 'step' */
    double lambda;        /* 'lambda' */
    double damping;       /* 'damping' as written; negated internally (:664) */
    double gravity[3];    /* 'gravity' */
    double cutoff;        /* 'cutoff' */
    double box_unit_cell; /* 'box_unit_cell' */
    double box[3];        /* 'box_size' */
    double wall_k;        /* 'box_wall_rep' */
    int bc_type;          /* 0 pbc, 1 finite (after the :2168 override) */
    int grid_update_freq; /* 'grid_update_freq' */
    double skin_ratio;    /* skin_radius = radius + skin_ratio (:1431) */
    int n_types;          /* number of 'type' lines */
    int periodic_mask;    /* extension: bit a = axis a periodic; -1 = bc_type */
} fn_settings;

/* One network's model, borrowed host arrays (model-file order).  Vectors
   are 3 doubles per bead.  Replaces the CreateBuffer<Bead/BeadInfo/
   SpringStructure/AngleBond/Pair> uploads of ReadBeadsData, ReadSpringData,
   ReadAngleData and LoadTypeAndPairInfo (SimulationManager.cpp:1461-1486,
   1572, 1650, 963). */
typedef struct fn_network_desc {
    fn_settings settings;
    const int* pair_kind;    /* n_types*(n_types+1)/2 entries, GETADRESS order */
    const double* pair_raw;  /* 4 per pair: the 'pair' line tokens 4..7 */
    int n_beads;
    const int* type;
    const int* tag;
    const int* loc_id;
    const double* radius;
    const double* mass;
    const double* pos;
    const double* vel;
    const double* vel_old;
    const double* force;
    const double* img;
    int n_springs;
    const int* s_type;       /* 0 HR, 1 HR_FL */
    const int* s_p1;
    const int* s_p2;
    const double* s_rest;
    const double* s_k;
    const double* s_c1;      /* HR_FL Young's modulus */
    const double* s_c2;      /* HR_FL failure stress */
    int n_angles;
    const int* a_type;       /* 0 HR, 1 HR_FL */
    const int* a_b1;
    const int* a_b2;
    const int* a_b3;
    const int* a_s1;
    const int* a_s2;
    const double* a_theta0;
    const double* a_k;
} fn_network_desc;

typedef struct fn_config {
    int device;         /* CUDA device ordinal */
    int cell_capacity;  /* beads kept per grid cell (reference: 64, kernel.cl:10) */
    int list_capacity;  /* contacts kept per bead (full list) */
    int reorder;        /* 1: renumber beads in Morton order of their fibre */
    int use_graphs;     /* 1: replay steps as CUDA graphs */
    int block_size;     /* threads per block for the step kernel; 0 = default
                           (128); at most 256 on the chain path */
    int chain_mode;     /* 0 auto: per-bead bond records when the model is in
                           chain form (fibres), the tile's data staged in
                           shared memory before use; 1 chain form without
                           staging; 2 never (incidence lists) */
    double verlet_skin; /* 0: the reference's cadence (rebuild every
                           grid_update_freq steps, counter local to each
                           fn_step call, SimulationManager.cpp:152-173).
                           > 0: cut-off pairs are listed out to cutoff + skin
                           and the list is rebuilt only when some bead has
                           moved more than 0.45 of the smallest skin (this one
                           for cut-off kinds, skin radius - radius for hs
                           kinds, both capped by the cell step minus the
                           acting radius) since the last rebuild, checked on
                           the device before every step: no pair within reach
                           is ever missed.  Not a reference mode. */
    int host_upload;    /* 0: fn_upload checks, orders and converts the model
                           on the device when it can (fibres stored bead
                           after bead, bonds in chain form), else on host
                           threads; 1: always on host threads.  Both give the
                           same device state bit for bit. */
} fn_config;

/* Counters read back from the device. */
typedef struct fn_stats {
    long long cell_overflow;   /* beads dropped because a cell was full */
    long long list_overflow;   /* contacts dropped because a list was full */
    long long rebuilds;        /* contact-list rebuilds done */
    long long steps;           /* time steps done */
    int block_size;            /* step-kernel block size in use */
    int bond_path;             /* 0 per-bead incidence, 1 per-tile incidence, 2 chain records */
    int n_networks;
    long long n_beads;
    long long device_bytes;    /* device memory held by the context */
    long long graph_launches;  /* step segments replayed as CUDA graphs */
    long long nonfinite;       /* bead-steps whose new force was NaN or inf */
    int items_per_thread;      /* staged chain kernel: contact items per thread
                                  and round (0: another step kernel) */
    long long stalls;          /* tiles skipped because a bounded wait for their
                                  staged data ran out (fn_sync then fails) */
    int upload_on_device;      /* 1: the last fn_upload checked, ordered and
                                  converted the model on the device */
    int list_by_bricks;        /* 1: contact lists built by bricks of cells
                                  (fn_set_list_build) */
    int list_build;            /* the list build in use: 0 bead by bead, 1 by
                                  bricks of cells, 2 by groups of lanes */
} fn_stats;

/* A device array of the context, for zero-copy readers (torch through
   __cuda_array_interface__).  Beads are in internal order (fn_get_permutation)
   with 4 components per bead (the 4th is packing: radius/type bits for
   positions, 1/mass for images, 0 for velocities and forces).  The pointer is
   valid until the next call that steps, uploads or restores state: positions
   alternate between two buffers from step to step. */
typedef struct fn_view {
    void* ptr;
    long long n;    /* beads */
    int elem_bytes; /* bytes of one component: 8 (FP64) or 4 (FP32) */
    int components; /* 4 */
} fn_view;

/* Per-network observables (FP64 reductions on the device). */
typedef struct fn_observables {
    double reaction[3];   /* sum of Bead.force over beads of the chosen type */
    long long broken;     /* springs with status 0 */
    long long angles_dead;/* angles with status 0 */
} fn_observables;

/* Energy and virial of one network (FP64 device reductions; the reference
   computes neither).  Each potential is the one whose negative gradient is the
   force the step applies: springs k/2 (L - L0)^2, angles k (theta - theta0)^2,
   hs K/2 p^2 (p = overlap), hsr K/2 p^2 + k/2 (rc - r)^2 below rc, lj and st
   the integrals of their (shifted) forces out to their cut-off, walls
   wall_k/2 d^2, gravity -g.x on image positions.  kinetic = m/2 |v|^2 of the
   step-end velocity (velocity_old) over beads of non-zero mass.  virial =
   sum r_ij (x) F_ij over springs, angles and contact pairs (row-major 3x3,
   r in minimum image for contacts, image positions for bonds). */
typedef struct fn_energy {
    double kinetic, spring, angle, contact, wall, gravity;
    double virial[9];
    long long contacts; /* contact pairs with a non-zero force */
} fn_energy;

/* OpenclManager::Initialize (OpenclManager.cpp:5-85) without the interactive
   platform/device prompt: binds cfg->device and creates the stream. */
FN_API int fn_create(const fn_config* cfg, fn_ctx** out);

/* Frees every device buffer (OpenclManager::Close). */
FN_API void fn_destroy(fn_ctx* ctx);

/* Text of the last error on this context ("" if none).  Replaces checkErr
   logging (OpenclManager.cpp:335-408). */
FN_API const char* fn_last_error(const fn_ctx* ctx);

/* Uploads n_networks independent networks (1 = the reference's single
   simulation; >1 = a batched ensemble run in the same launches).  Replaces
   the CreateBuffer/WriteBuffer calls of ReadInputFile and the argument binding
   of ReadKernelData (SimulationManager.cpp:1153-1307; OpenclManager.h:121-174). */
FN_API int fn_upload(fn_ctx* ctx, int n_networks, const fn_network_desc* nets);

/* RunSimulationLoop(nsteps) on every network (SimulationManager.cpp:151-181):
   kick/drift, springs, angles, contact rebuild at step 0 of the call and every
   grid_update_freq steps, contacts, velocity update.  Asynchronous with
   respect to the host; ExecuteKernel + RunKernels per step become one
   stream-ordered (optionally graph-replayed) sequence. */
FN_API int fn_step(fn_ctx* ctx, int nsteps);

/* ResetGrid + ResetContactList + FillGrid + BuildContactList at the current
   positions (kernel.cl:487-789). */
FN_API int fn_rebuild_contacts(fn_ctx* ctx);

/* ResetBeadEnergy (kernel.cl:468-483) on every network, as
   MinimizeSystemEnergy calls it (SimulationManager.cpp:120, 138). */
FN_API int fn_reset_energy(fn_ctx* ctx);

/* Waits for the context's stream (OpenclManager::RunKernels). */
/* Waits for the context's work.  Returns FN_ERR_NONFINITE once a step has
   produced a NaN or infinite force (the state is then unusable). */
FN_API int fn_sync(fn_ctx* ctx);

/* Blocking read of one bead field, 3 doubles per bead, all networks in upload
   order (OpenclManager::ReadBuffer as DumpData/DumpRestartData use it,
   SimulationManager.cpp:1996, 1884). */
FN_API int fn_download(fn_ctx* ctx, int field, double* host);

/* Overwrites one bead field (the read-modify-write of LoadBeadModifications
   and ReadRestartFile, SimulationManager.cpp:220-228, 403-411, 1739-1816). */
FN_API int fn_set_beads(fn_ctx* ctx, int field, const double* host);

/* Per-bead mass, all networks in upload order (modif_bead mass,
   SimulationManager.cpp:267-316): recomputes the inverse-mass constants. */
FN_API int fn_set_mass(fn_ctx* ctx, const double* mass);

/* Per-bead skin radius (modif_bead skin_radius, SimulationManager.cpp:356-391). */
FN_API int fn_set_skin(fn_ctx* ctx, const double* skin_radius);

/* Spring parameters, all networks in upload order (modif_spring
   rest_length/stiffness/c1/c2, SimulationManager.cpp:449-626).  A null
   pointer leaves that parameter unchanged. */
FN_API int fn_set_springs(fn_ctx* ctx, const double* rest, const double* k, const double* c1,
                          const double* c2);

/* Angle stiffness and rest angle (no reference counterpart; used by fitting). */
FN_API int fn_set_angles(fn_ctx* ctx, const double* theta0, const double* k);

/* Spring and angle status (1 alive, 0 broken/dead), all networks. */
FN_API int fn_download_status(fn_ctx* ctx, int* spring_status, int* angle_status);
FN_API int fn_set_status(fn_ctx* ctx, const int* spring_status, const int* angle_status);

/* Observables of network `net`; reaction sums the force on beads of type
   `reaction_type` (-1: none). */
FN_API int fn_observe(fn_ctx* ctx, int net, int reaction_type, fn_observables* out);

FN_API int fn_get_stats(fn_ctx* ctx, fn_stats* out);

/* ---- differentiation (no counterpart in the reference) ----------------
   Gradients of a loss on the recorded reaction force with respect to every
   spring stiffness and rest length, every angle stiffness and the initial
   positions and velocities, by the discrete adjoint of the step loop.

   fn_adjoint_forward runs nsamples fn_step(every) calls from the current
   state, records after each the reaction of every network (the force summed
   over its beads of type reaction_type) into reaction[nsamples][n_networks][3]
   (may be null), and keeps a device checkpoint every checkpoint_every steps
   (a multiple of every dividing nsamples * every).  Needs damping 0.

   fn_adjoint_backward takes dL/d reaction in the same layout and writes the
   gradients (any output may be null): per spring and per angle in upload
   order, per bead [n_beads][3] in upload order for the positions and
   velocities the forward pass started from.  Contact sets, the contact list
   of each rebuild interval and HR_FL break events are those of the forward
   pass; segments are recomputed from their checkpoints (checked bit for bit
   against the next checkpoint).  It leaves the state where the forward pass
   ended; any state change in between makes it fail with FN_ERR_STATE.
   Device memory, kept between calls until fn_adjoint_release: 112 B per
   bead per checkpoint; for the replay 64 B per bead per step of a
   checkpoint interval plus the contact lists of its rebuilds. */
FN_API int fn_adjoint_forward(fn_ctx* ctx, int nsamples, int every, int checkpoint_every,
                              int reaction_type, double* reaction);
FN_API int fn_adjoint_backward(fn_ctx* ctx, const double* dloss_dreaction, double* grad_spring_k,
                               double* grad_spring_rest, double* grad_angle_k, double* grad_pos0,
                               double* grad_vel0);
FN_API int fn_adjoint_release(fn_ctx* ctx);

/* Energy and virial of network `net` at the current state (after fn_step the
   state holds the positions its last forces were evaluated at). */
FN_API int fn_energy_eval(fn_ctx* ctx, int net, fn_energy* out);

/* The Run flow's time series without a host round trip per chunk: runs
   nsteps as fn_step(every) calls (the rebuild counter restarts with every
   chunk, SimulationManager.cpp:152) and after each chunk records, on the
   device, one row for network `net`: {steps done, reaction x, y, z, broken
   springs, dead angles} and, when with_energy != 0, the 16 fields of
   fn_energy (contacts as a double).  Rows are copied to host_rows
   (ceil(nsteps / every) rows of 6 or 22 doubles) once, at the end. */
FN_API int fn_step_series(fn_ctx* ctx, int nsteps, int every, int net, int reaction_type,
                          int with_energy, double* host_rows);

/* The observables of fn_observe for callers that cannot allocate device
   memory when they need them: a host loop or callback that must not
   synchronise the device (cudaMalloc and cudaFree may), or an application
   whose device memory all belongs to its own allocator.  No counterpart in
   the reference.  Writes
   {reaction x, y, z, broken springs, dead angles} as 5 doubles to the
   caller's device buffer out_device, asynchronously on the context's stream
   (read it after fn_sync).  Calls no cudaMalloc/cudaFree: its scratch is a
   fixed 40 KB array in the library (1,024 partial sums, the most that
   fn_observe's reduction uses; larger networks loop inside each block), which
   every GPU that loads the library keeps until exit.  Results equal
   fn_observe's bit for bit at every network size; a reduction that would need
   more partial sums than the array holds is rejected with FN_ERR_CAPACITY.
   The first call on a device looks up the scratch's device address; make it
   before any stream capture, and do not call it on a device after a
   cudaDeviceReset.  All calls share the scratch: calls that overlap on the
   GPU (other streams or contexts on the same device) race. */
FN_API int fn_observe_noalloc(fn_ctx* ctx, int net, int reaction_type, double* out_device);

/* Grid and contact-list inspection (tests): cell of each bead (-1 outside
   the grid or beyond the cell capacity), the raw count of each cell, and
   each bead's contacts (raw count and up to cap partner ids), all in upload
   numbering; cells are numbered per network like the reference
   (x + y*nx + z*nx*ny) plus the network's cell offset. */
FN_API int fn_get_cells(fn_ctx* ctx, int* bead_cell, int* cell_count, long long n_cells);
FN_API int fn_get_lists(fn_ctx* ctx, int* count, int* partners, int cap);
FN_API long long fn_n_cells(fn_ctx* ctx);

/* Forces alone at the current positions and contact list (zeroed first, no
   damping/gravity/wall term, no kick or drift): the per-step force of
   ResolveSprings + ResolveAngles + ResolveContacts (kernel.cl:268-441,
   792-1011) for one-step parity checks.  terms: bit 0 springs, 1 angles,
   2 contacts.  The result is read with fn_download(FN_FORCE). */
FN_API int fn_forces_only(fn_ctx* ctx, int terms);

/* Internal bead numbering: perm[internal] = upload index. */
FN_API int fn_get_permutation(fn_ctx* ctx, int* perm);

/* The device array of field (FN_POSITION, FN_IMAGE, FN_VELOCITY, FN_FORCE,
   FN_VELOCITY_OLD) without a copy; synchronises the context's stream first. */
FN_API int fn_device_view(fn_ctx* ctx, int field, fn_view* out);

/* Times steps_per_trial steps at each candidate shape of the step kernel
   (block size 64 .. 512; for the staged chain kernel also 2, 4 or 8 contact
   items per thread and round, or no staging) from one snapshot of the state,
   restored after every trial, keeps the fastest, then keeps the fastest of
   the three list builds (fn_set_list_build) at that shape; the simulation
   does not advance. */
FN_API int fn_autotune(fn_ctx* ctx, int steps_per_trial);

/* How contact lists are built (ResetGrid .. BuildContactList,
   kernel.cl:487-789): 0 (the default) one thread per bead reading its
   candidates from global memory; 1 by bricks of 8 x 4 x 4 grid cells whose
   beads and neighbouring beads are staged in shared memory; 2 by groups of 8
   lanes per bead (more threads in flight for small networks).  All give the
   same lists, entry for entry; fn_autotune keeps the fastest. */
FN_API int fn_set_list_build(fn_ctx* ctx, int mode);

/* Sets the step kernel's shape: threads per block (a multiple of 32; 64 ..
   256 on the chain path, whose tiles hold block - 4 beads) and, for the
   staged chain kernel (chain_mode 0), contact items per thread and round
   (1 .. 8; 0 runs the chain kernel without staging).  fn_autotune picks the
   same parameters by timing. */
FN_API int fn_set_kernel_shape(fn_ctx* ctx, int block, int items_per_thread);

/* Device-side snapshot of the dynamic state (positions, images, velocities,
   forces, bond statuses, counters; in displacement mode also the reference
   images and the rebuild gate), kept in one device buffer of the context.
   fn_state_restore puts the last snapshot back (the step count with it), so
   the same steps can be run again from the same state; a new fn_upload drops
   the snapshot.  No counterpart in the reference, whose restart files
   (SimulationManager.cpp:1739-1884) go through the host: fn_download /
   fn_set_beads / fn_set_status remain the file path. */
FN_API int fn_state_save(fn_ctx* ctx);
FN_API int fn_state_restore(fn_ctx* ctx);

/* fn_step bracketed by CUDA events on the context's stream: waits for the
   steps to finish and writes their device time (ms) to *ms. */
FN_API int fn_step_timed(fn_ctx* ctx, int nsteps, double* ms);

/* Average duration (ms) of the step kernel over the last fn_step call when
   timing is enabled, with the launch count. */
FN_API int fn_enable_timing(fn_ctx* ctx, int on);
FN_API int fn_kernel_time(fn_ctx* ctx, double* step_kernel_ms, long long* launches,
                          double* rebuild_ms, long long* rebuilds);

#ifdef __cplusplus
}
#endif
#endif
