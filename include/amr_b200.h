/* amr_b200.h -- C ABI of the B200 static-AMR cut-cell explicit time step.
 *
 * One header, plain C: fixed-width integers, plain pointers and sizes, no C++ or
 * torch types.  Two families of entry points live here:
 *
 *   amr_gpu_*    the single-case FP64 session.  Each entry point replaces one of the
 *                five functions of the reference's C++ session API
 *                (src/static_amr2d_gpu.h:17-24 in the reference):
 *                  amr_gpu_create    <- static_amr_gpu_create    (static_amr2d_gpu.h:17-18)
 *                  amr_gpu_advance   <- static_amr_gpu_advance   (static_amr2d_gpu.h:19-21)
 *                  amr_gpu_download  <- static_amr_gpu_download  (static_amr2d_gpu.h:22)
 *                  amr_gpu_stats     <- static_amr_gpu_stats     (static_amr2d_gpu.h:23)
 *                  amr_gpu_destroy   <- static_amr_gpu_destroy   (static_amr2d_gpu.h:24)
 *                The C++ adapter behind include/static_amr2d_gpu.h forwards the
 *                reference's signatures to these.
 *
 *   amr_batch_*  the batched form: many meshes in ragged device arrays, each case
 *                with its own time, dt, retry counter and status, advanced together
 *                by one persistent kernel per batch of trials.  It has no counterpart
 *                in the reference, which runs one case per session.
 *
 * Record layouts.  amr_cell_t, amr_face_t, amr_wall_t, amr_gradient_term_t,
 * amr_wall_sample_t, amr_face_geometry_t, amr_boundary_t and amr_transport_t have
 * the same field order, types and therefore the same byte layout as the reference's
 * AmrCell2D / AmrFace2D (src/static_amr2d.h:37-45), WallFragment2D
 * (src/euler2d.h:186-190), AmrGradientTerm2D / AmrWallSample2D /
 * AmrViscousFaceGeometry2D / AmrTransport2D (src/static_amr2d_viscous.h:15-25) and
 * AmrBoundary2D (src/static_amr2d_boundary.h:14-21) on LP64 targets, so a caller
 * holding the reference's std::vectors passes .data() without copying.
 *
 * Return codes: 0 success, 1 error (message in the caller's buffer), 2 wall-clock
 * budget expired with a resumable state (advance only), 3 no room (batch admission).
 */
#ifndef AMR_B200_H
#define AMR_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AMR_B200_ABI_VERSION 1

/* Boundary kinds (reference src/static_amr2d_boundary.h:11-12). */
enum {
  AMR_B200_BC_INHERIT = -1,
  AMR_B200_BC_TRANSMISSIVE = 1,
  AMR_B200_BC_REFLECT = 2,
  AMR_B200_BC_FARFIELD = 3,
  AMR_B200_BC_TOTAL_INLET = 4,
  AMR_B200_BC_PRESSURE_OUTLET = 5,
  AMR_B200_BC_NOSLIP = 6
};
/* Flow model, viscosity law and viscous time-step mode (src/static_amr2d_viscous.h:12-14). */
enum { AMR_B200_MODEL_EULER = 0, AMR_B200_MODEL_LAMINAR = 1 };
enum { AMR_B200_MU_CONSTANT = 0, AMR_B200_MU_SUTHERLAND = 1 };
enum { AMR_B200_VISCOUS_VOLUME = 0, AMR_B200_VISCOUS_SRD = 1 };
/* Numerical flux (src/types.h:6) and the only accepted limiter/integrator. */
enum { AMR_B200_FLUX_HLLC = 0, AMR_B200_FLUX_AUSMPUP = 1 };
enum { AMR_B200_LIMITER_FIRST_ORDER = 3 };
enum { AMR_B200_TIME_SSP_RK3 = 0 };
/* Device status codes (reference src/static_amr2d_cuda.cu:57,66,186,214). */
enum {
  AMR_B200_STATUS_OK = 0,
  AMR_B200_STATUS_NONPHYSICAL_BASE = 2,
  AMR_B200_STATUS_MAXSTEPS = 3,
  AMR_B200_STATUS_DT_UNDERFLOW = 4,
  AMR_B200_STATUS_REJECTIONS = 5,
  AMR_B200_STATUS_BARRIER_TIMEOUT = 9
};

typedef struct amr_cell_t {
  int32_t ix, iy, span, level;
  double x0, x1, y0, y1, volume, cx, cy;
  uint64_t wall_begin, wall_count;
} amr_cell_t;

typedef struct amr_face_t {
  int32_t left, right, axis, boundary; /* -1 outside; normal points +axis */
  double coordinate, lo, hi, length, centroid;
} amr_face_t;

typedef struct amr_wall_t {
  uint64_t owner_cell;
  int32_t source_edge_id, body_id, patch_id;
  double x0, y0, x1, y1, nx, ny, length; /* normal points fluid -> solid */
} amr_wall_t;

typedef struct amr_gradient_term_t {
  int32_t source, side; /* source >= 0 neighbour cell, -1 body wall, -2 exterior no-slip wall */
  double x, y;
} amr_gradient_term_t;

typedef struct amr_wall_sample_t {
  int32_t donor;
  double distance;
} amr_wall_sample_t;

typedef struct amr_face_geometry_t {
  double dx, dy, ex, ey, distance;
} amr_face_geometry_t;

typedef struct amr_boundary_t {
  int32_t kind;
  double reference[4]; /* rho,u,v,p; also the outlet backflow reservoir */
  double total_pressure, total_temperature, gas_constant;
  double direction[2];
  double outlet_pressure;
  double wall_velocity[2];
} amr_boundary_t;

typedef struct amr_transport_t {
  int32_t model, law, stabilization;
  double mu_ref, gas_constant, temperature_ref, sutherland, viscous_cfl;
  int32_t sa_model;
  double sa_nu_inf, sa_cfl;
  double wall_probe_min_h;
} amr_transport_t;

/* Solver parameters used by the time step (the subset of the reference's Params2D,
 * src/euler2d.h:137-151, that the static-AMR path reads). */
typedef struct amr_params_t {
  double gamma, cfl, dt_fixed, ausm_mco;
  int32_t flux, limiter, time_integrator;
  int32_t bc[4]; /* legacy kind for sides whose amr_boundary_t.kind is AMR_B200_BC_INHERIT */
} amr_params_t;

/* A static mesh as the reference's host builder leaves it (StaticAmrMesh2D,
 * src/static_amr2d.h:46-66, plus AmrViscousTable2D, src/static_amr2d_viscous.h:26-32).
 * Every pointer is borrowed for the duration of the call only. */
typedef struct amr_mesh_view_t {
  uint64_t n_cells, n_faces, n_walls;
  const amr_cell_t* cells;
  const amr_face_t* faces;
  const amr_wall_t* walls;
  const uint64_t* face_offsets;   /* n_cells + 1 */
  const uint64_t* cell_faces;     /* face_offsets[n_cells] */
  const uint64_t* group_offsets;  /* n_cells + 1 (SRD neighbourhoods) */
  const uint64_t* group_members;  /* group_offsets[n_cells] */
  const uint64_t* member_offsets; /* n_cells + 1 */
  const uint64_t* member_groups;  /* member_offsets[n_cells] */
  const double* group_volume;     /* n_cells */
  uint64_t small_cells;
  int32_t agglomerate_small;
  amr_boundary_t boundaries[4];   /* xmin, xmax, ymin, ymax */
  amr_transport_t transport;
  /* Viscous tables; required when transport.model == AMR_B200_MODEL_LAMINAR. */
  const uint64_t* visc_offsets;   /* n_cells + 1 */
  const amr_gradient_term_t* visc_terms;
  const amr_wall_sample_t* wall_samples;    /* n_walls */
  const amr_wall_sample_t* face_samples;    /* n_faces */
  const amr_face_geometry_t* face_geometry; /* n_faces */
  const double* wall_distance;              /* n_cells; required when transport.sa_model */
} amr_mesh_view_t;

typedef struct amr_gpu_options_t {
  int32_t batch_trials;  /* trials per status poll, 1..1024 (reference default 32) */
  int32_t graph;         /* replay the per-poll launch through a CUDA graph */
  int32_t fused;         /* accepted for API parity; the engine is always fused */
  int32_t event_timing;  /* accumulate CUDA-event time per poll */
  int32_t sa_fused;      /* accepted for API parity */
  int32_t device;        /* CUDA device ordinal */
  int32_t block_threads; /* 0 = autotuned */
  int32_t grid_blocks;   /* 0 = autotuned */
  int32_t launch_mode;   /* AMR_B200_LAUNCH_*; AUTO with block_threads = grid_blocks = 0 autotunes */
} amr_gpu_options_t;

/* Same fields, order and layout as the reference's AmrGpuStats (src/static_amr2d_gpu.h:9-16). */
typedef struct amr_gpu_stats_t {
  uint64_t allocated_bytes, pinned_bytes, geometry_h2d_bytes, state_h2d_bytes;
  uint64_t control_h2d_bytes;
  uint64_t control_d2h_bytes, state_d2h_bytes, status_polls, full_downloads;
  double setup_seconds, advance_seconds, download_seconds;
  double advance_event_seconds;
  uint64_t event_batches, graph_nodes_per_trial;
} amr_gpu_stats_t;

/* Host-visible metadata of a case (StaticAmrState2D time/steps/rejected, src/static_amr2d.h:67-71). */
typedef struct amr_state_meta_t {
  double time;
  int64_t steps, rejected;
  int32_t status;   /* AMR_B200_STATUS_* */
  int32_t finished; /* time reached the last advance target */
} amr_state_meta_t;

typedef struct amr_gpu_session amr_gpu_session;

void amr_gpu_default_options(amr_gpu_options_t* options);

/* Validates mesh and parameters, uploads the mesh tables and the initial state
 * u0[nv*n_cells] (SoA: u0[var*n_cells+cell], nv = 5 with SA else 4).  *out is NULL on
 * failure.  Replaces static_amr_gpu_create (reference src/static_amr2d_cuda.cu:274-325). */
int amr_gpu_create(const amr_mesh_view_t* mesh, const amr_params_t* params,
                   const double* u0, uint64_t u0_count, double time0, int64_t steps0,
                   int64_t rejected0, const amr_gpu_options_t* options,
                   amr_gpu_session** out, char* error, uint64_t error_size);

/* Advances until time == tend or a fatal status; maxsteps counts accepted steps since
 * the case began (steps0 included).  Returns 0 done, 1 fatal (last accepted state
 * kept on the device), 2 wall budget expired (resumable).  Replaces
 * static_amr_gpu_advance (reference src/static_amr2d_cuda.cu:327-353). */
int amr_gpu_advance(amr_gpu_session* session, double tend, int64_t maxsteps,
                    double wall_budget_seconds, amr_state_meta_t* meta,
                    char* error, uint64_t error_size);

/* Copies the accepted state to u_out[u_count] (u_count == nv*n_cells).  Replaces
 * static_amr_gpu_download (reference src/static_amr2d_cuda.cu:355-363). */
int amr_gpu_download(amr_gpu_session* session, double* u_out, uint64_t u_count,
                     amr_state_meta_t* meta, char* error, uint64_t error_size);

/* Zeros for a NULL session.  Replaces static_amr_gpu_stats (src/static_amr2d_cuda.cu:364). */
int amr_gpu_stats(const amr_gpu_session* session, amr_gpu_stats_t* out);

/* Synchronises and frees; accepts NULL.  Replaces static_amr_gpu_destroy (src/static_amr2d_cuda.cu:365). */
void amr_gpu_destroy(amr_gpu_session* session);

/* Residual dU/dt of the accepted state, r_out[nv*n_cells], computed on the device by the
 * same operators as the time step (the reference's static_amr2d_rhs, src/static_amr2d.cpp:369-377). */
int amr_gpu_residual(amr_gpu_session* session, double* r_out, uint64_t r_count,
                     char* error, uint64_t error_size);

/* Steady-state diagnostics of the accepted state, reduced on the device in FP64:
 * out[0..4] volume-weighted mean |R_v| over cells whose centroid lies in
 * [region[0],region[1]]x[region[2],region[3]] (the SA row divided by sa_nu_inf),
 * out[5..7] = Fx, Fy, Mz about (moment_x, moment_y) from wall pressure minus viscous
 * wall flux, as in the reference driver (src/quick_airfoil.cpp:189-199). */
int amr_gpu_diagnostics(amr_gpu_session* session, const double region[4], double moment_x,
                        double moment_y, double out[8], char* error, uint64_t error_size);

/* Residual dU/dt of the inviscid (Euler) model that allocates no device memory.  It has no
 * counterpart in the reference.  It is for callers that cannot call cudaMalloc at the point where
 * they need a residual: code running under another framework's memory pool or allocator, a
 * latency-critical loop in which an allocation would synchronise the device, or a plug-in that
 * is handed device buffers but may not own memory.  The caller passes device pointers to its own
 * copies of the mesh records (cells, faces, walls, face_offsets, cell_faces in the layout above),
 * the state u[4*n_cells] and the output r[4*n_cells]; boundaries[4] and params are host records;
 * stream is a cudaStream_t (NULL: the default stream).  The scratch (primitives and face fluxes)
 * lives in one static device array of 1.8 MB that every GPU loading the library holds until the
 * process exits, so meshes are limited to 16384 cells and 40960 faces; larger ones are rejected
 * with an error.  Every call looks up that array's device address on the current device and
 * synchronises `stream` to read its status word, so no call may be made while a stream is being
 * captured.  All calls on a device share the array: calls whose kernels overlap on the GPU (other
 * streams or host threads) race, so serialise them.  Returns 1 with a message for a nonphysical
 * state, like amr_gpu_residual, and for mesh records whose indices fall outside the arrays
 * passed (face cells, boundary side or axis, a cell's face range, face ids, wall ranges). */
int amr_euler_residual_static(const amr_cell_t* cells, uint64_t n_cells, const amr_face_t* faces, uint64_t n_faces,
                              const amr_wall_t* walls, uint64_t n_walls, const uint64_t* face_offsets,
                              const uint64_t* cell_faces, const amr_boundary_t* boundaries, const amr_params_t* params,
                              const double* u, double* r, void* stream, char* error, uint64_t error_size);

/* The same export for the single-case session (see amr_batch_export). */
int amr_gpu_export(amr_gpu_session* session, double* wall_rows, uint64_t wall_count, double* sa_rows,
                   uint64_t sa_count, double limits[2], char* error, uint64_t error_size);

/* ----------------------------------------------------------------------------------
 * Batched form.
 * ---------------------------------------------------------------------------------- */
enum { AMR_B200_PRECISION_FP64 = 64, AMR_B200_PRECISION_FP32 = 32 };
/* Launch modes: one persistent cooperative kernel per poll with grid barriers between phases;
 * one kernel per phase (a warp per tile of whole cells) replayed from a CUDA graph; or split,
 * also graph-replayed: gradients one thread per cell, each face flux once (one thread per face
 * or wall record), then one thread per cell gathering its records in order with the update; or
 * tiled, graph-replayed: one kernel per stage, each block working through block tiles of up to
 * 128 cells with the cell records and face fluxes of a tile kept in shared memory. */
enum {
  AMR_B200_LAUNCH_AUTO = 0,
  AMR_B200_LAUNCH_PERSISTENT = 1,
  AMR_B200_LAUNCH_PHASES = 2,
  AMR_B200_LAUNCH_SPLIT = 3,
  AMR_B200_LAUNCH_TILED = 4
};

typedef struct amr_batch_config_t {
  int32_t precision;      /* AMR_B200_PRECISION_FP32 or _FP64 */
  int32_t device;
  int32_t model;          /* AMR_B200_MODEL_*: one flow model per batch */
  int32_t sa_model;       /* 0 or 1 */
  int32_t flux;           /* AMR_B200_FLUX_*: one flux per batch */
  int32_t max_cases;
  uint64_t max_cells, max_faces, max_walls, max_terms, max_srd; /* arena capacities; 0 = sized from hbm_bytes */
  uint64_t hbm_bytes;     /* arena budget used when capacities are 0 */
  int32_t block_threads;  /* 0 = 256 until amr_batch_autotune */
  int32_t grid_blocks;    /* 0 = one wave of co-resident blocks */
  int32_t launch_mode;    /* AMR_B200_LAUNCH_*; AUTO starts persistent until amr_batch_autotune */
} amr_batch_config_t;

/* Per-case run control and the steady retirement rule (reference driver,
 * src/quick_airfoil.cpp:180-208). check_period <= 0 disables steady checks. */
typedef struct amr_case_control_t {
  double tend;             /* physical time cap */
  int64_t maxsteps;        /* accepted-step cap */
  double first_check, check_period;
  double min_time, raw_tol, load_tol;
  int32_t hold;
  double region[4];
  double moment_x, moment_y, mach, aoa_degrees;
} amr_case_control_t;

typedef struct amr_case_status_t {
  double time;
  int64_t steps, rejected;
  int32_t status, finished, converged, checks, hold;
  double residual[5];
  double cl, cd, cm;
} amr_case_status_t;

typedef struct amr_batch amr_batch;

int amr_batch_create(const amr_batch_config_t* config, amr_batch** out, char* error, uint64_t error_size);
/* Admits one case; *slot receives its id.  Returns 3 (no room) when the arena lacks cells,
 * faces, walls, terms or case slots for it.  u0 holds nv*n_cells values (SoA), or nv values for a
 * uniform start (the reference's static_amr2d_initialize from freestream primitives,
 * src/static_amr2d.cpp:360-367, in conserved form), which the device fills itself. */
int amr_batch_admit(amr_batch* batch, const amr_mesh_view_t* mesh, const amr_params_t* params,
                    const double* u0, uint64_t u0_count, const amr_case_control_t* control,
                    int32_t* slot, char* error, uint64_t error_size);
/* Admits `count` cases at once (entry i: meshes[i], params[i], u0[i][u0_counts[i]],
 * controls[i]), converting them into the engine layout on `threads` host threads (0 = up to
 * 16) with one stream synchronisation for the lot.  slots[i] receives the id or -1,
 * status[i] 0 (admitted), 1 (invalid; the first such message goes to error) or 3 (no room).
 * Ids and arena placement follow the request order whatever the thread count, so the result
 * equals `count` amr_batch_admit calls.  Returns 1 if any case was invalid, else 3 if any
 * found no room, else 0.  No counterpart in the reference, which sets up one case per
 * session. */
int amr_batch_admit_many(amr_batch* batch, uint64_t count, const amr_mesh_view_t* const* meshes,
                         const amr_params_t* const* params, const double* const* u0, const uint64_t* u0_counts,
                         const amr_case_control_t* const* controls, int32_t threads, int32_t* slots,
                         int32_t* status, char* error, uint64_t error_size);
/* Runs `trials` trials of every live case (one persistent launch, replayed from a CUDA
 * graph that is recaptured when the case set changes), then refreshes host-side status. */
int amr_batch_advance(amr_batch* batch, int32_t trials, char* error, uint64_t error_size);
/* amr_batch_advance in two halves: the first enqueues the trials on the batch's stream and returns
 * at once, the second waits for them and refreshes the host-side statuses.  One host thread can so
 * keep several batches' trials in flight together (each batch has its own stream).  Make no other
 * call on a batch between its two halves.  No counterpart in the reference. */
int amr_batch_advance_async(amr_batch* batch, int32_t trials, char* error, uint64_t error_size);
int amr_batch_wait(amr_batch* batch, char* error, uint64_t error_size);
/* Runs `trials` trials of every live case of `count` batches of one device with their work in
 * flight together: every batch's trials start after one start event, each on its own stream, so
 * the kernels of one batch fill the tails of another's.  Each batch ends exactly as after its own
 * amr_batch_advance.  *device_seconds (if not null) receives the device time from the start event,
 * recorded after every batch's host-side preparation (uploads, graph captures), to the last batch's
 * end.  Returns 1 with a message for a null or repeated batch, batches on
 * different devices or a failed advance (every advance that began is completed first).  No
 * counterpart in the reference. */
int amr_batch_group_advance(amr_batch* const* batches, int32_t count, int32_t trials, double* device_seconds,
                            char* error, uint64_t error_size);
/* Device bytes a batch allocated (arena, state, scratch and records). */
uint64_t amr_batch_device_bytes(const amr_batch* batch);
/* Free and total memory of CUDA device `device` (cudaMemGetInfo), for admission by free device
 * memory.  Returns 0, or 1 when the device cannot be queried.  No counterpart in the reference. */
int amr_device_memory(int32_t device, uint64_t* free_bytes, uint64_t* total_bytes);
/* Evaluates the steady criteria for every live case whose next check time has been reached. */
int amr_batch_check(amr_batch* batch, char* error, uint64_t error_size);
int amr_batch_status(const amr_batch* batch, int32_t slot, amr_case_status_t* out);
/* The accepted states of `count` cases, u_out[i][u_counts[i]] for slots[i] (u_counts[i] ==
 * nv * n_cells of that case), in one staged copy with one synchronisation.  No counterpart in the
 * reference, which downloads one session's state at a time. */
int amr_batch_download_many(amr_batch* batch, uint64_t count, const int32_t* slots, double* const* u_out,
                            const uint64_t* u_counts, char* error, uint64_t error_size);
int amr_batch_download(amr_batch* batch, int32_t slot, double* u_out, uint64_t u_count,
                       char* error, uint64_t error_size);
/* Compact results of one case, computed on the device from its accepted state, so a retired
 * case leaves the device without its full state: the wall-stress rows of the reference's viscous
 * snapshot (src/static_amr2d_viscous.cpp:155-160; 14 doubles per wall fragment, viscous models
 * only, else wall_count = 0), the SA cell rows (nutilde, eddy viscosity, wall distance; 3 per
 * cell, SA only, else sa_count = 0) and limits = {smallest convective dt, smallest viscous dt}.
 * Runs one residual pass of the live cases first.  No counterpart in the reference, which
 * downloads the state and evaluates these on the host. */
int amr_batch_export(amr_batch* batch, int32_t slot, double* wall_rows, uint64_t wall_count, double* sa_rows,
                     uint64_t sa_count, double limits[2], char* error, uint64_t error_size);
int amr_batch_release(amr_batch* batch, int32_t slot);
int amr_batch_live_cases(const amr_batch* batch);
uint64_t amr_batch_free_cells(const amr_batch* batch);
/* Device time of the last amr_batch_advance in seconds (CUDA events on the launch stream). */
double amr_batch_last_advance_seconds(const amr_batch* batch);
/* Times every launch mode and block size on the live cases (state and controls are restored
 * afterwards) and keeps the fastest. */
int amr_batch_autotune(amr_batch* batch, int32_t trials, char* error, uint64_t error_size);
/* Kernels launched by this batch so far. */
uint64_t amr_batch_kernel_launches(const amr_batch* batch);
void amr_batch_destroy(amr_batch* batch);

/* ----------------------------------------------------------------------------------
 * Host mesh builder.
 *
 * amr_mesh_build replaces the reference's two host calls that turn a body polygon into a
 * solver-ready mesh: static_amr2d_build (src/static_amr2d.h:80-82, src/static_amr2d.cpp:229)
 * followed by static_amr2d_prepare_viscous (src/static_amr2d_viscous.h, defined at
 * src/static_amr2d_viscous.cpp:40, which also runs static_amr2d_prepare_sa).  The tables it
 * returns are bit-identical to the reference's; the build is faster and amr_mesh_build_many
 * runs many builds on a pool of host threads (no reference counterpart), so that mesh
 * generation keeps up with a serving batch.
 * ---------------------------------------------------------------------------------- */
typedef struct amr_mesh_box_t {
  double x0, x1, y0, y1;
  int32_t level;
} amr_mesh_box_t;

/* StaticAmrOptions2D (src/static_amr2d.h:29-35). */
typedef struct amr_mesh_options_t {
  int32_t nx, ny, levels, buffer;
  double xmin, xmax, ymin, ymax;
  uint64_t max_cells;
  int32_t agglomerate_small;
  int32_t n_boxes;
  const amr_mesh_box_t* boxes;
} amr_mesh_options_t;

/* One build: options, the closed body polygon (no repeated closing vertex) with optional
 * per-edge patch ids, and the physics the tables depend on (boundary kinds, transport). */
typedef struct amr_mesh_request_t {
  const amr_mesh_options_t* options;
  const double* px;
  const double* py;
  const int32_t* patches; /* n_points or NULL */
  uint64_t n_points;
  const amr_boundary_t* boundaries; /* 4: xmin, xmax, ymin, ymax */
  const amr_transport_t* transport;
  const amr_params_t* params;       /* bc[] of sides whose kind is INHERIT */
} amr_mesh_request_t;

typedef struct amr_mesh_counts_t {
  uint64_t background_leaves, split_leaves, coarse_fine_faces, small_cells, n_terms;
} amr_mesh_counts_t;

typedef struct amr_mesh_t amr_mesh_t; /* opaque; owns every table of one mesh */

int amr_mesh_build(const amr_mesh_request_t* request, amr_mesh_t** out, char* error, uint64_t error_size);
/* Builds count meshes on `threads` host threads (0 = all cores).  out[i] and status[i] (0 or
 * 1) are set per request; a failed request's message goes to errors + i * error_stride.
 * Returns 1 if any request failed. */
int amr_mesh_build_many(uint64_t count, const amr_mesh_request_t* requests, int32_t threads, amr_mesh_t** out,
                        int32_t* status, char* errors, uint64_t error_stride);
/* A view of the mesh's tables, valid until amr_mesh_destroy; pass it to amr_gpu_create or
 * amr_batch_admit. */
int amr_mesh_view(const amr_mesh_t* mesh, amr_mesh_view_t* view);
int amr_mesh_get_counts(const amr_mesh_t* mesh, amr_mesh_counts_t* counts);

/* Build records the mesh files carry besides the tables: the agglomeration map (9 doubles per
 * original control volume: old id, new id, x0, x1, y0, y1, volume, cx, cy) and the (background
 * leaf, control volume) pairs of leaves split into several fluid loops. */
typedef struct amr_mesh_extras_t {
  uint64_t coarse_fine_faces, split_leaves;
  const double* agglomeration;     /* n_agglomeration x 9 */
  uint64_t n_agglomeration;
  const uint64_t* leaf_components; /* n_leaf_components x 2 */
  uint64_t n_leaf_components;
} amr_mesh_extras_t;
int amr_mesh_get_extras(const amr_mesh_t* mesh, amr_mesh_extras_t* extras);
void amr_mesh_destroy(amr_mesh_t* mesh);

/* ----------------------------------------------------------------------------------
 * Result files in the reference's formats (read by its pipeline/export.py).
 *
 * amr_write_mesh_files   <- static_amr_binary_mesh (src/static_amr2d_binary.cpp:25-49):
 *                           <prefix>.bc.json, .transport.json, .viscous_stabilization.json,
 *                           .gradient_table.csv, .wall_samples.csv (viscous), .cells.npy,
 *                           .faces.npy, .walls.npy, .leaf_components.npy, .agglomeration.npy,
 *                           .mesh.json
 * amr_write_snapshot_files <- static_amr_binary_snapshot (src/static_amr2d_binary.cpp:50-69):
 *                           <prefix>.state.npy, .json and, for viscous models,
 *                           .timestep_limits.json, .wall_stress.npy, .viscous_loads.json,
 *                           .sa.npy, .sa.json; the rows come from amr_gpu_export /
 *                           amr_batch_export.
 * amr_write_npy          <- static_amr_write_npy (src/static_amr2d_binary.cpp:14-24).
 * The files are byte-identical to the reference writer's for the same inputs.
 * ---------------------------------------------------------------------------------- */
typedef struct amr_export_rows_t {
  const double* wall_rows; /* n_walls x 14 (viscous models) */
  const double* sa_rows;   /* n_cells x 3 (SA) */
  double convective_dt, viscous_dt;
} amr_export_rows_t;

int amr_write_npy(const char* path, const double* values, uint64_t rows, uint64_t cols, char* error,
                  uint64_t error_size);
int amr_write_mesh_files(const char* prefix, const amr_mesh_view_t* mesh, const amr_mesh_options_t* options,
                         const amr_params_t* params, const amr_mesh_extras_t* extras, char* error,
                         uint64_t error_size);
int amr_write_snapshot_files(const char* prefix, const amr_mesh_view_t* mesh, const amr_mesh_options_t* options,
                             const amr_params_t* params, const double* u, double time, int64_t steps,
                             int64_t rejected, const char* backend, const amr_export_rows_t* rows, char* error,
                             uint64_t error_size);

/* Tuning and introspection.  None has a counterpart in the reference. */
/* Sets a case's advance target time and step cap (the driver's stop time and max steps). */
int amr_batch_set_target(amr_batch* batch, int32_t slot, double target, int64_t maxsteps, char* error,
                         uint64_t error_size);
/* Evaluates the residual of every live case's accepted state (no update) and copies case `slot`'s
 * (nv * n_cells values, SoA) to r. */
int amr_batch_residual(amr_batch* batch, int32_t slot, double* r, uint64_t count, char* error, uint64_t error_size);
/* Replays advances from CUDA graphs (on, the default) or launches their kernels directly. */
int amr_batch_set_graph(amr_batch* batch, int32_t on);
/* Split launch mode, viscous models without SRD: the live cases run as `lanes` (1..4, default 3)
 * independent chains of kernels, each on its own stream over about an equal share of the cells, so
 * that one chain's kernels fill the tails of the others'.  Lanes need every case of one lane to lie
 * below every case of the next in the arena (as after admissions in one order); otherwise one lane
 * runs.  Returns 1 for a count outside 1..4. */
int amr_batch_set_lanes(amr_batch* batch, int32_t lanes);
/* The launch configuration chosen (mode, block, grid, graph or direct, lanes) as text. */
int amr_batch_launch_config(const amr_batch* batch, char* out, uint64_t size);
int amr_gpu_launch_config(const amr_gpu_session* session, char* out, uint64_t size);
/* Kernels the session launched so far. */
uint64_t amr_gpu_kernel_launches(const amr_gpu_session* session);

#ifdef __cplusplus
}
#endif
#endif
