/*
 * rh3t.h — C ABI of the B200 implementation of the 3T_RH semi-discrete
 * operator l() and its SSP-RK3 driver (colinhu123/3T_RH, src/main.rs).
 *
 * The reference exposes this path only as private Rust functions of a binary
 * crate (main.rs:135 l, main.rs:351 rk3_ssp, main.rs:375 calc_global_dt,
 * ghost.rs:199 GhostGrid::update_values_parallel). Each entry point below
 * names the reference item it replaces. Plain pointers and sizes only.
 *
 * Layouts shared with the reference:
 *   - a field value array is nx*ny records of 6 doubles
 *     (rho, mom_x, mom_y, ee, ei, er) at linear index i*ny + j
 *     (field1.rs:205-215, state.rs:18-25);
 *   - a fluid mask is nx*ny bytes at the same linear index (field1.rs:112-122).
 *
 * Errors: every call returns an rh3t_status. The reference panics instead;
 * rh3t_last_error() returns the record a caller needs to re-raise the
 * reference's message (stage label, cell or ghost index).
 *
 * Threading: one context = one CUDA stream; a context must not be used from
 * two threads at once (the reference's l() takes &mut GhostGrid / &mut Scratch).
 */
#ifndef RH3T_H
#define RH3T_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RH3T_ABI_VERSION 2

typedef enum {
    RH3T_OK = 0,
    RH3T_ERR_NONPHYSICAL_STATE = 1, /* main.rs:30-33 assert_admissible panic */
    RH3T_ERR_NONFINITE_GHOST = 2,   /* ghost.rs:229-263 panic */
    RH3T_ERR_SINGULAR_ILW = 3,      /* bc1.rs:467-469 solve6 panic */
    RH3T_ERR_PERIODIC_WRAP = 4,     /* bc1.rs:594-604 panic */
    RH3T_ERR_STENCIL_FIT = 5,       /* bc1.rs:1429-1434 / 1466-1471 panic */
    RH3T_ERR_GEOMETRY = 6,          /* geometry.rs / ghost.rs build-time asserts */
    RH3T_ERR_INVALID_ARGUMENT = 7,
    RH3T_ERR_CUDA = 8,
    RH3T_ERR_NONPOSITIVE_DT = 9,    /* main.rs:464 assert!(dt > 0.0) */
    RH3T_ERR_NO_DEVICE = 10,
    RH3T_ERR_DEVICE_TIMEOUT = 11    /* a bounded device-side wait ran out (no reference counterpart) */
} rh3t_status;

/* field1.rs:6-15 GridInfo: node-centred x = x0 + i*dx, y = y0 + j*dy */
typedef struct {
    int32_t nx, ny;
    double dx, dy, x0, y0;
} rh3t_grid;

/* constant.rs:1-25 as runtime values (the reference's are compile-time
 * constants); rh3t_default_params() returns the reference values.
 * periodic_ly replaces the hardcoded ly = 0.5 of bc1.rs:577. */
typedef struct {
    double gamma_e, gamma_i, gamma_r;
    double cve, cvi, a_rad;
    double kappa_e, kappa_i, kappa_r;
    double omega_ei, omega_er;
    double lambda, weno_q, eps;
    double periodic_ly;
} rh3t_params;

/* bc1.rs:17-28 BCType */
typedef enum {
    RH3T_BC_REFLECTIVE_WALL = 0,
    RH3T_BC_WALL = 1,
    RH3T_BC_PERIODIC = 2,
    RH3T_BC_CONSTANT = 3,
    RH3T_BC_TIME_DEPENDENT = 4,
    RH3T_BC_OUTFLOW = 5,
    RH3T_BC_ZEROTH_ORDER = 6,
    RH3T_BC_FAR_FIELD = 7
} rh3t_bc_kind;

/* One BCType value. state: Constant / FarField state. p_inf, sigma, l_domain:
 * Outflow. TimeDependent carries the one closure the reference uses
 * (init.rs:61-65): state = P0.x <= td_x0 + td_speed*t ? td_left : td_right. */
typedef struct {
    int32_t kind;
    int32_t reserved;
    double state[6];
    double p_inf, sigma, l_domain;
    double td_x0, td_speed;
    double td_left[6], td_right[6];
} rh3t_bc;

/* geometry.rs:661-673 ArcOverride with the arc given by its three points
 * (geometry.rs:492-549 CircularArc::from_three_points). boundary: 0 outer, 1 inner. */
typedef struct {
    int32_t boundary;
    int32_t side_start, side_end;
    int32_t fluid_side; /* 0 Inside, 1 Outside */
    double start[2], mid[2], end[2];
} rh3t_arc;

/* ghost.rs:18-46 GhostGrid::info + bc1.rs:50-57 GhostBC, as SoA arrays.
 * Ghost g: idx[2g..2g+1] = (i, j); proj[5g..5g+4] = (P0.x, P0.y, n.x, n.y, D)
 * (the FINAL projection, ghost.rs:428-456); pre[g] = slot in the GhostBC
 * arrays or -1 (only Wall / Outflow / FarField ghosts have one).
 * GhostBC slot k: nearest[2k..], stencil[55k..] (linear indices i*ny+j),
 * s[979k..], w[225k..], d[5k..] with the offsets of bc1.rs:45-47. */
typedef struct {
    int32_t n_ghosts;
    const int32_t* idx;
    const int32_t* boundary;
    const int32_t* side;
    const double* proj;
    const int32_t* pre;
    int32_t n_heavy;
    const int32_t* nearest;
    const uint32_t* stencil;
    const double* s;
    const double* w;
    const double* d;
} rh3t_ghost_table;

typedef struct {
    int32_t code;     /* rh3t_status */
    int32_t stage;    /* 1..3 for RK stage states ("RK1 state" ...), 0 otherwise */
    int64_t step;     /* step of rh3t_advance in which it happened (0-based) */
    int32_t i, j;     /* cell index (code 1) or ghost grid index (code 2, 3, 4) */
    int32_t ghost;    /* ghost id (codes 2, 3, 4), else -1 */
    int32_t instance; /* failing instance of a batch context (0 for a plain one), -1 if none */
    char message[160];
} rh3t_error;

/* ------------------------------------------------------------------ */
/* Host mirror of Field::new + GhostGrid::build (field1.rs:95-136,     */
/* ghost.rs:50-118, bc1.rs:108-188). Host code, apart from the        */
/* least-squares step of rh3t_geom_build_ghosts_device.               */
/* ------------------------------------------------------------------ */
typedef struct rh3t_geom rh3t_geom;

/* outer_xy / inner_xy: polygon points (x, y) pairs; *_fluid_side 0 Inside,
 * 1 Outside; one rh3t_bc per polygon side (side k spans point k -> k+1).
 * Replaces Field::new (field1.rs:95-136) + the arc registration of
 * init.rs:461-467. */
int rh3t_geom_create(const rh3t_grid* grid, const rh3t_params* params,
                     int32_t n_outer, const double* outer_xy, int32_t outer_fluid_side, const rh3t_bc* outer_bcs,
                     int32_t n_inner, const double* inner_xy, int32_t inner_fluid_side, const rh3t_bc* inner_bcs,
                     int32_t n_arcs, const rh3t_arc* arcs, rh3t_geom** out);
/* field1.rs:112-122 fluid mask, nx*ny bytes */
int rh3t_geom_fluid_mask(const rh3t_geom* g, uint8_t* out);
/* ghost.rs:50-118 GhostGrid::build with ghost.rs:482-493 default offsets;
 * n_threads <= 0 uses all host cores. */
int rh3t_geom_build_ghosts(rh3t_geom* g, int32_t n_threads);
/* GhostGrid::build of n geometries (ghost.rs:50-118) with the GhostBC
 * least-squares tables (bc1.rs:108-188: E_r pseudo-inverses, S_r, w_r)
 * computed on GPU `device`, one warp per Wall / Outflow / FarField ghost,
 * all geometries in one pass. Discovery, projection and E_r stencils are
 * built on the host as by rh3t_geom_build_ghosts; the device tables are
 * bit-identical to that function's. Returns the first failing geometry's
 * status (its rh3t_geom_last_error has the text). n_threads as above. */
int rh3t_geom_build_ghosts_device(int32_t n, rh3t_geom* const* geoms, int32_t n_threads, int32_t device);
/* view of the built tables (valid until rh3t_geom_destroy) */
int rh3t_geom_ghost_table(const rh3t_geom* g, rh3t_ghost_table* view);
/* ghost.rs:71-107 access table, nx*ny*17 u32 (0 for non-fluid cells) */
int rh3t_geom_access_table(const rh3t_geom* g, uint32_t* out);
/* last build error text (NUL-terminated) */
const char* rh3t_geom_last_error(const rh3t_geom* g);
void rh3t_geom_destroy(rh3t_geom* g);

/* ------------------------------------------------------------------ */
/* Device solver                                                       */
/* A context holds one instance (rh3t_create, the drop-in for the      */
/* reference's single Field) or a batch of independent instances       */
/* (rh3t_batch_create). Whole-context calls (rh3t_advance,             */
/* rh3t_rk3_ssp, rh3t_profile_steps, rh3t_synchronize) act on every    */
/* instance with one launch per kernel phase; the single-instance      */
/* calls (rh3t_upload_state, rh3t_download_state, rh3t_l,              */
/* rh3t_calc_global_dt, rh3t_last_dt) act on instance 0.               */
/* ------------------------------------------------------------------ */
typedef struct rh3t_ctx rh3t_ctx;

void rh3t_default_params(rh3t_params* out);

/* Creates the device copy of a Field (grid, mask, BC lists) and its
 * GhostGrid. All tables are copied; the caller keeps ownership.
 * n_outer_bc / n_inner_bc: BC list lengths (field1.rs Field::bc_outer/bc_inner). */
int rh3t_create(const rh3t_grid* grid, const rh3t_params* params, const uint8_t* fluid,
                int32_t n_outer_bc, const rh3t_bc* outer_bcs, int32_t n_inner_bc, const rh3t_bc* inner_bcs,
                const rh3t_ghost_table* ghosts, int32_t device, rh3t_ctx** out);

/* One instance of a batch: the arguments of rh3t_create. */
typedef struct {
    const rh3t_grid* grid;
    const rh3t_params* params;
    const uint8_t* fluid;
    int32_t n_outer_bc;
    const rh3t_bc* outer_bcs;
    int32_t n_inner_bc;
    const rh3t_bc* inner_bcs;
    const rh3t_ghost_table* ghosts;
} rh3t_instance;

/* Batched solver (no reference counterpart: the reference advances one
 * Field per process). n independent instances of any sizes, parameters and
 * BCs, resident together; every kernel launch covers all of them, each
 * instance keeps its own dt reduction, time and error record, and one step
 * of the whole batch replays as one CUDA graph (rh3t_advance). */
int rh3t_batch_create(int32_t n, const rh3t_instance* instances, int32_t device, rh3t_ctx** out);
int32_t rh3t_instance_count(const rh3t_ctx* ctx);
/* values: the instances' Field::value arrays concatenated in instance order;
 * times: one Field::time per instance (may be NULL on download) */
int rh3t_upload_batch(rh3t_ctx* ctx, const double* values, const double* times);
int rh3t_download_batch(rh3t_ctx* ctx, double* values, double* times);
int rh3t_upload_instance(rh3t_ctx* ctx, int32_t k, const double* value, double time);
/* One time-loop iteration of every instance on host arrays (main.rs:460-466
 * for a batch): values / times as for rh3t_upload_batch, replaced by the
 * values and times after one step of dt = cfl_factor * dt_cfl per instance.
 * The instances are taken in n_groups groups of about equal cell counts
 * (n_groups <= 0: 8): the host -> device copy of one group, the step of
 * another and the device -> host copy of a third run at the same time. The
 * overlap needs page-locked host arrays (cudaHostAlloc or a pinned tensor);
 * with pageable ones the result is the same and the copies do not overlap.
 * The first call allocates two streams and a small page-locked buffer. */
int rh3t_step_host_batch(rh3t_ctx* ctx, double* values, double* times, double cfl_factor, int32_t n_groups);
int rh3t_download_instance(rh3t_ctx* ctx, int32_t k, double* value, double* time);
/* rh3t_l of instance k */
int rh3t_l_instance(rh3t_ctx* ctx, int32_t k, double* rhs, double* ghost_values);
/* calc_global_dt of every instance, dt_cfl[n] */
int rh3t_calc_global_dt_batch(rh3t_ctx* ctx, double* dt_cfl);
/* per-instance time, dt of the last step and steps taken (arrays of n, each may be NULL) */
int rh3t_instance_times(rh3t_ctx* ctx, double* t, double* dt, int64_t* steps);
/* per-instance status of the last synchronising call (codes[n]) */
int rh3t_instance_status(const rh3t_ctx* ctx, int32_t* codes);

/* Work-tile shapes (no reference counterpart). Each instance has three
 * shapes, given as log2 of the tile's j extent: x-face tiles of
 * (64 >> lg_fx) x (1 << lg_fx) faces, lg_fx in [2, 4]; y-face tiles of
 * (64 >> lg_fy) x (1 << lg_fy) faces, lg_fy in [4, 6]; RHS tiles of
 * (256 >> lg_rhs) x (1 << lg_rhs) cells, lg_rhs in [4, 6]. Shapes change
 * only the work decomposition: results are bit-identical for every shape.
 * k = -1 sets every instance. */
int rh3t_set_tile_shapes(rh3t_ctx* ctx, int32_t k, int32_t lg_fx, int32_t lg_fy, int32_t lg_rhs);
int rh3t_get_tile_shapes(const rh3t_ctx* ctx, int32_t k, int32_t* lg3);

/* Autotuner: instances are grouped into classes by (nx, ny, diffusion on);
 * for each class every admissible shape of each of the three tile kinds is
 * timed on the class's own instances (CUDA events, `reps` launches, the
 * minimum kept) and the fastest is applied. Results are cached per class in
 * the process and, when cache_path is not NULL, in that text file (read
 * first, rewritten after). out (may be NULL) receives up to max_out
 * entries, one per class. Time it after uploading a state. */
typedef struct {
    int32_t nx, ny, diffusion, n_instances;
    int32_t lg_fx, lg_fy, lg_rhs;
    int32_t from_cache;
    double ms_fx[3], ms_fy[3], ms_rhs[3]; /* per admissible shape, ascending lg; 0 if from cache */
} rh3t_tune_entry;
int rh3t_autotune(rh3t_ctx* ctx, const char* cache_path, int32_t reps, rh3t_tune_entry* out, int32_t max_out,
                  int32_t* n_out);

/* Adjoint (no reference counterpart: the reference has no derivative
 * code). Hand-written vector-Jacobian products of l() and of the SSP-RK3
 * step, for every BC kind (Wall: both ILW solves in reverse; Outflow: the
 * LODI row). Kinks follow the values: d|x|/dx = +1 at 0, max/min pass the
 * derivative to the first argument on ties, FarField rows switch on
 * lambda < 0, the Outflow row on lambda_1 < 0, dt's derivative goes to the
 * first minimising cell. Parameter cotangents per instance (8 doubles): the
 * FarField state (6, one for all FarField sides), omega_ei, omega_er (the
 * Outflow p_inf, sigma, l_domain and Constant / TimeDependent states are
 * held fixed). */
/* rbar: nx*ny*6 cotangent of l()'s result for instance k; ubar (out): the
 * cotangent of the resident state, pbar8 (out, may be NULL). */
int rh3t_l_vjp(rh3t_ctx* ctx, int32_t k, const double* rbar, double* ubar, double* pbar8);
/* Runs nsteps steps of every instance (dt = cfl_factor * dt_cfl, no
 * clipping) from the resident states, saving the states every ckpt_every
 * steps for rh3t_adjoint_backward. */
int rh3t_adjoint_forward(rh3t_ctx* ctx, int32_t nsteps, double cfl_factor, int32_t ckpt_every);
/* Segment records of the sweep (no reference counterpart): the forward run
 * keeps the full record (stage states and rhs of every step) of its last
 * segments, as many as fit in a quarter of the free device memory, so the
 * reverse sweep does not recompute them. rh3t_adjoint_records: the number
 * allocated; rh3t_adjoint_max_records: a cap (0: none) for the next
 * rh3t_adjoint_forward, which then allocates again. */
int32_t rh3t_adjoint_records(const rh3t_ctx* ctx);
int rh3t_adjoint_max_records(rh3t_ctx* ctx, int32_t n);
/* dJ_du: cotangent of the final states (all instances' value arrays
 * concatenated); dJ_du0 (out, same layout): gradient with respect to the
 * initial states; dJ_dparams (out, n x 8, may be NULL). Recomputes each
 * segment from its checkpoint; the resident states are those at the end of
 * the forward run afterwards. */
int rh3t_adjoint_backward(rh3t_ctx* ctx, const double* dJ_du, double* dJ_du0, double* dJ_dparams);

/* io.rs:25-99 save_data: instance k's resident state as an RH3TBIN1 file
 * (header: "RH3TBIN1", u32 version 1, u32 nvar 8, u64 nx, u64 ny, f64 time;
 * payload j-major / i-fastest, per node f64 x, y, rho, mom_x, mom_y, ee, ei,
 * er, the state NaN at non-fluid nodes; little endian). The payload is packed
 * on the device and copied to pinned host memory on the context's stream; a
 * host thread writes `path`.tmp and renames it to `path`, so the call
 * returns before the file is written. The next rh3t_snapshot or
 * rh3t_snapshot_wait joins that write and returns its status. */
int rh3t_snapshot(rh3t_ctx* ctx, int32_t k, const char* path);
int rh3t_snapshot_wait(rh3t_ctx* ctx);
/* io.rs:101-123 load_data: instance k's state and time from an RH3TBIN1
 * file; the header must match (magic, version, nvar, nx, ny) and every fluid
 * node's state must be finite (RH3T_ERR_INVALID_ARGUMENT with the
 * reference's message otherwise). */
int rh3t_restart(rh3t_ctx* ctx, int32_t k, const char* path);
/* py_utils/energy_split.py as a device reduction over instance k's fluid
 * nodes: out[0..2] max |ee - ei|, |ee - er|, |ei - er|; out[3..5] their
 * means; out[6..8] their root mean squares; out[9], out[10] (x, y) of the
 * first node (j-major order) of the maximum |ee - er|; out[11] the number of
 * fluid nodes. */
int rh3t_energy_split(rh3t_ctx* ctx, int32_t k, double* out);

/* Field::value host <-> device (values of non-fluid cells are ignored on
 * upload and returned as 0 on download), plus Field::time. */
int rh3t_upload_state(rh3t_ctx* ctx, const double* value, double time);
int rh3t_download_state(rh3t_ctx* ctx, double* value, double* time);

/* main.rs:135-305 l(): ghost update + fluxes + RHS of the resident state at
 * the resident time. rhs: nx*ny*6 (zero on non-fluid cells) or NULL;
 * ghost_values: n_ghosts*6 (ghost.rs GhostGrid::values) or NULL. */
int rh3t_l(rh3t_ctx* ctx, double* rhs, double* ghost_values);

/* main.rs:375-408 calc_global_dt of the resident state */
int rh3t_calc_global_dt(rh3t_ctx* ctx, double* dt_cfl);

/* Allocation-free calc_global_dt for callers that cannot allocate device
 * memory (a host framework or pool owns all device memory, or an allocation
 * would synchronise the device at that point). No counterpart in the
 * reference (it is a variant of rh3t_calc_global_dt for such callers).
 * d_value: device array of nx*ny records of 6 doubles (i*ny + j), d_fluid:
 * device nx*ny bytes, d_dt_cfl: device double receiving the minimum; the work
 * is queued on `stream` (a cudaStream_t, NULL = default stream) and nothing is
 * allocated or freed. The scratch (one partial minimum per 256 nodes) is a
 * static device array of RH3T_DT_NOALLOC_MAX_CELLS / 256 doubles (512 KiB)
 * that every GPU loading the library keeps until exit: grids of more than
 * RH3T_DT_NOALLOC_MAX_CELLS nodes are rejected with
 * RH3T_ERR_INVALID_ARGUMENT. The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) and keeps it for the life of the
 * process, so the entry point must not be used on a device after a
 * cudaDeviceReset of it: make the first call before any stream capture. All
 * calls share the array, so calls that overlap on the GPU race; calls
 * ordered on one stream are safe (each writes every entry it reads). */
#define RH3T_DT_NOALLOC_MAX_CELLS (65536 * 256)
int rh3t_calc_global_dt_noalloc(const rh3t_grid* grid, const rh3t_params* params, const double* d_value,
                                const uint8_t* d_fluid, double* d_dt_cfl, void* stream);

/* main.rs:351-373 rk3_ssp with a caller-given dt, resident state */
int rh3t_rk3_ssp(rh3t_ctx* ctx, double dt);

/* main.rs:459-477 time loop body repeated nsteps times on the device:
 * dt = cfl_factor * calc_global_dt, clipped to t_final (pass INFINITY for
 * none), then rk3_ssp. dt stays on the device; use_graph != 0 replays one
 * captured CUDA graph per step. */
int rh3t_advance(rh3t_ctx* ctx, int32_t nsteps, double cfl_factor, double t_final, int32_t use_graph);

/* Drop-in step with a host-owned Field::value (the reference's own loop
 * body, main.rs:460-466): upload value, dt = cfl_factor * calc_global_dt,
 * rk3_ssp, download value (in place). dt_out may be NULL. */
int rh3t_step_host(rh3t_ctx* ctx, double* value, double* time, double cfl_factor, double* dt_out);

/* dt of the last step of rh3t_advance / rh3t_step_host (host read) */
int rh3t_last_dt(rh3t_ctx* ctx, double* dt);

/* Instrumentation (no reference counterpart): runs nsteps steps of
 * rh3t_advance without graph capture, with CUDA events around every launch,
 * and returns the summed device time per kernel class in ms_out[0..4]:
 * ghost update, interface fluxes, RHS + stage update, dt reduction, and the
 * number of launches of each class in launches_out[0..4] (may be NULL). */
int rh3t_profile_steps(rh3t_ctx* ctx, int32_t nsteps, double cfl_factor, double* ms_out, int64_t* launches_out);

/* Measured FP64 FMA throughput of the device (TFLOP/s, 2 FLOP per FMA) from a
 * register-resident DFMA loop over all SMs; the FP64 roofline denominator. */
int rh3t_fp64_peak(int32_t device, double* tflops);

/* Diagnostic (no reference counterpart): the device power routines the solver
 * uses in place of the reference's two powf calls (state.rs:261 x^0.25,
 * bc1.rs:241 x^WENO_Q): out[3k] = x[k]^0.25, out[3k+1] = x[k]^10,
 * out[3k+2] = x[k]^q. */
int rh3t_math_check(int32_t device, const double* x, int32_t n, double q, double* out);

/* Diagnostic (no reference counterpart): the shared-reciprocal divisions
 * the solver uses in place of IEEE division where one divisor serves several
 * quotients (Markstein's correction step from y = RN(1/b); the constants 3
 * and 6) against the IEEE quotient, bit for bit, on n device-generated
 * operand pairs: counts[0..6] the mismatches per category (0 random,
 * 1 divisors with all-ones significands, 2 quotients next to a rounding
 * midpoint, 3 range edges and special values, 4 a / 3, 5 a / 6, 6 the
 * reciprocals of a face's 6 c^2 and 3 c^2, formed as 2 and 4 times
 * RN(1 / (12 c^2))); first[3] = a, b and the routine's quotient of one
 * mismatch. */
int rh3t_div_check(int32_t device, int64_t n, uint64_t seed, int64_t* counts, double* first);

/* Diagnostic (no reference counterpart): the bounded mbarrier wait of the
 * ghost update (2^18 try_wait rounds, about a second on a B200, then
 * RH3T_ERR_DEVICE_TIMEOUT) run by
 * one warp on a barrier whose phase completes (arrive != 0) or that nothing
 * completes (arrive == 0): *timed_out = 1 when the wait gave up, 0 when it
 * returned with the phase complete. */
int rh3t_wait_check(int32_t device, int32_t arrive, int32_t* timed_out);

int rh3t_synchronize(rh3t_ctx* ctx);
int rh3t_last_error(const rh3t_ctx* ctx, rh3t_error* out);
/* status of the last rh3t_create / rh3t_batch_create on the calling thread
 * (0 when it succeeded) and its message (the reference's panic text, e.g.
 * "instance 1: periodic wrapped point is not fluid"; bc1.rs:594-604); the
 * failed call returned no context to ask with rh3t_last_error. */
int rh3t_create_error(char* message, int32_t len);
/* number of kernels this context launched since creation (instrumentation) */
int64_t rh3t_kernel_launches(const rh3t_ctx* ctx);
/* the CUDA stream the context runs on (cudaStream_t) */
void* rh3t_stream(const rh3t_ctx* ctx);
void rh3t_destroy(rh3t_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
