/* gelios_b200 — B200-native (sm_100a) plasma time step of Gelios_2D behind a C ABI.
 *
 * The reference (SergeyMSU/Gelios_2D) exposes this path as member functions
 * of its grid class Setka (Setka.h:21-235); each entry point below names the
 * reference interface it stands in for.  The ABI carries only plain pointers,
 * sizes and POD structs: a C++ driver that holds a reference Setka converts
 * its Point/Cell/Gran/Rail pointers to indices (Point::number, Cell::number,
 * All_Gran / All_Gran_copy order) and calls these functions in place of the
 * member functions (a thin C++ shim over these entry points replaces the
 * bodies of Setka::Go_5_komponent__MK2, Go_stationary and
 * Go_stationary_5_komponent_inner_MK2).
 *
 * Conventions
 *   - return 0 on success, a negative GELIOS_E_* code on error; the message
 *     of the last error of the calling thread is gelios_last_error().
 *   - one context per host thread; calls on one context are not re-entrant.
 *   - device memory belongs to the context; host arrays belong to the caller
 *     and are only read/written during the call.
 *   - numbering: points in All_Points order, cells in All_Cells order, faces
 *     unified as All_Gran (main, [0, n_main)) followed by All_Gran_copy
 *     ([n_main, n_faces)); -1 stands for a null pointer.
 *   - enum values are the reference's: Gran_type (Gran.h:8-17), Cell_type
 *     (Cell.h:8-17), Point_type (Point.h:7-22), Rail_type (Rail.h:8-16).
 */
#ifndef GELIOS_B200_H
#define GELIOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GELIOS_ABI_VERSION 1

enum {
    GELIOS_OK = 0,
    GELIOS_E_ARG = -1,      /* bad argument / size */
    GELIOS_E_CUDA = -2,     /* CUDA runtime error */
    GELIOS_E_STATE = -3,    /* call order (e.g. step before topology) */
    GELIOS_E_NODEVICE = -4, /* no CUDA device */
    GELIOS_E_MESH = -5,     /* topology the kernels cannot take */
    GELIOS_E_LIMIT = -6     /* size beyond a stated maximum */
};

/* Step forms (which reference loop gelios_step replaces). */
enum {
    GELIOS_FORM_STATIONARY = 0, /* Setka::Go_stationary(int)                      Setka.h:177, Setka.cpp:5205-5343  */
    GELIOS_FORM_MK2 = 1,        /* Setka::Go_5_komponent__MK2(int)                Setka.h:186, Setka.cpp:10121-10482 */
    GELIOS_FORM_INNER_MK2 = 2,  /* Setka::Go_stationary_5_komponent_inner_MK2(int) Setka.h:176, Setka.cpp:6999-7212  */
    GELIOS_FORM_5_KOMPONENT = 3, /* Setka::Go_5_komponent(int): plasma + four hydrogen fluids, Setka.cpp:8269-8950 */
    GELIOS_FORM_MHD_PUI = 4     /* ion MHD fluid + pickup protons on the moving grid: no reference step (see below) */
};

/* Riemann-solver precision (geometry, accumulation and the dt reduction stay FP64).
 * GELIOS_PREC_FP32_FLUX: the approximate Riemann solvers in FP32.
 * GELIOS_PREC_FP32_WAVES: the plain form's HLLC (GELIOS_FORM_STATIONARY and
 * plain batches) with its sound speeds and wave-speed estimates SL, SR in
 * FP32 and every flux and star state in FP64, so that the FP32 rounding no
 * longer sets a residual floor; the other forms run it as FP64.  No
 * counterpart in the reference (FP64 throughout). */
enum { GELIOS_PREC_FP64 = 0, GELIOS_PREC_FP32_FLUX = 1, GELIOS_PREC_FP32_WAVES = 2 };

/* Runtime replacement of the reference's compile-time constants
 * (Help.h:39-114, Gran.cpp:216-281, Setka.cpp:3380/5256/10129/10169,
 * Solvers.cpp:1206).  gelios_params_reference() fills the reference values. */
typedef struct gelios_params {
    double gamma;        /* adiabatic index ga/ggg */
    double kurant;       /* CFL number */
    double chi;          /* inner-sphere wind speed (chi_real) */
    double inner_mach;   /* inner-sphere Mach number (10) */
    double in_ro, in_p, in_u, in_v, in_Q; /* Input BC state */
    double extern_u_par; /* outflow clamp of Get_par (-0.1) */
    double extern_u_tvd; /* outflow clamp of Get_par_TVD (-0.01) */
    double R11;          /* MK2: cells with centroid radius < R11 are not updated */
    double rad_stat;     /* Go_stationary: radial scaling below this radius (95) */
    double R1, R111, R5, Left; /* rail geometry of Move_Setka_Calculate_2 */
    double koef;         /* Move_surface damping (0.1) */
    double src_rmin, src_rmax; /* radial window of the source re-interpolation */
    double src_coef;     /* n_p_LISM_/Kn_ */
    double a_2;          /* charge-exchange cross-section coefficient */
    double ro_floor, p_floor; /* update clamps (1e-5, 1e-6) */
    double dt0;          /* dt of the first step of every call (1e-8) */
    int32_t n_inner;     /* rail points of the inner layer (20) */
    int32_t n_outer_shock; /* (13) */
    int32_t godunov_max_iter; /* Newton/bisection cap (1100); exceeded -> status flag, never a trap */
    int32_t precision;   /* GELIOS_PREC_* */
} gelios_params;

/* Topology + geometry of a Setka, as flat arrays (read during the call only). */
typedef struct gelios_mesh_view {
    int32_t dims[8]; /* N1..M4 passed to Setka(N1..M4), zeros for grids without rails */
    int32_t n_points;
    const double *x, *y;           /* Point::x, y */
    const int32_t *point_type;     /* Point::type */
    int32_t n_cells;
    const int32_t *cell_type;      /* Cell::type */
    const int32_t *contour_start;  /* n_cells+1, CSR of Cell::contour */
    const int32_t *contour;
    const int32_t *gran_start;     /* n_cells+1, CSR of Cell::Grans (order = flux summation order) */
    const int32_t *gran;
    const int32_t *cell_back, *cell_next; /* Cell::Back/Next (TVD_prepare), may be NULL */
    const double *r_istoch;        /* Cell::r_istoch, may be NULL */
    int32_t n_faces, n_main;
    const int32_t *face_A, *face_B, *face_type, *face_master, *face_sosed, *face_copy;
    const int32_t *face_sosed_up, *face_sosed_down; /* may be NULL: then computed like TVD_prepare */
    int32_t n_rails;               /* A_Rails, B_Rails, C_Rails, D_Rails concatenated */
    const int32_t *rail_type;
    const double *rail_s;
    const int32_t *rail_M;         /* 4 per rail: M1..M4 */
    const int32_t *rail_pstart, *rail_points; /* CSR of Rail::All_point */
    const int32_t *rail_kstart, *rail_keys;   /* CSR of Rail::Key_point */
    int32_t n_contact, n_inner_line, n_outer_line;
    const int32_t *line_contact, *line_inner, *line_outer; /* Line_Contact/Inner/Outer (sorted by polar angle) */
} gelios_mesh_view;

#define GELIOS_STATUS_WAVE_ORDER 32

typedef struct gelios_status {
    int32_t flags;      /* bit0 Newton/bisection cap, bit1 non-positive TVD state,
                           bit2 negative Newton pressure, bit3 broken source chain,
                           bit4 non-finite dt, bit5 MHD wave speeds out of order
                           (GELIOS_STATUS_WAVE_ORDER) */
    int32_t steps_done;
    int64_t n_ro_clamp; /* updates clamped to ro_floor */
    int64_t n_p_clamp;  /* updates clamped to p_floor */
    double dt;          /* dt computed by the last step (the one the next step would use) */
    int32_t result_buf; /* buffer (0/1) that holds the newest state, like par[] in the reference */
    int32_t pad_;
} gelios_status;

typedef struct gelios_ctx gelios_ctx;
typedef struct gelios_mesh gelios_mesh;

/* ---- parameters ---------------------------------------------------------- */
void gelios_params_reference(gelios_params *out);
const char *gelios_last_error(void);
int gelios_abi_version(void);

/* ---- native grid builders (host) -------------------------------------------
 * Setka::Setka(N1,N2,N3,N4,M1,M2,M3,M4), Setka.cpp:19-1076: same points,
 * cells, faces, rails and Line_* lists in the same order (bit-exact). */
gelios_mesh *gelios_mesh_build_setka(int N1, int N2, int N3, int N4, int M1, int M2, int M3, int M4);
/* Axisymmetric polar half-plane grid: n_theta x n_r quads, rays uniform in
 * 0..pi, radii log-spaced r_in..r_out; Axis faces on both rays, Inner_sphere
 * faces at r_in, Input faces on the outer arc for theta < pi/2, Extern beyond. */
gelios_mesh *gelios_mesh_build_polar(int n_theta, int n_r, double r_in, double r_out);
/* Setka::TVD_prepare, Setka.cpp:1294-1492: Sosed_up/Sosed_down of every face,
 * Back/Next/r_istoch of every cell (uses the reference's colliding face numbers). */
int gelios_mesh_tvd_prepare(gelios_mesh *m);
/* Setka::TVD_prepare on a caller's view: fills n_faces Sosed_up/Sosed_down
 * and n_cells Back/Next/r_istoch (any output pointer may be NULL). */
int gelios_tvd_prepare_view(const gelios_mesh_view *v, int32_t *sosed_up, int32_t *sosed_down, int32_t *back,
                            int32_t *next, double *r_istoch);
/* The same with the face numbering chosen: unique_face_numbers = 0 for a grid
 * built by the constructor (All_Gran and All_Gran_copy numbered from 0 each),
 * 1 for a grid loaded by Setka::Download_Setka_ALL_ALPHA_2_0 (main faces then
 * copies, Setka.cpp:3213-3224).  TVD_prepare compares these numbers
 * (Setka.cpp:1328, 1383), so the two grids get different TVD neighbours. */
int gelios_tvd_prepare_view_numbered(const gelios_mesh_view *v, int unique_face_numbers, int32_t *sosed_up,
                                     int32_t *sosed_down, int32_t *back, int32_t *next, double *r_istoch);
/* Cells whose centroid radius is <= r_max (All_Cells_Inner, Gelios_2D.cpp:152-231). */
int gelios_mesh_inner_cells(const gelios_mesh *m, double r_max, int32_t *out, int32_t cap);
/* Pointers into the mesh (valid until gelios_mesh_free). */
int gelios_mesh_get_view(const gelios_mesh *m, gelios_mesh_view *out);
void gelios_mesh_free(gelios_mesh *m);

/* ---- device context --------------------------------------------------------
 * gelios_create: stands in for the Setka instance that owns par[0/1] and the
 * points; it owns device buffers and one CUDA stream on `device`. */
int gelios_create(gelios_ctx **out, const gelios_params *prm, int device);
int gelios_set_params(gelios_ctx *ctx, const gelios_params *prm);
void gelios_destroy(gelios_ctx *ctx);
/* Copies the topology (and current point coordinates) to the device. */
int gelios_upload_topology(gelios_ctx *ctx, const gelios_mesh_view *mesh);
/* Cell::par[buf].ro/p/u/v/Q for all cells (host arrays of n_cells doubles). */
int gelios_upload_state(gelios_ctx *ctx, int buf, const double *ro, const double *p, const double *u,
                        const double *v, const double *Q);
int gelios_download_state(gelios_ctx *ctx, int buf, double *ro, double *p, double *u, double *v, double *Q);
/* The four hydrogen fluids of Cell::par[buf] (Cell.h:27-46) for
 * GELIOS_FORM_5_KOMPONENT: rows16 = ro_H1, p_H1, u_H1, v_H1, ..., v_H4, each
 * n_cells long (16 * n_cells doubles). */
int gelios_upload_hydrogen(gelios_ctx *ctx, int buf, const double *rows16);
int gelios_download_hydrogen(gelios_ctx *ctx, int buf, double *rows16);
/* Monte-Carlo moments left in Cell::par[0] by MK_start_new (Setka.cpp:12241-12449):
 * Hn/Hu/Hv/HT are [cell*4 + sort], ku/kv/kT are per cell. */
int gelios_upload_mc(gelios_ctx *ctx, const double *Hn, const double *Hu, const double *Hv, const double *HT,
                     const double *ku, const double *kv, const double *kT);
/* All_Cells_Inner for GELIOS_FORM_INNER_MK2. */
int gelios_set_inner_cells(gelios_ctx *ctx, const int32_t *cells, int32_t n);
/* Runs `nsteps` iterations of the chosen loop (each call restarts dt at dt0,
 * as the reference does).  Asynchronous on the context stream unless
 * `status` is non-NULL, in which case it synchronises and fills it. */
int gelios_step(gelios_ctx *ctx, int form, int nsteps, gelios_status *status);
/* Point::x,y (after motion) for all points. */
int gelios_download_points(gelios_ctx *ctx, double *x, double *y);
int gelios_synchronize(gelios_ctx *ctx);
/* Device-resident pointers of the state buffers (5 x n_cells doubles each,
 * rows ro,p,u,v,Q) for callers that keep data in HBM. */
int gelios_state_device_ptr(gelios_ctx *ctx, int buf, double **dptr);
/* The context's CUDA stream (cudaStream_t as void*). */
void *gelios_stream(gelios_ctx *ctx);
/* Kernel launches issued by the last gelios_step call. */
int64_t gelios_last_launch_count(gelios_ctx *ctx);
/* Phase timing: when enabled, gelios_step brackets each phase with CUDA
 * events on the context stream and accumulates, per phase, the device time
 * and the number of launches (phases: 0 centroids, 1 face fluxes,
 * 2 surface tracking + rail motion, 3 cell update, 4 commit/dt).  gelios_phase_times
 * synchronises, writes ms[5] and launches[5] accumulated since the last
 * reset, and resets when `reset` is non-zero. */
int gelios_set_phase_timing(gelios_ctx *ctx, int enabled);
int gelios_phase_times(gelios_ctx *ctx, double *ms, int64_t *launches, int reset);

/* ---- MHD + pickup-proton moving-grid step ---------------------------------
 * GELIOS_FORM_MHD_PUI has no counterpart among the reference's steps (the
 * reference steps gas dynamics only; its MHD solvers are never called).  It
 * is the moving-grid step of GELIOS_FORM_MK2 (same surface tracking and rail
 * motion, Setka.cpp:3378-3844 and 4324-4759, driven by the ion fluid's
 * gas-dynamic state) for two fluids:
 *   - ions, ideal MHD: ro, p, u, v, Q in the state rows of gelios_upload_state
 *     and w (u_phi), Bx, By, Bz (B_phi) in the extra rows; Gaussian units
 *     (magnetic pressure B^2/8pi).  Face flux: HLLD of Solvers::HLLDQ_Korolkov
 *     (Solvers.cpp:1642-2185, metod 3) in the face frame, the states shifted
 *     by the face speed, transformed back to the moving-face flux F - W U;
 *   - pickup protons, gas dynamics: ro, p, u, v in the extra rows; face flux
 *     HLLC of HLLC_2d_Korolkov_b_s (Setka.cpp:10484-10700).
 * Cell update: the MK2 update (Setka.cpp:10425-10468) extended with the
 * axisymmetric terms of both fluids (radial momentum p_T + ro w^2 -
 * B_phi^2/4pi, azimuthal momentum -(ro v w - B_r B_phi/4pi), B_phi (v B_phi -
 * w B_r)) and the caller's fixed charge-exchange sources of the ion
 * momentum and energy (gelios_upload_sources).
 * Extra rows (gelios_upload_mhd): w, Bx, By, Bz, ro_pui, p_pui, u_pui, v_pui,
 * each n_cells long (8 * n_cells doubles). */
typedef struct gelios_mhd_params {
    double lism_bx, lism_by, lism_bz; /* B of the Input boundary state */
    double inner_bphi;               /* B_phi of the inner-sphere state at r = R1 on the equator (falls as R1 sin(theta)/r) */
    double pui_in_ro, pui_in_p;      /* pickup protons of the Input boundary state (moving with the inflow) */
    double pui_inner_ro, pui_inner_p; /* pickup protons of the inner-sphere state, fractions of the wind's ro and p */
} gelios_mhd_params;

int gelios_set_mhd_params(gelios_ctx *ctx, const gelios_mhd_params *mp);
int gelios_upload_mhd(gelios_ctx *ctx, int buf, const double *rows8);
int gelios_download_mhd(gelios_ctx *ctx, int buf, double *rows8);
/* Fixed charge-exchange sources of the ion fluid per unit volume: x and y
 * momentum, energy (n_cells each); read by GELIOS_FORM_MHD_PUI. */
int gelios_upload_sources(gelios_ctx *ctx, const double *q1, const double *q2, const double *q3);

/* ---- residual (no counterpart in the reference: it has no residual) --------
 * gelios_residual: the L1 residual of the density over the last step,
 * sum |ro(n+1) - ro(n)| / sum |ro(n+1)| between the two state buffers
 * (result_buf is the newer one); deterministic device reduction.
 * gelios_run_to_residual: calls of `check_every` (even, > 0) steps of `form`
 * until the residual per unit time, residual / dt, is at most `tol` or
 * `max_steps` steps ran; each call restarts dt at dt0, as gelios_step does.
 * Returns the steps run, the last residual per unit time and the dt. */
int gelios_residual(gelios_ctx *ctx, int result_buf, double *residual);
int gelios_run_to_residual(gelios_ctx *ctx, int form, double tol, int64_t max_steps, int32_t check_every,
                           int64_t *steps_done, double *residual_per_time, double *dt);
/* gelios_operator_residual: the residual of a moving-grid operator
 * (form GELIOS_FORM_MK2 or GELIOS_FORM_MHD_PUI) at state par[buf] (and the
 * MHD form's extra rows of buffer buf) with the grid held still: every face
 * flux of the step (the same reconstructions and Riemann solvers) evaluated
 * at face speed 0 on the current points, then sum over updated cells of
 * |sum of the cell's (ion) mass fluxes F.S| / volume, divided by sum |ro|:
 * the L1 density change per unit time of the flow alone, without the volume
 * change of moving cells that the step residual above contains.  Writes
 * only scratch (the moved-point buffer is set to the current points); the
 * state, the points and the dt words stay. */
int gelios_operator_residual(gelios_ctx *ctx, int form, int buf, double *residual);
/* gelios_mk2_source_terms: the charge-exchange source terms the moving-grid
 * step adds per cell, Cell::Get_Sourse_MK1 (Cell.cpp:498-665) as
 * Go_5_komponent__MK2 calls it (Setka.cpp:10414-10420), for the state
 * par[buf], the current points' cell centres and the uploaded Monte-Carlo
 * moments (gelios_upload_mc): q1, q2, q3 (n_cells each, host arrays) = the
 * x-momentum, y-momentum and energy sources; 0 for the cells the step does
 * not update (centre radius < R11).  The step's own kernel, run alone (for
 * checking it and for callers that want the sources).  GELIOS_E_STATE where
 * an interpolation chain link the reference would follow is missing. */
int gelios_mk2_source_terms(gelios_ctx *ctx, int buf, double *q1, double *q2, double *q3);

/* ---- streamed host I/O (no counterpart in the reference) --------------------
 * For callers that feed a fresh state from host memory every step and read
 * every result back (a host code coupled to the step, or a driver timing
 * the step end to end).  Runs `nsteps` one-step calls of `form`, each like
 * gelios_step(ctx, form, 1, NULL) (dt restarts at dt0): call k copies
 * host_in[k] into par[0], steps, and copies par[1] into host_out[k].  A host
 * block holds gelios_io_rows(form) rows of n_cells doubles: ro, p, u, v, Q,
 * then the form's extra rows (the 16 hydrogen rows of
 * GELIOS_FORM_5_KOMPONENT, the 8 rows of GELIOS_FORM_MHD_PUI).  The copies
 * of call k+1's input and of call k-1's result run on two copy streams
 * while call k steps, through device staging buffers (two per direction,
 * allocated on first use); host blocks should be pinned for the copies to
 * overlap.  Returns once every result is in host memory. */
int gelios_io_rows(int form);
int gelios_run_streamed(gelios_ctx *ctx, int form, int nsteps, const double *const *host_in, double *const *host_out);

/* ---- batched instances (no counterpart in the reference) -------------------
 * Many independent instances of GELIOS_FORM_MHD_PUI (a parameter sweep: each
 * context its own grid, inflow, state and dt) advanced together: every
 * phase of a step (surface tracking, rails, face units, cell update,
 * commit) is one launch over all instances, the step a CUDA graph.  The
 * contexts must live on one device, have their topology, MHD data and
 * sources uploaded and one flux precision; the batch runs on the first
 * context's stream and leaves each context's results where gelios_step
 * would (par[nsteps % 2], points, dt).  statuses: n entries or NULL (then
 * the call does not wait for the GPU). */
typedef struct gelios_batch gelios_batch;
int gelios_batch_create(gelios_batch **out, gelios_ctx *const *ctxs, int n);
int gelios_batch_step(gelios_batch *batch, int form, int nsteps, gelios_status *statuses);
void gelios_batch_destroy(gelios_batch *batch);
/* How a batch runs its steps.  schedule 0: one launch per phase, each step
 * a captured CUDA graph (the default).  schedule k > 0: every step of a
 * call in ONE persistent cooperative kernel of k 128-thread blocks per SM,
 * the phases separated by grid barriers, the tiles of all instances dealt
 * to the blocks by grid stride; both schedules compute the same per-face
 * and per-cell bodies.  GELIOS_E_ARG if k blocks per SM cannot be
 * co-resident.  gelios_batch_autotune runs `steps` real steps of the sweep
 * for each schedule (0 and every k that fits; each advances every
 * instance, once untimed and once timed), keeps the fastest and returns it
 * with its time per step in ms (either pointer may be NULL); each_ms[k]
 * (k < n_each; each_ms may be NULL when n_each is 0) receives schedule k's
 * time per step, -1 where k blocks per SM do not fit. */
int gelios_batch_set_schedule(gelios_batch *batch, int32_t schedule);
int gelios_batch_get_schedule(gelios_batch *batch, int32_t *schedule);
int gelios_batch_autotune(gelios_batch *batch, int steps, int32_t *schedule, double *ms, double *each_ms, int n_each);

/* ---- batched plain-form instances (no counterpart in the reference) --------
 * Instances of GELIOS_FORM_STATIONARY that share one mesh (the contexts
 * were given the same gelios_mesh_view) and differ in parameters (inflow
 * and inner-wind states) and state: an inflow-parameter sweep marched to a
 * steady state.  All listed instances advance in one cooperative launch per
 * call (each with its own dt); results stay where gelios_step would leave
 * them (par[nsteps % 2] of each context).  Contexts must live on one device
 * and share one flux precision; the batch drains their streams before it
 * runs.
 * gelios_plain_batch_step: `nsteps` steps of every instance; statuses: n
 * entries or NULL.
 * gelios_plain_batch_run_to_residual: gelios_run_to_residual for every
 * instance at once: chunks of `check_every` (even) steps, after each chunk
 * the instances whose residual per unit time is at most `tol` (or whose
 * step reported a failure flag) stop; the others go on until `max_steps`.
 * Per instance (arrays of n, each may be NULL): steps run, last residual
 * per unit time, last dt. */
typedef struct gelios_plain_batch gelios_plain_batch;
int gelios_plain_batch_create(gelios_plain_batch **out, gelios_ctx *const *ctxs, int n);
int gelios_plain_batch_step(gelios_plain_batch *batch, int nsteps, gelios_status *statuses);
int gelios_plain_batch_run_to_residual(gelios_plain_batch *batch, double tol, int64_t max_steps,
                                       int32_t check_every, int64_t *steps_done, double *residual_per_time,
                                       double *dt);
void gelios_plain_batch_destroy(gelios_plain_batch *batch);

/* ---- warm-start network (no counterpart in the reference) ------------------
 * A coordinate MLP trained and evaluated on the GPU by the library's own
 * kernels: bf16 tensor-core GEMMs with fp32 accumulation, GELU, mean squared
 * error, Adam on fp32 master weights.  Rows of n_in raw inputs; the network
 * input is the raw row followed by sin(2^f pi s), cos(2^f pi s), f <
 * n_fourier, of its last two entries (the position), i.e. n_in + 4
 * n_fourier values; then `depth` hidden layers of `width` with GELU and a
 * linear output layer of n_out.  Parameters are one flat fp32 vector: per
 * layer the weight [out][in] (row-major) then the bias [out].
 * gelios_mlp_set_params also resets the Adam moments and step count.
 * gelios_mlp_loss_grad: mean squared error of M (<= max_batch) host rows
 * against host targets and (grad != NULL) its gradient, without an update.
 * gelios_mlp_set_data: the training set (host rows), kept on the device.
 * gelios_mlp_train: `iters` Adam steps on mini-batches of `batch` rows drawn
 * from the training set by a hash of (seed, step, row); learning rate linear
 * from 0 over `warmup` steps, then cosine from lr_max down to lr_min; the
 * batch loss of every step into loss_hist (iters floats, may be NULL).
 * gelios_mlp_predict: outputs of M host rows (in chunks of max_batch).
 * gelios_mlp_gemm_bf16: the GEMM alone (device pointers; C = A . B^T with
 * A[m][k] at A[m lda + k], B[n][k] at B[n ldb + k], C fp32 rows of ldc;
 * stream may be NULL), for checks. */
typedef struct gelios_mlp gelios_mlp;
int gelios_mlp_create(gelios_mlp **out, int device, int n_in, int n_fourier, int width, int depth, int n_out,
                      int max_batch);
void gelios_mlp_destroy(gelios_mlp *mlp);
int64_t gelios_mlp_param_count(const gelios_mlp *mlp);
int gelios_mlp_set_params(gelios_mlp *mlp, const float *params, int64_t n);
int gelios_mlp_get_params(const gelios_mlp *mlp, float *params, int64_t n);
int gelios_mlp_loss_grad(gelios_mlp *mlp, const float *x, const float *t, int M, double *loss, float *grad);
int gelios_mlp_set_data(gelios_mlp *mlp, const float *x, const float *t, int64_t n_rows);
int gelios_mlp_train(gelios_mlp *mlp, int iters, int batch, float lr_max, float lr_min, int warmup, uint64_t seed,
                     float *loss_hist);
int gelios_mlp_predict(gelios_mlp *mlp, const float *x, int64_t M, float *y);
int gelios_mlp_gemm_bf16(int M, int N, int K, const void *A, int64_t lda, const void *B, int64_t ldb, float *C,
                         int64_t ldc, void *stream);
/* gelios_mlp_time_layer: device time of one hidden layer of the network's
 * forward pass, an M x N x K bf16 GEMM with bias + GELU (seeded operands
 * allocated for the call): tma != 0 the TMA-staged GEMM applying bias + GELU
 * as the accumulator leaves tensor memory and storing the Z / H tiles
 * through shared memory with the TMA (what the forward pass uses), tma == 0
 * the cp.async-staged GEMM followed by a separate bias + GELU kernel.
 * `reps` layers back to back, captured in one CUDA graph and replayed once
 * untimed, then timed with CUDA events on a private stream; mean ms per
 * layer.  For measurements; no counterpart in the reference. */
int gelios_mlp_time_layer(int M, int N, int K, int reps, int tma, double *ms);

/* ---- autotuning of launch shapes (no counterpart in the reference) ---------
 * The dominant kernel of the MHD form (its face kernel) has
 * gelios_variant_count(form) launch shapes (threads per block x resident
 * blocks per SM, i.e. a register cap); the moving-grid form
 * (GELIOS_FORM_MK2) has as many variants of its face units + cell update:
 * a face kernel writing flux slots in global memory followed by an update
 * kernel (variants 0-3; 8-10 the same with every gather of a face unit
 * prefetched into L1), or one kernel per tile of cells with the slots in
 * shared memory (4-7, slower in the whole step; gelios_autotune for this
 * form times variants 0-3 and 8-10).  All give the same bits.
 * gelios_autotune times each shape on the context's grid and current state
 * (`reps` launches each, CUDA events on the context stream; only scratch
 * buffers are written, the state and the points are not touched), keeps the
 * fastest for the steps that follow and returns its index and mean time in
 * ms (either pointer may be NULL).  gelios_set_variant picks a shape by
 * hand (GELIOS_E_ARG outside [0, count)).  Forms without variants: count 1,
 * autotune returns variant 0. */
int gelios_variant_count(int form);
int gelios_autotune(gelios_ctx *ctx, int form, int reps, int32_t *variant, double *ms);
int gelios_set_variant(gelios_ctx *ctx, int form, int32_t variant);
/* The variant a context uses for `form` (set by hand or by gelios_autotune;
 * 0 for forms without variants). */
int gelios_get_variant(gelios_ctx *ctx, int form, int32_t *variant);
/* Pipelined moving-grid calls (on by default; no counterpart in the
 * reference): within a call of two or more GELIOS_FORM_MK2 steps, the next
 * step's surface tracking and rail motion (Setka::Move_surface,
 * Move_Setka_Calculate_2) run while the cells they do not read are still
 * being updated.  Same results bit for bit as one step after the other
 * (on = 0), which one-step calls, the tile variants (4-7) and phase timing
 * always use. */
int gelios_set_pipelined(gelios_ctx *ctx, int on);

/* ---- per-face solvers on the device (known-answer checks) ------------------
 * Batched HLLC_2d_Korolkov_b_s (Setka.cpp:10484-10700): in[n*16] =
 * roL,QL,pL,v1L,v2L, roR,QR,pR,v1R,v2R, W, n1, n2, rad, metod, nul_potok;
 * out[n*9] = time, P0..P3, PQ, Vl, Vc, Vp.  Host arrays. */
int gelios_hllc_batch(const gelios_params *prm, int n, const double *in, double *out);
/* Batched Godunov_Solver_Alexashov (Solvers.cpp:693-1172): in[n*15] =
 * q1[5] (ro,p,u,v,w), q2[5], n[3], w, dist; out[n*10] = time, q[5], dsl, dsp, dsc, status. */
int gelios_godunov_batch(const gelios_params *prm, int n, const double *in, double *out);
/* Batched Solvers::HLLDQ_Korolkov (Solvers.cpp:1642-2185), MHD flux with the
 * normal along a coordinate axis: in[n*23] = L[9], R[9] with states (ro, Q,
 * p, v1, v2, v3, Bx, By, Bz), n1, n2, n3, rad, metod (2: HLLC-type, 3:
 * HLLD); out[n*10] = time, P[8] (mass, momentum x3, B x3, energy), PQ. */
int gelios_hlldq_batch(const gelios_params *prm, int n, const double *in, double *out);
/* Batched Solvers::HLLD_Solver_Alexashov (Solvers.cpp:92-691): in[n*21] =
 * q1[8], q2[8] with q = (ro, p, u, v, w, bx, by, bz), n[3] (unit, any
 * direction), w (face speed), dist; out[n*13] = time, q[8] (mass, momentum
 * x3, B x3, energy), dsl, dsp, dsc, status (GELIOS_STATUS_WAVE_ORDER where
 * the reference exits). */
int gelios_hlld_batch(const gelios_params *prm, int n, const double *in, double *out);

/* ---- allocation-free plain step (no counterpart in the reference) ---------
 * For callers that cannot call cudaMalloc when they step (their device memory
 * is handed out up front by their own pool, or they step where the CUDA
 * allocator must not be touched): one step of the plain single-fluid form
 * (the same kernels as gelios_step with GELIOS_FORM_STATIONARY) on a grid
 * and state the caller already holds in device memory.  Nothing is
 * allocated: the step's scratch (face-slot fluxes, centroids, dt words) is
 * one fixed file-scope device array of about 6.0 MB that every GPU loading
 * the library holds until exit, so grids are limited to
 * GELIOS_NOALLOC_MAX_CELLS cells and GELIOS_NOALLOC_MAX_SLOTS face slots
 * (GELIOS_E_LIMIT beyond).  The array is reserved when the CUDA module of the
 * library loads on a device, which under lazy module loading (the default
 * since CUDA 12.2) is the first call on that device; the first call on a
 * device also resolves the array's device address (cached per device ordinal
 * for the life of the process, so it goes stale after cudaDeviceReset or a
 * different driver context on that device).  Make one call before any stream
 * capture and before handing the rest of the device memory to a pool.  All
 * calls share the array: calls that overlap on the GPU (other streams, other
 * threads) race.  Inputs: the grid arrays below, state_in[5] (ro, p, u, v, Q
 * per cell) and dt_in (one device double, the dt of this step); outputs:
 * state_out[5] (every cell: C_centr cells, which the step leaves unchanged,
 * are copied from state_in) and dt_out (the dt the next step would use).
 * Density / pressure floor counts and status flags are not reported (the
 * context path returns them in gelios_status).  Runs on `stream`
 * (cudaStream_t as void*, may be NULL) and returns without synchronising. */
#define GELIOS_NOALLOC_MAX_CELLS 32768
#define GELIOS_NOALLOC_MAX_SLOTS 131072

typedef struct gelios_device_grid {
    int32_t n_cells, n_slots, n_units;
    const double *x, *y;               /* point coordinates */
    const int32_t *contour_start;      /* n_cells+1 */
    const int32_t *contour;
    const int32_t *gran_start;         /* n_cells+1: face slots of cell c are gran_start[c].. */
    const uint32_t *cell_flags;        /* bit0 has an Axis face, bit1 C_1, bit2 C_centr */
    const int32_t *slot_A, *slot_B;    /* end points of the face in each slot */
    const int32_t *slot_nb;            /* Sosed of the face (-1 if none) */
    const uint32_t *slot_info;         /* Gran_type | 8 both ends tracked | 16 one end tracked */
    const int32_t *unit_slot, *unit_cell, *unit_twin; /* flux evaluations: owner slot, owner cell,
                                                           twin slot of an interior face or -1 */
} gelios_device_grid;

int gelios_stationary_step_noalloc(const gelios_params *prm, const gelios_device_grid *grid,
                                   const double *const *state_in, double *const *state_out, const double *dt_in,
                                   double *dt_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
