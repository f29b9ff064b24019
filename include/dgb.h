/*
 * dgb.h -- C ABI of the B200-native DG residual / time-step path for the 1D/2D
 * gamma-model multifluid Euler solver (drop-in for the reference's DG_SOLVER / RK /
 * Limiting path).
 *
 * Two layers:
 *   1. Host setup (C++; needs no GPU).  Replaces the setup sequence of the reference
 *      driver code/src/main.cc:75-906: deck parsing (code/src/deck/deck.cc:11), Gmsh 2.2
 *      mesh reading (code/src/mesh/simpleMesh.cc:141), interfaces/normals/neighbours
 *      (simpleMesh.cc:206, 664, 770), nodal Lagrange basis and Gauss quadrature
 *      (code/src/polynomials/polynomialBasis.cc:938, code/src/quadratures/Gauss*.cc),
 *      Jacobians and inverse mass matrices (code/src/dg/dg_functions.cc:33-174) and the
 *      limiter's Lagrange<->monomial transforms (main.cc:558-583, 1348-1524).
 *   2. Device context (CUDA, sm_100a).  Replaces the reference's device-side path:
 *      DG_SOLVER::dg_solver (code/src/dg/dg_solver.h:292), Lsolver
 *      (code/src/time_integration/rk_kernels.cu:182), Limiting::HRlimiting/M2limiting
 *      (code/src/limiting/limiting.cc:11, 123, 596-742), SENSOR::sensing (code/src/sensors/sensor.cc:11),
 *      RK::DtFromCFL (code/src/time_integration/rk.cc:250)
 *      and RK::RK_integration (rk.cc:11).
 *
 * Conventions (all entry points):
 *   - every call returns an int status (DGB_OK == 0); dgb_last_error() gives a message.
 *     The reference exits the process on these conditions (rk.cc:147-148, deck.cc:58-61,
 *     simpleMesh.cc:412-415); here they are returned.
 *   - state arrays in the reference layout: U[(e*N_F + f)*N_s + i], float64, element-major,
 *     field-major within the element, Gmsh node order fastest (main.cc:814-820).
 *   - the library owns all device memory of a context; calls on one context are not reentrant.
 *   - no CPU fallback: device entry points fail with DGB_ERR_NO_DEVICE / DGB_ERR_CUDA when the
 *     GPU path cannot run.
 */
#ifndef DGB_H
#define DGB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DGB_ABI_VERSION 2

enum dgb_status {
  DGB_OK = 0,
  DGB_ERR_ARG = 1,         /* bad argument, size or name */
  DGB_ERR_IO = 2,          /* deck / mesh / .pos file missing or malformed */
  DGB_ERR_MESH = 3,        /* interface without two sides, bad neighbour normal */
  DGB_ERR_UNSUPPORTED = 4, /* configuration outside the GPU path (see dgb_last_error) */
  DGB_ERR_CUDA = 5,        /* CUDA runtime error */
  DGB_ERR_NONFINITE = 6,   /* time step is NaN (reference rk.cc:148 exits) */
  DGB_ERR_DT_SMALL = 7,    /* time step < 1e-14 (reference rk.cc:147 exits) */
  DGB_ERR_TIMEOUT = 8,     /* a bounded device wait expired */
  DGB_ERR_NO_DEVICE = 9    /* no CUDA device / wrong architecture */
};

/* Riemann solver (compile-time FLUX=RUS|HLL|ROE in the reference Makefile:30-51). */
enum dgb_flux { DGB_FLUX_RUSANOV = 0, DGB_FLUX_HLL = 1, DGB_FLUX_ROE = 2 };

/* Limiter codes, same numbering as the reference deck strings (main.cc:167-175). */
enum dgb_limiter {
  DGB_LIM_NONE = 0, DGB_LIM_HRL = 1, DGB_LIM_M2L = 2, DGB_LIM_HRI = 3,
  DGB_LIM_M2I = 4, DGB_LIM_PRL = 5, DGB_LIM_PRI = 6, DGB_LIM_P0I = 7
};

/* Arithmetic of the residual kernels.  FP64: plain double precision (the parity form).  MIXED:
 * basis contractions, Rusanov flux and lift in FP32 on deviations from a per-element FP64 anchor;
 * state, pressure recovery, Roe solver and stage update in FP64 (structured 2D grids, p <= 3). */
enum dgb_form { DGB_FORM_FP64 = 0, DGB_FORM_MIXED = 1 };

/* Gamma model (GAMM of the reference Makefile): GAMNCON carries alpha = 1/(gamma-1) with a
 * non-conservative source, GAMCONS carries rho/(gamma-1) conservatively. */
enum dgb_gamma_model { DGB_GAMNCON = 0, DGB_GAMCONS = 1 };

/* Time integrators: classical RK4 (reference rk.h:44-57) and Shu-Osher SSP-RK3 (new). */
enum dgb_scheme { DGB_SSPRK3 = 3, DGB_RK4 = 4 };

/* Gmsh physical tags used for boundaries (simpleMesh.cc:842-845, 702; boundaries.cu:20). */
enum dgb_bc { DGB_BC_PERIODIC = 1, DGB_BC_TRANSMISSIVE = 2, DGB_BC_REFLECTIVE = 3, DGB_BC_FROZEN = 4 };

const char* dgb_last_error(void);
int dgb_abi_version(void);

/* ------------------------------------------------------------------------------------
 * Host setup
 * ------------------------------------------------------------------------------------ */
typedef struct dgb_problem dgb_problem;

/* Structured Cartesian mesh of the kind a Gmsh .geo "Transfinite ... Recombine" produces:
 * nx (x ny) elements of order `order`, elements numbered row-major (x fastest), boundary
 * elements carrying physical tags bc[] (1D: left,right; 2D: bottom,right,top,left). */
typedef struct {
  int dim;        /* 1 or 2 */
  int order;      /* polynomial order p >= 1 */
  int nx, ny;     /* elements per direction (ny ignored in 1D) */
  double x0, x1, y0, y1;
  int bc[4];
} dgb_mesh_spec;

/* Solver options that the reference takes from the deck and its compile-time flags. */
typedef struct {
  int flux;            /* enum dgb_flux */
  int limiter;         /* enum dgb_limiter */
  double cfl;          /* deck CFL; < 0 selects a fixed step (rk.cc:136-139) */
  double thresholds[3];/* sensor thresholds (sensor.h:35-45); n_thresholds of them are set */
  int n_thresholds;
  int n_mass;          /* passive mass fractions rho*Y_k appended to the state (MASS of the
                        * reference Makefile, 0..10; N_F = 4 (1D) / 5 (2D) + n_mass) */
  int gamma_model;     /* enum dgb_gamma_model */
} dgb_options;

/* Reads a reference input deck (format of code/src/deck/deck.cc:11-64) and the Gmsh 2.2 mesh
 * it names (path relative to the deck's directory).  The flux comes from the deck's optional
 * "#Make options" block (FLUX=ROE|RUS|HLL, the block tests/runtests.py:80-87 reads), else ROE;
 * MASS=n there gives n passive mass fractions, GAMM=GAMCONS the conservative gamma model. */
int dgb_problem_from_deck(const char* deck_path, dgb_problem** out);
/* Builds the same problem from an in-memory structured mesh (identical to reading the file
 * that dgb_mesh_write_msh writes for the same spec). */
int dgb_problem_structured(const dgb_mesh_spec* mesh, const dgb_options* opt, dgb_problem** out);
/* Writes a Gmsh 2.2 ASCII mesh for the spec (replaces running gmsh on a .geo file). */
int dgb_mesh_write_msh(const dgb_mesh_spec* mesh, const char* path);
void dgb_problem_destroy(dgb_problem* p);

typedef struct {
  int dim, order, n_fields;      /* D, p, N_F */
  int n_elem, n_s, n_g;          /* N_E, N_s, N_G */
  int n_ifaces, m_s, m_g, n_n;   /* M_T, M_s, M_G, N_N */
  int n_reflective;              /* reflective interfaces (M_B of buildBoundary) */
  int cartesian;                 /* iscartesian() (simpleMesh.cc:1102) */
  int gpu_supported;             /* 1 when the device path supports this problem */
  int flux, limiter;
  int nx, ny;                    /* structured extents when detected, else 0 */
  double cfl, dx_min, cfl_scaled;/* cfl_scaled = CFL*Dx/(2p+1) (main.cc:896-897) */
  double final_time;
  int n_output_times;
  int error_output;              /* deck "#Make options" ERRR=ERROR: error.dat after the run */
  int gamma_model;               /* enum dgb_gamma_model */
  int cons_output;               /* deck "#Make options" CONS=CONS: conservation.dat at each output */
} dgb_info;

int dgb_problem_info(const dgb_problem* p, dgb_info* out);

/* Copies a named host array, in the reference's own layout, into dst (nbytes must match).
 * Names: "phi","dphi","phi_w","dphi_w","psi","psi_w","weight","J","invJac","JF","normals",
 * "Minv","map","invmap","boundaryMap","neighbors","Lag2Mono","Mono2Lag","Lag2MonoX","MonoX2MonoY",
 * "MonoY2Lag","MonoX2Lag","Lag2MonoY","xyz_nodes","output_times". */
int dgb_problem_array_size(const dgb_problem* p, const char* name, size_t* nbytes);
int dgb_problem_get_array(const dgb_problem* p, const char* name, void* dst, size_t nbytes);

/* Seeded initial states (reference layout).  Names: "sodtube" (reference init_cond.cc:400),
 * "tube_noise" (two-fluid tube split at params[0] with +-params[1] uniform noise on rho),
 * "shock_bubble" (Mach-1.5 shock hitting a gamma=1.67 bubble, 1% seeded Fourier
 * perturbation of the radius), "quadrants" (four-quadrant Riemann problem, seeded states),
 * "riemann" (1D two-fluid Riemann problem split at params[0], seeded left/right states). */
int dgb_problem_init_state(const dgb_problem* p, const char* ic, const double* params, int nparams,
                           uint64_t seed, double* U);
/* (ic == NULL selects the deck's "#initial condition" and, when nparams == 0, its "#ic inputs".)
 * "sinegam" is the reference's smooth advection test (init_cond.cc:551-618). */

/* Output in the reference .pos format (code/src/mesh/simpleMesh.cc:322-376 via
 * code/src/printer/printer.cc:77): one file per primitive field, <dir>/<name><step>.pos. */
int dgb_write_pos(const dgb_problem* p, const double* U, int step, double time, const char* dir);
/* The ERROR diagnostic of the reference driver (main.cc:909-1038): out = [dx, L1 (N_F), L2 (N_F),
 * Linf (N_F)] of the cell averages of U against U_exact (both host, reference layout), after both
 * are turned into (rho, u, (E - rho u^2/2) alpha^-1, alpha) on fields 0..3 as the reference does. */
int dgb_problem_error_norms(const dgb_problem* p, const double* U, const double* U_exact, double* out);
/* Restart read of the same files (printer.cc:108, simpleMesh.cc:378). */
int dgb_read_pos(const dgb_problem* p, int step, const char* dir, double* time, double* U);

/* ------------------------------------------------------------------------------------
 * Device context
 * ------------------------------------------------------------------------------------ */
typedef struct dgb_ctx dgb_ctx;

/* Uploads geometry, basis and limiter data and allocates the resident state
 * (replaces the DG_SOLVER, Limiting and RK constructors: dg_solver.h:104, limiting.h:123/249). */
int dgb_create(const dgb_problem* p, int device, dgb_ctx** out);
void dgb_destroy(dgb_ctx* c);

/* Resident state from / to host memory (reference layout). */
int dgb_set_state(dgb_ctx* c, const double* U_host);
int dgb_get_state(dgb_ctx* c, double* U_host);
/* Same with device pointers in the reference layout (no host staging). */
int dgb_set_state_device(dgb_ctx* c, const double* U_dev);
int dgb_get_state_device(dgb_ctx* c, double* U_dev);

/* f = S + F + Q for the state U (DG_SOLVER::dg_solver, dg_solver.h:292-364).
 * Host arrays in the reference layout; the resident state is not touched. */
int dgb_residual(dgb_ctx* c, const double* U_host, double* f_host);
/* DU = dt * Minv * f(U) (Lsolver, rk_kernels.cu:182, applied to dg_solver's output). */
int dgb_solve(dgb_ctx* c, double dt, const double* U_host, double* DU_host);
/* In-place limiting with the problem's limiter (Limiting::*limiting, limiting.cc). */
int dgb_limit(dgb_ctx* c, double* U_host);
/* Troubled-cell flags of U with the deck's sensor thresholds (SENSOR::sensing, sensor.cc:11 with
 * calc_sensors, sensor_kernels.cu:19): flags[e] = 0 (not flagged) or 1..3 (contact, shock, gamma
 * sensor), identical to the reference's sequential CPU evaluation.  Needs thresholds in the
 * problem or a sensor-gated limiter (hri, m2i, pri, p0i). */
int dgb_sensors(dgb_ctx* c, const double* U_host, int* flags_host);
/* Selects the arithmetic of the residual kernels (enum dgb_form) for later calls; no counterpart
 * in the reference, which is FP64 only. */
int dgb_set_form(dgb_ctx* c, int form);
/* Poll budget of the first wait of the residual kernels on each tile copy (default 4194304 polls;
 * the copy is drained with the default budget before the kernel returns).  A budget that runs out
 * makes the step return DGB_ERR_TIMEOUT and leaves the context usable; a budget of 0 makes every
 * such wait give up at once, which tests of the timeout path use.  No counterpart in the
 * reference, whose kernels have no bounded waits. */
int dgb_set_wait_limit(dgb_ctx* c, long long polls);
/* CFL step of the context's current (device-resident) state, as dgb_dt_from_cfl computes it. */
int dgb_cfl_dt(dgb_ctx* c, double* dt);
/* Dt = CFL_scaled / max_nodes(|u|+a) (RK::DtFromCFL, rk.cc:250-272). */
int dgb_dt_from_cfl(dgb_ctx* c, const double* U_host, double* dt);

/* Advances the resident state by nsteps steps of `scheme`.
 * dt > 0: fixed step (the reference's CFL<0 mode, rk.cc:136-139);
 * dt <= 0: step from the CFL condition, computed on the device each step.
 * Limiter placement follows rk.cc:176-209 (stage inputs after the first, end of step).
 * *time is advanced by the steps taken.  Status DGB_ERR_NONFINITE / DGB_ERR_DT_SMALL when the
 * CFL step is NaN / < 1e-14 (checked after the run; the state then holds the failing step). */
int dgb_advance(dgb_ctx* c, int scheme, int nsteps, double dt, double* time);
/* The same time loop with the state of record in host memory (reference layout): every step
 * uploads the state from U_host, advances it one step and downloads the result into U_host, so
 * that U_host holds each step's result as it completes.  The copies go in element chunks on two
 * copy streams, a chunk's upload for the next step waiting only for its own download, so the host
 * link's two directions overlap.  U_host should be pinned (cudaHostAlloc / cudaHostRegister) for
 * the copies to run asynchronously.  The learned indicator scores the first step of the call.
 * Status and *time as dgb_advance; returns after the last download.  Refused (DGB_ERR_UNSUPPORTED)
 * while per-kernel profiling is on (dgb_set_profiling), which times eager launches.  No counterpart in the
 * reference, whose state lives in host memory between its per-stage device launches. */
int dgb_advance_host(dgb_ctx* c, double* U_host, int scheme, int nsteps, double dt, double* time);

/* Last step size used by dgb_advance (host copy). */
int dgb_last_dt(dgb_ctx* c, double* dt);

/* ------------------------------------------------------------------------------------
 * Slab mode: one y-slab of a larger structured 2D grid per context (the reference's MPI
 * decomposition, simpleMesh.cc:1006-1074, with its per-element ghost exchange,
 * communicator_cpu.cc:14-59, replaced by whole ghost rows).  The context's grid is the slab
 * plus `lo` ghost rows below and `hi` above (rows of elements, nx each); a stage reaches two rows
 * deep (residual, then the limiter's y pass), so a slab neighbour needs 2 ghost rows.  The caller
 * moves the rows between slabs (NCCL, peer copies, or in one process):
 *   dgb_step_begin                    local CFL wave speed over the owned rows
 *   [MAX-reduce the word of dgb_step_wavespeed_word over the slabs, as 64-bit integers]
 *   for k in 0 .. stages-1:           (SSP-RK3: 3, RK4: 4)
 *     [dgb_halo_pack both sides, send / receive, dgb_halo_unpack both sides]
 *     dgb_step_stage(k)                residual, stage update, limiter
 *   dgb_step_end                       status and the step's dt added to *time
 * Pack / unpack act on the buffer the next stage reads (outside a step: the resident state);
 * all work is queued on the context's stream (dgb_stream).  Interior slabs give the same
 * result as the whole grid advanced by dgb_advance. */
int dgb_slab_ghost_rows(dgb_ctx* c, int lo, int hi);
/* Replaces the CFL scale CFL * Dx / (2p+1) of the context's CFL step (main.cc:896-897): the slabs
 * of one grid take one value (their own meshes can give it one ulp apart). */
int dgb_set_cfl_scale(dgb_ctx* c, double cfl_scaled);
int dgb_step_begin(dgb_ctx* c, int scheme, double dt);
int dgb_step_wavespeed_word(dgb_ctx* c, void** umax_dev);  /* device uint64: bits of max |u|+a */
int dgb_step_stage(dgb_ctx* c, int k);
int dgb_step_end(dgb_ctx* c, double* time);
/* doubles per side (0 bottom, 1 top): ghost rows x nx x N_F x N_s, laid out
 * buf[((f * N_s + node) * rows + row) * nx + col] */
int dgb_halo_count(dgb_ctx* c, int side, size_t* n);
int dgb_halo_pack(dgb_ctx* c, int side, double* dst_dev);
int dgb_halo_unpack(dgb_ctx* c, int side, const double* src_dev);
int dgb_stream(dgb_ctx* c, void** stream);  /* the context's cudaStream_t */
/* Every slab of one grid in this process on one device (slabs[0] the bottom slab, in order;
 * periodic != 0: the bottom and top slabs are neighbours), advanced nsteps steps together: the
 * phase-level sequence above with the ghost rows copied device to device between the slabs, one
 * CUDA graph per step (captured on the first call for these slabs, scheme and step kind) replayed
 * on slabs[0]'s stream.  Same arithmetic as the phase-level step; *time += the time advanced,
 * dgb_last_timing(slabs[0]) gives the device time.  No reference counterpart: the reference
 * exchanges ghosts through MPI (communicator_cpu.cc:14-59). */
int dgb_slabs_advance_local(dgb_ctx* const* slabs, int n, int periodic, int scheme, int nsteps, double dt,
                            double* time);

/* Conserved totals sum_e sum_g U_g J w_g per field (DG_SOLVER::conservation, dg_solver.h:367). */
int dgb_conservation(dgb_ctx* c, double* totals /* N_F */);

/* Device time (ms) of the last dgb_advance measured with CUDA events on the library stream,
 * and the number of kernel launches it issued. */
int dgb_last_timing(dgb_ctx* c, double* ms, long long* launches);
/* Per-kernel device time of the last dgb_advance when profiling is on:
 * names "residual", "limiter", "dt", "indicator" (the learned indicator's scoring kernels);
 * ms and launches of that kernel class. */
int dgb_set_profiling(dgb_ctx* c, int on);
int dgb_kernel_timing(dgb_ctx* c, const char* name, double* ms, long long* launches);

/* ------------------------------------------------------------------------------------
 * Learned troubled-cell indicator (no counterpart in the reference)
 * ------------------------------------------------------------------------------------
 * A 225 -> 64 -> 64 -> 1 MLP (GELU, sigmoid) reads each element's and its four neighbours'
 * normalised scaled-Taylor modes (2D, p = 2; each input x soft-thresholded at the rounding floor
 * 5e-5 and compressed, sign(x) log(1 + max(|x| - 5e-5, 0) / 1e-5) / log(1 + 1e5)) and predicts
 * whether the problem's limiter would change the element (labels: a non-constant mode changed by
 * more than 1e-8 of the field scale, in an element whose own modes rise above the floor).  Parameters: one FP32 array of dgb_mlp_param_count() values laid out as
 * W1[64][225], b1[64], W2[64][64], b2[64], w3[64], b3.  Pointers marked _dev are device memory. */
int dgb_mlp_param_count(void);
/* Features [N_E][225] (FP32, row-major) of the context's current state. */
int dgb_indicator_features(dgb_ctx* c, float* X_dev);
/* Labels [N_E] (0 / 1) of the context's current state from the problem's own limiter. */
int dgb_indicator_labels(dgb_ctx* c, float* y_dev);
/* Training kernels (FP32).  forward: probabilities, and the activations needed by backward in
 * cache_dev ([n][256], may be NULL); backward: weighted binary cross-entropy (positive samples
 * weighted by pos_weight, mean over n) into *loss_dev and its gradient into grad_dev; work_dev
 * holds n*129 floats.  adam: one bias-corrected Adam update (beta 0.9 / 0.999), step t >= 1. */
int dgb_mlp_forward(const float* params_dev, const float* X_dev, int n, float* cache_dev, float* prob_dev,
                    void* stream);
int dgb_mlp_backward(const float* params_dev, const float* X_dev, const float* y_dev, float pos_weight, int n,
                     const float* cache_dev, const float* prob_dev, float* grad_dev, float* loss_dev,
                     float* work_dev, void* stream);
int dgb_mlp_adam(float* params_dev, const float* grad_dev, float* m_dev, float* v_dev, int t, float lr,
                 void* stream);
/* Gates the limiter with the network: the limiter (m2l problems, 2D, p = 2) then runs only on the
 * band -- elements scoring above `threshold` and their face neighbours -- with per-element m2
 * arithmetic.  Scores (BF16 tensor-core MMAs) are taken once per time step on the step's initial
 * state (a discontinuity moves well under one element per step at CFL < 1), and on the given
 * state by dgb_limit.  params_host = NULL switches back to the full limiter. */
int dgb_set_indicator(dgb_ctx* c, const float* params_host, float threshold);
/* Steps between scorings of the learned indicator in dgb_advance (default 1: every step); the
 * steps in between reuse the band (flagged elements and their face neighbours) of the last
 * scoring.  A discontinuity moves at most CFL / (2p + 1) of an element per step, so the band keeps
 * covering it for up to (2p + 1) / CFL steps (16 at p = 2, CFL 0.3).  Setting a state restarts the
 * count (the next step scores).  No counterpart in the reference. */
int dgb_set_indicator_interval(dgb_ctx* c, int steps);
/* Scores [N_E] of U (reference layout, host) with the indicator set, and the flagged count. */
int dgb_indicator_scores(dgb_ctx* c, const double* U_host, float* score_host, int* n_flagged);

/* ------------------------------------------------------------------------------------
 * Batched ensemble (no counterpart in the reference, which runs one problem per process)
 * ------------------------------------------------------------------------------------
 * Many independent problems advanced together with SSP-RK3, each with its own CFL step.  The
 * cases are contexts made by dgb_create (owned by the caller, all on one device, outliving the
 * batch; states set and read with dgb_set_state / dgb_get_state on each).  They are grouped by
 * (dimension, order, flux, limiter); per group and operator one persistent launch walks the work
 * items of all its cases, and one step of the whole ensemble is a CUDA graph whose group branches
 * run concurrently.  A case advanced in a batch matches dgb_advance on it alone: bit for bit in
 * 1D, to a few ulps in 2D (the same arithmetic, with fused multiply-adds formed differently).
 * Supported: plain FP64 form, limiter none / hrl / m2l, positive CFL; 2D cases on structured
 * row-major grids with p <= 2, nx a multiple of 32 and ny of 4 (DGB_ERR_UNSUPPORTED otherwise). */
typedef struct dgb_batch dgb_batch;
int dgb_batch_create(dgb_ctx* const* cases, int n_cases, dgb_batch** out);
void dgb_batch_destroy(dgb_batch* b);
/* Number of element groups and, per group k, info[10] = {dim, order, flux, limiter, cases,
 * tile width (2D; 1D: elements per CTA), tile height (1D: 1), quadrature-loop unrolling (2D),
 * CTAs per SM of the residual launch (0 = occupancy limit), tuned stage time in ns (0 = untuned)}. */
int dgb_batch_n_classes(dgb_batch* b);
int dgb_batch_class_info(dgb_batch* b, int k, int* info);
/* Autotuner: per group, times every candidate residual configuration (tile shape and unrolling
 * for 2D, elements per CTA for 1D, persistent grid size) `reps` times on the cases' current
 * states (left unchanged) and keeps the fastest. */
int dgb_batch_autotune(dgb_batch* b, int reps);
/* Sets group k's residual configuration by hand: 2D: a tile shape among the tuner's candidates
 * (tile_w x tile_h = 32x4, 32x2 or 16x8 dividing every case's grid; unroll 1, or 2 with 32x4);
 * 1D: tile_w = elements per CTA (64, 128 or 256), tile_h and unroll ignored.  ctas_per_sm caps the
 * persistent grid (0 = occupancy limit).  DGB_ERR_ARG for anything else. */
int dgb_batch_set_tuning(dgb_batch* b, int k, int tile_w, int tile_h, int unroll, int ctas_per_sm);
/* Up to nsteps steps of every case, each with its own CFL step; times restart at 0.  t_end > 0:
 * a case stops at time t_end (its last step shortened to land on it) and the run ends early once
 * every case has stopped.  *steps_run = graph steps launched.  A case whose step fails stops; the
 * first failure is the returned status (DGB_ERR_NONFINITE / _DT_SMALL / _TIMEOUT). */
int dgb_batch_advance(dgb_batch* b, int nsteps, double t_end, int* steps_run);
/* Per case of the last run: simulated time, steps taken, and (t_end > 0) device wall-clock ms
 * from the start of the run to the step at which the case stopped (-1 if it did not stop). */
int dgb_batch_case_stats(dgb_batch* b, double* time, int* steps, double* wall_ms);
/* Device time (ms, CUDA events) and kernel launches of the last dgb_batch_advance. */
int dgb_batch_last_timing(dgb_batch* b, double* ms, long long* launches);

/* ------------------------------------------------------------------------------------
 * Allocation-free limiter (no counterpart in the reference)
 * ------------------------------------------------------------------------------------
 * For callers that cannot allocate device memory themselves -- an application that manages a
 * fixed device-memory budget claimed at start-up, or a time loop that must not trigger
 * cudaMalloc (and the device synchronisation it implies) -- and therefore cannot call
 * dgb_create.  Applies the problem's limiter (hrl or m2l) to the state U_in_dev and writes the
 * result to U_out_dev (both in the caller's device memory, reference layout, may alias).  The
 * work is queued on the CUDA stream `stream` (0 = default stream) of the current device and the
 * call returns without waiting for it: the result is there once the stream has reached it.  On a
 * structured grid (a 1D chain or a row-major 2D grid, each side with one boundary rule) the call
 * copies nothing from the host; on any other element order it copies the neighbour table from
 * host memory every time, and that copy first waits for the stream.  Temporaries live in one library-owned device array of 128 MiB, which every GPU that loads
 * this library holds until the process exits; a problem that needs more (2D: above about 166k
 * elements at p=2, 94k at p=3) is rejected with DGB_ERR_ARG.  The first call on a device looks
 * up that array's device address and uploads the limiter tables; make it before any stream
 * capture.  All calls share the array and it keeps the last call's contents: two calls that
 * overlap on the GPU (different streams or host threads) race.  Nothing in it needs to start at
 * zero; every call writes what it reads. */
int dgb_limit_noalloc(const dgb_problem* p, const double* U_in_dev, double* U_out_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DGB_H */
