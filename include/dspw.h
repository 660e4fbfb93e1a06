/*
 * dspw.h -- C ABI of the B200 DSP-WENO / SP-WENO TeCNO finite-volume stage path.
 *
 * Plain C, no C++ or CUDA types: the reference's C++ driver (or any FFI) binds
 * it directly.  The library is libdspw.so, built from dsp-weno_b200/csrc.
 *
 * What it replaces.  The reference has no plugin API; its per-stage work is a
 * set of private members of class FV called from the time loop
 * (enflo/src/fv.cc:1262-1313, enflo_scalar/src_scalar/fv.cc:553-597):
 *
 *   compute_dt()        enflo/src/fv.cc:366-383       -> dspw_compute_dt / dspw_step
 *   prim_to_ent()       enflo/src/fv.cc:421-552       -> fused into every stage
 *   compute_residual(rk) enflo/src/fv.cc:591-767      -> dspw_stage / dspw_residual
 *   update_solution(rk) enflo/src/fv.cc:1163-1198     -> dspw_stage
 *   con_to_prim()+apply_bc() enflo/src/fv.cc:388-400,121-361 -> fused into every stage
 *   compute_global()    enflo/src/compute_global.cc:10-89 -> dspw_globals
 *   compute_error()     enflo/src/compute_errors.cc:9-33  -> dspw_errors
 *   Neural_Network::load_network enflo/src/neural_network.cc:82-130 -> desc.nn_w/nn_b
 *
 * Ownership: a handle owns all device memory, its CUDA stream and its CUDA
 * graphs.  Host pointers passed in are borrowed for the duration of the call.
 * Threading: one host thread at a time per handle; handles are independent.
 * Errors: every call returns an int status (DSPW_OK == 0); nothing aborts or
 * exits across the ABI.  dspw_error_string() names a status.
 *
 * Host array layout: interior cells only, FP64, component planes of shape
 * (nvar, Nz, Ny, Nx) with x fastest.  Primitive components are
 * (rho, u, v, w, p) for the Euler/NS models and the single value u for the
 * scalar models; conserved components are (rho, rho u, rho v, rho w, E).
 */
#ifndef DSPW_H
#define DSPW_H

#ifdef __cplusplus
extern "C" {
#endif

#define DSPW_ABI_VERSION 2

#if defined(__GNUC__)
#define DSPW_API __attribute__((visibility("default")))
#else
#define DSPW_API
#endif

/* models (enflo/src/ext_constants.h:23, enflo_scalar/src_scalar/ext_constants.h:19) */
enum dspw_model { DSPW_LINADV = 0, DSPW_BURGERS = 1, DSPW_EULER = 2, DSPW_NS_ES = 3, DSPW_NS_KEP = 4 };

/* numerical fluxes: scalar names from enflo_scalar/src_scalar/ext_constants.h:17,
 * system names from enflo/src/ext_constants.h:17-19 */
enum dspw_flux {
  DSPW_LIN_EC = 0, DSPW_LIN_EC4 = 1, DSPW_LIN_TECNO = 2, DSPW_LIN_TECNO4 = 3,
  DSPW_BUR_EC = 4, DSPW_BUR_EC4 = 5, DSPW_BUR_TECNO = 6, DSPW_BUR_TECNO4 = 7,
  DSPW_ROE = 10, DSPW_KEP = 11, DSPW_KEP4 = 12, DSPW_KEPEC = 13, DSPW_KEPEC4 = 14,
  DSPW_ROE_EC = 15, DSPW_ROE_EC4 = 16, DSPW_KEPS = 17, DSPW_KEPS4 = 18,
  DSPW_KEP_TECNO_ROE = 19, DSPW_KEPES_TECNO_ROE = 20, DSPW_KEPES_TECNO_RUSANOV = 21,
  DSPW_ROE_TECNO_ROE = 22, DSPW_KEPES_TECNO4_ROE = 23, DSPW_KEPES_TECNO4_RUSANOV = 24,
  DSPW_ROE_TECNO4_ROE = 25
};

/* reconstructions: param.in names sp_weno, sp_wenoc, sp_weno_corr2, sp_weno_dl
 * (enflo/src/parameter.cc:179-206) and the simpler schemes of
 * enflo/src/reconstruct.cc:14-110 */
enum dspw_recon {
  DSPW_REC_SP_WENO = 0, DSPW_REC_SP_WENOC = 1, DSPW_REC_SP_WENO_CORR2 = 2, DSPW_REC_SP_WENO_DL = 3,
  DSPW_REC_FIRST = 4, DSPW_REC_SECOND = 5, DSPW_REC_MINMOD = 6, DSPW_REC_MINABS = 7,
  DSPW_REC_ENO2 = 8,         /* point-wise ENO, eno_level 2 (param.in "reconstruct eno 2") */
  DSPW_REC_ENO3 = 9          /* point-wise ENO, eno_level 3 ("reconstruct eno 3"): three ghost
                                cells and six-cell face stencils, as the reference's
                                ng_cell = 3 (enflo/src/parameter.cc:178-184, fv.cc:26).  A
                                wall axis needs at least 3 cells. */
};

/* boundary conditions (enflo/src/ext_constants.h:25).  DIRICHLET is parsed but
 * not implemented by the reference (enflo/src/parameter.cc:558-562); here it
 * means: ghost cells hold the fixed primitive state desc.bc_state[face]. */
enum dspw_bc { DSPW_BC_PERIODIC = 0, DSPW_BC_DIRICHLET = 1, DSPW_BC_NEUMANN = 2, DSPW_BC_WALL = 3,
  /* No counterpart in the reference: the face borders another slab of the same
   * domain.  Its ghost layers (3 for eno 3, else 2) are stored beside the
   * interior and filled by the caller before every stage from the
   * neighbouring slab (dspw_halo_view).  Only on the faces of the problem's
   * last swept direction (y of a 2-D problem, z of a 3-D one, x of a 1-D one),
   * for the Euler and scalar models, without the per-step diagnostics.
   * Unless the handle is connected (dspw_slab_connect), dspw_step / dspw_run
   * do not exchange: a slab then steps through dspw_stage with its layers
   * filled before each call (the stored layers stay inside the slab's own
   * storage, so stale ones give wrong values, never bad reads). */
  DSPW_BC_HALO = 4 };

enum dspw_time { DSPW_RK1 = 0, DSPW_SSPRK3 = 1, DSPW_JAMESON_RK4 = 2, DSPW_RK4 = 3 };
enum dspw_mu { DSPW_MU_CONSTANT = 0, DSPW_MU_SUTHERLAND = 1, DSPW_MU_POWER = 2 };

/* arithmetic of the stage path */
enum dspw_precision {
  DSPW_FP64 = 0,       /* plain form: state, fluxes, reconstruction and network in FP64 */
  DSPW_FP32_BF16 = 1   /* FP32 state/fluxes/reconstruction; network layers as BF16
                          tensor-core tiles with FP32 accumulation.  Time, CFL max and
                          global sums stay FP64. */
};

enum dspw_status_code {
  DSPW_OK = 0,
  DSPW_ERR_ARG = 1,          /* bad argument or descriptor */
  DSPW_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  DSPW_ERR_NONFINITE = 3,    /* NaN/Inf found in the state */
  DSPW_ERR_NONPOSITIVE = 4,  /* density or pressure <= 0 */
  DSPW_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  DSPW_ERR_UNSUPPORTED = 6,  /* combination not implemented */
  DSPW_ERR_NOMEM = 7,        /* device allocation failed */
  DSPW_ERR_FINISHED = 8      /* the problem has reached final_time or max_iter */
};

/* One problem.  Mirrors the param.in surface (enflo/src/parameter.h:14-74). */
typedef struct dspw_desc {
  int abi_version;           /* DSPW_ABI_VERSION */
  int model;                 /* enum dspw_model */
  int flux;                  /* enum dspw_flux */
  int recon;                 /* enum dspw_recon */
  int time_scheme;           /* enum dspw_time */
  int precision;             /* enum dspw_precision */
  int nx, ny, nz;            /* cells; ny == 1 / nz == 1 switch that sweep off */
  int bc[6];                 /* xleft, xright, yleft, yright, zleft, zright */
  int ec1_fix;               /* EC1_fix yes/no (enflo/src/parameter.cc:396-406) */
  int mu_model;              /* enum dspw_mu */
  int max_iter;
  int t_stamps;              /* output time_stamps; dt is clipped to them like FV::run */
  int nn_use_box;            /* 1: the network has a training box (nn_feat_lo / nn_feat_hi); a
                                stencil whose network inputs fall outside it is reconstructed by
                                plain SP-WENO (FP32 form) */
  int generic_kernels;       /* 1: run this problem on the generic sweep kernels even when
                                specialised ones exist (validation) */
  int tile_staging;          /* y / z sweeps of the specialised kernels: 0 = tiles of 8 columns
                                staged by per-thread cp.async copies, or the variant dspw_tune
                                measures faster (Tensor Memory Accelerator loads, or tiles of 4
                                columns); 1 = 8 columns, cp.async always; 2 = 8 columns, TMA where
                                the problem allows it (nx a multiple of 8, 16-byte aligned rows and
                                planes); 3 = 4 columns (blocks of 4 warps), cp.async */
  int reserved_i[5];         /* zero */
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double gamma, gas_const, prandtl, mu_ref, T_ref, T_0, omega;
  double lin_vel[3];         /* linadv velocity */
  double cfl, final_time;
  double bc_state[6][5];     /* DIRICHLET ghost state, primitive (rho,u,v,w,p) or (u) */
  double nn_w[4][5][5];      /* DSP-WENO layer weights, row = output, col = input */
  double nn_b[4][5];         /* DSP-WENO layer biases */
  double nn_feat_lo[5];      /* training box of the five network inputs (tanh theta-, tanh theta+,
                                |del1|, |del2|, |del3| of the scaled stencil,
                                enflo/src/neural_network.cc:16-38); used when nn_use_box == 1,
                                e.g. filled from dspw_trainer_box after training */
  double nn_feat_hi[5];
  double cell_size[3];       /* when > 0: the cell sizes dx, dy, dz instead of (max - min) / n, for
                                the slabs of a decomposed domain (DSPW_BC_HALO), which keep the
                                domain's own */
  double reserved_d[5];      /* zero */
} dspw_desc;

typedef struct dspw_handle dspw_handle;

/* Global quantities of one problem, FP64 sums on the device.  total_entropy is
 * sum(-rho s/(gamma-1)) vol for systems (enflo/src/compute_global.cc:18-28) and
 * sum(u^2/2) vol for scalar laws (enflo_scalar/src_scalar/compute_global.cc:12-21). */
typedef struct dspw_globals_out {
  double time;
  double dt;
  int iter;
  int finished;
  double total_entropy;
  double conserved[5];       /* sum(U) vol per component */
  double kinetic_energy;     /* sum(rho |u|^2/2) vol (systems) */
} dspw_globals_out;

/* Device-side health word, accumulated since the last dspw_last_status call. */
typedef struct dspw_status_out {
  int code;                  /* first error seen, DSPW_OK if none */
  long long nonfinite_cells;
  long long nonpositive_cells;
  long long sign_violations;  /* reconstructions whose jump Zji-Zij opposes Z_{i+1}-Z_i by
                                 more than rounding (64 ulps of the stencil's magnitude) */
  long long faces_checked;    /* component-face reconstructions checked */
  long long limiter_acts;     /* FP32 form: opposing jumps zeroed by the sign-preserving limiter */
} dspw_status_out;

DSPW_API const char* dspw_error_string(int code);
DSPW_API int dspw_version(void);

/* Create a handle for one problem / for nprob independent problems advanced
 * together (one launch per kernel over all problems, per-problem dt). */
DSPW_API int dspw_create(const dspw_desc* desc, dspw_handle** out);
DSPW_API int dspw_create_batch(const dspw_desc* descs, int nprob, dspw_handle** out);
DSPW_API int dspw_destroy(dspw_handle* h);

/* Interior primitive state of problem p in, conserved/primitive state out.
 * dspw_upload_prim checks the state on the device after the copy: density or
 * pressure <= 0 (or NaN) gives DSPW_ERR_NONPOSITIVE, another non-finite value
 * DSPW_ERR_NONFINITE, and the problem keeps its previous state. */
DSPW_API int dspw_upload_prim(dspw_handle* h, int p, const double* prim);
DSPW_API int dspw_download_prim(dspw_handle* h, int p, double* prim);
DSPW_API int dspw_download_cons(dspw_handle* h, int p, double* cons);

/* CFL time step cfl*min(h)/max|speed| of the current state (FV::compute_dt). */
DSPW_API int dspw_compute_dt(dspw_handle* h, int p, double* dt);

/* Residual of the current state (compute_residual(rk), reference sign). */
DSPW_API int dspw_residual(dspw_handle* h, int p, double* res);

/* One time-integration stage rk with step dt on every problem (dt <= 0 keeps
 * the per-problem dt of the current step); rk runs 0..0 for rk1, 0..2 for
 * ssprk3 and 0..3 for jameson_rk4 / rk4, the stages of FV::run's loop
 * (enflo/src/fv.cc:1268-1310), which a caller issues in order. */
DSPW_API int dspw_stage(dspw_handle* h, int rk, double dt);

/* Up to nsteps steps of the FV::run loop body on every unfinished problem:
 * CFL dt, clipping to the next time stamp, all stages, time += dt.  With
 * fixed_dt > 0 the CFL step is replaced by fixed_dt.  Steps run as one CUDA
 * graph per step; nothing is copied to the host.  After the final
 * synchronisation the call returns the first health error the device has
 * recorded since the last dspw_last_status (DSPW_ERR_NONFINITE or
 * DSPW_ERR_NONPOSITIVE from the last stage's check of every cell), DSPW_OK if
 * none; dspw_stage does the same after its stage. */
DSPW_API int dspw_step(dspw_handle* h, int nsteps, double fixed_dt);

/* Advance every problem until final_time/max_iter, checking completion every
 * `chunk` steps.  Returns the number of steps of the longest problem. */
DSPW_API int dspw_run(dspw_handle* h, int chunk, int* steps);

DSPW_API int dspw_globals(dspw_handle* h, int p, dspw_globals_out* g);
DSPW_API int dspw_last_status(dspw_handle* h, dspw_status_out* s);

/* L1/L2/Linf error of problem p against host values `exact` (same layout as
 * dspw_download_prim, component comp), volume-weighted like
 * enflo_scalar/src_scalar/compute_errors.cc:9-30. */
DSPW_API int dspw_errors(dspw_handle* h, int p, int comp, const double* exact, double err[3]);

/* Run one step outside the CUDA graph with a CUDA event pair around every
 * kernel launch on the handle's stream and return the launch durations in
 * milliseconds (kernel_ms, up to max_k entries, launch order: begin-step,
 * per stage the sweeps x/y/z [and the viscous kernels], end-step) and a short
 * name per launch (names: max_k rows of 16 chars).  For measurement only. */
/* Launch autotuner (no counterpart in the reference, whose loops are
   serial): for every kernel class and sweep direction of the handle, times the
   sweep on the current state (a residual evaluation, which writes only the
   residual buffer) with its default grid and with persistent grids of 1, 2 and
   4 times the resident blocks of the GPU, for the specialised y / z sweeps
   also with tiles of 8 and of 4 columns and, where tensor maps exist, with
   cp.async and TMA staging (within what tile_staging allows); keeps the
   fastest, and drops the step graph so that the next step is captured with
   the choice.  Every candidate computes the same bits.  The state, the
   problems' clocks and the status counters are unchanged.  reps: timed
   launches per candidate (their median is compared, 1..1000).
   before_ms / after_ms (nullable): summed sweep times with the default and the
   chosen launches. */
DSPW_API int dspw_tune(dspw_handle* h, int reps, double* before_ms, double* after_ms);

DSPW_API int dspw_profile_step(dspw_handle* h, double* kernel_ms, char* names, int max_k, int* nk);

/* Reconstruct n independent 4-cell stencils u4[4*i..4*i+3] at their middle
 * face with desc->recon in desc->precision, on the GPU, with the same device
 * code as the stage kernels (reconstruct(), enflo/src/reconstruct.cc:192-239).
 * limiter_acts receives how often the FP32 form's sign-preserving limiter
 * acted.  Allocates its own temporary device buffers.  DSPW_REC_ENO3 reads
 * six-cell stencils and returns DSPW_ERR_UNSUPPORTED here. */
DSPW_API int dspw_reconstruct_batch(const dspw_desc* desc, const double* u4, long long n, double* recl,
                                    double* recr, long long* limiter_acts);

/* Global sums of a state the caller owns, with no device allocation.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc: a
 * driver that keeps every device buffer in its own pool, a component that may
 * not grow the device footprint, or a loop that must not synchronise the device
 * through an allocation.  d_cons: conserved component planes on the current
 * device (stride elements apart, elem_bytes 8 or 4, the layout of
 * dspw_device_state); d_out: 7 device doubles receiving total entropy, kinetic
 * energy and the 5 conserved totals (dspw_globals_out order), each times the
 * cell volume.  Work is enqueued on `stream` (a cudaStream_t, may be NULL); the
 * call does not synchronise.  Scratch is one fixed 256 KiB device array in the
 * library, shared by all calls: states above 16,777,216 cells are rejected with
 * DSPW_ERR_ARG, and calls that overlap on the GPU race on it.  The first call
 * on each device looks up the array's device address and should not be made
 * during stream capture. */
DSPW_API int dspw_globals_noalloc(const dspw_desc* desc, const void* d_cons, long long stride, int elem_bytes,
                                  double* d_out, void* stream);

/* Discrete entropy inequality, checked every step on the device: the total
 * entropy E = sum U(u) vol of each new state (U = -rho s / (gamma - 1) with
 * s = ln p - gamma ln rho for systems, u^2 / 2 for scalar laws; the
 * reference's compute_global, enflo/src/compute_global.cc:18-28,
 * enflo_scalar/src_scalar/compute_global.cc:12-21), taken in the state's own
 * arithmetic type, against the state before the step.  *max_rise is the
 * largest relative one-step increase (E_{n+1} - E_n) / |E_n| since the last
 * upload (negative when E only fell), *steps (may be NULL) the steps checked.
 * An entropy-stable TeCNO run keeps *max_rise at rounding level. */
DSPW_API int dspw_entropy_check(dspw_handle* h, int p, double* max_rise, long long* steps);

/* ---- per-step diagnostics ----------------------------------------------
 * The global quantities FV::run computes every step, evaluated on the device
 * inside the step graph and kept in a device ring of `capacity` rows per
 * problem, which dspw_step / dspw_run drain to host memory as they go
 * (replaces compute_global, compute_residual_norm and find_vorticity,
 * enflo/src/compute_global.cc:10-89, enflo/src/fv.cc:1204-1226,
 * enflo/src/find_vort.cc:9-29, enflo_scalar/src_scalar/compute_global.cc:10-39,
 * enflo_scalar/src_scalar/fv.cc:505-517).  One row per problem and step:
 *   systems: iter, time, total entropy, KE, KE_diss_pr, KE_diss_stress (NS,
 *     else 0), enstrophy -- the values compute_global writes at stage 0, of
 *     U^n at t^n -- then the residual norm of the step's last stage per
 *     component (mass, x/y/z momentum, energy);
 *   scalar: iter and time after the step, the total entropy sum u^2/2 vol of
 *     U^(n+1), zeros, the residual norm sqrt(sum R^2), zeros.
 * Sums are taken in a different order than the reference's loops: they agree
 * to rounding. */
enum dspw_diag_col {
  DSPW_DIAG_ITER = 0, DSPW_DIAG_TIME = 1, DSPW_DIAG_ENTROPY = 2, DSPW_DIAG_KE = 3, DSPW_DIAG_KE_DISS_PR = 4,
  DSPW_DIAG_KE_DISS_STRESS = 5, DSPW_DIAG_ENSTROPHY = 6, DSPW_DIAG_RES = 7 /* 7..11 */, DSPW_DIAG_COLS = 12
};

/* capacity > 0: record a row every step from now on (the ring holds capacity
 * steps between drains); 0: stop recording.  Either way pending rows are
 * discarded.  Allocates device memory; not during stream capture. */
DSPW_API int dspw_diag_enable(dspw_handle* h, int capacity);

/* Rows of problem p recorded and not yet read; *ndropped (may be NULL) counts
 * rows lost because more than `capacity` steps ran between drains (dspw_stage
 * does not drain). */
DSPW_API int dspw_diag_pending(dspw_handle* h, int p, int* nrows, long long* ndropped);

/* Copy up to max_rows of problem p's oldest pending rows (DSPW_DIAG_COLS
 * doubles each) into rows and remove them; *nread is the number copied. */
DSPW_API int dspw_diag_read(dspw_handle* h, int p, double* rows, int max_rows, int* nread);

/* ---- snapshots at the output time stamps -----------------------------
 * FV::run writes the solution whenever a step ends on a time stamp
 * (enflo/src/fv.cc:1309-1313, enflo_scalar/src_scalar/fv.cc:586-590).  With
 * snapshots enabled the step graph copies the state of every problem that
 * reached a stamp into a device ring of `slots` state buffers; dspw_step and
 * dspw_run drain the ring every `slots` steps into host memory (primitive
 * planes, FP64), from where dspw_snap_read hands them out oldest first.  The
 * writer of the reference's files stays with the caller (the command-line
 * driver writes sol/omg VTK and 1Dsol files, enflo/src/output.cc:10-172). */

/* slots > 0: take snapshots from now on; 0: stop.  Pending snapshots are
 * discarded.  Allocates slots x the state size on the device; not during
 * stream capture. */
DSPW_API int dspw_snap_enable(dspw_handle* h, int slots);

/* Snapshots of problem p taken and not yet read; *ndropped (may be NULL)
 * counts those lost because more than `slots` stamps were reached between
 * drains (dspw_stage does not drain). */
DSPW_API int dspw_snap_pending(dspw_handle* h, int p, int* n, long long* ndropped);

/* Copy problem p's oldest pending snapshot into prim (nvar x nz x ny x nx
 * doubles, the layout of dspw_download_prim), its time and iteration count
 * into *time and *iter (either may be NULL), and remove it.  DSPW_ERR_ARG when
 * none is pending. */
DSPW_API int dspw_snap_read(dspw_handle* h, int p, double* prim, double* time, int* iter);

/* Synchronise the handle's stream; returns the first error recorded. */
DSPW_API int dspw_sync(dspw_handle* h);

/* The handle's CUDA stream (a cudaStream_t) so callers can order their own work. */
DSPW_API void* dspw_stream(dspw_handle* h);

/* Halo layers of problem p in the state that stage rk reads (the state of the
 * step's start for rk 0): per component c (0 .. ncomp-1) the `count`
 * contiguous elements at recv_lo + c * comp_stride are the ghost layers below
 * the first interior layer, those at recv_hi + c * comp_stride the ghost
 * layers above the last; send_lo / send_hi are the first / last `ng` interior
 * layers, which the lower / upper neighbour receives into its recv_hi /
 * recv_lo.  Elements are elem_bytes wide (the handle's precision); pointers
 * are device pointers of the handle's GPU.  A slab decomposition exchanges
 * these before every dspw_stage and gives every slab the same dt (the minimum
 * of their dspw_compute_dt).  DSPW_ERR_ARG unless a face of p is DSPW_BC_HALO. */
typedef struct dspw_halo_out {
  void* recv_lo;
  void* recv_hi;
  void* send_lo;
  void* send_hi;
  long long count;           /* elements per component and side: ng x layer cells */
  long long comp_stride;     /* elements between component planes */
  int ncomp;
  int elem_bytes;
  int ng;                    /* ghost layers per side */
  int layer_cells;           /* cells of one layer across the decomposed direction */
} dspw_halo_out;
DSPW_API int dspw_halo_view(dspw_handle* h, int p, int rk, dspw_halo_out* out);

/* A new NCCL unique id (128 bytes) for dspw_slab_connect: one rank makes it
 * and the caller hands it to every rank.  NCCL is opened at run time
 * (libnccl.so.2); DSPW_ERR_UNSUPPORTED without it. */
DSPW_API int dspw_nccl_id(unsigned char id[128]);

/* Make the one-problem handle h slab `rank` of `nranks` (one GPU each) of a
 * decomposed domain.  From then on every step of dspw_step / dspw_run, and
 * dspw_stage, fills the halo layers from the neighbouring ranks with NCCL
 * sends and receives on the handle's stream before every stage (inside the
 * step graph), and a step's CFL dt is the domain's: an NCCL all-reduce(max)
 * of the wave speed.  Those calls are then collective: every rank makes them
 * in the same order with the same arguments.  Residuals, dspw_compute_dt and
 * dspw_tune stay local.  Neighbours: rank - 1 below and rank + 1 above through
 * the DSPW_BC_HALO faces, wrapping around when the first slab's lower face
 * (and the last's upper face) is a halo face. */
DSPW_API int dspw_slab_connect(dspw_handle* h, const unsigned char id[128], int rank, int nranks);

/* Raw device pointer to the conserved state planes of problem p (component
 * stride in elements returned in *stride) and the element size in bytes (8 or 4). */
DSPW_API int dspw_device_state(dspw_handle* h, int p, void** ptr, long long* stride, int* elem_bytes);

/* ---- DSP-WENO network training (no counterpart in the reference's C++; the
 * reference trains with PyTorch in DSP-WENO_trainer/DSP-WENO_network_trainer.py) */

typedef struct dspw_trainer dspw_trainer;

/* Adam settings follow DSP-WENO_trainer/config.py:25-31. */
typedef struct dspw_train_cfg {
  double lr, beta1, beta2, weight_decay, eps;
  int batch;
  int seed;
  int compute_bf16;    /* 1: weights and activations rounded to BF16 before each product (FP32 accumulation) */
  int collect_stride;  /* dspw_trainer_collect keeps every collect_stride-th reconstruction (>= 1) */
  int reserved_i[6];
} dspw_train_cfg;

DSPW_API int dspw_trainer_create(const dspw_train_cfg* cfg, const double* w_init /* 4*25 */,
                        const double* b_init /* 4*5 */, dspw_trainer** out);
DSPW_API int dspw_trainer_destroy(dspw_trainer* t);
/* Device-resident data set: n samples of 4 cell values and 2 target interface
 * values (left, right), host FP64 in. */
DSPW_API int dspw_trainer_set_data(dspw_trainer* t, const double* stencils /* n*4 */,
                          const double* targets /* n*2 */, long long n);
/* Generate stencil/target pairs on the GPU from the current state of a solver
 * handle: every face of every component contributes its 4-cell stencil and the
 * plain SP-WENO interface values as targets.  Appends up to max_pairs. */
DSPW_API int dspw_trainer_collect(dspw_trainer* t, dspw_handle* h, long long max_pairs, long long* added);
/* One epoch of minibatch Adam on the device; loss = (MSE_left + MSE_right)/2. */
DSPW_API int dspw_trainer_epoch(dspw_trainer* t, double* mean_loss);
/* Loss and gradients for one explicit batch (FP64 host in/out), for checks. */
DSPW_API int dspw_trainer_loss_grad(dspw_trainer* t, const double* stencils, const double* targets, int n,
                           double* loss, double* grad_w /* 4*25 */, double* grad_b /* 4*5 */);
DSPW_API int dspw_trainer_get_params(dspw_trainer* t, double* w /* 4*25 */, double* b /* 4*5 */);
/* Mean loss over the trainer's data set with the current parameters, no update. */
DSPW_API int dspw_trainer_eval(dspw_trainer* t, double* mean_loss);
/* Number of samples and the largest |feature| of each of the 5 network inputs
 * over the valid samples. */
DSPW_API int dspw_trainer_info(dspw_trainer* t, long long* nsamples, double* feature_max /* 5 */);
/* The training box of the network: the smallest and largest value of each of
 * the 5 network inputs over the trainer's valid samples, ready for a
 * descriptor's nn_feat_lo / nn_feat_hi (with nn_use_box = 1), so that the
 * solver reconstructs stencils outside the data the network was fitted on by
 * plain SP-WENO.  No counterpart in the reference, whose network is applied
 * to every stencil (enflo/src/reconstruct.cc:138-157).  DSPW_ERR_ARG when the
 * trainer holds no valid sample. */
DSPW_API int dspw_trainer_box(dspw_trainer* t, double lo[5], double hi[5]);
/* The trainer's valid samples as rows of the reference trainer's data file
 * (23 doubles each, the column order its reader slices with tanh_theta,
 * DSP-WENO_trainer/DSP-WENO_network_trainer.py:305-333: cell values u0..u3,
 * theta-, theta+, tanh theta-, tanh theta+, del1..del3, vertex x 0..4,
 * vertex y 0..4, target left, target right).  rows == NULL: *nrows is the
 * number of valid samples; else at most max_rows are copied. */
DSPW_API int dspw_trainer_export(dspw_trainer* t, double* rows, long long max_rows, long long* nrows);

#ifdef __cplusplus
}
#endif
#endif /* DSPW_H */
