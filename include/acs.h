/*
 * acs.h -- C ABI of the B200 artificial-compressibility (AC) pseudo-time solver.
 *
 * Drop-in for the pseudo-time loop of the Fortran reference (paths relative to the reference
 * project, OpenMp_Multicore/):
 *   solve_U   equations.f90:244-301   ->  acs_solve_u
 *   solve_V   equations.f90:546-603   ->  acs_solve_v
 *   solve_P   equations.f90:607-665   ->  acs_solve_p
 *   solve_Z   equations.f90:669-719   ->  acs_solve_z
 *   solve_C   equations.f90:769-819   ->  acs_solve_c
 *   bcUV/bcP/bcZ/bcC boundary.f90:1-159 (called inside the routines above, as in the reference)
 *   pseudo loop + convergence check main.f90:116-186 -> acs_physical_steps / acs_batch_run
 *   mesh      nonsymetric_mesh.f90:1-218 -> acs_mesh_reference, acs_mesh_channel (host helpers),
 *             acs_mesh_channel_device (device arrays)
 *   comp_mean comp_mean.f90:1-25 (+ the velocity magnitude of transient.f90:69-74)
 *             -> acs_cell_fields / acs_batch_cell_fields
 *
 * Conventions (those of the Fortran caller):
 *   - every field is a caller-owned host array in Fortran order (column-major, i fastest):
 *       um, um_tau, um_n_tau : (imax+1) x jmax
 *       vm, vm_tau, vm_n_tau : imax x (jmax+1)
 *       p, pn, T, T_*, C, C_*: imax x jmax
 *   - 1-D metric arrays: x[imax], y[jmax], xm[imax+1], ym[jmax+1] (Fortran x(1) is x[0]);
 *   - return value 0 = ACS_OK, otherwise an ACS_E_* code; no exception crosses the ABI;
 *     acs_last_error() gives a message for the calling thread;
 *   - a handle is used by one host thread at a time.
 * All arithmetic is FP64.  Nothing here falls back to the CPU: without a CUDA device every
 * call that needs one returns ACS_E_CUDA.
 */
#ifndef ACS_H
#define ACS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum acs_status {
  ACS_OK = 0,
  ACS_E_ARG = 1,         /* null pointer or invalid parameter */
  ACS_E_SIZE = 2,        /* grid too small/large, or size over a stated maximum */
  ACS_E_CUDA = 3,        /* CUDA runtime error or no device */
  ACS_E_NOMEM = 4,       /* device allocation failed */
  ACS_E_STATE = 5,       /* call out of order */
  ACS_E_UNSUPPORTED = 6  /* option not available for this input */
};

/* convection scheme */
enum acs_scheme { ACS_SCHEME_QUICK = 0, ACS_SCHEME_UPWIND = 1 };
/* boundary passes */
enum acs_bc { ACS_BC_REFERENCE = 0, ACS_BC_CHANNEL = 1 };
/* arithmetic: EXACT keeps the reference's operation order with every product and sum
 * separately rounded (bit-identical to a -ffp-contract=off CPU build); FAST uses fused
 * multiply-adds and precomputed reciprocals of the metric (results differ in the last bits). */
enum acs_arith { ACS_ARITH_EXACT = 0, ACS_ARITH_FAST = 1 };

/* per-case status word */
enum acs_case_status { ACS_CASE_RUNNING = 0, ACS_CASE_DONE = 1, ACS_CASE_FAILED = 2 };

/* Constants read by the loop (comum.f90:29-31, 79-85, 112-115; iterations.dat; main.f90:105-106).
 * Same layout as the oracle's parameter block. */
typedef struct acs_params {
  int imax, jmax;      /* p-node counts (comum.f90:44-46) */
  int scheme;          /* acs_scheme */
  int bc;              /* acs_bc */
  int solve_scalars;   /* 1: solve_Z and solve_C run inside the loop (main.f90:130-132) */
  int itc_max;         /* pseudo-iteration cap per physical step (main.f90:120) */
  double Re, Pe, Sc;   /* Reynolds, Peclet (T diffusion 1/Pe), Schmidt (C diffusion 1/(Re Sc)) */
  double Da, Cf;       /* Darcy number, Forchheimer coefficient */
  double g;            /* body force on u: RU -= g*epsilon1 (equations.f90:104) */
  double InvFr2;       /* buoyancy: RV += InvFr2*(1 - 1/Tbar) (equations.f90:405) */
  double v_in;         /* inflow velocity (v_i at the bottom for ACS_BC_REFERENCE, u on the left
                          for ACS_BC_CHANNEL) */
  double T_in;         /* T on the inflow boundary (Tinf, boundary.f90:86) */
  double C_in;         /* C on the inflow boundary (0 in boundary.f90:129) */
  double b_art;        /* artificial bulk viscosity */
  double beta;         /* artificial compressibility */
  double dt, dtau;     /* physical and pseudo time steps */
  double eps;          /* tolerance on max(res_u, res_v, res_p) (main.f90:139-142) */
  int arith;           /* acs_arith (solver option, no reference counterpart) */
  int continuity;      /* 0: RP = -(face-flux balance) as in equations.f90:623-625;
                          1: RP divided by the p-cell volume vol_p (nonsymetric_mesh.f90:234-238),
                          i.e. the velocity divergence (used by the channel configurations) */
} acs_params;

/* Grid and porous fields (module comum: x, y, xm, ym, epsilon1, liga_poros).  Host or device
 * pointers: acs_create / acs_batch_create copy the arrays they are given. */
typedef struct acs_grid {
  int imax, jmax;
  const double *x, *y, *xm, *ym;      /* [imax], [jmax], [imax+1], [jmax+1] */
  const double *epsilon1, *liga_poros;/* [imax*jmax] column-major */
} acs_grid;

/* field identifiers for get/set (main.f90:15-20) */
enum acs_field {
  ACS_UM = 0, ACS_VM, ACS_UM_TAU, ACS_VM_TAU, ACS_UM_N_TAU, ACS_VM_N_TAU,
  ACS_P, ACS_PN, ACS_T, ACS_T_TAU, ACS_T_N_TAU, ACS_C, ACS_C_TAU, ACS_C_N_TAU,
  ACS_NFIELDS
};

typedef struct acs_handle acs_handle;  /* one case */
typedef struct acs_batch acs_batch;    /* many independent cases in one launch */

const char* acs_last_error(void);
const char* acs_version(void);
int acs_device_count(int* n);

/* ---- mesh helper (the reference driver's `CALL mesh`, nonsymetric_mesh.f90:1-218) ---------- */
/* jmax of the compiled-in reference domain for a given imax (comum.f90:40-46). */
int acs_reference_jmax(int imax);
/* Reference domain 12 x 20, y stretched (Py=1.6, Q=1), porous block x<=-4, y>=0.5 dilated by
 * the flag rule; eps = porosity in flagged cells.  flag may be NULL. */
int acs_mesh_reference(int imax, double porosity, double* x, double* y, double* xm, double* ym,
                       int* flag, double* epsilon1, double* liga_poros);
/* Channel domain [0,Lx] x [0,Ly]: uniform x, y = Ly/2 (1 + tanh(s(2xi-1))/tanh(s)); up to two
 * rectangular porous blocks (box = {x0,x1,y0,y1}; NULL or x0 > x1 disables a block). */
int acs_mesh_channel(int imax, int jmax, double Lx, double Ly, double s, const double* box1,
                     const double* box2, double porosity, double* x, double* y, double* xm,
                     double* ym, int* flag, double* epsilon1, double* liga_poros);
/* acs_mesh_channel generated on the device, for batches of synthetic cases built without host
 * arrays (no reference counterpart beyond nonsymetric_mesh.f90, which it follows): every array is
 * a DEVICE pointer (x: imax, y: jmax, xm: imax+1, ym: jmax+1, flag / epsilon1 / liga_poros:
 * imax x jmax column-major).  The 1-D arrays are computed on the host as acs_mesh_channel does and
 * copied; the porous flag with its dilation sweeps and epsilon1 / liga_poros are computed by
 * kernels on `cuda_stream` (NULL: the legacy default stream), which the call synchronises.  The
 * results equal acs_mesh_channel's bit for bit; an acs_grid may point at them directly. */
int acs_mesh_channel_device(int imax, int jmax, double Lx, double Ly, double stretch, const double* box1,
                            const double* box2, double porosity, double* x, double* y, double* xm, double* ym,
                            int* flag, double* epsilon1, double* liga_poros, void* cuda_stream);
/* Seeded uniform noise in [-amp, amp): splitmix64 of (seed, case, field, index). */
double acs_noise(uint64_t seed, uint64_t case_id, uint64_t field, uint64_t index, double amp);
/* out[k] = acs_noise(seed, case_id, field, index[k], amp) for k < n. */
int acs_noise_array(uint64_t seed, uint64_t case_id, uint64_t field, const uint64_t* index, long long n,
                    double amp, double* out);

/* ---- single case -------------------------------------------------------------------------- */
int acs_create(const acs_grid* g, const acs_params* p, acs_handle** out);
int acs_destroy(acs_handle* h);
/* Launch on this cudaStream_t (NULL = the library's own stream). */
int acs_set_stream(acs_handle* h, void* cuda_stream);

/* Per-routine entry points: host arrays in, host arrays out (one H2D/D2H each call).
 * solve_U: mirrors solve_U(um,vm,um_n,um_tau,vm_tau,um_n_tau,p,residual_u); like the reference,
 * its boundary pass rewrites the boundary values of vm_tau (in/out). */
int acs_solve_u(acs_handle* h, const double* um, const double* um_tau, double* vm_tau,
                const double* p, double* um_n_tau, double* residual_u);
/* solve_V(um,vm,vm_n,um_tau,vm_tau,vm_n_tau,p,T,residual_v); rewrites um_tau's boundary. */
int acs_solve_v(acs_handle* h, const double* vm, double* um_tau, const double* vm_tau,
                const double* p, const double* T, double* vm_n_tau, double* residual_v);
/* solve_P(p,um_n,vm_n,pn,residual_p) */
int acs_solve_p(acs_handle* h, const double* p, const double* um_n_tau, const double* vm_n_tau,
                double* pn, double* residual_p);
/* solve_Z(um_n,vm_n,Z,Z_n_tau,Z_tau): temperature, diffusion 1/Pe */
int acs_solve_z(acs_handle* h, const double* um_n_tau, const double* vm_n_tau, const double* T,
                double* T_n_tau, const double* T_tau);
/* solve_C(um_n,vm_n,C,C_n_tau,C_tau): concentration, diffusion 1/(Re Sc) */
int acs_solve_c(acs_handle* h, const double* um_n_tau, const double* vm_n_tau, const double* Cc,
                double* C_n_tau, const double* C_tau);

/* Device-resident loop state (main.f90:15-20). */
int acs_set_field(acs_handle* h, int field, const double* host);
int acs_get_field(acs_handle* h, int field, double* host);
/* acs_batch_cell_fields of the handle's case */
int acs_cell_fields(acs_handle* h, double* u, double* v, double* vel_mag);
/* n_steps physical steps of main.f90:116-186 on the device, the whole pseudo loop in one CUDA
 * graph.  *itc is the reference's pseudo counter carried across calls (1 before the first step).
 * iters[n_steps] and err[n_steps] (may be NULL) receive each step's pseudo-iteration count and
 * final max residual.  Returns ACS_OK, or ACS_E_STATE with *status = ACS_CASE_FAILED when the
 * residual became NaN/Inf. */
int acs_physical_steps(acs_handle* h, int n_steps, int* itc, int* iters, double* err, int* status);

/* ---- batch of independent cases ----------------------------------------------------------- */
int acs_batch_create(const acs_grid* grids, const acs_params* params, int n_cases, acs_batch** out);
int acs_batch_destroy(acs_batch* b);
int acs_batch_set_stream(acs_batch* b, void* cuda_stream);
int acs_batch_set_field(acs_batch* b, int case_id, int field, const double* host);
int acs_batch_get_field(acs_batch* b, int case_id, int field, double* host);
/* comp_mean (comp_mean.f90:1-25) of case case_id's physical-step velocities computed on the device:
 * u(i,j) = (um(i+1,j) + um(i,j))/2, v(i,j) = (vm(i,j+1) + vm(i,j))/2 and sqrt(u^2 + v^2), the
 * velocity magnitude of the ParaView output (transient.f90:69-74); host arrays imax x jmax,
 * Fortran order.  Uses the batch's stage scratch, so call it between runs. */
int acs_batch_cell_fields(acs_batch* b, int case_id, double* u, double* v, double* vel_mag);
/* Runs every case for n_steps physical steps in one graph launch; converged cases drop out of
 * the launch through per-case masks.  itc[n_cases] in/out; iters/err are [n_cases*n_steps]
 * (case-major, may be NULL); status[n_cases] (may be NULL). */
int acs_batch_run(acs_batch* b, int n_steps, int* itc, int* iters, double* err, int* status);
/* Measurement helper (no reference counterpart): times `reps` back-to-back launches of one
 * kernel of the pseudo-iteration over every case of the batch with CUDA events on the batch's
 * stream and writes the mean duration of one launch in milliseconds.  kernel: 0 = u-momentum
 * (first stage, or the whole fused routine on the FAST path), 1 = v-momentum, 2 = pressure,
 * 3 = temperature, 4 = concentration (per-stage kernels); 5 = the tile engine's U/V Runge-Kutta
 * stage 2, 6 = its P/T/C kernel (FAST batches; sets the tile engine up if needed).  Only stage
 * scratch is written (the output buffers of the pressure and P/T/C kernels are saved and
 * restored), so the loop state is unchanged.  *cells receives the nodes one launch updates. */
int acs_batch_time_kernel(acs_batch* b, int kernel, int reps, double* ms_mean, long long* cells);

/* ---- solve_U without device allocation --------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc (their device memory
 * belongs to another allocator, or they must not allocate once running): solve_U of
 * acs_solve_u, with every array a DEVICE pointer in the Fortran layout (um, um_tau, um_n_tau:
 * (imax+1) x jmax; vm_tau: imax x (jmax+1); pn and the grid's epsilon1/liga_poros: imax x jmax;
 * the grid's x, y, xm, ym as in acs_grid) and no handle.  Its scratch is one static device array
 * of ACS_STATIC_SCRATCH_BYTES that every GPU loading this library holds until exit; sizes beyond
 * ACS_STATIC_MAX_DIM per direction or round_up(imax+1,4)*(jmax+1) > ACS_STATIC_MAX_NODES are
 * rejected with ACS_E_SIZE.  The parameter block is checked as acs_create checks it (ACS_E_ARG
 * for Re, Pe, Sc or Da <= 0, itc_max < 2, an unknown scheme, bc or continuity), and arith must be
 * ACS_ARITH_EXACT, the arithmetic it computes in.  The scratch address is looked up on the first
 * call made on each device, so make that first call before any stream capture; the address is
 * kept for the life of the process and does not survive cudaDeviceReset (do not call this entry
 * point again after a reset).  All calls share the scratch, which each call clears before use:
 * calls that overlap on the GPU race.  The call synchronises `cuda_stream` (NULL = legacy default
 * stream) and writes *residual_u on the host. */
#define ACS_STATIC_MAX_DIM 4096
#define ACS_STATIC_MAX_NODES 65536
#define ACS_STATIC_SCRATCH_BYTES (5 * 1024 * 1024)
int acs_solve_u_static(const acs_params* p, const acs_grid* grid_dev, const double* um, const double* um_tau,
                       double* vm_tau, const double* pn, double* um_n_tau, double* residual_u, void* cuda_stream);

/* Solver options (no reference counterpart). */
enum acs_option {
  ACS_OPT_ENGINE = 1,        /* 0 (default): persistent cluster engine, one thread-block cluster
                                per case runs whole physical steps in one launch;
                                1: CUDA graph of per-stage kernels with a device WHILE node;
                                2: tile engine, ACS_ARITH_FAST only (ACS_E_UNSUPPORTED otherwise):
                                   32 x 32-node tiles of every active case loaded into shared
                                   memory by TMA, four stage kernels per pseudo-iteration in a CUDA graph
                                   with a device WHILE node -- the fastest for many cases.  Setting
                                   it builds the tile table and tensor maps (device memory).  With
                                   the environment variable ACS_NO_CONDITIONAL_GRAPH set, engines 1
                                   and 2 loop from the host instead (one graph launch per
                                   pseudo-iteration), which profilers can look inside */
  ACS_OPT_NODES_PER_CTA = 2, /* engine: target nodes per CTA when sizing a case's cluster */
  ACS_OPT_L1_LOADS = 3,      /* FAST engine: 1 (default) reads cluster-written arrays through L1 */
  ACS_OPT_THREADS = 4,       /* FAST engine: threads per CTA, 256 or 512 (default) */
  ACS_OPT_CTAS_PER_SM = 5,   /* FAST engine, 256 threads: 2 caps registers so two CTAs share an SM */
  ACS_OPT_STAGED = 6,        /* FAST engine: 1 (default) copies each phase's stencil arrays (the
                                CTA's rows plus two halo rows) into shared memory first, where
                                they fit in 220 KB; 0 reads them from L1/L2 */
  ACS_OPT_EXTRAP_ORDER = 7   /* warm start: the extrapolated candidate of acs_batch_set_start is
                                x + inc (1, default) or x + (2 inc - inc_prev), the quadratic
                                through the last three step starts (2; linear until three
                                acs_batch_ws_features calls have given two increments) */
};
int acs_batch_set_option(acs_batch* b, int option, long long value);
/* Persistent cluster engine (no reference counterpart): the number of CTAs (1..16) of case
 * case_id's cluster, overriding ACS_OPT_NODES_PER_CTA for that case; 0 restores the default.
 * A batched step lasts as long as its slowest case, so a caller that knows which cases need the
 * most pseudo-iterations (e.g. from the previous step) can give them more CTAs.  Still capped at
 * (jmax+1)/4 (strips of at least 4 rows).  Results do not depend on it. */
int acs_batch_set_cluster_size(acs_batch* b, int case_id, int ctas);
/* The pseudo-time residual tolerance of case case_id for the following steps: the `eps` of the
 * exit test `error < eps` (main.f90:142; read from input/iterations.dat), initially the
 * case's acs_params.eps.  A warm-start policy may iterate warm-started steps to a tighter
 * tolerance than the plain ones.  eps must be positive and finite (ACS_E_ARG otherwise). */
int acs_batch_set_tolerance(acs_batch* b, int case_id, double eps);
int acs_set_option(acs_handle* h, int option, long long value);

/* ---- learned warm start (no counterpart in the reference) ------------------------------------
 * Each case is drawn on a common H x W canvas (H >= jmax+1, W >= imax+1): node (i, j) of um, vm,
 * p, T and C sits at pixel (j-1, i-1); pixels outside a field's shape are 0.  All tensors are
 * DEVICE pointers, NHWC FP32, case-major, and ordered on the batch's stream.
 *   acs_batch_ws_enable     allocates the per-case history (previous fields, last increment).
 *   acs_batch_ws_features   updates the history (inc = fields - previous fields; 0 on the first
 *                           call after acs_batch_ws_enable; fields uploaded in between count as
 *                           the new fields), computes per case and field the
 *                           RMS s of inc over the field's nodes (1 where inc is 0) and writes
 *                           X[n][H][W][11] = u, v, p, T, C, porous indicator, inc_u/s_u, ...,
 *                           inc_C/s_C.  inc_scale[n][8] (may be NULL) receives s.
 *   acs_batch_ws_target     after a step: T[n][H][W][8] = (increment of this step - inc) / s
 *                           (channels 0..4), Wt = 1 where the node exists, else 0.
 *   acs_batch_set_start     start of the next pseudo-time loop.  Candidates: 0 plain (the stale
 *                           pseudo-iterate the reference starts from), 1 extrapolated
 *                           (fields + inc), 2 learned (fields + a[f] inc + s scale[f] Y[..][f]
 *                           with a[f] = scale[8+f]; only when Y != NULL; scale has 16 entries),
 *                           each with the boundary passes applied.
 *                           policy 0 commits the candidate with the smallest initial residual
 *                           (dtau-scaled max-norm of the U, V stage-1 and P updates); 1 the
 *                           prediction (2 if Y, else 1); 2 plain.  chosen[n] (host, may be NULL)
 *                           = the committed candidate; res0[3n] (host, may be NULL) = the three
 *                           initial residuals (NaN for a candidate that was not built).
 * The pseudo-time loop then iterates to the same tolerance from whichever start was kept. */
#define ACS_WS_IN_CHANNELS 11
#define ACS_WS_OUT_CHANNELS 8
int acs_batch_ws_enable(acs_batch* b, int H, int W);
int acs_batch_ws_features(acs_batch* b, float* X, float* inc_scale);
int acs_batch_ws_target(acs_batch* b, float* T, float* Wt);
int acs_batch_set_start(acs_batch* b, const float* Y, int ldy, const float* scale, int policy, int* chosen,
                        double* res0);

/* Number of kernel launches issued by the last acs_batch_run / acs_physical_steps. */
int acs_batch_launch_count(acs_batch* b, long long* launches);
int acs_launch_count(acs_handle* h, long long* launches);

#ifdef __cplusplus
}
#endif
#endif /* ACS_H */
