/*
 * maxichem_b200: the per-call chemistry solve of imalsky/maxichem as a C-ABI library for NVIDIA B200 (sm_100a).
 *
 * One call advances B independent 0-D gas cells by their own dt with Rodas3 (order 3, L-stable), the exact
 * mass-action Jacobian, adaptive steps, and a guard/recovery pass; it is the device-side body of the reference's
 * CudaSolver call (maxichem/kincuda.py:230-320). Python's CudaSolver (maxichem_b200/solver.py) rebuilds the
 * reference's Python surface on top of these entry points through ctypes.
 *
 * Conventions: all array arguments of mx_call are DEVICE pointers on the solver's device, row-major, float64 unless
 * stated; a call allocates nothing except when its B exceeds every earlier call's (the solver's recompute list then
 * grows, once); errors come back as a nonzero status and a message in err (never an exception across the ABI).
 * Inputs and outputs must not alias. Calls on one solver run one at a time on the given stream (its scratch, queues
 * and list are shared), as the reference's do (maxichem/kincuda.py:114-116).
 */
#ifndef MAXICHEM_B200_H
#define MAXICHEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Settings, with the reference's values (maxichem/_constants.py:12-78); maxichem_b200/constants.py holds the same. */
#define MX_T_MIN 300.0
#define MX_T_MAX 3000.0
#define MX_X_SUM_TOL 1e-10
#define MX_DRIFT 1e-6
#define MX_REC_STEPS 10
#define MX_H_MIN 1e-12
#define MX_CALL_END (1.0 - 1e-14)
#define MX_STEP_SAFETY 0.9
#define MX_ERR_FLOOR 1e-10
#define MX_FAC_NONFINITE 0.1
#define MX_FACACC 0.2
#define MX_FACREJ 0.2
#define MX_FACMAX 20.0
#define MX_FAC_AFTER_REJECT 0.5
#define MX_SECMIN 1e-4
#define MX_SECANT_MIN_ORDER 0.05
#define MX_SECANT_MAX_ORDER 3.0
#define MX_SECANT_TARGET 0.5
#define MX_PIVTAU 0.1
#define MX_ELEMENT_PIVOT_MIN 1e-10
#define MX_REC_RETRIES 3
#define MX_REC_RETRY_SPLIT 0.5
#define MX_GMAX 1e-3
#define MX_KB 1.380649e-16
#define MX_P0 1.0e6
#define MX_NASA_SPLIT_T 1000.0
#define MX_K_COLL 1e-9
#define MX_MAX_SPECIES 254
#define MX_MAX_ELEMENTS 8

/* Count slots of the device count array (maxichem/_constants.py:100-113). */
enum {
  MX_COUNT_QUEUE = 0,
  MX_COUNT_BAD_INPUT,
  MX_COUNT_COLD,
  MX_COUNT_HOT,
  MX_COUNT_NONFINITE,
  MX_COUNT_UNFINISHED,
  MX_COUNT_DRIFT,
  MX_COUNT_RECOMPUTED,
  MX_COUNT_RECOVERED,
  MX_COUNT_STILL_FAILED,
  MX_COUNT_NONFINITE_H,
  MX_COUNT_RECOVERY_QUEUE,
  MX_COUNT_SLOTS
};

/* Status codes (maxichem/kernels/common.cuh:260-262). */
enum { MX_STATUS_OK = 0, MX_REFUSED_COLD = 1, MX_REFUSED_BAD_INPUT = 2, MX_REFUSED_HOT = 3 };

/* Return codes of the entry points. */
enum { MX_OK = 0, MX_ERR_ARGUMENT = 1, MX_ERR_CUDA = 2, MX_ERR_NETWORK = 3, MX_ERR_CLOSED = 4 };

/*
 * A network's tables in host memory, as maxichem_b200/tables.py builds them. Rows are in elimination order (the
 * reference's minimum-degree order, maxichem/_tables.py:35-50) except atoms, which is in the network's species order.
 */
typedef struct mx_network {
  int32_t ns, nr, nrt, nj, nel;  /* species, reactions (thermal then photolysis), thermal, photolysis, elements */
  int32_t n_entries;             /* Jacobian entries */
  int32_t has_troe, has_eff;
  const int32_t* perm;           /* [ns] network species of elimination row i */
  const uint8_t* rx;             /* [nr][6] reactants 0-2, products 3-5 (elimination rows, padding ns) */
  const double* rc;              /* [nr][14] ln A0 B0 C0, ln A1 B1 C1, ln Ai Bi Ci, Troe a T3 T1 T2, efficiency */
  const int32_t* rf;             /* [nr] law flags */
  const double* nasa;            /* [2][ns][9] NASA-9 ranges below and above MX_NASA_SPLIT_T */
  const double* atoms;           /* [ns][nel] network species order */
  const int32_t* sv_ptr;         /* [ns + 1] */
  const uint32_t* sv_term;       /* reaction | coefficient code << 16 */
  const int32_t* jac_ptr;        /* [n_entries + 1] */
  const uint32_t* jac_entry;     /* row << 16 | column */
  const uint32_t* jac_term;      /* rate index | code << 12 | a << 16 | b << 24 */
  const uint8_t* fill;           /* [ns][ns] pattern of L + U (the oracle's sparse factorisation) */
  /* S v rows in pieces of sv_piece terms (the last may be shorter; a row with no terms has one empty piece): row i
   * is the sum, in order, of pieces sv_row_ptr[i] .. sv_row_ptr[i + 1] - 1, each summed in ascending reaction order. */
  int32_t sv_piece, n_pieces;
  const int32_t* sv_row_ptr;     /* [ns + 1] */
  /* Per-thread streams of the same sums for the call kernel's thread groups (maxichem_b200/tables.py
   * thread_streams): [0] the CTA of 128 threads, [1] its last 96 threads. Word q of thread t at q * threads + t. */
  int32_t stream_threads[2];
  int32_t sv_rounds[2], sv_nrows[2], jac_rounds[2], jac_nents[2];
  const uint16_t* sv_stream[2];  /* reaction | code << 11 | end << 13 (padding: nr) */
  const uint16_t* sv_rows[2];    /* the pieces each thread sums */
  const uint32_t* jac_stream[2]; /* rate | code << 12 | end << 14 | a << 16 | b << 24 (padding: rate 2 nr) */
  const uint16_t* jac_dst[2];    /* dense index p ld + q of each thread's entries, ld = ns | 1 */
} mx_network;

typedef struct mx_solver mx_solver;

/*
 * Build a solver for one network on one CUDA device (replaces CudaSolver.__init__/_setup, maxichem/kincuda.py:130-227):
 * copies the tables to the device, sizes the persistent launches and allocates the solver-owned scratch.
 * drift: the guard's element-drift allowance (finite, >= 0).
 */
int mx_create(const mx_network* net, double drift, int device, mx_solver** out, char* err, size_t errlen);

/*
 * One call (replaces CudaSolver.launch's three launches, maxichem/kincuda.py:279-317, without the host read of the
 * counts): screening, rates, Rodas3 steps and the guard in one persistent kernel, then the recovery of the cells the
 * guard listed, then total += count. No host synchronisation.
 * Inputs:  x [B][ns], T, P, dt, h_in [B], J [B][nj] (NULL when nj == 0).
 * Outputs: x_out [B][ns], h_out [B], done [B] (int32 0/1), steps [B], flag [B] (int32 0/1/2), status [B] (int32).
 * count: int32[MX_COUNT_SLOTS], zeroed and filled by the call; total: int64[MX_COUNT_SLOTS], incremented.
 * stream: a cudaStream_t (NULL: the legacy default stream).
 */
int mx_call(mx_solver* s, const double* x, const double* T, const double* P, const double* dt, const double* h_in,
            const double* J, int64_t B, double rtol, double atol, int32_t max_steps, double* x_out, double* h_out,
            int32_t* done, double* steps, int32_t* flag, int32_t* status, int32_t* count, int64_t* total,
            void* stream, char* err, size_t errlen);

/* Cells of one mx_call_static call at most: the size of its static recompute list (4 MiB of device memory). */
#define MX_STATIC_MAX_CELLS 1048576

/*
 * mx_call for callers that cannot allocate device memory. No counterpart in the reference. Such callers are, for
 * instance, a GCM whose framework reserved the GPU's memory for its own pool at start-up (a cudaMalloc during the
 * time loop then fails or fragments that pool), or a time loop that cannot afford the device-wide synchronisation
 * that cudaMalloc and cudaFree may imply. Same arguments, results, errors and kernels as mx_call, but the call's
 * only scratch (the recompute list, one int32 per cell) is a file-scope static device array of MX_STATIC_MAX_CELLS
 * entries instead of solver-owned memory, so the call never calls cudaMalloc, cudaFree or any allocating library
 * routine (the solver handle itself still comes from mx_create, once, at set-up).
 * - B above MX_STATIC_MAX_CELLS is refused with MX_ERR_ARGUMENT and a message naming the limit.
 * - Each call looks up the array's address on the solver's device (cudaGetSymbolAddress, with that device current)
 *   and passes it to the kernels: the array's name is only a host-side stand-in in host code. The first call on a
 *   device may load the library's module there; make that first call before any stream capture on the device.
 * - Every call of every solver in the process shares the array, which keeps the last call's contents. Nothing in it
 *   must start at zero (a call writes each entry before reading it); the queue and list counters that must start at
 *   zero are in count, which the call clears. Calls that overlap on the GPU (other streams, other threads) race on
 *   the array: run them one after another.
 */
int mx_call_static(mx_solver* s, const double* x, const double* T, const double* P, const double* dt,
                   const double* h_in, const double* J, int64_t B, double rtol, double atol, int32_t max_steps,
                   double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag, int32_t* status,
                   int32_t* count, int64_t* total, void* stream, char* err, size_t errlen);

/* Precisions of mx_set_precision. */
#define MX_PRECISION_FP64 0
#define MX_PRECISION_MIXED 1
#define MX_MIXED_MAX_SWEEPS 4
/* The mixed path's default trust bound: a try whose last refinement moved a stage vector by more than this share of
 * the error-control scale (rtol |N| + atol) has its cell redone in FP64. */
#define MX_MIXED_TOL 1.0

/*
 * The arithmetic of later mx_call calls of this solver (mixed precision; no counterpart in the reference, whose
 * solve is FP64 throughout). MX_PRECISION_FP64 (the default): the plain path. MX_PRECISION_MIXED: each try's matrix
 * M0 = I / (gamma h) - Jn is row-scaled by powers of two, factored in FP32 and every stage solve is refined `sweeps`
 * times (1..MX_MIXED_MAX_SWEEPS) against an FP64 residual formed from the rate tables (no FP64 matrix is stored);
 * rates, equilibrium constants, right-hand sides, stage vectors, the error estimate, step control and the guard stay
 * FP64. An accepted try whose last correction exceeds tol (> 0) times the error-control scale hands its cell to the
 * plain FP64 kernel, which redoes it from its inputs in the same call. Results, counts and flags have mx_call's meaning.
 * mx_call_static always runs the plain path.
 */
int mx_set_precision(mx_solver* s, int32_t precision, int32_t sweeps, double tol);

/* Register a device int64[1] that later mixed-precision calls add the number of cells they handed to the FP64 kernel
 * to (NULL stops counting). No counterpart in the reference. */
int mx_set_escalation_counter(mx_solver* s, int64_t* counter);

/* One fresh try of one cell (device x [ns], J [nj]) at try size h through the mixed path with `sweeps` refinements
 * (0..MX_MIXED_MAX_SWEEPS): out = K1, K2, K3, K4, N' [ns each, elimination order], err, ok, the largest last
 * correction and the largest first correction on the error-control scale. No counterpart in the reference: a test
 * hook, against mx_debug_try's FP64 stages. */
int mx_debug_try_mixed(mx_solver* s, const double* x, double T, double P, double h, const double* J, double rtol,
                       double atol, int32_t sweeps, double* out, void* stream);

/* Tangent directions of one mx_jvp call at most (the reference's DMAX, maxichem/_constants.py:29). */
#define MX_JVP_MAX_DIRECTIONS 16

/*
 * One call and its tangent along D directions (replaces ADSolver.jvp's launches, maxichem/kincuda_ad.py:325-453):
 * the call's screening, rates, Rodas3 steps, guard and recovery, with the derivative of x_out and h_out along each
 * direction. The primal is mx_call's bit for bit when lm and rc are NULL.
 * Inputs as mx_call's, and lm [B][nr] per-cell log rate multipliers (NULL: none; a multiplier scales both directions
 * of a reaction after the collision limit, a photolysis branch has kf = J e^lm), rc [nr][14] the rate table (NULL:
 * the network's). adapt: 1 differentiates the step control too (rejected tries included, h carried in and out), 0
 * holds every accepted try's size fixed (no tangent through dt, h or the error; dh_out 0).
 * Tangents, device arrays with a leading axis of D directions: dx [D][B][ns], dT, dP, ddt, dh [D][B], dlm [D][B][nr],
 * drc [D][nr][9] (the nine Arrhenius columns), dJ [D][B][nj]; dlm, drc and dJ NULL for zero.
 * Outputs as mx_call's, and dx_out [D][B][ns], dh_out [D][B]: the tangents of the result before the guard's
 * element-share correction (conservation makes the correction's own sensitivity zero). A cell the guard recomputes
 * is differentiated along the recovery's path; one that still fails (flag 2) has NaN tangents. A non-finite log
 * multiplier is not a refusal: the cell takes no step and fails. Errors as mx_call's, and D outside
 * 1..MX_JVP_MAX_DIRECTIONS or adapt not 0/1 (MX_ERR_ARGUMENT). Allocates the tangent kernels' scratch at the first
 * call and when a call needs more. Calls run one at a time.
 */
int mx_jvp(mx_solver* s, const double* x, const double* T, const double* P, const double* dt, const double* h_in,
           const double* J, const double* lm, const double* rc, int64_t B, double rtol, double atol, int32_t max_steps,
           int32_t adapt, int32_t D, const double* dx, const double* dT, const double* dP, const double* ddt,
           const double* dh, const double* dlm, const double* drc, const double* dJ, double* x_out, double* h_out,
           int32_t* done, double* steps, int32_t* flag, int32_t* status, double* dx_out, double* dh_out,
           int32_t* count, int64_t* total, void* stream, char* err, size_t errlen);

/*
 * One call and its adjoint (replaces ADSolver.vjp's launches, maxichem/kincuda_ad.py:455-556): the call, guard and
 * recovery as mx_jvp's, then the cotangents of the inputs for the cotangents gx [B][ns] of x_out and gh [B] of h_out
 * (NULL for zero; used with adapt 1 only). The forward pass stores each try's state, beyond 2 cap tries a checkpoint
 * every ceil(n / 2 cap) tries whose segments are recomputed; max_steps may be at most (2 cap)^2 / MX_REC_STEPS.
 * Outputs as mx_call's, and gx0 [B][ns], gT, gP, gdt, gh0 [B], glm [B][nr], gJ [B][nj] (NULL when nj == 0) per cell,
 * and grc [nr][9], the rate table's nine Arrhenius columns, summed over the cells in a fixed order. A cell that still
 * fails (flag 2) has NaN cotangents and is left out of grc, as is a refused cell. Results do not depend on the batch
 * order or on the launch: no atomics enter the arithmetic (grc is summed over fixed chunks of 64 consecutive cells
 * and then over the chunks in order, so it keeps its bits for a given batch). Allocates the adjoint's scratch at the
 * first call and when a call needs more: per CTA 17 nr + 4 cap (ns + 8) doubles, per chunk of 64 cells 9 nr doubles
 * (the chunk's partial sum of the rate table's cotangent: 0.5 GB at 1,048,576 cells of 438 reactions), and 3 nr
 * doubles per cell the recovery redoes; one small host read of the count of those cells (a synchronisation of
 * the stream). Calls run one at a time.
 */
int mx_vjp(mx_solver* s, const double* x, const double* T, const double* P, const double* dt, const double* h_in,
           const double* J, const double* lm, const double* rc, int64_t B, double rtol, double atol, int32_t max_steps,
           int32_t adapt, int32_t cap, const double* gx, const double* gh, double* x_out, double* h_out, int32_t* done,
           double* steps, int32_t* flag, int32_t* status, double* gx0, double* gT, double* gP, double* gdt,
           double* gh0, double* glm, double* grc, double* gJ, int32_t* count, int64_t* total, void* stream,
           char* err, size_t errlen);

/* The guard alone on given states (replaces a launch of the reference's guard kernel, maxichem/kernels/guard.cuh:114):
 * counts refused cells from status, checks and corrects the others in x_out, writes flag 0/1 and the recompute list
 * count. Device pointers; used by tests of the guard's thresholds. */
int mx_guard(mx_solver* s, const double* x, double* x_out, const int32_t* done, const double* steps,
             const int32_t* status, int64_t B, double atol, int32_t* flag, int32_t* count, void* stream, char* err,
             size_t errlen);

/* Launch layout of the solver, for reports: warps per cell, rows per lane of the solves, shared bytes per cell,
 * call and recovery CTAs per SM at full occupancy, SMs, the matrix's leading dimension, the call grid's CTAs per SM
 * (0: one CTA per cell), the cells the solver-owned recompute list holds (0 until an mx_call or mx_guard sized it),
 * the mixed kernel's shared bytes per cell and CTAs per SM, the precision (MX_PRECISION_*) and refinement sweeps. */
int mx_info(const mx_solver* s, int32_t* values, int32_t n);

/* The call kernel's grid for later calls: ctas_per_sm from 1 to the occupancy limit (the larger of the plain and the
 * mixed kernel's; each kernel takes at most its own) runs that many persistent CTAs per SM over the cell queue; 0
 * launches one CTA per cell (a static launch); -1 restores the default (the occupancy limit). Results do not depend
 * on it. No counterpart in the reference, which picks its cells per block by
 * recompiling (maxichem/kincuda.py:184-218); maxichem_b200/autotune.py times the choices. */
int mx_set_grid(mx_solver* s, int32_t ctas_per_sm);

/* One fresh try of one cell (device x [ns], J [nj]) at try size h, with every stage written to the device array out:
 * kf, kr [nr each], F, u0 [ns each], -Jn [ns][ns], w [ns], LU factors [ns][ns], dinv, K1, K2, K3, K4, N' [ns each],
 * err, ok (elimination order). No counterpart in the reference: a test hook that runs the call kernel's own device
 * functions, so each stage can be checked against the CPU oracle. */
int mx_debug_try(mx_solver* s, const double* x, double T, double P, double h, const double* J, double rtol,
                 double atol, double* out, void* stream);

/* Register a device int64[3] that later calls of this solver add their tries to: [0] the call kernel's tries, [1] those
 * that followed a rejection, [2] the recovery's tries (NULL stops counting). No counterpart in the reference: it
 * feeds the measured roofline (algorithmic FLOPs per try are a property of the network's tables). */
int mx_set_try_counter(mx_solver* s, int64_t* tries);

/* Register a device int64[8] that later calls add per-phase SM cycles to (clock64 on one thread per cell): rates, F
 * and Jacobian, LU, stages 1-2, stage 3, stage 4, step control, output and guard; NULL returns to the plain kernel.
 * No counterpart in the reference: it attributes the call kernel's time for tuning. */
int mx_set_phase_counter(mx_solver* s, int64_t* cycles);

/* Average SM cycles of each device function of one try, each repeated reps times on one cell in each of ctas CTAs
 * (device x [ns], J [nj]): rates, F, Jacobian and w, LU, two-vector solve, one-vector solve, Sherman-Morrison, error,
 * guard test, into the device int64[9] cycles. No counterpart in the reference: a tuning hook. */
int mx_time_phases(mx_solver* s, const double* x, double T, double P, double h, const double* J, int32_t reps,
                   int32_t ctas, int64_t* cycles, void* stream);

/* FP64 fused multiply-add throughput of a device in GFLOP/s, from independent fma chains on every SM (synchronises
 * the device). No counterpart in the reference: the roofline's FP64 denominator, which the driver-measured peaks
 * file does not hold. */
int mx_probe_fp64(int device, int64_t iters, double* gflops);

/* A solver from a folder that CudaSolver.export wrote (meta.txt and tables/<name>.bin: the network's tables and the
 * drift allowance), for a caller without Python; replaces the reference's export loader (cpp/maxichem.cpp:40-171).
 * The folder is read and checked completely before any CUDA work: a missing or malformed table returns
 * MX_ERR_NETWORK. */
int mx_create_from_export(const char* folder, int device, mx_solver** out, char* err, size_t errlen);

/* The GCM step's conversions either side of a call (replace maxichem/coupling/composition.py:102-183), on device
 * arrays of B cells, asynchronous on stream; one pass over [B][ns] each, one warp per cell, row sums in the warp's
 * order (lane l adds entries l, l + 32, ..., then a butterfly).
 * mx_mass_to_mole: mass mixing ratios q -> mole fractions x = (q / mw) / sum(q / mw). *bad (device int32, zeroed by
 * the call) gets bit 1 for a non-finite q, and unless signed_ok bit 2 for a negative q and bit 4 for a cell whose
 * sum is not above 0. With signed_ok (signed_mole_fractions, composition.py:130-151) negatives pass through.
 * mx_mole_to_mass: x and each cell's tracer mass -> q = x mw (mass / sum(x mw)); *bad gets bit 1 for a non-finite x,
 * 2 for a negative x, 4 for a cell whose sum of x mw is not above 0, 8 for a mass negative or not finite. */
int mx_mass_to_mole(const double* q, const double* mw, int64_t B, int32_t ns, int32_t signed_ok, double* x,
                    int32_t* bad, void* stream);
int mx_mole_to_mass(const double* x, const double* mw, const double* mass, int64_t B, int32_t ns, double* q,
                    int32_t* bad, void* stream);

/*
 * The learned part of the call (no counterpart in the reference). A BF16 MLP surrogate of the
 * per-call solve: features of a cell (log10 x per species floored at 1e-30, log10 T, P, dt and the carried h,
 * log10(J + 1e-30) per branch, standardised, zero-padded to a multiple of 64: kin) -> `layers` hidden layers of width `hidden` (SiLU) ->
 * `heads` output blocks of nt = ns + 1 values (log10 x_out - log10 x_in per species, log10 h_out; standardised),
 * padded to kout (a multiple of 64). Every layer is a tcgen05 GEMM with its bias and activation fused; training on
 * the GPU by the same GEMMs (backward dX with the SiLU derivative fused, dW), bias sums and Adam.
 */
typedef struct mx_surrogate mx_surrogate;

/* A surrogate for a network of ns species, nj photolysis branches and nel elements (atoms [ns][nel], host, network
 * order), with zero weights and unit scaling, on one device. */
int mx_sur_create(int32_t ns, int32_t nj, int32_t nel, const double* atoms, int32_t hidden, int32_t layers,
                  int32_t heads, int32_t device, mx_surrogate** out, char* err, size_t errlen);

/* Sizes: nf (features), kin, nt, kout, P (FP32 parameters), layers, hidden, heads, training steps taken. */
int mx_sur_info(const mx_surrogate* s, int64_t* values, int32_t n);

/* The standardisation (host float arrays): feature mean, deviation and training range [lo, hi] ([nf] each), target
 * mean and deviation ([nt] each). A cell with a feature outside its range is never accepted. */
int mx_sur_set_scaling(mx_surrogate* s, const float* feat_mean, const float* feat_std, const float* feat_lo,
                       const float* feat_hi, const float* tgt_mean, const float* tgt_std);

/* Features of B cells (device inputs as mx_call's) into feat (device BF16 [B][kin]) and in_range (device int32 [B],
 * nullable: 1 when every feature is inside the training range). Asynchronous on stream. */
int mx_sur_features(mx_surrogate* s, const double* x, const double* T, const double* P, const double* dt,
                    const double* h, const double* J, int64_t B, void* feat, int32_t* in_range, void* stream);

/* The network on B rows of features (device BF16 [B][kin]) into pred (device FP32 [B][kout]), in chunks of 65,536
 * rows. Asynchronous on stream. */
int mx_sur_forward(mx_surrogate* s, const void* feat, int64_t B, float* pred, void* stream);

/* One Adam step (lr, betas 0.9 / 0.999, eps 1e-8) on a batch of M rows (a multiple of 64): features feat (BF16
 * [M][kin]), standardised targets tgt (FP32 [M][nt]) and per-row head weights wts (FP32 [M][heads], the heads'
 * bootstrap draw). The loss is the weighted mean over rows, heads and targets of the square error (delta 0) or of
 * the Huber loss of width delta (> 0, in standardised units); *loss (device FP32, nullable) is incremented by it.
 * Asynchronous on stream; lr 0 computes the gradients only (mx_sur_params 1). */
int mx_sur_train_step(mx_surrogate* s, const void* feat, const float* tgt, const float* wts, int64_t M, float lr,
                      float delta, float* loss, void* stream);

/* The FP32 parameters (which 0) or the last step's gradients (which 1) into a host array of P floats, layer by layer:
 * W_l [out][in] then b_l [out]. Synchronises. mx_sur_set_params writes them (and restarts Adam). */
int mx_sur_params(mx_surrogate* s, int32_t which, float* host, int64_t n);
int mx_sur_set_params(mx_surrogate* s, const float* host, int64_t n);

/* The GEMMs' error flag (1 when a wait on the tensor-core pipeline gave up), read and cleared. Synchronises. */
int mx_sur_error(mx_surrogate* s, int32_t* flag);

/*
 * The gated call: for B cells (device arrays as mx_call's) the network proposes each cell's end-of-call state (the
 * heads' mean) and step size. A proposal is accepted only if every feature is inside the training range, the heads'
 * largest deviation over species above 1e-20 is at most spread_max (dex), and projecting it onto the input's element
 * shares (the guard's multiplicative correction, twice) moves no species by more than proj_max (relative) and leaves
 * the guard's drift test passed. Accepted cells take the proposal (steps 0, done 1, flag 0). Rejected cells, and a
 * seeded draw of one accepted cell in audit_every (0: none), are solved by the solver's Rodas3 path (its precision)
 * with its guard and recovery, in the same call, with no host synchronisation. The audited cells' proposals go to
 * audit_x [audit_cap][ns] (their cells to audit_cells, *audit_count of them, at most audit_cap) and their relative
 * error against Rodas3 per species above 1e-20 (else 0) to audit_err [audit_cap][ns]. stats (device uint64[6]) is
 * incremented by: accepted, audited, refused for range, for spread, for the projection, unusable inputs. count and
 * total as mx_call's (the queue slot counts every cell).
 */
int mx_sur_call(mx_surrogate* s, mx_solver* solver, const double* x, const double* T, const double* P,
                const double* dt, const double* h_in, const double* J, int64_t B, double rtol, double atol,
                int32_t max_steps, double spread_max, double proj_max, int32_t audit_every, uint32_t seed,
                double* x_out, double* h_out, int32_t* done, double* steps, int32_t* flag, int32_t* status,
                int32_t* count, int64_t* total, uint64_t* stats, int32_t* audit_cells, double* audit_x,
                float* audit_err, int32_t* audit_count, int32_t audit_cap, void* stream, char* err, size_t errlen);

/* The gate's measures without a decision (for calibrating the thresholds on held-out cells and for tests): for B
 * cells the projected proposal into x_prop [B][ns] and, per cell, diag [B][4]: the heads' spread (dex), the
 * projection's size (infinite when the projected proposal fails the drift test with allowance drift), 1 when the
 * inputs are usable and inside the training range (else 0), and the proposed h. Asynchronous on stream. */
int mx_sur_propose(mx_surrogate* s, const double* x, const double* T, const double* P, const double* dt,
                   const double* h_in, const double* J, int64_t B, double drift, double atol, double* x_prop,
                   double* diag, void* stream);

int mx_sur_destroy(mx_surrogate* s);

/* The surrogate's GEMM alone (a building block, exported for tests): C[M, N] = A[M, K] B[N, K]^T, A and B device BF16
 * row-major with leading dimensions lda, ldb (K and N multiples of 64). mode 0: out FP32 = C; 1: out FP32 = C + bias;
 * 2: z = C + bias (FP32 [M][ldz] when z is not null), out BF16 = silu(z); 3: out BF16 = C * silu'(z), z read.
 * Every pointer (A, B, out, bias, z) and row pitch in bytes must be a multiple of 16, or MX_ERR_ARGUMENT is returned
 * with nothing launched. *err_flag (device int32) is set when a wait gave up. Asynchronous on stream. */
int mx_gemm_bf16(const void* A, int32_t lda, const void* B, int32_t ldb, int64_t M, int32_t N, int32_t K,
                 int32_t mode, const float* bias, float* z, int32_t ldz, void* out, int32_t ldo, int32_t* err_flag,
                 void* stream);

/* The weight gradients' product alone (exported for tests): out[M][N] FP32 (pitch ldo) = A B^T as mx_gemm_bf16's
 * mode 0, with K (the batch) split across the SMs when the output has fewer 128 x 64..256 tiles than the device has
 * SMs: each split's partial product goes to workspace (mx_gemm_split_workspace(M, N, K) floats; NULL when that is 0)
 * and a second kernel adds them in split order, so the result is the same bits run to run (not those of the unsplit
 * product: the partial sums group the terms differently). */
int mx_gemm_bf16_split(const void* A, int32_t lda, const void* B, int32_t ldb, int64_t M, int32_t N, int32_t K,
                       float* workspace, float* out, int32_t ldo, int32_t* err_flag, void* stream);
int64_t mx_gemm_split_workspace(int64_t M, int32_t N, int32_t K);

/* Release the solver's device memory. Safe on NULL. */
int mx_destroy(mx_solver* s);

/* The library's build identity (architecture and version), a static string. */
const char* mx_version(void);

/* Warps per cell of the call kernel by default: mx_network's stream groups have 32 x that and 32 x (that - 1) threads
 * (maxichem_b200/tables.py stream_groups). The call, recovery and mixed kernels also take 2 warps per cell (tables
 * built for 64 and 32 threads; mx_warps_supported), which fits twice the cells per SM when registers, not shared
 * memory, bound the occupancy; results are the same bits either way. The derivative kernels take the default only.
 * No counterpart in the reference, whose warps per cell follow the network's size (maxichem/_constants.py:70-72). */
int mx_warps_per_cell(void);
int mx_warps_supported(int32_t warps);

/* Cells of the network n that fit one SM of device by shared memory (one cell per CTA, the CTA's reserved shared
 * memory included), or -MX_ERR_NETWORK / -MX_ERR_CUDA. Allocates nothing and needs no solver: a caller chooses the
 * warps per cell with it before building the tables (maxichem_b200/solver.py takes 2 warps when at least 6 cells fit,
 * so that the 2-warp kernels, 8 CTAs per SM by registers, hold at least half again as many cells as the 4-warp ones).
 * n's stream fields are not read. No counterpart in the reference (its choice: maxichem/_constants.py:67-72). */
int mx_cells_per_sm(const mx_network* n, int32_t device);

#ifdef __cplusplus
}
#endif
#endif
