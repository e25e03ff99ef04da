/*
 * fame.h — C ABI of the B200 (sm_100a) eigensolver hot path for the 6D
 * null-space-free Maxwell projection method.
 *
 * Conventions
 *  - Every entry point returns an int status (FAME_OK == 0).  No exceptions
 *    cross the boundary.  fame_last_error() gives the message of the last
 *    failure on the calling thread.
 *  - Arrays are DEVICE pointers unless a parameter says "host".  Complex data
 *    is interleaved (re,im): complex128 for FAME_F64, complex64 for FAME_F32.
 *    Matrices are column-major (MATLAB layout); a vector of NF rows is the
 *    column-major 6D grid of (2N)^6 Fourier modes in FFT order
 *    [0..N-1, -N..-1] per axis; 2NF/3NF vectors are component-stacked.
 *  - Buffers are caller-owned; handles own their workspace.  A handle is used
 *    from one host thread at a time.  Work is ordered on the context's stream
 *    (fame_ctx_set_stream); calls that return host values synchronise it.
 *  - The reference functions each entry point replaces are cited as
 *    file:line inside the reference project (MATLAB).
 */
#ifndef FAME_H
#define FAME_H
#include <stdint.h>
#if defined(__GNUC__)
#define FAME_API __attribute__((visibility("default")))
#else
#define FAME_API
#endif
#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (mirror the reference's error identifiers) ---- */
#define FAME_OK 0
#define FAME_ERR_INVALID 1       /* *:BadSize / *:BadInput (e.g. exp1/rank1_exact_fft_scatter.m:5-7) */
#define FAME_ERR_CUDA 2          /* CUDA runtime failure */
#define FAME_ERR_OOM 3           /* allocation failed (exp1/classify_exp1_exception.m:20-38 "oom") */
#define FAME_ERR_NOT_CONVERGED 4 /* PCG flag!=0 and relres>10*tol (exp2/make_krinv_instrumented.m:72-77) */
#define FAME_ERR_NONFINITE 5     /* NaN/Inf input/output (exp2/make_krinv_instrumented.m:38-40) */
#define FAME_ERR_BUDGET 6        /* iteration budget (exp1/make_run_budget.m:29-83 EXP1:IterationLimit) */
#define FAME_ERR_SINGULAR 7      /* zero projected mode, Gamma point (exp1/assemble_K_and_nullspace_free_basis.m:36-42) */
#define FAME_ERR_UNSUPPORTED 8   /* size outside the supported range (2N <= 14) */
#define FAME_ERR_BREAKDOWN 9     /* Lanczos breakdown (exp2/Lanczos.m:75-79) */

#define FAME_F64 0
#define FAME_F32 1

/* mass-operator modes: the four handles of exp1/build_mass_backend_large_scalar.m:28-31 */
#define FAME_MASS_SCALAR 0 /* MscalarOp: NF -> NF          */
#define FAME_MASS_FULL3 1  /* Mop:       3NF -> 3NF        */
#define FAME_MASS_COL3 2   /* Mcol3op:   NF -> 3NF [0;0;M]x */
#define FAME_MASS_COLS12 3 /* Mcols12op: 2NF -> 3NF diag(M,M,0) */

/* K_r^{-1} realisations */
#define FAME_KRINV_EXPLICIT 0 /* exp1/make_explicit_krinv_compact.m */
#define FAME_KRINV_NESTED 1   /* exp1/make_nested_krinv_instrumented.m */

/* precision forms of the inner solves */
#define FAME_PREC_FP64 0  /* plain FP64 throughout */
#define FAME_PREC_MIXED 1 /* FP32 mass + PCG inside FP64 iterative refinement */

typedef struct fame_ctx fame_ctx;
typedef struct fame_mass fame_mass;
typedef struct fame_basis fame_basis;
typedef struct fame_krinv fame_krinv;

FAME_API const char* fame_status_string(int status);
FAME_API const char* fame_last_error(void);
FAME_API int fame_version(void);
/* Kernels launched by this library since load (instrumentation for benchmarks). */
FAME_API long long fame_kernel_launches(void);
/* (No reference counterpart) the library takes its device memory from a memory pool it
 * creates per device (the device's default pool and its settings are left alone) and keeps
 * freed blocks cached for its next handles (a free still waits for the device, as cudaFree
 * does); this returns the cached memory of a device to the driver. */
FAME_API int fame_device_trim_memory(int device);

/* ---- context (replaces gpu_initialize / wait_for_gpu: exp1/wait_for_gpu.m:5-11) ---- */
FAME_API int fame_ctx_create(int device, fame_ctx** out);
FAME_API int fame_ctx_destroy(fame_ctx* ctx);
/* Order all work of the context on `stream` (a cudaStream_t; NULL is the legacy
 * default stream).  A new context uses its own non-blocking stream. */
FAME_API int fame_ctx_set_stream(fame_ctx* ctx, void* stream);
/* Return to the context's own non-blocking stream. */
FAME_API int fame_ctx_use_own_stream(fame_ctx* ctx);
FAME_API int fame_ctx_sync(fame_ctx* ctx);

/* ---- 6D Fourier mass operator ---- */
/* Replaces applyMij_fft(x,Eij,sz,n) — exp1/applyMij_fft.m:1-24.
 * y = fftn(E .* ifftn(x)) column by column; E real, NF=(2N)^6, 1 <= N <= 7. */
FAME_API int fame_applyMij_fft(fame_ctx* ctx, int N, const double* E, const void* x, void* y,
                      int nrhs, int prec);

/* Mass handle: replaces the mass struct of exp1/build_mass_backend_large_scalar.m:27-46.
 * E is the real-space permittivity on the (2N)^6 grid (device, FP64). */
FAME_API int fame_mass_create(fame_ctx* ctx, int N, const double* E, fame_mass** out);
FAME_API int fame_mass_destroy(fame_mass* m);
/* mode: FAME_MASS_*; prec: FAME_F64 / FAME_F32 (x,y complex128 / complex64) */
FAME_API int fame_mass_apply(fame_mass* m, int mode, const void* x, void* y, int nrhs, int prec);

/* (No reference counterpart) fault-path self-test of the bounded device-side waits: runs
 * pass B of the FP32 chain with every stage barrier armed for bytes that no copy delivers
 * (no copy is issued), so each CTA's wait runs out after poll_limit polls (1..2^20), sets
 * the device's fault word and returns.  Returns what the next synchronisation reports:
 * FAME_ERR_CUDA when the timeout was detected (the expected outcome); the fault word is
 * cleared and the context stays usable.  The mass handle's scratch field is overwritten. */
FAME_API int fame_selftest_bounded_wait(fame_mass* m, unsigned poll_limit);

/* Replaces applyMij_rank1_exact(x,kernelFFT,plan) — exp1/applyMij_rank1_exact.m:1-6
 * with rank1_exact_fft_scatter / rank1_exact_ifft_gather
 * (exp1/rank1_exact_fft_scatter.m:1-13, exp1/rank1_exact_ifft_gather.m:1-11).
 * inputIdx/targetIdx are the plan's 1-based uint32 code vectors (device, NF each) of
 * exp1/build_radix_exact_rank1_plan_scalar.m:57-58 and M the plan length.  The plan is
 * verified against the radix construction (FAME_ERR_INVALID if it is not that plan);
 * the action is the algebraically identical 6D convolution. */
FAME_API int fame_applyMij_rank1_exact(fame_mass* m, const uint32_t* inputIdx, const uint32_t* targetIdx,
                              long long M, const void* x, void* y, int nrhs);

/* Replaces rank1_exact_fft_scatter(x,plan) — exp1/rank1_exact_fft_scatter.m:1-13.
 * Xfft (M x nrhs, column-major, device complex128) = the length-M DFT (MATLAB fft) of the
 * embedding of x (NF x nrhs) at the plan's 1-based inputIdx (device uint32, NF entries).
 * M may be any product of factors <= 27 (the radix plans' M = nGrid (2 nGrid - 1)^5 are);
 * FAME_ERR_UNSUPPORTED otherwise.  FAME_ERR_INVALID for an index outside [1, M]
 * (rank1_exact_fft_scatter:BadSize is the caller's check of x's NF rows).  Uses
 * M complex128 of context workspace; synchronises the context's stream. */
FAME_API int fame_rank1_exact_fft_scatter(fame_ctx* ctx, const void* x, int nrhs, const uint32_t* inputIdx,
                                          long long NF, long long M, void* Xfft);
/* Replaces rank1_exact_ifft_gather(Yfft,plan) — exp1/rank1_exact_ifft_gather.m:1-11.
 * y (NF x nrhs) = ifft(Yfft)(targetIdx) for Yfft (M x nrhs, device complex128, read only)
 * and the plan's 1-based targetIdx (device uint32, NF).  Same M rule and errors as the
 * scatter; uses 2 M complex128 of context workspace; synchronises the stream. */
FAME_API int fame_rank1_exact_ifft_gather(fame_ctx* ctx, const void* Yfft, int nrhs, const uint32_t* targetIdx,
                                          long long NF, long long M, void* y);

/* ---- block-diagonal basis maps (complex128, n modes, nrhs columns) ---- */
/* exp1/apply_V_blockdiag.m:1-17: y(3n x nrhs) = V x(2n x nrhs) */
FAME_API int fame_apply_V_blockdiag(fame_ctx* ctx, const void* x, const void* V11, const void* V12,
                           const void* V21, const void* V22, const void* V31, const void* V32,
                           long long n, int nrhs, void* y);
/* exp1/apply_VH_blockdiag.m:1-16: y(2n x nrhs) = V^* x(3n x nrhs) */
FAME_API int fame_apply_VH_blockdiag(fame_ctx* ctx, const void* x, const void* V11, const void* V12,
                            const void* V21, const void* V22, const void* V31, const void* V32,
                            long long n, int nrhs, void* y);
/* exp1/solveV1_blockdiag.m:1-10: y = V1^{-1} x */
FAME_API int fame_solveV1_blockdiag(fame_ctx* ctx, const void* x, const void* V11, const void* V12,
                           const void* V21, const void* V22, const void* det, long long n,
                           int nrhs, void* y);
/* exp1/solveV1H_blockdiag.m:1-10: y = V1^{-*} x */
FAME_API int fame_solveV1H_blockdiag(fame_ctx* ctx, const void* x, const void* V11, const void* V12,
                            const void* V21, const void* V22, const void* det, long long n,
                            int nrhs, void* y);

/* ---- null-space-free basis (exp1/assemble_K_and_nullspace_free_basis.m:18-105,
 *      exp1/build_experiment1_q_system.m:7-24, exp1/build_inner_system_operators.m:10-14) ---- */
/* P: host, 6x3 column-major; q: host, 3.  kLift = P (P^T P)^{-1} q. */
FAME_API int fame_basis_create(fame_ctx* ctx, int N, const double* P, const double* q, fame_basis** out);
FAME_API int fame_basis_destroy(fame_basis* b);
typedef struct {
  long long NF;
  int N;
  int nsingular;       /* modes handled by the singular branch (:75-91) */
  double minQq;        /* min |q_xi|^2 */
  double minAbsDetV1;  /* exp1/build_experiment1_q_system.m:16 */
  double kLift[6];
  int pivot;           /* component forming the V3 row of the explicit split: 2 as in the
                          reference, else the largest |q_c| when that V1 block is singular */
} fame_basis_info;
FAME_API int fame_basis_info_get(fame_basis* b, fame_basis_info* out);
/* Export one modewise diagonal into a caller buffer (device):
 *  complex128: 0..5 = V11,V21,V31,V12,V22,V32; 6 = detV1; 7 = W1; 8 = W2
 *  float64:    9 = invC; 10 = |q|^2; 11,12,13 = q1,q2,q3 */
FAME_API int fame_basis_get(fame_basis* b, int which, void* dst);

/* exp1/apply_Mhat_C_scalar_compact.m:8-21 (with the basis' W1, W2, invC):
 * y = C^{-1}(M z + W1^* M(W1 z) + W2^* M(W2 z)), z = C^{-1} x; x,y NF-vectors
 * (complex128 for FAME_F64, complex64 for FAME_F32). */
FAME_API int fame_apply_Mhat_C_scalar_compact(fame_basis* b, fame_mass* m, const void* x, void* y,
                                              int prec);

/* Same action as fame_apply_Mhat_C_scalar_compact, with no device allocation: no
 * counterpart in the reference.  For callers that cannot let a library allocate
 * GPU memory (hosts that own all device memory through their own pool, loops that
 * must not pay the device synchronisation of cudaMalloc/cudaFree).  The three-field
 * scratch is a static 32 MiB device array held by every GPU that loads this library
 * until exit, so 3*NF*sizeof(element) must fit: FP32 up to N=5, FP64 up to N=4;
 * larger sizes return FAME_ERR_INVALID.  The first call on a device looks up the
 * array's device address (make it before any stream capture).  All calls share the
 * array: calls that overlap on the GPU (e.g. on different streams) race. */
FAME_API int fame_apply_Mhat_C_scalar_compact_noalloc(fame_basis* b, fame_mass* m, const void* x,
                                                      void* y, int prec);

/* ---- Yee-field physical validation (LWRQ) ---- */
/* exp3/compute_yee_lwrq_metrics_exp4.m + compute_lwrq_exp4.m + apply_cropped_A_exp3.m +
   separable_conv3_same_exp4.m + sample_scalar_yee_material_exp4.m.  u1..u3: device complex128
   fields on the plus-grid, (2n+3)^3 each, x fastest.  P: cut matrix, column-major 6 x 3.
   material_kind 0: eps = mp0 exp(mp1/6 sum_l cos(P_l.x)) (epsC, alpha); 1: eps = 1 + mp0 prod_l
   (1 + cos(P_l.x))/2 (delta).  metrics (host, 10): lambdaCrop, lambda3D, eta3D, etaUsing6DLambda,
   deltaLambda, VLWRQ, nuLWRQ, deltaPart, deltaLWRQIdentity, croppedMass.  slice_z0 / slice_x0
   (host, (2n+1)^2 each, or NULL): |rho - lambda3D| / |lambda3D| on z = 0 (x fastest) and on
   x = 0 (y fastest). */
FAME_API int fame_yee_lwrq_metrics(fame_ctx* ctx, const void* u1, const void* u2, const void* u3, int n,
                                   double h, const double* P, int material_kind, double mp0, double mp1,
                                   double lambda6D, double* metrics, double* slice_z0, double* slice_x0);

/* ---- K_r^{-1} actions ---- */
typedef struct {
  int kind;        /* FAME_KRINV_EXPLICIT | FAME_KRINV_NESTED */
  int prec_mode;   /* FAME_PREC_FP64 | FAME_PREC_MIXED */
  double tolCG;    /* explicit: Mhat PCG tolerance (1e-10) */
  int maxitCG;     /* explicit: Mhat PCG max iterations (1200) */
  double tolKr;    /* nested: outer K_r PCG tolerance (1e-10) */
  double tolM;     /* nested: inner M PCG tolerance (1e-12) */
  int maxitKr;     /* nested (600) */
  int maxitM;      /* nested (1600) */
  double epsC;     /* nested preconditioner scale epsC*r./sigma_r (4) */
  int useKrPreconditioner; /* nested (1) */
  double tolInner32; /* mixed: relative tolerance of each FP32 correction solve (3e-6) */
  int maxRefine;     /* mixed: max FP64 refinement steps per solve (20) */
  int checkEvery;    /* PCG iterations queued between host convergence checks (4) */
  int verifyTrueResidual; /* confirm convergence on the true residual, as MATLAB pcg (1) */
  int useGraphs;     /* replay PCG iterations as captured CUDA graphs (1) */
  int mhatPreconditioner; /* explicit: precondition the Mhat PCG with the same operator on the
                             material 1/eps, C^{-1} B^H (I3 (x) M^{-1}) B C^{-1}; the stopping
                             test stays ||b - Mhat u|| <= tolCG ||b|| (1).  0: plain CG as the
                             reference's pcg(Mhat, ...) in exp1/make_explicit_krinv_compact.m:43 */
  int passColumns; /* columns per CTA of the inner solves' pass A/C kernels: 0 = built-in default;
                      alternatives 2, 4 (2N = 10), 2, 4 (2N = 8), 4, 6 (2N = 6); other values
                      fall back to the default (fame_b200.autotune picks it per problem) */
  double refineTarget; /* explicit, mixed: the FP64 refinement of each Mhat solve stops once
                          ||bhat - Mhat u|| <= refineTarget * tolCG * ||bhat||, in (0, 1] (0.1).
                          1 is the stopping rule of the reference's pcg (relres <= tolCG); the
                          default stops a decade lower, so that the Lanczos eigenvalues before
                          any Rayleigh-Ritz step stay within tolCG of those of the FP64 form */
} fame_krinv_opts;
FAME_API int fame_krinv_default_opts(fame_krinv_opts* o);
FAME_API int fame_krinv_create(fame_basis* b, fame_mass* m, const fame_krinv_opts* o, fame_krinv** out);
FAME_API int fame_krinv_destroy(fame_krinv* k);
/* y = K_r^{-1} b column by column; b,y complex128 (2NF x ncols) */
FAME_API int fame_krinv_apply(fame_krinv* k, const void* b, void* y, int ncols);
/* Mirrors init_stats of exp1/make_explicit_krinv_compact.m:100-105 and
 * exp1/make_nested_krinv_instrumented.m:154-174 (totals only). */
typedef struct {
  long long inverseCalls;
  long long totalIterations;      /* Mhat PCG (explicit) or outer K_r PCG (nested) */
  long long maxIterations;
  double maxRelativeResidual;
  long long massSolveCalls;       /* nested: inner M solves */
  long long totalMassIterations;  /* nested */
  long long refineSteps;          /* mixed: FP64 refinement steps */
  long long fp32Iterations;       /* mixed: FP32 PCG iterations */
  long long massApplies;          /* scalar-equivalent mass actions */
  double totalInverseSeconds;
} fame_krinv_stats;
FAME_API int fame_krinv_stats_get(fame_krinv* k, fame_krinv_stats* out);
FAME_API int fame_krinv_stats_reset(fame_krinv* k);

/* Eigenvector recovery, exp2/recover_original_eigenvectors_exp2.m:12-50:
 * X(:,j) = M^{-1} V Y(:,j) by PCG on diag(M,M,M) (tol, maxit; FAME_PREC_MIXED uses FP64
 * refinement around FP32 PCG), M-normalised; MX = M X.  Y: 2NF x k, X, MX: 3NF x k
 * (device, complex128).  iterations/relres: host arrays of k (may be NULL). */
FAME_API int fame_recover_eigvecs(fame_basis* b, fame_mass* m, const void* Y, int k, double tol,
                                  int maxit, int prec_mode, void* X, void* MX, int* iterations,
                                  double* relres);
/* exp2/compute_fourier_diagnostics_exp2.m:10-19: original-GEVP residual
 * ||Kx-lam Mx||/(||Kx||+|lam| ||Mx||), divergence ||D0 U0^H Mx||/||Mx||, Rayleigh
 * quotient, for k columns; lambda and the outputs are host arrays of k. */
FAME_API int fame_fourier_diagnostics(fame_basis* b, const void* X, const void* MX,
                                      const double* lambda, int k, double* resGEVP,
                                      double* divRelative2, double* rayleigh);

/* ---- Yee-field reconstruction (complex128 coefficients, FP64) ---- */
/* exp2/reconstruct_field_direct_blocked_exp3.m:8-15: u = exp(i R Q^T) c.
 * coeff: NF; qModes: NF x 3 (column-major); rPoints: M x 3 (column-major); u: M. */
FAME_API int fame_reconstruct_direct(fame_ctx* ctx, const void* coeff, const double* qModes,
                                     long long NF, const double* rPoints, long long M, void* u);
/* The same sum for an axis-block cut matrix P = [diag(d1); diag(d2)] (the basis' P)
 * and points on the tensor grid xs (nx) x ys (ny) x zs (nz), u ordered x fastest
 * (the Yee point order of exp2/build_yee_edge_points_plus.m:11-17): three complex
 * GEMMs against per-axis phase tables.  FAME_ERR_UNSUPPORTED for a dense P. */
FAME_API int fame_reconstruct_direct_grid(fame_basis* b, const void* coeff, const double* xs, int nx,
                                          const double* ys, int ny, const double* zs, int nz,
                                          void* u);
/* (No reference counterpart) the same factorised sum with the three complex GEMMs as
 * split-FP32 (3xTF32) tcgen05 tensor-core products (phase tables and result FP64;
 * relative field error ~2e-6 against fame_reconstruct_direct_grid).  The operands are
 * split once into TF32 head/tail panels held in the context's workspace (about twice
 * the FP64 intermediates: ~0.3 GB at N=5 on a 83^3 window, ~2.5 GB on 403^3). */
FAME_API int fame_reconstruct_direct_grid_3xtf32(fame_basis* b, const void* coeff, const double* xs, int nx,
                                                 const double* ys, int ny, const double* zs, int nz,
                                                 void* u);
/* The factorised direct sum for ncomp (1..3) field components at once: coeff component-
 * stacked (ncomp x NF), xs/ys/zs the components' axes stacked (ncomp x nx, ...; equal sizes,
 * as the three staggered Yee plus-grids have), u component-stacked (ncomp x nx ny nz).  The
 * three GEMMs run as single launches batched over the components (the reference
 * reconstructs the components one after another, exp2/reconstruct_three_components_exp3.m);
 * tensor_cores != 0 runs them as split-FP32 (3xTF32) tcgen05 products. */
FAME_API int fame_reconstruct_direct_grid_fields(fame_basis* b, const void* coeff, int ncomp, const double* xs,
                                                 int nx, const double* ys, int ny, const double* zs, int nz,
                                                 int tensor_cores, void* u);
/* exp2/taylor_on_blocks_exp3.m:8-79 (multi-center Taylor, order p <= 12).  Blocks in
 * CSR form: point indices blockIds[blockPtr[b] .. blockPtr[b+1]) (0-based, device);
 * fixedCenter: host 3-vector or NULL (then each block's bounding-box midpoint). */
FAME_API int fame_taylor_on_blocks(fame_ctx* ctx, const void* coeff, const double* qModes,
                                   long long NF, const double* rPoints, long long M, int p,
                                   const long long* blockPtr, const long long* blockIds,
                                   int nBlocks, const double* fixedCenter, void* u);
/* Same reconstruction with the block moments (the dense contraction over the NF modes) as
   split-FP32 tensor-core products: each FP32 operand is split into TF32 head + tail and the
   moments are head*head + head*tail + tail*head (3xTF32), computed by hand-written tcgen05
   kind::tf32 MMAs on operands generated in shared memory from qModes and coeff (slices of at
   most 512 modes, FP32 accumulation in TMEM) and summed over slices in FP64.  Relative field
   error vs the FP64 form ~2e-6 (the tensor cores' FP32 accumulation sets it).
   No counterpart in the reference (its Taylor moments are FP64 gpuArray products). */
FAME_API int fame_taylor_on_blocks_3xtf32(fame_ctx* ctx, const void* coeff, const double* qModes, long long NF,
                                          const double* rPoints, long long M, int p, const long long* blockPtr,
                                          const long long* blockIds, int nBlocks, const double* fixedCenter,
                                          void* u);

/* ---- mass-operator adjoint (no reference function; eigenvalue gradients) ---- */
/* out[j*nparams + t] = X(:,j)^H (dM/dtheta_t) X(:,j) for the 3-component mass
 * diag(M,M,M) with dM/dtheta_t = fftn(dEps_t .* ifftn(.)): X 3NF x nmodes (device,
 * complex128), dEps NF x nparams (device, real, column-major), out host. */
FAME_API int fame_mass_adjoint(fame_mass* m, const void* X, int nmodes, const double* dEps,
                               int nparams, double* out);

/* ---- restarted Lanczos on K_r^{-1} (exp2/Lanczos.m:1-148, fncB = fncBinv = I) ---- */
typedef struct {
  int steps;      /* total Lanczos steps (iter) */
  int restarts;   /* restart cycles run */
  int converged;  /* nconv >= k */
  int nconv;
  double maxWantedResidual;
} fame_lanczos_info;
/* n = 2NF; theta: host, k values (descending); Y: device n x k complex128 (may be NULL) */
FAME_API int fame_lanczos(fame_krinv* k, int nev, double tol, int maxiter, int p, const void* v0,
                 double* theta, void* Y, fame_lanczos_info* info);

/* (No reference counterpart; the reference reports lambda = 1/theta of the Lanczos Ritz
 * values, exp2/Lanczos.m:140-147, whose error follows the inner tolerance of K_r^{-1}.)
 * Rayleigh-Ritz refinement of k (1..32) approximate eigenvectors Y (device, 2NF x k,
 * complex128, e.g. the Y of fame_lanczos) with the exact K_r = V^* M^{-1} V: on the (2N)^6
 * grid M^{-1} is the mass chain on the material 1/eps, so K_r applies to rounding error.
 * Solves Y^H K_r Y u = lambda Y^H Y u, overwrites Y with the refined vectors (Y u) and
 * returns lambda (host, k, ascending) and, if relres is not NULL, ||K_r y - lambda y|| /
 * ||K_r y|| per refined vector (host, k).  The eigenvalue error is quadratic in the
 * eigenvector error of the input. */
FAME_API int fame_rayleigh_ritz(fame_basis* b, fame_mass* m, void* Y, int k, double* lambda, double* relres);

/* ---- Method A: original shift-invert without the null-space-free basis ----
 * exp1/build_experiment1_q_system_A_only.m, exp1/build_original_shift_preconditioner_A_only.m,
 * exp1/make_A_eigs_top_preconditioned.m, exp1/run_method_A_fig1a.m.  The operator of the
 * reference's eigs call, T x = (K - sigma M)^{-1} M x on 3NF vectors (components stacked,
 * natural order), with K the per-mode symbol |q|^2 I - q q^T and the shifted system solved
 * by preconditioned MINRES (preconditioner (K + tau I)^{-1}, exact per mode; the reference
 * uses tau = sigma * mean(eps)); the basis handle supplies q (its V blocks are unused). */
typedef struct fame_osi fame_osi;
typedef struct fame_osi_stats {
  long long topApplications;  /* shifted solves (one per T application) */
  long long minresIterations; /* all MINRES iterations, correction cycles included */
  long long cycles;           /* MINRES cycles (1 + residual corrections per solve) */
  double maxTrueRelres;       /* largest final ||b - A x|| / ||b|| */
  int failures;               /* solves that missed the tolerance and the plateau ceiling */
  int plateauAccepts;         /* solves whose residual stalled between the tolerance and 1e-9 */
} fame_osi_stats;
FAME_API int fame_osi_create(fame_basis* b, fame_mass* m, double sigma, double tau, double tolMinres,
                             int maxitMinres, fame_osi** out);
FAME_API int fame_osi_destroy(fame_osi* A);
/* y = T x for ncols 3NF columns. */
FAME_API int fame_osi_apply(fame_osi* A, const void* x, void* y, int ncols);
/* The nev eigenvalues of K x = lambda M x above the shift closest to it (the largest
 * theta of T; lambda = sigma + 1/theta, ascending) by the restarted Lanczos on the
 * Hermitian M^(1/2) (K - sigma M)^{-1} M^(1/2); X (3NF x nev, optional) M-normalised. */
FAME_API int fame_osi_eigs(fame_osi* A, int nev, double tol, int maxiter, int p, const void* v0,
                           double* lambda, void* X, fame_lanczos_info* info);
FAME_API int fame_osi_stats_get(fame_osi* A, fame_osi_stats* out);
/* exp1/build_experiment1_q_system_A_only.m:61-73 (applyK): y = K x, ncols 3NF columns. */
FAME_API int fame_apply_K_original(fame_basis* b, const void* x, void* y, int ncols);

/* Batched Bloch path: solve `count` independent instances (N[i], eps E[i] on the
 * (2N_i)^6 grid (device), Bloch vector q[3i..3i+2]) for their nev largest theta of
 * K_r^{-1}, concurrently on one device (one context, stream and host thread per
 * instance).  theta: host count x nev; info, status: host arrays of count (may be
 * NULL).  The reference solves Bloch points sequentially (exp4/run_exp4_medium.m:37-109).
 * Returns the first failing instance's status. */
FAME_API int fame_solve_batch(int device, int count, const int* N, const double* const* E,
                              const double* q, const double* P, const fame_krinv_opts* o, int nev,
                              double tol, int maxiter, int p, unsigned long long seed,
                              double* theta, fame_lanczos_info* info, int* status);
/* (No reference counterpart) the same with one K_r^{-1} options struct per instance
 * (opts: count entries), e.g. the launch schedule and pass tile shape the autotuner
 * chose for each instance's N. */
FAME_API int fame_solve_batch_each(int device, int count, const int* N, const double* const* E,
                                   const double* q, const double* P, const fame_krinv_opts* opts, int nev,
                                   double tol, int maxiter, int p, unsigned long long seed,
                                   double* theta, fame_lanczos_info* info, int* status);
/* Start vector of the shared counter-based generator (complex128, device). */
FAME_API int fame_start_vector(fame_ctx* ctx, unsigned long long seed, long long n, void* v);

#ifdef __cplusplus
}
#endif
#endif /* FAME_H */
