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

/* ---- context (replaces gpu_initialize / wait_for_gpu: exp1/wait_for_gpu.m:5-11) ---- */
FAME_API int fame_ctx_create(int device, fame_ctx** out);
FAME_API int fame_ctx_destroy(fame_ctx* ctx);
/* stream: a cudaStream_t (NULL = the context's own stream) */
FAME_API int fame_ctx_set_stream(fame_ctx* ctx, void* stream);
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

/* Replaces applyMij_rank1_exact(x,kernelFFT,plan) — exp1/applyMij_rank1_exact.m:1-6
 * with rank1_exact_fft_scatter / rank1_exact_ifft_gather
 * (exp1/rank1_exact_fft_scatter.m:1-13, exp1/rank1_exact_ifft_gather.m:1-11).
 * inputIdx/targetIdx are the plan's 1-based uint32 code vectors (device, NF each) of
 * exp1/build_radix_exact_rank1_plan_scalar.m:57-58 and M the plan length.  The plan is
 * verified against the radix construction (FAME_ERR_INVALID if it is not that plan);
 * the action is the algebraically identical 6D convolution. */
FAME_API int fame_applyMij_rank1_exact(fame_mass* m, const uint32_t* inputIdx, const uint32_t* targetIdx,
                              long long M, const void* x, void* y, int nrhs);

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
  double tolInner32; /* mixed: relative tolerance of each FP32 correction solve (1e-5) */
  int maxRefine;     /* mixed: max FP64 refinement steps per solve (20) */
  int checkEvery;    /* PCG iterations queued between host convergence checks (8) */
  int verifyTrueResidual; /* confirm convergence on the true residual, as MATLAB pcg (1) */
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
/* Start vector of the shared counter-based generator (complex128, device). */
FAME_API int fame_start_vector(fame_ctx* ctx, unsigned long long seed, long long n, void* v);

#ifdef __cplusplus
}
#endif
#endif /* FAME_H */
