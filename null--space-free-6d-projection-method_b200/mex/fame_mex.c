/*
 * fame_mex.c -- MATLAB gateway to libfame_b200.so (include/fame.h) for the reference's
 * hot-path functions.  Complex data cross as interleaved complex gpuArrays (the layout of
 * double2 / float2), so no copies are made: device pointers go straight to the C ABI.
 *
 * Build (MATLAB R2018a or later with the Parallel Computing Toolbox, interleaved complex API):
 *   mex -R2018a fame_mex.c -I<repo>/include -L<repo>/null--space-free-6d-projection-method_b200/fame_b200 \
 *       -lfame_b200 -lcudart -lmwgpu
 *
 * Usage (the .m wrappers in this folder keep the reference signatures):
 *   h = fame_mex('mass_create', N, E)                 E: real gpuArray, (2N)^6
 *   y = fame_mex('mass_apply', h, mode, x)           mode 0..3 = MscalarOp / Mop / Mcol3op / Mcols12op
 *   y = fame_mex('applyMij_fft', x, E, N)
 *   b = fame_mex('basis_create', N, P, q)            P: 6x3 double, q: 3 doubles (host)
 *   k = fame_mex('krinv_create', b, h, kind, opts)   kind 0 explicit / 1 nested; opts struct (fame_krinv_opts names)
 *   y = fame_mex('krinv_apply', k, q)                q: 2NF x ncols complex gpuArray
 *   s = fame_mex('krinv_stats', k)                   struct with the init_stats totals
 *   [ev, ew, iter, info] = fame_mex('lanczos', k, nev, tol, maxiter, p, v0)
 *   [lambda, relres] = fame_mex('rayleigh_ritz', b, h, Y)   Y refined in place (returned as 3rd output)
 *   X = fame_mex('rank1_exact_fft_scatter', x, plan)  plan: struct with M, NF, inputIdx (uint32, 1-based)
 *   y = fame_mex('rank1_exact_ifft_gather', Y, plan)  plan: struct with M, NF, targetIdx
 *   fame_mex('destroy', handle)                      any handle made above
 * Handles are uint64 scalars; all work is ordered on the legacy default stream (as MATLAB's
 * GPU operations) and synchronised before the gateway returns.
 */
#include <stdint.h>
#include <string.h>
#include "mex.h"
#include "gpu/mxGPUArray.h"
#include "fame.h"

enum { H_MASS = 1, H_BASIS = 2, H_KRINV = 3 };
typedef struct {
  int kind;
  void* p;
} handle_t;

static fame_ctx* g_ctx = NULL;

/* Map a status to the reference's error identifiers (exp2/make_krinv_instrumented.m:38-77,
 * exp1/rank1_exact_fft_scatter.m:5-7, exp1/assemble_K_and_nullspace_free_basis.m:36-42). */
static void check(int st) {
  const char* id = "fame:CUDA";
  if (st == FAME_OK) return;
  switch (st) {
    case FAME_ERR_INVALID: id = "fame:BadSize"; break;
    case FAME_ERR_NOT_CONVERGED: id = "make_krinv_instrumented:InnerCGFailure"; break;
    case FAME_ERR_NONFINITE: id = "make_krinv_instrumented:NonFiniteInput"; break;
    case FAME_ERR_SINGULAR: id = "assemble_K_and_nullspace_free_basis:SingularQ"; break;
    case FAME_ERR_OOM: id = "fame:OutOfMemory"; break;
    case FAME_ERR_BUDGET: id = "EXP1:IterationLimit"; break;
    case FAME_ERR_BREAKDOWN: id = "Lanczos:Breakdown"; break;
    default: break;
  }
  mexErrMsgIdAndTxt(id, "%s: %s", fame_status_string(st), fame_last_error());
}

static void cleanup(void) {
  if (g_ctx) fame_ctx_destroy(g_ctx);
  g_ctx = NULL;
}

static fame_ctx* ctx(void) {
  if (!g_ctx) {
    int dev = 0;
    mxInitGPU();
    check(fame_ctx_create(dev, &g_ctx));
    check(fame_ctx_set_stream(g_ctx, NULL));  /* legacy default stream */
    mexAtExit(cleanup);
  }
  return g_ctx;
}

static mxArray* wrap(int kind, void* p) {
  handle_t* h = (handle_t*)mxMalloc(sizeof(handle_t));
  mxArray* out = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
  mexMakeMemoryPersistent(h);
  h->kind = kind;
  h->p = p;
  *(uint64_t*)mxGetData(out) = (uint64_t)(uintptr_t)h;
  return out;
}

static handle_t* unwrap(const mxArray* a, int kind) {
  handle_t* h;
  if (!mxIsUint64(a) || mxGetNumberOfElements(a) != 1) mexErrMsgIdAndTxt("fame:BadHandle", "expected a handle");
  h = (handle_t*)(uintptr_t)(*(uint64_t*)mxGetData(a));
  if (!h || (kind && h->kind != kind)) mexErrMsgIdAndTxt("fame:BadHandle", "wrong handle kind");
  return h;
}

/* A complex double (or single) gpuArray: its device pointer, rows and columns. */
static const mxGPUArray* gpu_in(const mxArray* a, mxClassID cls, mxComplexity cx, const void** ptr,
                                 mwSize* rows, mwSize* cols) {
  const mxGPUArray* g = mxGPUCreateFromMxArray(a);
  const mwSize* d = mxGPUGetDimensions(g);
  if (mxGPUGetClassID(g) != cls || mxGPUGetComplexity(g) != cx)
    mexErrMsgIdAndTxt("fame:BadSize", "unexpected class or complexity of a gpuArray input");
  *ptr = mxGPUGetDataReadOnly(g);
  *rows = d[0];
  *cols = mxGPUGetNumberOfDimensions(g) > 1 ? mxGPUGetNumberOfElements(g) / d[0] : 1;
  return g;
}

static mxGPUArray* gpu_out(mwSize rows, mwSize cols, mxClassID cls, void** ptr) {
  mwSize dims[2];
  mxGPUArray* g;
  dims[0] = rows;
  dims[1] = cols;
  g = mxGPUCreateGPUArray(2, dims, cls, mxCOMPLEX, MX_GPU_DoNotInitialize);
  *ptr = mxGPUGetData(g);
  return g;
}

static double field_or(const mxArray* s, const char* name, double dflt) {
  const mxArray* f = s ? mxGetField(s, 0, name) : NULL;
  return f ? mxGetScalar(f) : dflt;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  char cmd[64];
  if (nrhs < 1 || mxGetString(prhs[0], cmd, sizeof(cmd))) mexErrMsgIdAndTxt("fame:Usage", "fame_mex('command', ...)");
  (void)ctx();

  if (!strcmp(cmd, "mass_create")) { /* build_mass_backend_large_scalar.m:27-46 */
    const void* E;
    mwSize r, c;
    fame_mass* m = NULL;
    const mxGPUArray* gE = gpu_in(prhs[2], mxDOUBLE_CLASS, mxREAL, &E, &r, &c);
    check(fame_mass_create(ctx(), (int)mxGetScalar(prhs[1]), (const double*)E, &m));
    check(fame_ctx_sync(ctx()));
    mxGPUDestroyGPUArray(gE);
    plhs[0] = wrap(H_MASS, m);
  } else if (!strcmp(cmd, "mass_apply")) { /* mass.MscalarOp / Mop / Mcol3op / Mcols12op */
    handle_t* h = unwrap(prhs[1], H_MASS);
    const int mode = (int)mxGetScalar(prhs[2]);
    const mxGPUArray* probe = mxGPUCreateFromMxArray(prhs[3]);
    const int single = mxGPUGetClassID(probe) == mxSINGLE_CLASS;  /* complex64 input: the FP32 operator */
    const mxClassID cls = single ? mxSINGLE_CLASS : mxDOUBLE_CLASS;
    const void* x;
    void* y;
    mwSize r, c, rows_out;
    const mxGPUArray* gx;
    mxGPUArray* gy;
    mxGPUDestroyGPUArray(probe);
    gx = gpu_in(prhs[3], cls, mxCOMPLEX, &x, &r, &c);
    rows_out = (mode == FAME_MASS_SCALAR) ? r : (mode == FAME_MASS_FULL3 ? r : (mode == FAME_MASS_COL3 ? 3 * r : 3 * r / 2));
    gy = gpu_out(rows_out, c, cls, &y);
    check(fame_mass_apply((fame_mass*)h->p, mode, x, y, (int)c, single ? FAME_F32 : FAME_F64));
    check(fame_ctx_sync(ctx()));
    plhs[0] = mxGPUCreateMxArrayOnGPU(gy);
    mxGPUDestroyGPUArray(gx);
    mxGPUDestroyGPUArray(gy);
  } else if (!strcmp(cmd, "applyMij_fft")) { /* exp1/applyMij_fft.m:1-24 */
    const void *x, *E;
    void* y;
    mwSize r, c, re, ce;
    const mxGPUArray* gx = gpu_in(prhs[1], mxDOUBLE_CLASS, mxCOMPLEX, &x, &r, &c);
    const mxGPUArray* gE = gpu_in(prhs[2], mxDOUBLE_CLASS, mxREAL, &E, &re, &ce);
    mxGPUArray* gy = gpu_out(r, c, mxDOUBLE_CLASS, &y);
    check(fame_applyMij_fft(ctx(), (int)mxGetScalar(prhs[3]), (const double*)E, x, y, (int)c, FAME_F64));
    check(fame_ctx_sync(ctx()));
    plhs[0] = mxGPUCreateMxArrayOnGPU(gy);
    mxGPUDestroyGPUArray(gx);
    mxGPUDestroyGPUArray(gE);
    mxGPUDestroyGPUArray(gy);
  } else if (!strcmp(cmd, "basis_create")) { /* build_experiment1_q_system.m:4-24 */
    fame_basis* b = NULL;
    if (mxGetNumberOfElements(prhs[2]) != 18 || mxGetNumberOfElements(prhs[3]) != 3)
      mexErrMsgIdAndTxt("fame:BadSize", "P must be 6x3 and q must have 3 entries");
    check(fame_basis_create(ctx(), (int)mxGetScalar(prhs[1]), mxGetDoubles(prhs[2]), mxGetDoubles(prhs[3]), &b));
    check(fame_ctx_sync(ctx()));
    plhs[0] = wrap(H_BASIS, b);
  } else if (!strcmp(cmd, "krinv_create")) { /* make_explicit_krinv_compact.m / make_nested_krinv_instrumented.m */
    handle_t* b = unwrap(prhs[1], H_BASIS);
    handle_t* m = unwrap(prhs[2], H_MASS);
    const mxArray* o = nrhs > 4 ? prhs[4] : NULL;
    fame_krinv_opts opts;
    fame_krinv* k = NULL;
    check(fame_krinv_default_opts(&opts));
    opts.kind = (int)mxGetScalar(prhs[3]);
    opts.prec_mode = (int)field_or(o, "prec_mode", opts.prec_mode);
    opts.tolCG = field_or(o, "tolCG", opts.tolCG);
    opts.maxitCG = (int)field_or(o, "maxitCG", opts.maxitCG);
    opts.tolKr = field_or(o, "tolKr", opts.tolKr);
    opts.tolM = field_or(o, "tolM", opts.tolM);
    opts.maxitKr = (int)field_or(o, "maxitKr", opts.maxitKr);
    opts.maxitM = (int)field_or(o, "maxitM", opts.maxitM);
    opts.epsC = field_or(o, "epsC", opts.epsC);
    opts.useKrPreconditioner = (int)field_or(o, "useKrPreconditioner", opts.useKrPreconditioner);
    opts.mhatPreconditioner = (int)field_or(o, "mhatPreconditioner", opts.mhatPreconditioner);
    opts.refineTarget = field_or(o, "refineTarget", opts.refineTarget);
    check(fame_krinv_create((fame_basis*)b->p, (fame_mass*)m->p, &opts, &k));
    plhs[0] = wrap(H_KRINV, k);
  } else if (!strcmp(cmd, "krinv_apply")) { /* KrInvOp(q) */
    handle_t* k = unwrap(prhs[1], H_KRINV);
    const void* q;
    void* y;
    mwSize r, c;
    const mxGPUArray* gq = gpu_in(prhs[2], mxDOUBLE_CLASS, mxCOMPLEX, &q, &r, &c);
    mxGPUArray* gy = gpu_out(r, c, mxDOUBLE_CLASS, &y);
    check(fame_krinv_apply((fame_krinv*)k->p, q, y, (int)c));
    check(fame_ctx_sync(ctx()));
    plhs[0] = mxGPUCreateMxArrayOnGPU(gy);
    mxGPUDestroyGPUArray(gq);
    mxGPUDestroyGPUArray(gy);
  } else if (!strcmp(cmd, "krinv_stats")) { /* getStats(): init_stats field names */
    static const char* names[] = {"inverseCalls", "totalMhatIterations", "maxMhatIterations", "maxMhatRelativeResidual",
                                  "massSolveCalls", "totalMassIterations", "refineSteps", "fp32Iterations",
                                  "totalInverseTime", "averageMhatIterations"};
    handle_t* k = unwrap(prhs[1], H_KRINV);
    fame_krinv_stats s;
    mxArray* out = mxCreateStructMatrix(1, 1, 10, names);
    check(fame_krinv_stats_get((fame_krinv*)k->p, &s));
    mxSetField(out, 0, "inverseCalls", mxCreateDoubleScalar((double)s.inverseCalls));
    mxSetField(out, 0, "totalMhatIterations", mxCreateDoubleScalar((double)s.totalIterations));
    mxSetField(out, 0, "maxMhatIterations", mxCreateDoubleScalar((double)s.maxIterations));
    mxSetField(out, 0, "maxMhatRelativeResidual", mxCreateDoubleScalar(s.maxRelativeResidual));
    mxSetField(out, 0, "massSolveCalls", mxCreateDoubleScalar((double)s.massSolveCalls));
    mxSetField(out, 0, "totalMassIterations", mxCreateDoubleScalar((double)s.totalMassIterations));
    mxSetField(out, 0, "refineSteps", mxCreateDoubleScalar((double)s.refineSteps));
    mxSetField(out, 0, "fp32Iterations", mxCreateDoubleScalar((double)s.fp32Iterations));
    mxSetField(out, 0, "totalInverseTime", mxCreateDoubleScalar(s.totalInverseSeconds));
    mxSetField(out, 0, "averageMhatIterations",
               mxCreateDoubleScalar(s.inverseCalls ? (double)s.totalIterations / (double)s.inverseCalls : mxGetNaN()));
    plhs[0] = out;
  } else if (!strcmp(cmd, "lanczos")) { /* exp2/Lanczos.m with fncA = KrInvOp, fncB = fncBinv = I */
    handle_t* k = unwrap(prhs[1], H_KRINV);
    const int nev = (int)mxGetScalar(prhs[2]);
    const void* v0;
    void* Y;
    mwSize r, c;
    fame_lanczos_info info;
    static const char* inames[] = {"steps", "restarts", "converged", "nconv", "maxWantedResidual"};
    const mxGPUArray* gv = gpu_in(prhs[6], mxDOUBLE_CLASS, mxCOMPLEX, &v0, &r, &c);
    mxGPUArray* gY = gpu_out(r, (mwSize)nev, mxDOUBLE_CLASS, &Y);
    mxArray* ew = mxCreateDoubleMatrix((mwSize)nev, 1, mxREAL);
    mxArray* inf = mxCreateStructMatrix(1, 1, 5, inames);
    check(fame_lanczos((fame_krinv*)k->p, nev, mxGetScalar(prhs[3]), (int)mxGetScalar(prhs[4]),
                       (int)mxGetScalar(prhs[5]), v0, mxGetDoubles(ew), Y, &info));
    check(fame_ctx_sync(ctx()));
    mxSetField(inf, 0, "steps", mxCreateDoubleScalar(info.steps));
    mxSetField(inf, 0, "restarts", mxCreateDoubleScalar(info.restarts));
    mxSetField(inf, 0, "converged", mxCreateLogicalScalar(info.converged != 0));
    mxSetField(inf, 0, "nconv", mxCreateDoubleScalar(info.nconv));
    mxSetField(inf, 0, "maxWantedResidual", mxCreateDoubleScalar(info.maxWantedResidual));
    plhs[0] = mxGPUCreateMxArrayOnGPU(gY);
    plhs[1] = ew;
    if (nlhs > 2) plhs[2] = mxCreateDoubleScalar(info.steps);
    if (nlhs > 3) plhs[3] = inf;
    else mxDestroyArray(inf);
    mxGPUDestroyGPUArray(gv);
    mxGPUDestroyGPUArray(gY);
  } else if (!strcmp(cmd, "rayleigh_ritz")) { /* no reference counterpart */
    handle_t* b = unwrap(prhs[1], H_BASIS);
    handle_t* m = unwrap(prhs[2], H_MASS);
    mxGPUArray* gY = mxGPUCopyFromMxArray(prhs[3]);
    const mwSize* d = mxGPUGetDimensions(gY);
    const int k = mxGPUGetNumberOfDimensions(gY) > 1 ? (int)d[1] : 1;
    mxArray* lam = mxCreateDoubleMatrix((mwSize)k, 1, mxREAL);
    mxArray* rel = mxCreateDoubleMatrix((mwSize)k, 1, mxREAL);
    check(fame_rayleigh_ritz((fame_basis*)b->p, (fame_mass*)m->p, mxGPUGetData(gY), k, mxGetDoubles(lam),
                             mxGetDoubles(rel)));
    check(fame_ctx_sync(ctx()));
    plhs[0] = lam;
    if (nlhs > 1) plhs[1] = rel;
    else mxDestroyArray(rel);
    if (nlhs > 2) plhs[2] = mxGPUCreateMxArrayOnGPU(gY);
    mxGPUDestroyGPUArray(gY);
  } else if (!strcmp(cmd, "rank1_exact_fft_scatter") || !strcmp(cmd, "rank1_exact_ifft_gather")) {
    /* exp1/rank1_exact_fft_scatter.m:1-13, exp1/rank1_exact_ifft_gather.m:1-11 */
    const int scatter = !strcmp(cmd, "rank1_exact_fft_scatter");
    const mxArray* plan = prhs[2];
    const mxArray* fi = mxGetField(plan, 0, scatter ? "inputIdx" : "targetIdx");
    const long long M = (long long)field_or(plan, "M", -1), NF = (long long)field_or(plan, "NF", -1);
    const void *x, *idx;
    void* y;
    mwSize r, c;
    const mxGPUArray* gx = gpu_in(prhs[1], mxDOUBLE_CLASS, mxCOMPLEX, &x, &r, &c);
    const mxGPUArray* gi;
    mxGPUArray* gy;
    if (!fi || M <= 0 || NF <= 0) mexErrMsgIdAndTxt("fame:BadPlan", "plan needs M, NF and the index vector");
    if ((long long)r != (scatter ? NF : M))
      mexErrMsgIdAndTxt(scatter ? "rank1_exact_fft_scatter:BadSize" : "rank1_exact_ifft_gather:BadSize",
                        scatter ? "x must have plan.NF rows." : "Yfft must have plan.M rows.");
    gi = mxGPUCreateFromMxArray(fi);  /* a host index vector is copied to the device */
    if (mxGPUGetClassID(gi) != mxUINT32_CLASS || (long long)mxGPUGetNumberOfElements(gi) != NF)
      mexErrMsgIdAndTxt("fame:BadPlan", "the plan's index vector must be uint32 with NF entries");
    idx = mxGPUGetDataReadOnly(gi);
    gy = gpu_out((mwSize)(scatter ? M : NF), c, mxDOUBLE_CLASS, &y);
    if (scatter)
      check(fame_rank1_exact_fft_scatter(ctx(), x, (int)c, (const uint32_t*)idx, NF, M, y));
    else
      check(fame_rank1_exact_ifft_gather(ctx(), x, (int)c, (const uint32_t*)idx, NF, M, y));
    check(fame_ctx_sync(ctx()));
    plhs[0] = mxGPUCreateMxArrayOnGPU(gy);
    mxGPUDestroyGPUArray(gx);
    mxGPUDestroyGPUArray(gi);
    mxGPUDestroyGPUArray(gy);
  } else if (!strcmp(cmd, "destroy")) {
    handle_t* h = unwrap(prhs[1], 0);
    check(fame_ctx_sync(ctx()));
    if (h->kind == H_MASS) fame_mass_destroy((fame_mass*)h->p);
    if (h->kind == H_BASIS) fame_basis_destroy((fame_basis*)h->p);
    if (h->kind == H_KRINV) fame_krinv_destroy((fame_krinv*)h->p);
    h->p = NULL;
    h->kind = 0;
    mxFree(h);
  } else {
    mexErrMsgIdAndTxt("fame:Usage", "unknown command '%s'", cmd);
  }
}
