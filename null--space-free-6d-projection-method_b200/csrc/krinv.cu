// K_r^{-1} actions.
//  explicit (method C), exp1/make_explicit_krinv_compact.m:24-80:
//    r = V1^{-*} q;  mr_c = M r_c;  bhat = -C^{-1}(W1^* mr1 + W2^* mr2)
//    u = PCG(Mhat, bhat);  z = C^{-1} u;  y = V1^{-1}[mr1 + M(W1 z); mr2 + M(W2 z)]
//  Each bracketed line is one fused pass-A/B/C chain; PCG scalars stay on the
//  device.  FAME_PREC_MIXED solves Mhat u = bhat by FP64 iterative refinement
//  whose corrections come from an FP32 (complex64) PCG on an FP32 mass operator.
//  nested (method B), exp1/make_nested_krinv_instrumented.m:33-126: see nested.cu.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include "internal.cuh"
#include "krinv_impl.cuh"

namespace fame {

// pre chain: fields r1, r2 of r = V1^{-*} q (q, V, det in natural order)
struct ProKrPre {
  static constexpr bool natural = true;
  const double2* q;
  const double2 *V11, *V12, *V21, *V22, *det;
  long long NF;
  __device__ __forceinline__ void load(long long, long long i, double2* v) const {
    const double2 q1 = q[i], q2 = q[NF + i];
    const double2 d = cconj<double>(det[i]);
    v[0] = cdiv<double>(csub<double>(cmulc<double>(V22[i], q1), cmulc<double>(V21[i], q2)), d);
    v[1] = cdiv<double>(csub<double>(cmulc<double>(V11[i], q2), cmulc<double>(V12[i], q1)), d);
  }
};
// keep mr1, mr2; form bhat (= PCG rhs b and initial residual r), x = 0, PCG state
// (all line order)
struct EpiKrPre {
  using Acc = double;
  static constexpr int K = 1;
  MhatCoef<double> c;
  double2 *mr1, *mr2, *b, *r, *x;
  PcgState* st;
  double tol;
  int maxit;
  double* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long i, long long, const double2* v, Red<double, 1>& acc) const {
    mr1[i] = v[0];
    mr2[i] = v[1];
    const double2 s = cadd<double>(cmulc<double>(c.W1[i], v[0]), cmulc<double>(c.W2[i], v[1]));
    const double2 bb = cscale<double>(s, -c.invC[i]);
    b[i] = bb;
    r[i] = bb;
    x[i] = make_double2(0.0, 0.0);
    acc.v[0] += cabs2<double>(bb);
  }
  __device__ __forceinline__ void finalize(const Red<double, 1>& tot) const {
    pcg_init_state(st, tot.v[0], tol, maxit);
  }
};
// post chain: fields W1 z, W2 z with z = C^{-1} u
struct ProKrPost {
  MhatCoef<double> c;
  const double2* u;
  __device__ __forceinline__ void load(long long i, long long, double2* v) const {
    const double2 z = cscale<double>(u[i], c.invC[i]);
    v[0] = cmul<double>(c.W1[i], z);
    v[1] = cmul<double>(c.W2[i], z);
  }
};
// y = V1^{-1}[mr1 + M W1 z; mr2 + M W2 z] (y, V, det natural; mr line order);
// counts non-finite outputs into st->aux
struct EpiKrPost {
  using Acc = double;
  static constexpr int K = 1;
  static constexpr bool natural = true;
  const double2 *mr1, *mr2, *V11, *V12, *V21, *V22, *det;
  double2* y;
  long long NF;
  PcgState* st;
  double* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long ia, long long i, const double2* v, Red<double, 1>& acc) const {
    const double2 t1 = cadd<double>(mr1[ia], v[0]), t2 = cadd<double>(mr2[ia], v[1]);
    const double2 d = det[i];
    const double2 y1 = cdiv<double>(csub<double>(cmul<double>(V22[i], t1), cmul<double>(V12[i], t2)), d);
    const double2 y2 = cdiv<double>(csub<double>(cmul<double>(V11[i], t2), cmul<double>(V21[i], t1)), d);
    y[i] = y1;
    y[NF + i] = y2;
    const bool bad = !(isfinite(y1.x) && isfinite(y1.y) && isfinite(y2.x) && isfinite(y2.y));
    acc.v[0] += bad ? 1.0 : 0.0;
  }
  __device__ __forceinline__ void finalize(const Red<double, 1>& tot) const { st->aux = tot.v[0]; }
};

__global__ void k_zero_c(double2* x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = make_double2(0.0, 0.0);
}

template <> MhatCoef<double> coef_of<double>(fame_basis* b) { return MhatCoef<double>{b->invC, b->W1, b->W2}; }
template <> MhatCoef<float> coef_of<float>(fame_basis* b) { return MhatCoef<float>{b->invCf, b->W1f, b->W2f}; }
template <> MhatCoef<double> coef_line_of<double>(fame_basis* b) { return MhatCoef<double>{b->invC_l, b->W1_l, b->W2_l}; }
template <> MhatCoef<float> coef_line_of<float>(fame_basis* b) { return MhatCoef<float>{b->invCf_l, b->W1f_l, b->W2f_l}; }
template <> const double* es_of<double>(fame_mass* m) { return m->Et64; }
template <> const float* es_of<float>(fame_mass* m) { return m->Et32; }

// NaN/Inf test of the last explicit K_r^{-1} output (the post chain's count in aux).
int krinv_output_check(fame_krinv* K) {
  if (K->o.kind != FAME_KRINV_EXPLICIT) return FAME_OK;
  PcgState h{};
  FAME_TRY(read_back(K->ctx, K->st64, &h, sizeof(PcgState)));
  if (h.aux != 0.0) return fail(FAME_ERR_NONFINITE, "Explicit K_r^{-1} output contains NaN/Inf");
  return FAME_OK;
}

int krinv_explicit_apply_one(fame_krinv* K, const double2* q, double2* y) {
  fame_basis* bs = K->b;
  cudaStream_t s = K->ctx->stream;
  const long long NF = K->NF;
  const MhatCoef<double> c64 = coef_line_of<double>(bs);
  PcgBuf<double>& B = K->b64;
  PcgState* st = K->st64;
  const double tolMhat = K->o.tolCG;
  // ---- pre: r = V1^{-*} q ; mr = M r ; bhat ; PCG / refinement init
  {
    ProKrPre pro{q, bs->V1(0, 0), bs->V1(0, 1), bs->V1(1, 0), bs->V1(1, 1), bs->det, NF};
    EpiKrPre epi{c64, K->mr1, K->mr2, K->bhat, B.r, B.x, st, tolMhat,
                 K->o.prec_mode == FAME_PREC_MIXED ? K->o.maxRefine : K->o.maxitCG,
                 K->partials, K->counter};
    FAME_TRY((run_chain<double, 2>(K->n, pro, epi, B.work, K->m->Et64, NF, s)));
    K->stats.massApplies += 2;
  }
  PcgState h{};
  double relres = 0.0;
  int iters = 0;
  if (K->o.prec_mode == FAME_PREC_FP64) {
    if (K->o.mhatPreconditioner) {
      FAME_TRY(pcg_iterate<double>(K, OpMhatPre<double>{coef_line_of<double>(bs), es_of<double>(K->m), K->m->EtInv64},
                                   B, st, K->lastIt64, h, K->o.verifyTrueResidual != 0, K->bhat));
    } else {
      FAME_TRY(pcg_iterate<double>(K, OpMhat<double>{coef_line_of<double>(bs), es_of<double>(K->m)}, B, st,
                                   K->lastIt64, h, K->o.verifyTrueResidual != 0, K->bhat));
    }
    if (h.flag == -1) return fail(FAME_ERR_NONFINITE, "Mhat right-hand side contains NaN/Inf");
    iters = h.iter;
    relres = h.bnorm2 > 0 ? std::sqrt(h.rho / h.bnorm2) : 0.0;
    if (h.flag != 0 && relres > 10 * tolMhat)
      return fail(FAME_ERR_NOT_CONVERGED, "Mhat CG failed: flag=" + std::to_string(h.flag) +
                                              " relres=" + std::to_string(relres) +
                                              " iter=" + std::to_string(h.iter));
  } else {
    // FP64 iterative refinement: u (=B.x, zero) ; r64 (=B.r) = bhat.  The first two
    // rounds always run, so ||bhat||^2 is read with the second round's residual instead
    // of here (a zero bhat gives converged FP32 solves and a zero residual; NaN/Inf in
    // bhat reaches the FP32 solve's initial norm).
    double bn2 = 1.0, rn2 = 1.0;
    bool first = true;
    PcgBuf<float>& F = K->b32;
    PcgState* st32 = K->st32;
    float* partials32 = reinterpret_cast<float*>(K->partials);
    const MhatCoef<double> c = c64;
    int refine = 0;
    // refine to refineTarget*tolCG: at 1 the reference's pcg rule (relres <= tolCG); the
    // FP32 corrections leave no FP64-PCG overshoot below it, so the default of 0.1 keeps
    // the Lanczos eigenvalues within tolCG of the FP64 form's before any Rayleigh-Ritz step
    const double tolIR = K->o.refineTarget * tolMhat;
    while (first || (rn2 > tolIR * tolIR * bn2 && bn2 > 0)) {
      if (refine >= K->o.maxRefine) break;
      ++refine;
      first = false;
      // a round needs only the reduction that takes the residual to the target: the FP32
      // solve is asked for half of it, never for less than tolInner32 (its accuracy floor);
      // k_pcg_init takes it on the device from the FP64 state (residual and ||bhat||)
      // the first chunk of queued iterations is sized from this round of the previous call
      int& hint = K->lastIt32Round[std::min(refine, kRoundHints) - 1];
      k_pcg_init<float, double><<<vec_blocks(NF), 256, 0, s>>>(B.r, F.r, F.x, NF, st32,
                                                              K->o.tolInner32, K->o.maxitCG,
                                                              partials32, K->counter, st, tolIR);
      ::fame::count_launch();
      PcgState h32{};
      if (K->o.mhatPreconditioner) {
        FAME_TRY(pcg_iterate<float>(K, OpMhatPre<float>{coef_line_of<float>(bs), es_of<float>(K->m), K->m->EtInv32},
                                    F, st32, hint, h32, false, nullptr, true));
      } else {
        FAME_TRY(pcg_iterate<float>(K, OpMhat<float>{coef_line_of<float>(bs), es_of<float>(K->m)}, F, st32,
                                    hint, h32, false, nullptr, true));
      }
      if (h32.flag == -1) return fail(FAME_ERR_NONFINITE, "Mhat right-hand side contains NaN/Inf");
      if (h32.flag == 4) return fail(FAME_ERR_NOT_CONVERGED, "FP32 correction solve broke down");
      K->stats.fp32Iterations += h32.iter;
      iters += h32.iter;
      // u += dx ; r64 = bhat - Mhat u  (FP64 residual); the FP32 solve's last update of
      // dx is still pending and is applied here (the FP32 residual is not needed again)
      ProResidMhat<double, float, true> pro{c, B.x, F.x, F.p, st32};
      EpiResidMhat<double> epi{c, K->bhat, B.r, &st->rho, K->partials, K->counter};
      FAME_TRY((run_chain_lin<double, 3>(K->n, pro, epi, B.work, K->m->Et64, NF, s)));
      K->stats.massApplies += 3;
      // a second round always follows the first (one FP32 round reaches ~3e-6), and it
      // takes its tolerance on the device, so the host reads the residual from then on
      if (refine == 1 && K->o.maxRefine > 1) {
        first = true;
        continue;
      }
      FAME_TRY(read_back(K->ctx, st, &h, sizeof(PcgState)));
      if (h.flag == -1) return fail(FAME_ERR_NONFINITE, "Mhat right-hand side contains NaN/Inf");
      bn2 = h.bnorm2;
      rn2 = h.rho;
      if (!std::isfinite(rn2)) return fail(FAME_ERR_NONFINITE, "refinement residual is NaN/Inf");
    }
    K->stats.refineSteps += refine;
    relres = bn2 > 0 ? std::sqrt(rn2 / bn2) : 0.0;
    if (relres > 10 * tolMhat)
      return fail(FAME_ERR_NOT_CONVERGED, "Mhat refinement failed: relres=" + std::to_string(relres) +
                                              " steps=" + std::to_string(refine));
  }
  // ---- post: y = V1^{-1}[mr1 + M W1 z ; mr2 + M W2 z]
  {
    ProKrPost pro{c64, B.x};
    EpiKrPost epi{K->mr1, K->mr2, bs->V1(0, 0), bs->V1(0, 1), bs->V1(1, 0), bs->V1(1, 1), bs->det, y, NF, st,
                  K->partials, K->counter};
    FAME_TRY((run_chain<double, 2>(K->n, pro, epi, B.work, K->m->Et64, NF, s)));
    K->stats.massApplies += 2;
  }
  if (!K->deferOutputCheck) FAME_TRY(krinv_output_check(K));
  K->stats.inverseCalls += 1;
  K->stats.totalIterations += iters;
  K->stats.maxIterations = std::max<long long>(K->stats.maxIterations, iters);
  K->stats.maxRelativeResidual = std::max(K->stats.maxRelativeResidual, relres);
  return FAME_OK;
}

template <typename T> int alloc_pcgbuf(PcgBuf<T>& B, long long NF, int nvec) {
  FAME_TRY(dalloc((void**)&B.work, 3 * NF * sizeof(C<T>)));
  FAME_TRY(dalloc((void**)&B.x, nvec * NF * sizeof(C<T>)));
  FAME_TRY(dalloc((void**)&B.r, nvec * NF * sizeof(C<T>)));
  FAME_TRY(dalloc((void**)&B.p, nvec * NF * sizeof(C<T>)));
  FAME_TRY(dalloc((void**)&B.Ap, nvec * NF * sizeof(C<T>)));
  if (nvec == 1) FAME_TRY(dalloc((void**)&B.z, NF * sizeof(C<T>)));
  return FAME_OK;
}
template <typename T> void free_pcgbuf(PcgBuf<T>& B) {
  dfree(B.work); dfree(B.x); dfree(B.r); dfree(B.p); dfree(B.Ap); dfree(B.z);
  B = PcgBuf<T>{};
}

}  // namespace fame

using namespace fame;

extern "C" {

int fame_apply_Mhat_C_scalar_compact(fame_basis* b, fame_mass* m, const void* x, void* y, int prec) {
  if (!b || !m || !x || !y) return fail(FAME_ERR_INVALID, "apply_Mhat arguments");
  if (b->N != m->N) return fail(FAME_ERR_INVALID, "basis and mass have different N");
  double2* work = nullptr;
  const size_t el = prec == FAME_F32 ? sizeof(float2) : sizeof(double2);
  if (prec != FAME_F64 && prec != FAME_F32) return fail(FAME_ERR_INVALID, "prec must be FAME_F64 or FAME_F32");
  if (b->work_bytes < 3 * b->NF * el) {
    dfree(b->work);
    b->work = nullptr;
    b->work_bytes = 0;
    FAME_TRY(dalloc((void**)&b->work, 3 * b->NF * el));
    b->work_bytes = 3 * b->NF * el;
  }
  work = (double2*)b->work;
  cudaStream_t s = b->ctx->stream;
  if (prec == FAME_F64) {
    const MhatCoef<double> c = coef_of<double>(b);
    return run_chain_lin<double, 3>(b->n, ProMhat<double, false>{c, (const double2*)x}, EpiMhat<double, false>{c, (double2*)y},
                                work, m->Et64, b->NF, s);
  }
  const MhatCoef<float> c = coef_of<float>(b);
  return run_chain_lin<float, 3>(b->n, ProMhat<float, false>{c, (const float2*)x}, EpiMhat<float, false>{c, (float2*)y},
                             (float2*)work, m->Et32, b->NF, s);
}

int fame_krinv_default_opts(fame_krinv_opts* o) {
  if (!o) return fail(FAME_ERR_INVALID, "opts is NULL");
  o->kind = FAME_KRINV_EXPLICIT;
  o->prec_mode = FAME_PREC_FP64;
  o->tolCG = 1e-10;
  o->maxitCG = 1200;
  o->tolKr = 1e-10;
  o->tolM = 1e-12;
  o->maxitKr = 600;
  o->maxitM = 1600;
  o->epsC = 4.0;
  o->useKrPreconditioner = 1;
  o->tolInner32 = 3e-6;
  o->maxRefine = 20;
  o->checkEvery = 4;
  o->verifyTrueResidual = 1;
  o->useGraphs = 1;
  o->mhatPreconditioner = 1;
  o->passColumns = 0;
  o->refineTarget = 0.1;
  return FAME_OK;
}

int fame_krinv_create(fame_basis* b, fame_mass* m, const fame_krinv_opts* o, fame_krinv** out) {
  if (!b || !m || !out) return fail(FAME_ERR_INVALID, "fame_krinv_create arguments");
  *out = nullptr;
  if (b->N != m->N) return fail(FAME_ERR_INVALID, "basis and mass have different N");
  fame_krinv* K = new fame_krinv();
  fame_krinv_default_opts(&K->o);
  if (o) K->o = *o;
  if (K->o.kind != FAME_KRINV_EXPLICIT && K->o.kind != FAME_KRINV_NESTED) {
    delete K;
    return fail(FAME_ERR_INVALID, "unknown K_r^{-1} kind");
  }
  if (K->o.prec_mode != FAME_PREC_FP64 && K->o.prec_mode != FAME_PREC_MIXED) {
    delete K;
    return fail(FAME_ERR_INVALID, "unknown precision mode");
  }
  if (!(K->o.refineTarget > 0.0 && K->o.refineTarget <= 1.0)) {
    delete K;
    return fail(FAME_ERR_INVALID, "refineTarget must lie in (0, 1]");
  }
  K->b = b;
  K->m = m;
  K->ctx = b->ctx;
  K->NF = b->NF;
  K->n = b->n;
  const long long NF = K->NF;
  const bool nested = K->o.kind == FAME_KRINV_NESTED;
  int s = alloc_pcgbuf<double>(K->b64, NF, nested ? 3 : 1);
  if (s == FAME_OK && K->o.prec_mode == FAME_PREC_MIXED) s = alloc_pcgbuf<float>(K->b32, NF, nested ? 3 : 1);
  if (s == FAME_OK && !nested) s = dalloc((void**)&K->mr1, NF * sizeof(double2));
  if (s == FAME_OK && !nested) s = dalloc((void**)&K->mr2, NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&K->bhat, (nested ? 3 : 1) * NF * sizeof(double2));
  const long long nparts = std::max<long long>(passC_blocks(K->n), kVecBlocksMax) * 8;
  if (s == FAME_OK) s = dalloc((void**)&K->partials, nparts * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&K->counter, sizeof(unsigned));
  if (s == FAME_OK) s = dalloc((void**)&K->st64, sizeof(PcgState));
  if (s == FAME_OK) s = dalloc((void**)&K->st32, sizeof(PcgState));
  if (s == FAME_OK && nested) s = nested_alloc(K);
  if (s != FAME_OK) {
    fame_krinv_destroy(K);
    return s;
  }
  cudaMemsetAsync(K->counter, 0, sizeof(unsigned), K->ctx->stream);
  cudaMemsetAsync(K->st64, 0, sizeof(PcgState), K->ctx->stream);
  cudaMemsetAsync(K->st32, 0, sizeof(PcgState), K->ctx->stream);
  *out = K;
  return FAME_OK;
}

int fame_krinv_destroy(fame_krinv* K) {
  if (!K) return FAME_OK;
  cudaStreamSynchronize(K->ctx->stream);
  free_pcgbuf(K->b64);
  free_pcgbuf(K->b32);
  dfree(K->mr1); dfree(K->mr2); dfree(K->bhat);
  dfree(K->partials); dfree(K->counter); dfree(K->st64); dfree(K->st32);
  nested_free(K);
  lanczos_ws_free(K);
  for (auto& g : K->graphs)
    if (g) cudaGraphExecDestroy(g);
  delete K;
  return FAME_OK;
}

int fame_krinv_apply(fame_krinv* K, const void* b, void* y, int ncols) {
  if (!K || !b || !y || ncols < 0) return fail(FAME_ERR_INVALID, "fame_krinv_apply arguments");
  const long long nr = 2 * K->NF;
  auto t0 = std::chrono::steady_clock::now();
  for (int j = 0; j < ncols; ++j) {
    const double2* bj = (const double2*)b + nr * j;
    double2* yj = (double2*)y + nr * j;
    if (K->o.kind == FAME_KRINV_EXPLICIT) {
      FAME_TRY(krinv_explicit_apply_one(K, bj, yj));
    } else {
      FAME_TRY(krinv_nested_apply_one(K, bj, yj));
    }
  }
  auto t1 = std::chrono::steady_clock::now();
  K->stats.totalInverseSeconds += std::chrono::duration<double>(t1 - t0).count();
  return FAME_OK;
}

int fame_recover_eigvecs(fame_basis* b, fame_mass* m, const void* Y, int k, double tol, int maxit,
                         int prec_mode, void* X, void* MX, int* iterations, double* relres) {
  if (!b || !m || !Y || !X || !MX || k < 0) return fail(FAME_ERR_INVALID, "fame_recover_eigvecs arguments");
  fame_krinv_opts o;
  fame_krinv_default_opts(&o);
  o.kind = FAME_KRINV_NESTED;
  o.prec_mode = prec_mode;
  o.tolM = tol;
  o.maxitM = maxit;
  fame_krinv* K = nullptr;
  FAME_TRY(fame_krinv_create(b, m, &o, &K));
  const long long NF = b->NF;
  int s = FAME_OK;
  for (int j = 0; j < k && s == FAME_OK; ++j) {
    int it = 0;
    double rr = 0.0;
    s = recover_one(K, (const double2*)Y + 2 * NF * j, (double2*)X + 3 * NF * j, (double2*)MX + 3 * NF * j,
                    &it, &rr);
    if (iterations) iterations[j] = it;
    if (relres) relres[j] = rr;
    if (s == FAME_OK && rr > 10 * tol)
      s = fail(FAME_ERR_NOT_CONVERGED, "recover_original_eigenvectors_exp2:RecoveryCGFailure relres=" +
                                           std::to_string(rr));
  }
  fame_krinv_destroy(K);
  return s;
}

int fame_krinv_stats_get(fame_krinv* K, fame_krinv_stats* out) {
  if (!K || !out) return fail(FAME_ERR_INVALID, "fame_krinv_stats_get arguments");
  *out = K->stats;
  return FAME_OK;
}

int fame_krinv_stats_reset(fame_krinv* K) {
  if (!K) return fail(FAME_ERR_INVALID, "krinv is NULL");
  K->stats = fame_krinv_stats{};
  return FAME_OK;
}

}  // extern "C"
