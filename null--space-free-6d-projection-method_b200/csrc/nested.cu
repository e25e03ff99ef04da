// Nested K_r^{-1} (method B), exp1/make_nested_krinv_instrumented.m:33-126:
//   solve K_r x = b by PCG (tolKr, maxitKr, preconditioner epsC*r./sigma_r),
//   K_r z = V^* M3^{-1} V z with an inner PCG on M3 = diag(M,M,M) (tolM, maxitM)
//   for every outer matvec.  Outer scalars live in an OuterState on the device;
//   the host reads it once per outer iteration.  In FAME_PREC_MIXED the inner
//   M3 solves are FP64 iterative refinement around an FP32 PCG.
#include <cstdio>
#include <algorithm>
#include <cmath>
#include <string>
#include "internal.cuh"
#include "krinv_impl.cuh"

namespace fame {

static inline int nb(long long n) { return vec_blocks(n); }

__global__ void k_outer_init(const double2* b, double2* x, double2* r, long long n, OuterState* st,
                             double tol, double* partials, unsigned* counter) {
  Red<double, 1> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 bi = b[i];
    x[i] = make_double2(0.0, 0.0);
    r[i] = bi;
    acc.v[0] += cabs2<double>(bi);
  }
  grid_sum_finalize<double, 1>(acc, partials, counter, [&](const Red<double, 1>& t) {
    st->bnorm2 = t.v[0];
    st->tolb2 = tol * tol * t.v[0];
    st->rr = t.v[0];
    st->rho = 1.0;
    st->rho1 = 1.0;
    st->beta = 0.0;
    st->iter = 0;
    st->pad = 0;
  });
}

// z = M1 r (epsC * r ./ sigma_r or identity); rho = r^H z; beta = rho/rho1
__global__ void k_outer_precond(const double2* r, double2* z, const double* sigma, long long NF,
                                double epsC, int usePre, OuterState* st, double* partials,
                                unsigned* counter) {
  Red<double, 1> acc{};
  const long long n = 2 * NF;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 ri = r[i];
    const double w = usePre ? epsC / sigma[i % NF] : 1.0;
    const double2 zi = cscale<double>(ri, w);
    z[i] = zi;
    acc.v[0] += w * cabs2<double>(ri);
  }
  grid_sum_finalize<double, 1>(acc, partials, counter, [&](const Red<double, 1>& t) {
    st->rho1 = st->rho;
    st->rho = t.v[0];
    st->beta = st->iter > 0 ? st->rho / st->rho1 : 0.0;
    if (!(t.v[0] > 0.0) || !isfinite(t.v[0])) st->pad = 4;  // breakdown flag
  });
}

// p = z (first iteration) or z + beta p
__global__ void k_outer_dir(const double2* z, double2* p, long long n, const OuterState* st) {
  const bool first = st->iter == 0;
  const double beta = st->beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = first ? z[i] : cadd<double>(z[i], cscale<double>(p[i], beta));
}

// b3 = V p (2NF -> 3NF, b3 in line order), ||b3||^2 -> inner PCG state
__device__ __forceinline__ long long line_index(long long i, int n) {
  const long long n3 = (long long)n * n * n;
  const long long cb = i - i % n3;
  const long long g = i - cb;
  return cb + g / n + (long long)n * n * (g % n);
}

template <typename T>
__global__ void k_inner_init(const double2* p, const double2* V11, const double2* V12,
                             const double2* V21, const double2* V22, const double2* V31,
                             const double2* V32, long long NF, int n, double2* b3, PcgState* st,
                             double tol, int maxit, double* partials, unsigned* counter) {
  Red<double, 1> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    const double2 x1 = p[i], x2 = p[NF + i];
    const double2 y1 = cadd<double>(cmul<double>(V11[i], x1), cmul<double>(V12[i], x2));
    const double2 y2 = cadd<double>(cmul<double>(V21[i], x1), cmul<double>(V22[i], x2));
    const double2 y3 = cadd<double>(cmul<double>(V31[i], x1), cmul<double>(V32[i], x2));
    const long long il = line_index(i, n);
    b3[il] = y1;
    b3[NF + il] = y2;
    b3[2 * NF + il] = y3;
    acc.v[0] += cabs2<double>(y1) + cabs2<double>(y2) + cabs2<double>(y3);
  }
  grid_sum_finalize<double, 1>(acc, partials, counter, [&](const Red<double, 1>& t) {
    pcg_init_state(st, t.v[0], tol, maxit);
  });
}

__global__ void k_copy_zero(const double2* b, double2* r, double2* x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    r[i] = b[i];
    x[i] = make_double2(0.0, 0.0);
  }
}

// q = V^* u (3NF line order -> 2NF natural); with DOT, pq = p^H q -> alpha = rho/pq
template <bool DOT>
__global__ void k_outer_VH(const double2* u, const double2* V11, const double2* V12,
                           const double2* V21, const double2* V22, const double2* V31,
                           const double2* V32, long long NF, int n, double2* q, const double2* p,
                           OuterState* st, double* partials, unsigned* counter) {
  Red<double, 2> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    const long long il = line_index(i, n);
    const double2 x1 = u[il], x2 = u[NF + il], x3 = u[2 * NF + il];
    const double2 y1 = cadd<double>(cadd<double>(cmulc<double>(V11[i], x1), cmulc<double>(V21[i], x2)), cmulc<double>(V31[i], x3));
    const double2 y2 = cadd<double>(cadd<double>(cmulc<double>(V12[i], x1), cmulc<double>(V22[i], x2)), cmulc<double>(V32[i], x3));
    q[i] = y1;
    q[NF + i] = y2;
    if (DOT) {
      const double2 d1 = cmulc<double>(p[i], y1), d2 = cmulc<double>(p[NF + i], y2);
      acc.v[0] += d1.x + d2.x;
      acc.v[1] += d1.y + d2.y;
    }
  }
  if (DOT) {
    grid_sum_finalize<double, 2>(acc, partials, counter, [&](const Red<double, 2>& t) {
      st->pq_re = t.v[0];
      st->pq_im = t.v[1];
      if (!(t.v[0] > 0.0) || !isfinite(t.v[0])) {
        st->pad = 4;
        st->alpha_re = st->alpha_im = 0.0;
        return;
      }
      const double d = t.v[0] * t.v[0] + t.v[1] * t.v[1];
      st->alpha_re = st->rho * t.v[0] / d;
      st->alpha_im = -st->rho * t.v[1] / d;
    });
  }
}

// x += alpha p ; r -= alpha q ; rr = ||r||^2 ; iter++
__global__ void k_outer_update(double2* x, double2* r, const double2* p, const double2* q, long long n,
                               OuterState* st, double* partials, unsigned* counter) {
  const double2 a = make_double2(st->alpha_re, st->alpha_im);
  Red<double, 1> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] = cadd<double>(x[i], cmul<double>(a, p[i]));
    const double2 ri = csub<double>(r[i], cmul<double>(a, q[i]));
    r[i] = ri;
    acc.v[0] += cabs2<double>(ri);
  }
  grid_sum_finalize<double, 1>(acc, partials, counter, [&](const Red<double, 1>& t) {
    st->rr = t.v[0];
    st->iter += 1;
  });
}

// r = b - q ; rr = ||r||^2 (true outer residual)
__global__ void k_outer_resid(const double2* b, const double2* q, double2* r, long long n,
                              OuterState* st, double* partials, unsigned* counter) {
  Red<double, 1> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 ri = csub<double>(b[i], q[i]);
    r[i] = ri;
    acc.v[0] += cabs2<double>(ri);
  }
  grid_sum_finalize<double, 1>(acc, partials, counter, [&](const Red<double, 1>& t) { st->rr = t.v[0]; });
}

// Inner solve M3 u = b3 (b3 in K->bhat, u in K->b64.x); state in K->st64.
static int inner_m3_solve(fame_krinv* K) {
  cudaStream_t s = K->ctx->stream;
  const long long NF = K->NF, n3 = 3 * NF;
  PcgBuf<double>& B = K->b64;
  PcgState h{};
  const double tolM = K->o.tolM;
  if (K->o.prec_mode == FAME_PREC_FP64) {
    FAME_TRY(pcg_iterate<double>(K, OpM3<double>{K->m->Et64}, B, K->st64, K->lastIt64, h,
                                 K->o.verifyTrueResidual != 0, K->bhat));
    if (h.flag == -1) return fail(FAME_ERR_NONFINITE, "nested inner right-hand side is NaN/Inf");
    const double rr = h.bnorm2 > 0 ? std::sqrt(h.rho / h.bnorm2) : 0.0;
    K->stats.massSolveCalls += 1;
    K->stats.totalMassIterations += h.iter;
    if (h.flag != 0 && rr > 10 * tolM)
      return fail(FAME_ERR_NOT_CONVERGED, "Nested M solve failed: flag=" + std::to_string(h.flag) +
                                              " relres=" + std::to_string(rr));
    return FAME_OK;
  }
  // mixed: FP64 refinement, FP32 PCG corrections
  FAME_TRY(read_back(K->ctx, K->st64, &h, sizeof(PcgState)));
  if (h.flag == -1) return fail(FAME_ERR_NONFINITE, "nested inner right-hand side is NaN/Inf");
  const double bn2 = h.bnorm2;
  double rn2 = h.rho;
  PcgBuf<float>& F = K->b32;
  float* partials32 = reinterpret_cast<float*>(K->partials);
  int refine = 0, its = 0;
  while (rn2 > tolM * tolM * bn2 && bn2 > 0 && refine < K->o.maxRefine) {
    ++refine;
    k_pcg_init<float, double><<<nb(n3), 256, 0, s>>>(B.r, F.r, F.x, n3, K->st32, K->o.tolInner32,
                                                    K->o.maxitM, partials32, K->counter);
    ::fame::count_launch();
    PcgState h32{};
    FAME_TRY(pcg_iterate<float>(K, OpM3<float>{K->m->Et32}, F, K->st32, K->lastIt32, h32, false, nullptr));
    if (h32.flag == -1 || h32.flag == 4) return fail(FAME_ERR_NOT_CONVERGED, "FP32 correction solve broke down");
    its += h32.iter;
    K->stats.fp32Iterations += h32.iter;
    ProResidM3<double, float, true> pro{B.x, F.x, NF};
    EpiResidM3<double> epi{K->bhat, B.r, &K->st64->rho, NF, K->partials, K->counter};
    FAME_TRY((run_chain<double, 3>(K->n, pro, epi, B.work, K->m->Et64, NF, s)));
    K->stats.massApplies += 3;
    FAME_TRY(read_back(K->ctx, K->st64, &h, sizeof(PcgState)));
    rn2 = h.rho;
    if (!std::isfinite(rn2)) return fail(FAME_ERR_NONFINITE, "refinement residual is NaN/Inf");
  }
  K->stats.refineSteps += refine;
  K->stats.massSolveCalls += 1;
  K->stats.totalMassIterations += its;
  const double rr = bn2 > 0 ? std::sqrt(rn2 / bn2) : 0.0;
  if (rr > 10 * tolM) {
    char msg[96];
    std::snprintf(msg, sizeof(msg), "Nested M refinement failed: relres=%.3e after %d refinements", rr, refine);
    return fail(FAME_ERR_NOT_CONVERGED, msg);
  }
  return FAME_OK;
}

// out = K_r in = V^* M3^{-1} V in ; with DOT also p^H out -> alpha
template <bool DOT>
static int apply_Kr(fame_krinv* K, const double2* in, double2* out) {
  fame_basis* b = K->b;
  cudaStream_t s = K->ctx->stream;
  const long long NF = K->NF;
  PcgBuf<double>& B = K->b64;
  // b3 = V in ; inner state init (r3 = b3, x3 = 0 done below)
  k_inner_init<double><<<nb(NF), 256, 0, s>>>(in, b->V[0], b->V[3], b->V[1], b->V[4], b->V[2],
                                              b->V[5], NF, K->n, K->bhat, K->st64, K->o.tolM,
                                              K->o.prec_mode == FAME_PREC_MIXED ? K->o.maxRefine : K->o.maxitM,
                                              K->partials, K->counter);
  ::fame::count_launch();
  k_copy_zero<<<nb(3 * NF), 256, 0, s>>>(K->bhat, B.r, B.x, 3 * NF);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  FAME_TRY(inner_m3_solve(K));
  k_outer_VH<DOT><<<nb(NF), 256, 0, s>>>(B.x, b->V[0], b->V[3], b->V[1], b->V[4], b->V[2], b->V[5],
                                         NF, K->n, out, K->op, K->ost, K->partials, K->counter);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int krinv_nested_apply_one(fame_krinv* K, const double2* b, double2* x) {
  cudaStream_t s = K->ctx->stream;
  const long long NF = K->NF, n2 = 2 * NF;
  const double tolKr = K->o.tolKr;
  k_outer_init<<<nb(n2), 256, 0, s>>>(b, x, K->orr, n2, K->ost, tolKr, K->partials, K->counter);
  ::fame::count_launch();
  OuterState h{};
  FAME_TRY(read_back(K->ctx, K->ost, &h, sizeof(OuterState)));
  if (!std::isfinite(h.bnorm2)) return fail(FAME_ERR_NONFINITE, "Nested K_r^{-1} input contains NaN/Inf");
  int flag = 1, moresteps = 0;
  if (h.bnorm2 == 0.0) flag = 0;
  while (flag != 0 && h.iter < K->o.maxitKr) {
    k_outer_precond<<<nb(n2), 256, 0, s>>>(K->orr, K->oz, K->sigma, NF, K->o.epsC,
                                           K->o.useKrPreconditioner, K->ost, K->partials, K->counter);
    ::fame::count_launch();
    k_outer_dir<<<nb(n2), 256, 0, s>>>(K->oz, K->op, n2, K->ost);
    ::fame::count_launch();
    FAME_TRY(apply_Kr<true>(K, K->op, K->oq));
    k_outer_update<<<nb(n2), 256, 0, s>>>(x, K->orr, K->op, K->oq, n2, K->ost, K->partials, K->counter);
    ::fame::count_launch();
    FAME_CUDA_TRY(cudaGetLastError());
    FAME_TRY(read_back(K->ctx, K->ost, &h, sizeof(OuterState)));
    if (h.pad == 4) {
      flag = 4;
      break;
    }
    if (h.rr <= h.tolb2) {
      // confirm on the true residual b - K_r x (MATLAB pcg semantics)
      FAME_TRY(apply_Kr<false>(K, x, K->oq));
      k_outer_resid<<<nb(n2), 256, 0, s>>>(b, K->oq, K->orr, n2, K->ost, K->partials, K->counter);
      ::fame::count_launch();
      FAME_TRY(read_back(K->ctx, K->ost, &h, sizeof(OuterState)));
      if (h.rr <= h.tolb2 || !K->o.verifyTrueResidual) {
        flag = 0;
        break;
      }
      if (++moresteps >= 3) {
        flag = 3;
        break;
      }
    }
  }
  const double relres = h.bnorm2 > 0 ? std::sqrt(h.rr / h.bnorm2) : 0.0;
  K->stats.inverseCalls += 1;
  K->stats.totalIterations += h.iter;
  K->stats.maxIterations = std::max<long long>(K->stats.maxIterations, h.iter);
  K->stats.maxRelativeResidual = std::max(K->stats.maxRelativeResidual, relres);
  if (flag != 0 && relres > 10 * tolKr)
    return fail(FAME_ERR_NOT_CONVERGED, "Nested K_r solve failed: flag=" + std::to_string(flag) +
                                            " relres=" + std::to_string(relres) +
                                            " iter=" + std::to_string(h.iter));
  return FAME_OK;
}

// ---------------------------------------------------------------- recovery
// x (3NF, line order) -> M3 x written in natural order, x^H M3 x -> *out
struct ProM3x {
  const double2* x;
  long long NF;
  __device__ __forceinline__ void load(long long ia, long long, double2* v) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = x[c * NF + ia];
  }
};
struct EpiM3Norm {
  using Acc = double;
  static constexpr int K = 1;
  const double2* x;
  double2* MX;
  long long NF;
  double* out;
  double* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long ia, long long in, const double2* v, Red<double, 1>& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      MX[c * NF + in] = v[c];
      const double2 d = cmulc<double>(x[c * NF + ia], v[c]);
      acc.v[0] += d.x;
    }
  }
  __device__ __forceinline__ void finalize(const Red<double, 1>& t) const { *out = t.v[0]; }
};

// X = x / sqrt(n2) (x line order -> X natural), MX /= sqrt(n2)
__global__ void k_recover_scale(const double2* x, double2* X, double2* MX, long long NF, int n,
                                const double* n2) {
  const double s = 1.0 / sqrt(*n2);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    const long long il = line_index(i, n);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      X[c * NF + i] = cscale<double>(x[c * NF + il], s);
      MX[c * NF + i] = cscale<double>(MX[c * NF + i], s);
    }
  }
}

int recover_one(fame_krinv* K, const double2* y, double2* X, double2* MX, int* iters, double* relres) {
  fame_basis* b = K->b;
  cudaStream_t s = K->ctx->stream;
  const long long NF = K->NF;
  PcgBuf<double>& B = K->b64;
  const long long it0 = K->stats.totalMassIterations;
  // rhs = V y (line order), then x = M3^{-1} rhs
  k_inner_init<double><<<nb(NF), 256, 0, s>>>(y, b->V[0], b->V[3], b->V[1], b->V[4], b->V[2], b->V[5],
                                              NF, K->n, K->bhat, K->st64, K->o.tolM,
                                              K->o.prec_mode == FAME_PREC_MIXED ? K->o.maxRefine : K->o.maxitM,
                                              K->partials, K->counter);
  ::fame::count_launch();
  k_copy_zero<<<nb(3 * NF), 256, 0, s>>>(K->bhat, B.r, B.x, 3 * NF);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  FAME_TRY(inner_m3_solve(K));
  PcgState h{};
  FAME_TRY(read_back(K->ctx, K->st64, &h, sizeof(PcgState)));
  *iters = (int)(K->stats.totalMassIterations - it0);
  *relres = h.bnorm2 > 0 ? std::sqrt(h.rho / h.bnorm2) : 0.0;
  // M x and x^H M x (the mass action the normalisation needs anyway)
  ProM3x pro{B.x, NF};
  EpiM3Norm epi{B.x, MX, NF, &K->st64->aux, K->partials, K->counter};
  FAME_TRY((run_chain<double, 3>(K->n, pro, epi, B.work, K->m->Et64, NF, s)));
  FAME_TRY(read_back(K->ctx, K->st64, &h, sizeof(PcgState)));
  if (!(h.aux > 0.0) || !std::isfinite(h.aux))
    return fail(FAME_ERR_NONFINITE, "recover_original_eigenvectors_exp2:BadMassNorm");
  k_recover_scale<<<nb(NF), 256, 0, s>>>(B.x, X, MX, NF, K->n, &K->st64->aux);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int nested_alloc(fame_krinv* K) {
  const long long n2 = 2 * K->NF;
  FAME_TRY(dalloc((void**)&K->orr, n2 * sizeof(double2)));
  FAME_TRY(dalloc((void**)&K->oz, n2 * sizeof(double2)));
  FAME_TRY(dalloc((void**)&K->op, n2 * sizeof(double2)));
  FAME_TRY(dalloc((void**)&K->oq, n2 * sizeof(double2)));
  FAME_TRY(dalloc((void**)&K->ost, sizeof(OuterState)));
  K->sigma = K->b->Qq;  // sigma_r = [|q|^2; |q|^2] (exp1/assemble_K_and_nullspace_free_basis.m:93)
  return FAME_OK;
}

void nested_free(fame_krinv* K) {
  dfree(K->orr); dfree(K->oz); dfree(K->op); dfree(K->oq); dfree(K->ost);
  K->orr = K->oz = K->op = K->oq = nullptr;
  K->ost = nullptr;
}

}  // namespace fame
