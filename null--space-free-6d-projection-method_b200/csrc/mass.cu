// 6D Fourier mass operator: handle creation, the four mass modes of the
// reference (exp1/build_mass_backend_large_scalar.m:28-31), the raw
// applyMij_fft entry and the rank-1-lattice drop-in.
#include <algorithm>
#include "internal.cuh"
#include "mass_chain.cuh"

namespace fame {

__global__ void k_scale_E(const double* E, long long NF, double s, double* o64, float* o32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = E[i] * s;
    o64[i] = v;
    o32[i] = (float)v;
  }
}

// Verify that (inputIdx, targetIdx, M) is the radix rank-1 plan of
// exp1/build_radix_exact_rank1_plan_scalar.m:18-43 (1-based indices).
__global__ void k_check_rank1(const uint32_t* in, const uint32_t* tg, long long NF, int n,
                              long long B, long long M, long long shift, unsigned* bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF;
       i += (long long)gridDim.x * blockDim.x) {
    long long tmp = i, code = 0, z = 1;
    for (int j = 0; j < 6; ++j) {
      code += (tmp % n) * z;
      tmp /= n;
      z *= B;
    }
    const long long target = (code + shift) % M;
    if ((long long)in[i] != code + 1 || (long long)tg[i] != target + 1) atomicAdd(bad, 1u);
  }
}

template <typename T>
int mass_scalar_cols(int n, long long NF, const C<T>* x, C<T>* y, int ncols, const double* Es64,
                     const float* Es32, double escale, cudaStream_t st) {
  for (int j = 0; j < ncols; ++j) {
    ProCols<T, 1> pro;
    pro.x[0] = x + (long long)j * NF;
    EpiCols<T, 1> epi;
    epi.y[0] = y + (long long)j * NF;
    if constexpr (sizeof(T) == 8) {
      FAME_TRY((run_chain<T, 1>(n, pro, epi, y + (long long)j * NF, Es64, escale, NF, st)));
    } else {
      if (Es32) {
        FAME_TRY((run_chain<T, 1>(n, pro, epi, y + (long long)j * NF, Es32, (float)escale, NF, st)));
      } else {
        FAME_TRY((run_chain<T, 1>(n, pro, epi, y + (long long)j * NF, Es64, escale, NF, st)));
      }
    }
  }
  return FAME_OK;
}

// out[t] = (1/NF) sum_y g_t(y) sum_c |w_c(y)|^2, w_c the unnormalised inverse DFT
// of component c, i.e. NF sum_y g_t(y) sum_c |ifftn(x_c)(y)|^2 = x^H (dM/dtheta_t) x.
constexpr int kMaxAdjParams = 8;
__global__ void k_adjoint_reduce(const double2* w, long long NF, const double* g, int np,
                                 double* partials, unsigned* counter, double* out) {
  Red<double, kMaxAdjParams> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    const double d = cabs2<double>(w[i]) + cabs2<double>(w[NF + i]) + cabs2<double>(w[2 * NF + i]);
#pragma unroll
    for (int t = 0; t < kMaxAdjParams; ++t)
      if (t < np) acc.v[t] += g[(long long)t * NF + i] * d;
  }
  const double inv = 1.0 / (double)NF;
  grid_sum_finalize<double, kMaxAdjParams>(acc, partials, counter, [&](const Red<double, kMaxAdjParams>& tot) {
    for (int t = 0; t < kMaxAdjParams; ++t) out[t] = tot.v[t] * inv;
  });
}

template <int n>
int adjoint_inverse_n(const double2* x, double2* work, long long NF, cudaStream_t st) {
  using Q = Cube<n, double>;
  ProCols<double, 3> pro;
  for (int c = 0; c < 3; ++c) pro.x[c] = x + c * NF;
  FAME_TRY((launch_passA<n, double, 3>(pro, work, NF, st, Gate{nullptr})));
  constexpr int TT = PassBTile<double>::TT;
  const size_t smem = (size_t)TT * Q::size * sizeof(double2);
  static int attr = ensure_smem(k_passB_inv<n, double, TT>, smem);
  if (attr != FAME_OK) return attr;
  k_passB_inv<n, double, TT><<<dim3(Q::n3 / TT, 3), std::min(512, std::max(64, round32(TT * Q::n2))), smem, st>>>(work, NF);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int check_N(int N) {
  if (N < 1 || N > 7) return fail(FAME_ERR_UNSUPPORTED, "N must be in [1,7] (2N <= 14)");
  return FAME_OK;
}

long long grid_NF(int N) {
  long long n = 2 * N, NF = 1;
  for (int d = 0; d < 6; ++d) NF *= n;
  return NF;
}

// mode dispatch on a typed pointer pair
template <typename T>
int mass_apply_typed(fame_mass* m, int mode, const C<T>* x, C<T>* y, int nrhs) {
  const long long NF = m->NF;
  cudaStream_t st = m->ctx->stream;
  const double* E64 = m->Es64;
  const float* E32 = m->Es32;
  switch (mode) {
    case FAME_MASS_SCALAR:
      return mass_scalar_cols<T>(m->n, NF, x, y, nrhs, E64, E32, 1.0, st);
    case FAME_MASS_FULL3:
      // 3NF x nrhs, column-major: each column holds three components
      return mass_scalar_cols<T>(m->n, NF, x, y, 3 * nrhs, E64, E32, 1.0, st);
    case FAME_MASS_COL3:
      for (int j = 0; j < nrhs; ++j) {
        C<T>* yj = y + 3LL * NF * j;
        FAME_CUDA_TRY(cudaMemsetAsync(yj, 0, 2 * NF * sizeof(C<T>), st));
        FAME_TRY(mass_scalar_cols<T>(m->n, NF, x + NF * j, yj + 2 * NF, 1, E64, E32, 1.0, st));
      }
      return FAME_OK;
    case FAME_MASS_COLS12:
      for (int j = 0; j < nrhs; ++j) {
        C<T>* yj = y + 3LL * NF * j;
        FAME_TRY(mass_scalar_cols<T>(m->n, NF, x + 2 * NF * j, yj, 2, E64, E32, 1.0, st));
        FAME_CUDA_TRY(cudaMemsetAsync(yj + 2 * NF, 0, NF * sizeof(C<T>), st));
      }
      return FAME_OK;
    default:
      return fail(FAME_ERR_INVALID, "unknown mass mode");
  }
}

}  // namespace fame

using namespace fame;

extern "C" {

int fame_applyMij_fft(fame_ctx* ctx, int N, const double* E, const void* x, void* y, int nrhs,
                      int prec) {
  if (!ctx || !E || !x || !y || nrhs < 0) return fail(FAME_ERR_INVALID, "applyMij_fft arguments");
  FAME_TRY(check_N(N));
  const long long NF = grid_NF(N);
  const double escale = 1.0 / (double)NF;
  if (prec == FAME_F64)
    return mass_scalar_cols<double>(2 * N, NF, (const double2*)x, (double2*)y, nrhs, E, nullptr,
                                    escale, ctx->stream);
  if (prec == FAME_F32)
    return mass_scalar_cols<float>(2 * N, NF, (const float2*)x, (float2*)y, nrhs, E, nullptr,
                                   escale, ctx->stream);
  return fail(FAME_ERR_INVALID, "prec must be FAME_F64 or FAME_F32");
}

int fame_mass_create(fame_ctx* ctx, int N, const double* E, fame_mass** out) {
  if (!ctx || !E || !out) return fail(FAME_ERR_INVALID, "fame_mass_create arguments");
  *out = nullptr;
  FAME_TRY(check_N(N));
  fame_mass* m = new fame_mass();
  m->ctx = ctx;
  m->N = N;
  m->n = 2 * N;
  m->NF = grid_NF(N);
  int s = dalloc((void**)&m->Es64, m->NF * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&m->Es32, m->NF * sizeof(float));
  if (s != FAME_OK) {
    dfree(m->Es64);
    delete m;
    return s;
  }
  const int blocks = (int)std::min<long long>((m->NF + 255) / 256, 148 * 16);
  k_scale_E<<<blocks, 256, 0, ctx->stream>>>(E, m->NF, 1.0 / (double)m->NF, m->Es64, m->Es32);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  *out = m;
  return FAME_OK;
}

int fame_mass_destroy(fame_mass* m) {
  if (!m) return FAME_OK;
  cudaStreamSynchronize(m->ctx->stream);
  dfree(m->Es64);
  dfree(m->Es32);
  delete m;
  return FAME_OK;
}

int fame_mass_apply(fame_mass* m, int mode, const void* x, void* y, int nrhs, int prec) {
  if (!m || !x || !y || nrhs < 0) return fail(FAME_ERR_INVALID, "fame_mass_apply arguments");
  if (prec == FAME_F64) return mass_apply_typed<double>(m, mode, (const double2*)x, (double2*)y, nrhs);
  if (prec == FAME_F32) return mass_apply_typed<float>(m, mode, (const float2*)x, (float2*)y, nrhs);
  return fail(FAME_ERR_INVALID, "prec must be FAME_F64 or FAME_F32");
}

int fame_mass_adjoint(fame_mass* m, const void* X, int nmodes, const double* dEps, int nparams,
                      double* out) {
  if (!m || !X || !dEps || !out || nmodes < 0 || nparams < 1 || nparams > kMaxAdjParams)
    return fail(FAME_ERR_INVALID, "fame_mass_adjoint arguments (1 <= nparams <= 8)");
  const long long NF = m->NF;
  cudaStream_t st = m->ctx->stream;
  double2* work = nullptr;
  double* red = nullptr;
  unsigned* counter = nullptr;
  const int blocks = (int)std::min<long long>((NF + 255) / 256, 148 * 8);
  int s = dalloc((void**)&work, 3 * NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&red, ((size_t)blocks * kMaxAdjParams + kMaxAdjParams) * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&counter, sizeof(unsigned));
  if (s == FAME_OK) cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
  for (int j = 0; j < nmodes && s == FAME_OK; ++j) {
    const double2* xj = (const double2*)X + 3 * NF * j;
    switch (m->n) {
      case 2: s = adjoint_inverse_n<2>(xj, work, NF, st); break;
      case 4: s = adjoint_inverse_n<4>(xj, work, NF, st); break;
      case 6: s = adjoint_inverse_n<6>(xj, work, NF, st); break;
      case 8: s = adjoint_inverse_n<8>(xj, work, NF, st); break;
      case 10: s = adjoint_inverse_n<10>(xj, work, NF, st); break;
      case 12: s = adjoint_inverse_n<12>(xj, work, NF, st); break;
      case 14: s = adjoint_inverse_n<14>(xj, work, NF, st); break;
      default: s = fail(FAME_ERR_UNSUPPORTED, "adjoint: unsupported N");
    }
    if (s != FAME_OK) break;
    k_adjoint_reduce<<<blocks, 256, 0, st>>>(work, NF, dEps, nparams, red + kMaxAdjParams, counter, red);
    ::fame::count_launch();
    double h[kMaxAdjParams];
    s = cudaGetLastError() == cudaSuccess ? read_back(m->ctx, red, h, sizeof(h)) : fail(FAME_ERR_CUDA, "adjoint launch");
    for (int t = 0; t < nparams && s == FAME_OK; ++t) out[(size_t)j * nparams + t] = h[t];
  }
  dfree(work);
  dfree(red);
  dfree(counter);
  return s;
}

int fame_applyMij_rank1_exact(fame_mass* m, const uint32_t* inputIdx, const uint32_t* targetIdx,
                              long long M, const void* x, void* y, int nrhs) {
  if (!m || !inputIdx || !targetIdx || !x || !y || nrhs < 0)
    return fail(FAME_ERR_INVALID, "applyMij_rank1_exact arguments");
  const long long n = m->n, B = 2 * n - 1;
  long long Mexp = n;
  for (int j = 0; j < 5; ++j) Mexp *= B;
  if (M != Mexp) return fail(FAME_ERR_INVALID, "rank1_exact_fft_scatter:BadSize (plan.M mismatch)");
  long long sumz = 0, z = 1;
  for (int j = 0; j < 6; ++j) {
    sumz += z;
    z *= B;
  }
  const long long shift = ((n - 1) * sumz) % M;
  unsigned* bad = nullptr;
  FAME_TRY(dalloc((void**)&bad, sizeof(unsigned)));
  cudaStream_t st = m->ctx->stream;
  cudaMemsetAsync(bad, 0, sizeof(unsigned), st);
  const int blocks = (int)std::min<long long>((m->NF + 255) / 256, 148 * 16);
  k_check_rank1<<<blocks, 256, 0, st>>>(inputIdx, targetIdx, m->NF, m->n, B, M, shift, bad);
  ::fame::count_launch();
  unsigned hbad = 0;
  int s = read_back(m->ctx, bad, &hbad, sizeof(unsigned));
  dfree(bad);
  FAME_TRY(s);
  if (hbad != 0) return fail(FAME_ERR_INVALID, "rank-1 plan index vectors are not the radix plan");
  return mass_apply_typed<double>(m, FAME_MASS_SCALAR, (const double2*)x, (double2*)y, nrhs);
}

}  // extern "C"
