// 6D Fourier mass operator: handle creation, the four mass modes of the
// reference (exp1/build_mass_backend_large_scalar.m:28-31), the raw
// applyMij_fft entry and the rank-1-lattice drop-in.
#include <algorithm>
#include "internal.cuh"
#include "mass_chain.cuh"

namespace fame {

// Pass-B tile width of the chains in precision T for a runtime axis length n.
template <typename T> int work_tt(int n) {
  switch (n) {
    case 2: return WorkTile<2, T>::TT;
    case 4: return WorkTile<4, T>::TT;
    case 6: return WorkTile<6, T>::TT;
    case 8: return WorkTile<8, T>::TT;
    case 10: return WorkTile<10, T>::TT;
    case 12: return WorkTile<12, T>::TT;
    default: return WorkTile<14, T>::TT;
  }
}

// E*scale in the pass-B tile order of the chains in precision T.
template <typename T> int tile_E(const double* E, int n, long long NF, double scale, T* out, cudaStream_t st,
                                  int invert = 0) {
  const int blocks = (int)std::min<long long>((NF + 255) / 256, 148 * 16);
  k_tile_E<T><<<blocks, 256, 0, st>>>(E, n, work_tt<T>(n), NF, scale, invert, out);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
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

// Scalar mass action on ncols columns.  work: one NF-field of scratch that
// must not alias x or y (pass C reads it tile-major while writing y by columns).
template <typename T>
int mass_scalar_cols(int n, long long NF, const C<T>* x, C<T>* y, int ncols, const T* Et, C<T>* work,
                     cudaStream_t st) {
  for (int j = 0; j < ncols; ++j) {
    ProCols<T, 1> pro;
    pro.x[0] = x + (long long)j * NF;
    EpiCols<T, 1> epi;
    epi.y[0] = y + (long long)j * NF;
    FAME_TRY((run_chain<T, 1>(n, pro, epi, work, Et, NF, st)));
  }
  return FAME_OK;
}

// out[t] = (1/NF) sum_y g_t(y) sum_c |w_c(y)|^2, w_c the unnormalised inverse DFT
// of component c, i.e. NF sum_y g_t(y) sum_c |ifftn(x_c)(y)|^2 = x^H (dM/dtheta_t) x.
constexpr int kMaxAdjParams = 8;
__global__ void k_adjoint_reduce(const double2* w, long long NF, int n, int TT, const double* g, int np,
                                 double* partials, unsigned* counter, double* out) {
  const long long n3 = (long long)n * n * n;
  Red<double, kMaxAdjParams> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    // w is tile-major (WorkTile): element i holds grid point c123 + n^3*c456
    const long long rr = i / TT, c456 = rr % n3, c123 = (rr / n3) * TT + i % TT;
    const long long y = c123 + n3 * c456;
    const double d = cabs2<double>(w[i]) + cabs2<double>(w[NF + i]) + cabs2<double>(w[2 * NF + i]);
#pragma unroll
    for (int t = 0; t < kMaxAdjParams; ++t)
      if (t < np) acc.v[t] += g[(long long)t * NF + y] * d;
  }
  const double inv = 1.0 / (double)NF;
  grid_sum_finalize<double, kMaxAdjParams>(acc, partials, counter, [&](const Red<double, kMaxAdjParams>& tot) {
    for (int t = 0; t < kMaxAdjParams; ++t) out[t] = tot.v[t] * inv;
  });
}

template <int n>
int adjoint_inverse_n(const double2* x, double2* work, long long NF, cudaStream_t st) {
  using G = PassBGeom<n, double>;
  ProCols<double, 3> pro;
  for (int c = 0; c < 3; ++c) pro.x[c] = x + c * NF;
  FAME_TRY((launch_passA<n, double, 3>(pro, work, NF, st, Gate{nullptr})));
  const size_t smem = (size_t)G::stage * sizeof(double2);
  static int attr = ensure_smem(k_passB_inv<n, double>, smem);
  if (attr != FAME_OK) return attr;
  k_passB_inv<n, double><<<dim3(G::n3 / G::TT, 3), G::threads, smem, st>>>(work, NF);
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
template <typename T> const T* et_of(fame_mass* m);
template <> const double* et_of<double>(fame_mass* m) { return m->Et64; }
template <> const float* et_of<float>(fame_mass* m) { return m->Et32; }

// mode dispatch on a typed pointer pair
template <typename T>
int mass_apply_typed(fame_mass* m, int mode, const C<T>* x, C<T>* y, int nrhs) {
  const long long NF = m->NF;
  cudaStream_t st = m->ctx->stream;
  const T* Et = et_of<T>(m);
  C<T>* work = reinterpret_cast<C<T>*>(m->work);
  switch (mode) {
    case FAME_MASS_SCALAR:
      return mass_scalar_cols<T>(m->n, NF, x, y, nrhs, Et, work, st);
    case FAME_MASS_FULL3:
      // 3NF x nrhs, column-major: each column holds three components
      return mass_scalar_cols<T>(m->n, NF, x, y, 3 * nrhs, Et, work, st);
    case FAME_MASS_COL3:
      for (int j = 0; j < nrhs; ++j) {
        C<T>* yj = y + 3LL * NF * j;
        FAME_CUDA_TRY(cudaMemsetAsync(yj, 0, 2 * NF * sizeof(C<T>), st));
        FAME_TRY(mass_scalar_cols<T>(m->n, NF, x + NF * j, yj + 2 * NF, 1, Et, work, st));
      }
      return FAME_OK;
    case FAME_MASS_COLS12:
      for (int j = 0; j < nrhs; ++j) {
        C<T>* yj = y + 3LL * NF * j;
        FAME_TRY(mass_scalar_cols<T>(m->n, NF, x + 2 * NF * j, yj, 2, Et, work, st));
        FAME_CUDA_TRY(cudaMemsetAsync(yj + 2 * NF, 0, NF * sizeof(C<T>), st));
      }
      return FAME_OK;
    default:
      return fail(FAME_ERR_INVALID, "unknown mass mode");
  }
}

// One-shot applyMij_fft with a caller's natural-order E: a temporary tiled E/NF.
template <typename T>
int apply_fft_raw(fame_ctx* ctx, int n, long long NF, const double* E, const C<T>* x, C<T>* y, int nrhs) {
  T* Et = nullptr;
  C<T>* work = nullptr;
  FAME_TRY(dalloc((void**)&Et, NF * sizeof(T)));
  int s = dalloc((void**)&work, NF * sizeof(C<T>));
  if (s == FAME_OK) s = tile_E<T>(E, n, NF, 1.0 / (double)NF, Et, ctx->stream);
  if (s == FAME_OK) s = mass_scalar_cols<T>(n, NF, x, y, nrhs, Et, work, ctx->stream);
  if (s == FAME_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) s = fail(FAME_ERR_CUDA, "applyMij_fft");
  dfree(Et);
  dfree(work);
  return s;
}

}  // namespace fame

using namespace fame;

extern "C" {

int fame_applyMij_fft(fame_ctx* ctx, int N, const double* E, const void* x, void* y, int nrhs,
                      int prec) {
  if (!ctx || !E || !x || !y || nrhs < 0) return fail(FAME_ERR_INVALID, "applyMij_fft arguments");
  FAME_TRY(check_N(N));
  const long long NF = grid_NF(N);
  if (prec == FAME_F64) return apply_fft_raw<double>(ctx, 2 * N, NF, E, (const double2*)x, (double2*)y, nrhs);
  if (prec == FAME_F32) return apply_fft_raw<float>(ctx, 2 * N, NF, E, (const float2*)x, (float2*)y, nrhs);
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
  int s = dalloc((void**)&m->Et64, m->NF * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&m->Et32, m->NF * sizeof(float));
  if (s == FAME_OK) s = dalloc(&m->work, m->NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&m->EtInv64, m->NF * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&m->EtInv32, m->NF * sizeof(float));
  const double scale = 1.0 / (double)m->NF;
  if (s == FAME_OK) s = tile_E<double>(E, m->n, m->NF, scale, m->Et64, ctx->stream);
  if (s == FAME_OK) s = tile_E<float>(E, m->n, m->NF, scale, m->Et32, ctx->stream);
  if (s == FAME_OK) s = tile_E<double>(E, m->n, m->NF, scale, m->EtInv64, ctx->stream, 1);
  if (s == FAME_OK) s = tile_E<float>(E, m->n, m->NF, scale, m->EtInv32, ctx->stream, 1);
  if (s != FAME_OK) {
    dfree(m->Et64);
    dfree(m->Et32);
    dfree(m->work);
    dfree(m->EtInv64);
    dfree(m->EtInv32);
    delete m;
    return s;
  }
  *out = m;
  return FAME_OK;
}

int fame_mass_destroy(fame_mass* m) {
  if (!m) return FAME_OK;
  cudaStreamSynchronize(m->ctx->stream);
  dfree(m->Et64);
  dfree(m->Et32);
  dfree(m->work);
  dfree(m->EtInv64);
  dfree(m->EtInv32);
  delete m;
  return FAME_OK;
}

int fame_selftest_bounded_wait(fame_mass* m, unsigned poll_limit) {
  if (!m) return fail(FAME_ERR_INVALID, "fame_selftest_bounded_wait: mass is NULL");
  if (poll_limit < 1 || poll_limit > (1u << 20)) return fail(FAME_ERR_INVALID, "poll_limit must be in [1, 2^20]");
  fame_ctx* ctx = m->ctx;
  FAME_TRY(check_fault(ctx));  // start from a clear fault word
  // one FP32 field in the handle's scratch (8 NF bytes of its 16 NF); every stage barrier
  // expects bytes that no copy delivers, so each CTA's first wait runs out and returns
  float2* w = reinterpret_cast<float2*>(m->work);
  const Gate g{nullptr};
  int s = FAME_OK;
  switch (m->n) {
    case 2: s = launch_passB<2, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
    case 4: s = launch_passB<4, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
    case 6: s = launch_passB<6, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
    case 8: s = launch_passB<8, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
    case 10: s = launch_passB<10, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
    case 12: s = launch_passB<12, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
    default: s = launch_passB<14, float, float>(w, 1, m->Et32, m->NF, ctx->stream, g, poll_limit, 1); break;
  }
  FAME_TRY(s);
  FAME_CUDA_TRY(cudaGetLastError());
  return check_fault(ctx);  // FAME_ERR_CUDA: the timeout was detected and reported
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
    k_adjoint_reduce<<<blocks, 256, 0, st>>>(work, NF, m->n, work_tt<double>(m->n), dEps, nparams,
                                             red + kMaxAdjParams, counter, red);
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
