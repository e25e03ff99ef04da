// The rank-1 lattice pieces of the Fourier mass block as their own entry points:
//   rank1_exact_fft_scatter  (exp1/rank1_exact_fft_scatter.m:1-13)
//     Xfft = fft(xEmbed), xEmbed = zeros(M) with xEmbed(inputIdx) = x
//   rank1_exact_ifft_gather  (exp1/rank1_exact_ifft_gather.m:1-11)
//     y = ifft(Yfft)(targetIdx)
// M = nGrid * B^(dim-1) (B = 2 nGrid - 1, exp1/build_radix_exact_rank1_plan_scalar.m:24-27),
// 24,760,990 at N = 5.  The length-M DFT is a mixed-radix Stockham transform: M is
// factored into radices R <= 27 (the plan's nGrid and B, e.g. 19^5 * 10), and each pass
// reads the array with stride M/R, twiddles, runs a register DFT of length R and writes
// in sorted order, ping-ponging between two arrays of M complex128 (one of them the
// caller's output).  Twiddles exp(+-2 pi i r k / (Ns R)) come from one sincospi per
// thread and complex powers of it.  The composed operator applyMij_rank1_exact runs on
// the algebraically identical 6D convolution instead (mass.cu); these entry points are
// for callers that use the lattice transform itself.
#include "fft6d.cuh"
#include "internal.cuh"

namespace fame {
namespace {

// radices a pass may use (descending: the factorisation takes the largest first)
constexpr int kRadices[] = {27, 23, 19, 16, 15, 14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
constexpr int kMaxPasses = 64;

// one Stockham pass of radix R over an array of M values: sub-transforms of length Ns
// so far become length Ns*R
template <int R, int SIGN>
__global__ void __launch_bounds__(256) k_stockham(const double2* __restrict__ in, double2* __restrict__ out,
                                                  long long M, long long Ns) {
  const long long T = M / R;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < T; j += (long long)gridDim.x * blockDim.x) {
    const long long k = j % Ns;
    double re[R], im[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double2 v = in[j + r * T];
      re[r] = v.x;
      im[r] = v.y;
    }
    if (Ns > 1) {  // x_r *= w^r, w = exp(SIGN 2 pi i k / (Ns R))
      double s, c;
      sincospi((double)(2 * k) / (double)(Ns * R), &s, &c);
      const double wr = c, wi = SIGN * s;
      double pr = wr, pi = wi;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const double xr = re[r], xi = im[r];
        re[r] = fmadd(xr, pr, -xi * pi);
        im[r] = fmadd(xr, pi, xi * pr);
        const double t = fmadd(pr, wr, -pi * wi);
        pi = fmadd(pr, wi, pi * wr);
        pr = t;
      }
    }
    Dft<R, SIGN, double>::run(re, im);
    const long long d = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[d + r * Ns] = make_double2(re[r], im[r]);
  }
}

// The first pass (Ns = 1): thread j's R outputs are the contiguous run [j R, j R + R), so a
// warp's direct stores would touch 32 separate segments.  The block's 128 R outputs form one
// contiguous run: they go through shared memory and leave with consecutive threads on
// consecutive addresses.
constexpr int kFirstThreads = 128;
template <int R, int SIGN>
__global__ void __launch_bounds__(kFirstThreads) k_stockham_first(const double2* __restrict__ in,
                                                                  double2* __restrict__ out, long long M) {
  extern __shared__ double2 stage[];  // [kFirstThreads * R]
  const long long T = M / R;
  for (long long j0 = blockIdx.x * (long long)kFirstThreads; j0 < T; j0 += (long long)gridDim.x * kFirstThreads) {
    const long long j = j0 + threadIdx.x;
    if (j < T) {
      double re[R], im[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double2 v = in[j + r * T];
        re[r] = v.x;
        im[r] = v.y;
      }
      Dft<R, SIGN, double>::run(re, im);
#pragma unroll
      for (int r = 0; r < R; ++r) stage[threadIdx.x * R + r] = make_double2(re[r], im[r]);
    }
    __syncthreads();
    const long long base = j0 * R, len = (T - j0 < kFirstThreads ? T - j0 : kFirstThreads) * R;
    for (int t = threadIdx.x; t < len; t += kFirstThreads) out[base + t] = stage[t];
    __syncthreads();  // the stage is rewritten by the next chunk
  }
}

// emb (M) = 0 except emb[inputIdx[i] - 1] = x[i]; bad index -> flag (the write is skipped)
__global__ void k_rank1_scatter(const double2* __restrict__ x, const uint32_t* __restrict__ idx, long long NF,
                                long long M, double2* __restrict__ emb, unsigned* bad) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    const long long t = (long long)idx[i] - 1;
    if (t < 0 || t >= M) {
      atomicOr(bad, 1u);
      continue;
    }
    emb[t] = x[i];
  }
}

// y[i] = Y[targetIdx[i] - 1] / M
__global__ void k_rank1_gather(const double2* __restrict__ Y, const uint32_t* __restrict__ idx, long long NF,
                               long long M, double2* __restrict__ y, unsigned* bad) {
  const double s = 1.0 / (double)M;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    const long long t = (long long)idx[i] - 1;
    if (t < 0 || t >= M) {
      atomicOr(bad, 1u);
      y[i] = make_double2(0.0, 0.0);
      continue;
    }
    const double2 v = Y[t];
    y[i] = make_double2(v.x * s, v.y * s);
  }
}

int factor(long long M, int* rad) {
  int np = 0;
  while (M > 1) {
    int r = 0;
    for (int c : kRadices)
      if (M % c == 0) {
        r = c;
        break;
      }
    if (r == 0 || np == kMaxPasses) return -1;
    rad[np++] = r;
    M /= r;
  }
  return np;
}

template <int SIGN, int I = 0>
int launch_pass(int R, const double2* in, double2* out, long long M, long long Ns, cudaStream_t s) {
  if constexpr (I < (int)(sizeof(kRadices) / sizeof(int))) {
    constexpr int RR = kRadices[I];
    if (R != RR) return launch_pass<SIGN, I + 1>(R, in, out, M, Ns, s);
    const long long T = M / RR;
    if (Ns == 1) {
      constexpr size_t smem = (size_t)kFirstThreads * RR * sizeof(double2);
      static int attr = cudaFuncSetAttribute(k_stockham_first<RR, SIGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem) == cudaSuccess
                            ? FAME_OK
                            : fail(FAME_ERR_CUDA, "rank-1 FFT: shared-memory limit");
      FAME_TRY(attr);
      const int blocks = (int)std::min<long long>((T + kFirstThreads - 1) / kFirstThreads, (long long)num_sms() * 8);
      k_stockham_first<RR, SIGN><<<blocks, kFirstThreads, smem, s>>>(in, out, M);
    } else {
      const int blocks = (int)std::min<long long>((T + 255) / 256, (long long)num_sms() * 8);
      k_stockham<RR, SIGN><<<blocks, 256, 0, s>>>(in, out, M, Ns);
    }
    ::fame::count_launch();
    FAME_CUDA_TRY(cudaGetLastError());
    return FAME_OK;
  } else {
    return fail(FAME_ERR_UNSUPPORTED, "rank-1 FFT radix");
  }
}

// DFT of length M (SIGN -1: fft, +1: ifft without 1/M) of src into dst: the passes
// alternate between dst and tmp so that the last one writes dst.  Only the first pass
// reads src; src may be dst when the pass count is even (the first pass writes tmp).
int stockham(const int* rad, int np, int SIGN, const double2* src, double2* dst, double2* tmp, long long M,
             cudaStream_t s) {
  const double2* in = src;
  long long Ns = 1;
  for (int p = 0; p < np; ++p) {
    double2* out = ((np - 1 - p) % 2 == 0) ? dst : tmp;
    FAME_TRY(SIGN < 0 ? launch_pass<-1>(rad[p], in, out, M, Ns, s) : launch_pass<+1>(rad[p], in, out, M, Ns, s));
    in = out;
    Ns *= rad[p];
  }
  return FAME_OK;
}

int check_args(fame_ctx* ctx, const void* idx, long long NF, long long M, const void* a, const void* b, int nrhs,
               int* rad, int* np) {
  if (!ctx || !idx || !a || !b || nrhs < 0 || NF <= 0 || M < NF) return fail(FAME_ERR_INVALID, "rank-1 FFT arguments");
  *np = factor(M, rad);
  if (*np < 0) return fail(FAME_ERR_UNSUPPORTED, "rank-1 FFT: M has a prime factor above 27");
  return FAME_OK;
}

int read_flag(fame_ctx* ctx, unsigned* bad, const char* what) {
  unsigned h = 0;
  FAME_TRY(read_back(ctx, bad, &h, sizeof(h)));
  if (h) return fail(FAME_ERR_INVALID, what);
  return FAME_OK;
}

}  // namespace
}  // namespace fame

using namespace fame;

extern "C" {

int fame_rank1_exact_fft_scatter(fame_ctx* ctx, const void* x, int nrhs, const uint32_t* inputIdx, long long NF,
                                 long long M, void* Xfft) {
  int rad[kMaxPasses], np = 0;
  FAME_TRY(check_args(ctx, inputIdx, NF, M, x, Xfft, nrhs, rad, &np));
  if (nrhs == 0) return FAME_OK;
  void* ws = nullptr;
  FAME_TRY(ctx_workspace(ctx, (size_t)M * sizeof(double2) + 256, &ws));
  double2* tmp = static_cast<double2*>(ws);
  unsigned* bad = reinterpret_cast<unsigned*>(static_cast<char*>(ws) + (size_t)M * sizeof(double2));
  cudaStream_t s = ctx->stream;
  FAME_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned), s));
  const int eb = (int)std::min<long long>((NF + 255) / 256, (long long)num_sms() * 8);
  for (int c = 0; c < nrhs; ++c) {
    double2* X = static_cast<double2*>(Xfft) + (size_t)c * M;
    // the embedding starts in X when the pass count is even (the first pass then writes
    // tmp), in tmp when it is odd (the first pass then writes X)
    double2* emb = (np % 2 == 1) ? tmp : X;
    FAME_CUDA_TRY(cudaMemsetAsync(emb, 0, (size_t)M * sizeof(double2), s));
    k_rank1_scatter<<<eb, 256, 0, s>>>(static_cast<const double2*>(x) + (size_t)c * NF, inputIdx, NF, M, emb, bad);
    ::fame::count_launch();
    FAME_CUDA_TRY(cudaGetLastError());
    FAME_TRY(stockham(rad, np, -1, emb, X, tmp, M, s));
  }
  return read_flag(ctx, bad, "rank1_exact_fft_scatter: inputIdx outside [1, M]");
}

int fame_rank1_exact_ifft_gather(fame_ctx* ctx, const void* Yfft, int nrhs, const uint32_t* targetIdx, long long NF,
                                 long long M, void* y) {
  int rad[kMaxPasses], np = 0;
  FAME_TRY(check_args(ctx, targetIdx, NF, M, Yfft, y, nrhs, rad, &np));
  if (nrhs == 0) return FAME_OK;
  void* ws = nullptr;
  FAME_TRY(ctx_workspace(ctx, 2 * (size_t)M * sizeof(double2) + 256, &ws));
  double2* t0 = static_cast<double2*>(ws);
  double2* t1 = t0 + M;
  unsigned* bad = reinterpret_cast<unsigned*>(t1 + M);
  cudaStream_t s = ctx->stream;
  FAME_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(unsigned), s));
  const int eb = (int)std::min<long long>((NF + 255) / 256, (long long)num_sms() * 8);
  for (int c = 0; c < nrhs; ++c) {
    // the caller's spectrum is only read: the passes alternate between t0 and t1, the last in t0
    const double2* Yc = static_cast<const double2*>(Yfft) + (size_t)c * M;
    FAME_TRY(stockham(rad, np, +1, Yc, t0, t1, M, s));
    k_rank1_gather<<<eb, 256, 0, s>>>(np > 0 ? t0 : Yc, targetIdx, NF, M, static_cast<double2*>(y) + (size_t)c * NF,
                                      bad);
    ::fame::count_launch();
    FAME_CUDA_TRY(cudaGetLastError());
  }
  return read_flag(ctx, bad, "rank1_exact_ifft_gather: targetIdx outside [1, M]");
}

}  // extern "C"
