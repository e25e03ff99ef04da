// Yee-field reconstruction of a Fourier eigenvector component,
//   u(r) = sum_j c_j exp(i q_j . r)                (exp2/reconstruct_field_direct_blocked_exp3.m:8-15)
// and its multi-center Taylor approximation
//   u(r) ~ sum_{|a|<=p} gamma_a(r_c) (r - r_c)^a,
//   gamma_a(r_c) = i^|a|/a! sum_j c_j exp(i q_j . r_c) q_j^a   (exp2/taylor_on_blocks_exp3.m:1-79)
//
// Three device paths:
//  * k_direct_sum: the plain sum for any cut matrix (FP64 sincos per term);
//  * the factorised sum for an axis-block cut matrix P = [diag(d1); diag(d2)]
//    and points on a tensor grid: q_x depends only on (xi_1, xi_4), q_y on
//    (xi_2, xi_5), q_z on (xi_3, xi_6), so u = C x1 Ex x2 Ey x3 Ez is three
//    complex GEMMs against per-axis phase tables (exact in exact arithmetic);
//  * the Taylor moments (one CTA per mode chunk and center, one thread per
//    multi-index) and the per-block polynomial evaluation.
#include <algorithm>
#include <cmath>
#include <vector>
#include "internal.cuh"

namespace fame {

static inline int rblocks(long long n, int t = 256) { return (int)std::min<long long>((n + t - 1) / t, 148 * 32); }

// ------------------------------------------------------------------ direct
constexpr int kDirectPts = 128;
constexpr int kDirectModes = 256;
__global__ void __launch_bounds__(kDirectPts) k_direct_sum(const double2* __restrict__ c, const double* __restrict__ Q,
                                                          long long NF, const double* __restrict__ R, long long M,
                                                          double2* __restrict__ u) {
  __shared__ double sq[3][kDirectModes];
  __shared__ double2 sc[kDirectModes];
  const long long i = (long long)blockIdx.x * kDirectPts + threadIdx.x;
  const bool act = i < M;
  const double rx = act ? R[i] : 0.0, ry = act ? R[M + i] : 0.0, rz = act ? R[2 * M + i] : 0.0;
  double ar = 0.0, ai = 0.0;
  for (long long j0 = 0; j0 < NF; j0 += kDirectModes) {
    const int nj = (int)std::min<long long>(kDirectModes, NF - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < nj; t += blockDim.x) {
      sq[0][t] = Q[j0 + t];
      sq[1][t] = Q[NF + j0 + t];
      sq[2][t] = Q[2 * NF + j0 + t];
      sc[t] = c[j0 + t];
    }
    __syncthreads();
    if (act) {
      for (int t = 0; t < nj; ++t) {
        double s, co;
        sincos(sq[0][t] * rx + sq[1][t] * ry + sq[2][t] * rz, &s, &co);
        ar += sc[t].x * co - sc[t].y * s;
        ai += sc[t].x * s + sc[t].y * co;
      }
    }
  }
  if (act) u[i] = make_double2(ar, ai);
}

// -------------------------------------------------------------- factorised
// phase table T[x + nx*a] = exp(i q(a) xs[x]),  a = j_lo + n j_hi,
// q(a) = d1 (xi(j_lo) + k_lo) + d2 (xi(j_hi) + k_hi)
__global__ void k_phase_table(const double* xs, int nx, int N, double d1, double k1, double d2, double k2,
                              double2* T) {
  const int n = 2 * N, n2 = n * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nx * n2;
       t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % nx), a = (int)(t / nx);
    const int jl = a % n, jh = a / n;
    const double xl = (jl < N ? jl : jl - n) + k1, xh = (jh < N ? jh : jh - n) + k2;
    double s, c;
    sincos((d1 * xl + d2 * xh) * xs[x], &s, &c);
    T[t] = make_double2(c, s);
  }
}

// Cp[a + n^2 (b + n^2 c)] = coeff[j1 + n j2 + n^2 j3 + n^3 j4 + n^4 j5 + n^5 j6]
// with a = j1 + n j4, b = j2 + n j5, c = j3 + n j6
__global__ void k_pair_permute(const double2* coeff, int n, double2* Cp) {
  const long long n2 = (long long)n * n, NF = n2 * n2 * n2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF; i += (long long)gridDim.x * blockDim.x) {
    long long t = i;
    int j[6];
    for (int d = 0; d < 6; ++d) {
      j[d] = (int)(t % n);
      t /= n;
    }
    const long long a = j[0] + n * j[3], b = j[1] + n * j[4], c = j[2] + n * j[5];
    Cp[a + n2 * (b + n2 * c)] = coeff[i];
  }
}

// Batched complex GEMM C(m,n) = sum_k A(m,k) B(k,n) with element strides, FP64.
// 16 x 16 threads; each thread owns RM x RN outputs (rows tx + 16 a, columns ty + 16 b), so
// a CTA covers (16 RM) x (16 RN); the tile shape follows the GEMM's shape (zgemm).  k runs in
// tiles of 8 through two shared-memory buffers: the global loads of tile t + 1 are issued
// before the products of tile t, and each operand is read along whichever of its two
// dimensions is contiguous in memory.
struct GemmArgs {
  const double2* A;
  const double2* B;
  double2* C;
  int M, N, K;
  long long sam, sak, sbk, sbn, scm, scn;
  long long bA, bB, bC;  // batch strides (blockIdx.z)
  int bdivB = 1;         // B advances by bB every bdivB batch entries
};
constexpr int kGKT = 8;
template <int RM, int RN>
__global__ void __launch_bounds__(256) k_zgemm(GemmArgs g) {
  constexpr int TM = 16 * RM, TN = 16 * RN;
  constexpr int AE = TM * kGKT / 256, BE = TN * kGKT / 256;  // elements per thread and k tile
  static_assert(AE * 256 == TM * kGKT && BE * 256 == TN * kGKT, "tile loads divide over the threads");
  __shared__ double2 As[2][kGKT][TM + 1];
  __shared__ double2 Bs[2][kGKT][TN + 1];
  const double2* A = g.A + g.bA * blockIdx.z;
  const double2* B = g.B + g.bB * (blockIdx.z / g.bdivB);
  double2* Cm = g.C + g.bC * blockIdx.z;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const bool aMfast = g.sam == 1, bNfast = g.sbn == 1;
  // element e of this thread in the A (TM x 8) and B (8 x TN) tiles
  auto a_at = [&](int e, int& mm, int& kk) {
    const int t = threadIdx.x + 256 * e;
    mm = aMfast ? t % TM : t / kGKT;
    kk = aMfast ? t / TM : t % kGKT;
  };
  auto b_at = [&](int e, int& nn, int& kk) {
    const int t = threadIdx.x + 256 * e;
    nn = bNfast ? t % TN : t / kGKT;
    kk = bNfast ? t / TN : t % kGKT;
  };
  double2 ra[AE], rb[BE];
  auto load = [&](int k0) {
#pragma unroll
    for (int e = 0; e < AE; ++e) {
      int mm, kk;
      a_at(e, mm, kk);
      const int m = m0 + mm, k = k0 + kk;
      ra[e] = (m < g.M && k < g.K) ? A[m * g.sam + k * g.sak] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int e = 0; e < BE; ++e) {
      int nn, kk;
      b_at(e, nn, kk);
      const int n = n0 + nn, k = k0 + kk;
      rb[e] = (n < g.N && k < g.K) ? B[k * g.sbk + n * g.sbn] : make_double2(0.0, 0.0);
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int e = 0; e < AE; ++e) {
      int mm, kk;
      a_at(e, mm, kk);
      As[buf][kk][mm] = ra[e];
    }
#pragma unroll
    for (int e = 0; e < BE; ++e) {
      int nn, kk;
      b_at(e, nn, kk);
      Bs[buf][kk][nn] = rb[e];
    }
  };
  double2 acc[RM][RN];
#pragma unroll
  for (int a = 0; a < RM; ++a)
#pragma unroll
    for (int b = 0; b < RN; ++b) acc[a][b] = make_double2(0.0, 0.0);
  load(0);
  stash(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < g.K; k0 += kGKT) {
    const bool more = k0 + kGKT < g.K;
    if (more) load(k0 + kGKT);
#pragma unroll
    for (int kk = 0; kk < kGKT; ++kk) {
      double2 a[RM], b[RN];
#pragma unroll
      for (int q = 0; q < RM; ++q) a[q] = As[buf][kk][tx + 16 * q];
#pragma unroll
      for (int q = 0; q < RN; ++q) b[q] = Bs[buf][kk][ty + 16 * q];
#pragma unroll
      for (int qa = 0; qa < RM; ++qa)
#pragma unroll
        for (int qb = 0; qb < RN; ++qb) {
          acc[qa][qb].x = fma(a[qa].x, b[qb].x, fma(-a[qa].y, b[qb].y, acc[qa][qb].x));
          acc[qa][qb].y = fma(a[qa].x, b[qb].y, fma(a[qa].y, b[qb].x, acc[qa][qb].y));
        }
    }
    if (more) stash(buf ^ 1);  // buffer buf ^ 1 was last read before the previous barrier
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int qa = 0; qa < RM; ++qa)
#pragma unroll
    for (int qb = 0; qb < RN; ++qb) {
      const int m = m0 + tx + 16 * qa, n = n0 + ty + 16 * qb;
      if (m < g.M && n < g.N) Cm[m * g.scm + n * g.scn] = acc[qa][qb];
    }
}

template <int RM, int RN> int zgemm_t(const GemmArgs& g, int batch, cudaStream_t s) {
  dim3 grid((g.M + 16 * RM - 1) / (16 * RM), (g.N + 16 * RN - 1) / (16 * RN), batch);
  if (grid.y > 65535) return fail(FAME_ERR_UNSUPPORTED, "zgemm: N too large");
  k_zgemm<RM, RN><<<grid, 256, 0, s>>>(g);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

// 64-wide tiles along a dimension of 256 or more, 32-wide otherwise (the factorised
// direct sum's GEMMs: T1 = 83 x 10^4, T2 = 83 x 83 batched, u = 6889 x 83 at n = 40, N = 5)
int zgemm(const GemmArgs& g, int batch, cudaStream_t s) {
  const bool wm = g.M >= 256, wn = g.N >= 256;
  if (wm && wn) return zgemm_t<4, 4>(g, batch, s);
  if (wm) return zgemm_t<4, 2>(g, batch, s);
  if (wn) return zgemm_t<2, 4>(g, batch, s);
  return zgemm_t<2, 2>(g, batch, s);
}

// ------------------------------------------------------------------ Taylor
// centers: per block the midpoint of the bounding box of its points
__global__ void k_block_centers(const double* R, long long M, const long long* ptr, const long long* ids,
                                const double* fixed, double* centers) {
  __shared__ double mn[3][256], mx[3][256];
  const int b = blockIdx.x;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (long long t = ptr[b] + threadIdx.x; t < ptr[b + 1]; t += blockDim.x) {
    const long long i = ids[t];
    for (int d = 0; d < 3; ++d) {
      lo[d] = fmin(lo[d], R[d * M + i]);
      hi[d] = fmax(hi[d], R[d * M + i]);
    }
  }
  for (int d = 0; d < 3; ++d) {
    mn[d][threadIdx.x] = lo[d];
    mx[d][threadIdx.x] = hi[d];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int d = 0; d < 3; ++d) {
        mn[d][threadIdx.x] = fmin(mn[d][threadIdx.x], mn[d][threadIdx.x + s]);
        mx[d][threadIdx.x] = fmax(mx[d][threadIdx.x], mx[d][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) centers[3 * b + d] = fixed ? fixed[d] : 0.5 * (mn[d][0] + mx[d][0]);
}

constexpr int kTaySub = 64;     // modes staged per sub-chunk
constexpr int kTayChunk = 4096; // modes per CTA
constexpr int kMaxP = 12;
// partial[(chunk * nB + b) * L + alpha] = sum_{j in chunk} c_j e^{i q_j.r_c} q_j^alpha
__global__ void __launch_bounds__(512) k_taylor_moments(const double2* __restrict__ c, const double* __restrict__ Q,
                                                       long long NF, const double* __restrict__ centers,
                                                       const int* __restrict__ alist, int L, int p, int nB,
                                                       double2* __restrict__ partial) {
  __shared__ double2 w[kTaySub];
  __shared__ double pw[3][kTaySub][kMaxP + 1];
  const int chunk = blockIdx.x, b = blockIdx.y;
  const double cx = centers[3 * b], cy = centers[3 * b + 1], cz = centers[3 * b + 2];
  const int al = threadIdx.x;
  const bool act = al < L;
  const int a1 = act ? alist[3 * al] : 0, a2 = act ? alist[3 * al + 1] : 0, a3 = act ? alist[3 * al + 2] : 0;
  double ar = 0.0, ai = 0.0;
  const long long j0c = (long long)chunk * kTayChunk;
  const long long j1c = std::min<long long>(NF, j0c + kTayChunk);
  for (long long j0 = j0c; j0 < j1c; j0 += kTaySub) {
    const int nj = (int)std::min<long long>(kTaySub, j1c - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < nj; t += blockDim.x) {
      const long long j = j0 + t;
      const double qx = Q[j], qy = Q[NF + j], qz = Q[2 * NF + j];
      double s, co;
      sincos(qx * cx + qy * cy + qz * cz, &s, &co);
      const double2 cj = c[j];
      w[t] = make_double2(cj.x * co - cj.y * s, cj.x * s + cj.y * co);
      double px = 1.0, py = 1.0, pz = 1.0;
      for (int k = 0; k <= p; ++k) {
        pw[0][t][k] = px;
        pw[1][t][k] = py;
        pw[2][t][k] = pz;
        px *= qx;
        py *= qy;
        pz *= qz;
      }
    }
    __syncthreads();
    if (act) {
      for (int t = 0; t < nj; ++t) {
        const double mono = pw[0][t][a1] * pw[1][t][a2] * pw[2][t][a3];
        ar += w[t].x * mono;
        ai += w[t].y * mono;
      }
    }
  }
  if (act) partial[((long long)chunk * nB + b) * L + al] = make_double2(ar, ai);
}

// gamma[b*L + a] = coef[a] * sum_chunks partial (fixed order)
__global__ void k_taylor_reduce(const double2* partial, int nChunks, int nB, int L, const double2* coef,
                                double2* gamma) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nB * L) return;
  double ar = 0.0, ai = 0.0;
  for (int ch = 0; ch < nChunks; ++ch) {
    const double2 v = partial[(long long)ch * nB * L + t];
    ar += v.x;
    ai += v.y;
  }
  const double2 cf = coef[t % L];
  gamma[t] = make_double2(cf.x * ar - cf.y * ai, cf.x * ai + cf.y * ar);
}

// u(ids[t]) = sum_a gamma[b, a] (r - r_c)^a for the block's points
__global__ void __launch_bounds__(256) k_taylor_eval(const double* __restrict__ R, long long M,
                                                    const long long* __restrict__ ptr, const long long* __restrict__ ids,
                                                    const double* __restrict__ centers, const double2* __restrict__ gamma,
                                                    const int* __restrict__ alist, int L, int p, double2* __restrict__ u) {
  extern __shared__ double2 sg[];
  int* sa = reinterpret_cast<int*>(sg + L);
  const int b = blockIdx.y;
  for (int t = threadIdx.x; t < L; t += blockDim.x) {
    sg[t] = gamma[(long long)b * L + t];
    sa[3 * t] = alist[3 * t];
    sa[3 * t + 1] = alist[3 * t + 1];
    sa[3 * t + 2] = alist[3 * t + 2];
  }
  __syncthreads();
  const long long t = ptr[b] + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ptr[b + 1]) return;
  const long long i = ids[t];
  const double dx = R[i] - centers[3 * b], dy = R[M + i] - centers[3 * b + 1], dz = R[2 * M + i] - centers[3 * b + 2];
  double px[kMaxP + 1], py[kMaxP + 1], pz[kMaxP + 1];
  px[0] = py[0] = pz[0] = 1.0;
  for (int k = 1; k <= p; ++k) {
    px[k] = px[k - 1] * dx;
    py[k] = py[k - 1] * dy;
    pz[k] = pz[k - 1] * dz;
  }
  double ar = 0.0, ai = 0.0;
  for (int a = 0; a < L; ++a) {
    const double mono = px[sa[3 * a]] * py[sa[3 * a + 1]] * pz[sa[3 * a + 2]];
    ar += sg[a].x * mono;
    ai += sg[a].y * mono;
  }
  u[i] = make_double2(ar, ai);
}

}  // namespace fame

using namespace fame;

extern "C" {

int fame_reconstruct_direct(fame_ctx* ctx, const void* coeff, const double* qModes, long long NF,
                            const double* rPoints, long long M, void* u) {
  if (!ctx || !coeff || !qModes || !rPoints || !u || NF <= 0 || M < 0)
    return fail(FAME_ERR_INVALID, "reconstruct_direct arguments");
  if (M == 0) return FAME_OK;
  k_direct_sum<<<(int)((M + kDirectPts - 1) / kDirectPts), kDirectPts, 0, ctx->stream>>>(
      (const double2*)coeff, qModes, NF, rPoints, M, (double2*)u);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

// The factorised direct sum for ncomp components at once (component-stacked coeff, axes
// and u; equal grid sizes): each of the three GEMMs is one launch batched over the
// components (and, for the second, over its contraction slices), so the launches are
// ncomp times larger.  No host synchronisation: the results are ordered on the stream.
static int direct_grid_impl(fame_basis* bs, const void* coeff, int ncomp, const double* xs, int nx, const double* ys,
                            int ny, const double* zs, int nz, void* u, bool tc) {
  if (!bs || !coeff || !xs || !ys || !zs || !u || nx <= 0 || ny <= 0 || nz <= 0 || ncomp < 1 || ncomp > 3)
    return fail(FAME_ERR_INVALID, "reconstruct_direct_grid arguments");
  const double* P = bs->P;  // column-major 6 x 3
  for (int l = 0; l < 6; ++l)
    for (int c = 0; c < 3; ++c)
      if (l % 3 != c && P[c * 6 + l] != 0.0)
        return fail(FAME_ERR_UNSUPPORTED, "factorised reconstruction needs an axis-block cut matrix [diag; diag]");
  const int N = bs->N, n = 2 * N;
  const long long n2 = (long long)n * n, NF = bs->NF;
  if ((long long)ncomp * n2 > 65535) return fail(FAME_ERR_UNSUPPORTED, "reconstruct_direct_grid: too many slices");
  cudaStream_t s = bs->ctx->stream;
  // workspace pieces (per component, consecutive): phase tables, permuted coefficients,
  // two GEMM intermediates
  // 3xTF32 operand panels (zgemm_tc.cu): Tx (A of T1), Cp (B of T1), Ty (B of T2), Tz (B of
  // u), split together before T1; T1 (A of T2) and then T2 (A of u) share one region
  const int in2 = (int)n2;
  ZPanelJob jTx{nullptr, 1, nx, (long long)nx * n2, nx, in2, ncomp, true, 0, nullptr};
  ZPanelJob jCp{nullptr, n2, 1, NF, (int)(n2 * n2), in2, ncomp, false, (int)(n2 * n2), nullptr};
  ZPanelJob jTy{nullptr, 1, ny, (long long)ny * n2, ny, in2, ncomp, false, ny, nullptr};
  ZPanelJob jTz{nullptr, 1, nz, (long long)nz * n2, nz, in2, ncomp, false, nz, nullptr};
  ZPanelJob jT1{nullptr, 1, nx, (long long)nx * n2, nx, in2, ncomp * in2, true, 0, nullptr};
  ZPanelJob jT2{nullptr, 1, (long long)nx * ny, (long long)nx * ny * n2, nx * ny, in2, ncomp, true, 0, nullptr};
  const size_t pbig = tc ? std::max(zpanel_bytes(jT1), zpanel_bytes(jT2)) : 0;
  auto carve = [&](Carve& cv, double2** Tx, double2** Ty, double2** Tz, double2** Cp, double2** T1, double2** T2,
                   unsigned char** Pn) {
    *Tx = cv.take<double2>((size_t)ncomp * nx * n2);
    *Ty = cv.take<double2>((size_t)ncomp * ny * n2);
    *Tz = cv.take<double2>((size_t)ncomp * nz * n2);
    *Cp = cv.take<double2>((size_t)ncomp * NF);
    *T1 = cv.take<double2>((size_t)ncomp * nx * n2 * n2);
    *T2 = cv.take<double2>((size_t)ncomp * nx * ny * n2);
    if (tc) {  // panel buffers start on 1024-byte boundaries of the actual addresses (sizes
               // are multiples of 1024); the sizing pass reserves the largest padding
      const uintptr_t at = reinterpret_cast<uintptr_t>(cv.base) + cv.used;
      cv.used += cv.base ? (1024 - (at & 1023)) & 1023 : 1024;
      for (ZPanelJob* j : {&jTx, &jCp, &jTy, &jTz}) {
        j->out = cv.take<unsigned char>((zpanel_bytes(*j) + 1023) / 1024 * 1024);
      }
      *Pn = cv.take<unsigned char>(pbig);
    } else {
      *Pn = nullptr;
    }
  };
  double2 *Tx, *Ty, *Tz, *Cp, *T1, *T2;
  unsigned char* Pn;
  Carve size_only;
  carve(size_only, &Tx, &Ty, &Tz, &Cp, &T1, &T2, &Pn);
  void* ws = nullptr;
  int st = ctx_workspace(bs->ctx, size_only.used, &ws);
  Carve cv;
  cv.base = static_cast<char*>(ws);
  carve(cv, &Tx, &Ty, &Tz, &Cp, &T1, &T2, &Pn);
  const double* k = bs->info.kLift;
  if (st == FAME_OK) {
    for (int c = 0; c < ncomp; ++c) {
      k_phase_table<<<rblocks((long long)nx * n2), 256, 0, s>>>(xs + (long long)c * nx, nx, N, P[0], k[0], P[3], k[3],
                                                                Tx + (long long)c * nx * n2);
      k_phase_table<<<rblocks((long long)ny * n2), 256, 0, s>>>(ys + (long long)c * ny, ny, N, P[6 + 1], k[1], P[6 + 4],
                                                                k[4], Ty + (long long)c * ny * n2);
      k_phase_table<<<rblocks((long long)nz * n2), 256, 0, s>>>(zs + (long long)c * nz, nz, N, P[12 + 2], k[2],
                                                                P[12 + 5], k[5], Tz + (long long)c * nz * n2);
      k_pair_permute<<<rblocks(NF), 256, 0, s>>>((const double2*)coeff + (long long)c * NF, n, Cp + (long long)c * NF);
      ::fame::count_launch(4);
    }
    // T1[x, (b,c)] = sum_a Tx[x, a] Cp[a, (b,c)]                   (batched over components)
    GemmArgs g1{Tx, Cp, T1, nx, (int)(n2 * n2), (int)n2, 1, nx, 1, n2, 1, nx,
                (long long)nx * n2, NF, (long long)nx * n2 * n2};
    // T2[x, y, c] = sum_b T1[x, b, c] Ty[y, b]   (batched over components x c; Ty per component)
    GemmArgs g2{T1, Ty, T2, nx, ny, (int)n2, 1, nx, ny, 1, 1, nx, (long long)nx * n2, (long long)ny * n2,
                (long long)nx * ny, (int)n2};
    // u[(x,y), z] = sum_c T2[(x,y), c] Tz[z, c]                    (batched over components)
    GemmArgs g3{T2, Tz, (double2*)u, nx * ny, nz, (int)n2, 1, (long long)nx * ny, nz, 1, 1, (long long)nx * ny,
                (long long)nx * ny * n2, (long long)nz * n2, (long long)nx * ny * nz};
    const GemmArgs* gs[3] = {&g1, &g2, &g3};
    const int batches[3] = {ncomp, (int)(ncomp * n2), ncomp};
    if (!tc) {
      for (int t = 0; t < 3 && st == FAME_OK; ++t) st = zgemm(*gs[t], batches[t], s);
    } else {
      jTx.src = Tx;
      jCp.src = Cp;
      jTy.src = Ty;
      jTz.src = Tz;
      jT1.src = T1;
      jT2.src = T2;
      jT1.out = jT2.out = Pn;
      const ZPanelJob first[4] = {jTx, jCp, jTy, jTz};
      st = zsplit_panels(first, 4, s);
      if (st == FAME_OK)
        st = zgemm_3xtf32_panels(jTx.out, jCp.out, T1, g1.M, g1.N, g1.K, g1.scm, g1.scn, g1.bC, ncomp, 1, s);
      if (st == FAME_OK) st = zsplit_panels(&jT1, 1, s);
      if (st == FAME_OK)
        st = zgemm_3xtf32_panels(Pn, jTy.out, T2, g2.M, g2.N, g2.K, g2.scm, g2.scn, g2.bC, ncomp * in2, in2, s);
      if (st == FAME_OK) st = zsplit_panels(&jT2, 1, s);
      if (st == FAME_OK)
        st = zgemm_3xtf32_panels(Pn, jTz.out, (double2*)u, g3.M, g3.N, g3.K, g3.scm, g3.scn, g3.bC, ncomp, 1, s);
    }
  }
  return st;
}

int fame_reconstruct_direct_grid(fame_basis* bs, const void* coeff, const double* xs, int nx, const double* ys, int ny,
                                 const double* zs, int nz, void* u) {
  return direct_grid_impl(bs, coeff, 1, xs, nx, ys, ny, zs, nz, u, false);
}

int fame_reconstruct_direct_grid_3xtf32(fame_basis* bs, const void* coeff, const double* xs, int nx, const double* ys,
                                        int ny, const double* zs, int nz, void* u) {
  return direct_grid_impl(bs, coeff, 1, xs, nx, ys, ny, zs, nz, u, true);
}

int fame_reconstruct_direct_grid_fields(fame_basis* bs, const void* coeff, int ncomp, const double* xs, int nx,
                                        const double* ys, int ny, const double* zs, int nz, int tensor_cores,
                                        void* u) {
  return direct_grid_impl(bs, coeff, ncomp, xs, nx, ys, ny, zs, nz, u, tensor_cores != 0);
}

}  // extern "C"

namespace fame {

// Multi-center Taylor reconstruction (exp2/taylor_on_blocks_exp3.m:1-97); the block
// moments either in FP64 on the CUDA cores or as 3xTF32 products on the tensor cores
// (taylor_tc.cu).
// Whether the nB centers (x, y, z per block) form a tensor grid in block order
// b = i + m1 (j + m2 k) with axis values X[i], Y[j], Z[k] (exact equality); on success
// grid.m1..m3 are set and ax = [X, Y, Z].
static bool tensor_grid_of(const std::vector<double>& c, int nB, TaylorTcGrid& grid, std::vector<double>& ax) {
  int m1 = 1, m2 = 1;
  while (m1 < nB && c[3 * m1 + 1] == c[1] && c[3 * m1 + 2] == c[2]) ++m1;
  while (m1 * m2 < nB && c[3 * (m1 * m2) + 2] == c[2]) ++m2;
  if (nB % (m1 * m2) != 0) return false;
  const int m3 = nB / (m1 * m2);
  if (m1 + m2 + m3 > kTaylorTcMaxAxis) return false;
  for (int b = 0; b < nB; ++b) {
    const int i = b % m1, j = (b / m1) % m2, k = b / (m1 * m2);
    if (c[3 * b] != c[3 * i] || c[3 * b + 1] != c[3 * (m1 * j) + 1] || c[3 * b + 2] != c[3 * (m1 * m2 * k) + 2])
      return false;
  }
  ax.clear();
  for (int i = 0; i < m1; ++i) ax.push_back(c[3 * i]);
  for (int j = 0; j < m2; ++j) ax.push_back(c[3 * (m1 * j) + 1]);
  for (int k = 0; k < m3; ++k) ax.push_back(c[3 * (m1 * m2 * k) + 2]);
  grid.m1 = m1;
  grid.m2 = m2;
  grid.m3 = m3;
  return true;
}

static int taylor_impl(fame_ctx* ctx, const void* coeff, const double* qModes, long long NF, const double* rPoints,
                       long long M, int p, const long long* blockPtr, const long long* blockIds, int nBlocks,
                       const double* fixedCenter, void* u, bool tc) {
  if (!ctx || !coeff || !qModes || !rPoints || !u || !blockPtr || !blockIds || NF <= 0 || M < 0 ||
      nBlocks < 1)
    return fail(FAME_ERR_INVALID, "taylor_on_blocks arguments");
  if (p < 0 || p > kMaxP) return fail(FAME_ERR_UNSUPPORTED, "Taylor order must be in [0,12]");
  // multi-indices |a| <= p, a1 outer, a3 inner (exp2/build_multi_index_list_3d_exp3.m:3-14)
  std::vector<int> al;
  std::vector<double2> cf;
  for (int a1 = 0; a1 <= p; ++a1)
    for (int a2 = 0; a2 <= p - a1; ++a2)
      for (int a3 = 0; a3 <= p - a1 - a2; ++a3) {
        al.push_back(a1);
        al.push_back(a2);
        al.push_back(a3);
        const int s = a1 + a2 + a3;
        const double mag = std::exp(-(std::lgamma(a1 + 1.0) + std::lgamma(a2 + 1.0) + std::lgamma(a3 + 1.0)));
        const double re[4] = {1, 0, -1, 0}, im[4] = {0, 1, 0, -1};  // i^s
        cf.push_back(make_double2(mag * re[s % 4], mag * im[s % 4]));
      }
  const int L = (int)cf.size();
  if (L > 512) return fail(FAME_ERR_UNSUPPORTED, "too many Taylor terms");
  const int nChunks = (int)((NF + kTayChunk - 1) / kTayChunk);
  const TaylorTcPlan tp = tc ? taylor_tc_plan(NF, nBlocks, L, p) : TaylorTcPlan{};
  std::vector<int> packed, tcol;
  if (tc) {
    for (int a = 0; a < L; ++a) packed.push_back(al[3 * a] | al[3 * a + 1] << 8 | al[3 * a + 2] << 16);
    tcol.resize(tp.Npad);
    taylor_tc_columns(tp, al.data(), L, p, tcol.data());
  }
  cudaStream_t s = ctx->stream;
  int *dal, *dpk, *dcol;
  double2 *dcf, *partial, *gamma;
  double *centers, *dfix, *dax;
  float* tout;
  auto carve = [&](Carve& cv) {
    dal = cv.take<int>(al.size());
    dpk = cv.take<int>(tc ? packed.size() : 1);
    dcol = cv.take<int>(tc ? tcol.size() : 1);
    dcf = cv.take<double2>(cf.size());
    partial = cv.take<double2>(tc ? 1 : (size_t)nChunks * nBlocks * L);
    gamma = cv.take<double2>((size_t)nBlocks * L);
    centers = cv.take<double>((size_t)nBlocks * 3);
    dfix = cv.take<double>(3);
    dax = cv.take<double>(kTaylorTcMaxAxis);
    tout = cv.take<float>(tc ? tp.out_floats : 1);
  };
  Carve size_only;
  carve(size_only);
  void* ws = nullptr;
  int st = ctx_workspace(ctx, size_only.used, &ws);
  Carve cv;
  cv.base = static_cast<char*>(ws);
  carve(cv);
  if (!fixedCenter) dfix = nullptr;
  if (st == FAME_OK) {
    cudaMemcpyAsync(dal, al.data(), al.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dcf, cf.data(), cf.size() * sizeof(double2), cudaMemcpyHostToDevice, s);
    if (fixedCenter) cudaMemcpyAsync(dfix, fixedCenter, 3 * sizeof(double), cudaMemcpyHostToDevice, s);
    k_block_centers<<<nBlocks, 256, 0, s>>>(rPoints, M, blockPtr, blockIds, dfix, centers);
    ::fame::count_launch();
    if (!tc) {
      dim3 gm(nChunks, nBlocks);
      k_taylor_moments<<<gm, std::max(32, (L + 31) / 32 * 32), 0, s>>>((const double2*)coeff, qModes, NF, centers,
                                                                       dal, L, p, nBlocks, partial);
      ::fame::count_launch();
      k_taylor_reduce<<<(nBlocks * L + 255) / 256, 256, 0, s>>>(partial, nChunks, nBlocks, L, dcf, gamma);
      ::fame::count_launch();
    } else {
      cudaMemcpyAsync(dpk, packed.data(), packed.size() * sizeof(int), cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(dcol, tcol.data(), tcol.size() * sizeof(int), cudaMemcpyHostToDevice, s);
      // centers on a tensor grid (the Yee block partition's are): the moment kernel then
      // factorises the phases per axis
      TaylorTcGrid grid;
      std::vector<double> hc((size_t)nBlocks * 3), hax;
      if (cudaMemcpyAsync(hc.data(), centers, hc.size() * sizeof(double), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
          cudaStreamSynchronize(s) == cudaSuccess && tensor_grid_of(hc, nBlocks, grid, hax)) {
        cudaMemcpyAsync(dax, hax.data(), hax.size() * sizeof(double), cudaMemcpyHostToDevice, s);
        grid.ax = dax;
      }
      cudaGetLastError();
      st = taylor_moments_tc(tp, s, (const double2*)coeff, qModes, NF, centers, nBlocks, dpk, dcol, L, p, dcf, tout,
                             gamma, grid);
    }
    // one grid column per block; x-extent covers the largest block
    std::vector<long long> hp(nBlocks + 1);
    cudaMemcpyAsync(hp.data(), blockPtr, (nBlocks + 1) * sizeof(long long), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && st == FAME_OK) st = fail(FAME_ERR_CUDA, "taylor sync");
    long long maxPts = 0;
    for (int b = 0; b < nBlocks && st == FAME_OK; ++b) maxPts = std::max(maxPts, hp[b + 1] - hp[b]);
    if (st == FAME_OK && maxPts > 0) {
      dim3 ge((unsigned)((maxPts + 255) / 256), nBlocks);
      const size_t smem = L * sizeof(double2) + 3 * L * sizeof(int);
      k_taylor_eval<<<ge, 256, smem, s>>>(rPoints, M, blockPtr, blockIds, centers, gamma, dal, L, p,
                                          (double2*)u);
      ::fame::count_launch();
    }
    if (st == FAME_OK && cudaGetLastError() != cudaSuccess) st = fail(FAME_ERR_CUDA, "taylor launch");
    if (st == FAME_OK && cudaStreamSynchronize(s) != cudaSuccess) st = fail(FAME_ERR_CUDA, "taylor sync");
  }
  return st;
}

}  // namespace fame

extern "C" {

int fame_taylor_on_blocks(fame_ctx* ctx, const void* coeff, const double* qModes, long long NF,
                          const double* rPoints, long long M, int p, const long long* blockPtr,
                          const long long* blockIds, int nBlocks, const double* fixedCenter, void* u) {
  return taylor_impl(ctx, coeff, qModes, NF, rPoints, M, p, blockPtr, blockIds, nBlocks, fixedCenter, u, false);
}

int fame_taylor_on_blocks_3xtf32(fame_ctx* ctx, const void* coeff, const double* qModes, long long NF,
                                 const double* rPoints, long long M, int p, const long long* blockPtr,
                                 const long long* blockIds, int nBlocks, const double* fixedCenter, void* u) {
  return taylor_impl(ctx, coeff, qModes, NF, rPoints, M, p, blockPtr, blockIds, nBlocks, fixedCenter, u, true);
}

}  // extern "C"
