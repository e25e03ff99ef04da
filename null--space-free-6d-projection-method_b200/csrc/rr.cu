// Rayleigh-Ritz refinement of approximate eigenvectors of K_r = V^* M^{-1} V
// (no counterpart in the reference; its eigenvalues are 1/theta of the
// Lanczos Ritz values of the inexact K_r^{-1}, exp2/Lanczos.m:140-147).
//
// On the (2N)^6 grid the mass operator is M = F diag(eps) F^{-1} exactly
// (exp1/applyMij_fft.m:11 is a circular convolution), so M^{-1} is the same
// pass A/B/C chain on the material 1/eps and K_r applies to rounding error.
// Given k approximate eigenvectors Y (2NF x k) -- e.g. the Ritz vectors of a
// Lanczos run on an inner-tolerance K_r^{-1} -- this computes Z = K_r Y in one
// fused FP64 chain per column (V y in pass A's prologue, V^* in pass C's
// epilogue), the Gram matrices G = Y^H Z and B = Y^H Y, solves G u = lambda B u
// on the host (Cholesky + complex Hermitian Jacobi), rotates Y in place to the
// refined vectors and reports ||K_r y - lambda y|| / ||K_r y|| per vector.  The
// eigenvalue error is then quadratic in the eigenvector error of Y: Ritz vectors
// from a K_r^{-1} at inner tolerance 1e-10 give eigenvalues at the rounding
// level instead of ~1e-9.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>
#include "internal.cuh"
#include "mass_chain.cuh"

namespace fame {

constexpr int kRRMaxK = 32;        // columns refined together
constexpr int kGramThreads = 256;
constexpr int kGramRows = 32;       // rows staged per iteration
constexpr int kGramPairs = 8;       // (i, j) pairs per thread: 2 k^2 <= 256 * 8
constexpr int kGramBlocksMax = 296;

// V y (prologue): field c = V_c1 y1 + V_c2 y2, natural order.
struct ProVy {
  static constexpr bool natural = true;
  const double2* V[6];  // V11, V21, V31, V12, V22, V32
  const double2* y;
  long long NF;
  __device__ __forceinline__ void load(long long, long long i, double2* v) const {
    const double2 y1 = y[i], y2 = y[NF + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = cadd<double>(cmul<double>(V[c][i], y1), cmul<double>(V[c + 3][i], y2));
  }
};
// V^* w (epilogue): z1 = sum_c conj(V_c1) w_c, z2 = sum_c conj(V_c2) w_c.
struct EpiVHz {
  using Acc = double;
  static constexpr int K = 0;
  static constexpr bool natural = true;
  const double2* V[6];
  double2* z;
  long long NF;
  double* partials = nullptr;
  unsigned* counter = nullptr;
  __device__ __forceinline__ void store(long long, long long i, const double2* w, Red<double, 1>&) const {
    double2 z1 = mk<double>(0, 0), z2 = mk<double>(0, 0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      z1 = cadd<double>(z1, cmulc<double>(V[c][i], w[c]));
      z2 = cadd<double>(z2, cmulc<double>(V[c + 3][i], w[c]));
    }
    z[i] = z1;
    z[NF + i] = z2;
  }
  __device__ __forceinline__ void finalize(const Red<double, 1>&) const {}
};

// Partial Gram sums of one block of rows: part[b][p] for the 2k^2 pairs
// p < k^2: G(i,j) = sum conj(Y_i) Z_j, p >= k^2: B(i,j) = sum conj(Y_i) Y_j.
__global__ void __launch_bounds__(kGramThreads) k_rr_gram(const double2* __restrict__ Y, const double2* __restrict__ Z,
                                                         long long n, int k, double2* __restrict__ part) {
  __shared__ double2 ys[kGramRows][kRRMaxK], zs[kGramRows][kRRMaxK];
  const int npair = 2 * k * k;
  double2 acc[kGramPairs];
#pragma unroll
  for (int a = 0; a < kGramPairs; ++a) acc[a] = mk<double>(0, 0);
  const long long rows_per_block = (n + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * rows_per_block, r1 = min(n, r0 + rows_per_block);
  for (long long rb = r0; rb < r1; rb += kGramRows) {
    __syncthreads();
    for (int e = threadIdx.x; e < kGramRows * k; e += blockDim.x) {
      const int rr = e % kGramRows, c = e / kGramRows;
      const long long row = rb + rr;
      const bool in = row < r1;
      ys[rr][c] = in ? Y[row + n * c] : mk<double>(0, 0);
      zs[rr][c] = in ? Z[row + n * c] : mk<double>(0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < kGramPairs; ++a) {
      const int p = threadIdx.x + a * kGramThreads;
      if (p < npair) {
        const int q = p % (k * k), i = q % k, j = q / k;
        const bool gram = p < k * k;
        double2 s = acc[a];
        for (int rr = 0; rr < kGramRows; ++rr) {
          const double2 yi = ys[rr][i], w = gram ? zs[rr][j] : ys[rr][j];
          s.x += yi.x * w.x + yi.y * w.y;
          s.y += yi.x * w.y - yi.y * w.x;
        }
        acc[a] = s;
      }
    }
  }
#pragma unroll
  for (int a = 0; a < kGramPairs; ++a) {
    const int p = threadIdx.x + a * kGramThreads;
    if (p < npair) part[(long long)blockIdx.x * npair + p] = acc[a];
  }
}

// out[p] = sum_b part[b][p] in block order (deterministic)
__global__ void k_rr_gram_reduce(const double2* part, int nblk, int npair, double2* out) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npair; p += gridDim.x * blockDim.x) {
    double2 s = mk<double>(0, 0);
    for (int b = 0; b < nblk; ++b) s = cadd<double>(s, part[(long long)b * npair + p]);
    out[p] = s;
  }
}

// Yr = Y R and, per column j, ||Z R_j - lambda_j Y R_j||^2 and ||Z R_j||^2 as
// block partials (res[b][2j], res[b][2j+1]); R is k x k column-major.  Output
// columns are produced in chunks of kRotCols (the row's inputs are re-read per
// chunk from L2) so that the accumulators stay in registers.
constexpr int kRotCols = 8;
__global__ void __launch_bounds__(256) k_rr_rotate(const double2* __restrict__ Y, const double2* __restrict__ Z,
                                                   long long n, int k, const double2* __restrict__ R,
                                                   const double* __restrict__ lam, double2* __restrict__ Yr,
                                                   double* __restrict__ res) {
  __shared__ double2 Rs[kRRMaxK * kRRMaxK];
  __shared__ double red[8][2 * kRotCols];
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) Rs[e] = R[e];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int j0 = 0; j0 < k; j0 += kRotCols) {
    const int nc = min(kRotCols, k - j0);
    double acc[2 * kRotCols];
#pragma unroll
    for (int j = 0; j < 2 * kRotCols; ++j) acc[j] = 0.0;
    for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < n;
         row += (long long)gridDim.x * blockDim.x) {
      double2 yj[kRotCols], zj[kRotCols];
#pragma unroll
      for (int j = 0; j < kRotCols; ++j) yj[j] = zj[j] = mk<double>(0, 0);
      for (int i = 0; i < k; ++i) {
        const double2 y = Y[row + n * i], z = Z[row + n * i];
#pragma unroll
        for (int j = 0; j < kRotCols; ++j) {
          if (j < nc) {
            const double2 r = Rs[i + k * (j0 + j)];
            yj[j] = cadd<double>(yj[j], cmul<double>(y, r));
            zj[j] = cadd<double>(zj[j], cmul<double>(z, r));
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kRotCols; ++j) {
        if (j < nc) {
          Yr[row + n * (j0 + j)] = yj[j];
          const double2 d = csub<double>(zj[j], cscale<double>(yj[j], lam[j0 + j]));
          acc[2 * j] += cabs2<double>(d);
          acc[2 * j + 1] += cabs2<double>(zj[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 2 * kRotCols; ++j) {
      double v = acc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[wid][j] = v;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 2 * nc; j += blockDim.x) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][j];
      res[(long long)blockIdx.x * 2 * k + 2 * j0 + j] = s;
    }
    __syncthreads();
  }
}

using cd = std::complex<double>;

// Eigen-decomposition of a Hermitian k x k matrix A (column-major) by cyclic
// complex Jacobi rotations: A = U diag(w) U^H, w ascending.
void herm_jacobi(std::vector<cd> A, int k, std::vector<double>& w, std::vector<cd>& U) {
  U.assign((size_t)k * k, cd(0, 0));
  for (int i = 0; i < k; ++i) U[i + (size_t)k * i] = 1.0;
  auto at = [&](int i, int j) -> cd& { return A[i + (size_t)k * j]; };
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < k; ++j)
      for (int i = 0; i < k; ++i) {
        const double a = std::norm(at(i, j));
        tot += a;
        if (i != j) off += a;
      }
    if (off <= 1e-32 * tot) break;
    for (int p = 0; p < k - 1; ++p)
      for (int q = p + 1; q < k; ++q) {
        const cd apq = at(p, q);
        const double m = std::abs(apq);
        if (m < 1e-300) continue;
        const cd e = apq / m;  // A' = D^H A D with D = diag(1, conj(e)) makes a_pq real
        const double theta = (std::real(at(q, q)) - std::real(at(p, p))) / (2.0 * m);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
        // J = [[c, s], [-s conj(e), c conj(e)]] on rows/columns (p, q); A <- J^H A J, U <- U J
        const cd jpp = c, jpq = s, jqp = -s * std::conj(e), jqq = c * std::conj(e);
        for (int r = 0; r < k; ++r) {  // columns: A J
          const cd ap = at(r, p), aq = at(r, q);
          at(r, p) = ap * jpp + aq * jqp;
          at(r, q) = ap * jpq + aq * jqq;
          const cd up = U[r + (size_t)k * p], uq = U[r + (size_t)k * q];
          U[r + (size_t)k * p] = up * jpp + uq * jqp;
          U[r + (size_t)k * q] = up * jpq + uq * jqq;
        }
        for (int col = 0; col < k; ++col) {  // rows: J^H (A J)
          const cd ap = at(p, col), aq = at(q, col);
          at(p, col) = std::conj(jpp) * ap + std::conj(jqp) * aq;
          at(q, col) = std::conj(jpq) * ap + std::conj(jqq) * aq;
        }
        at(p, q) = 0.0;
        at(q, p) = 0.0;
      }
  }
  std::vector<int> ord(k);
  for (int i = 0; i < k; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return std::real(at(a, a)) < std::real(at(b, b)); });
  std::vector<cd> Us((size_t)k * k);
  w.resize(k);
  for (int j = 0; j < k; ++j) {
    w[j] = std::real(at(ord[j], ord[j]));
    for (int i = 0; i < k; ++i) Us[i + (size_t)k * j] = U[i + (size_t)k * ord[j]];
  }
  U.swap(Us);
}

// Solve G u = lambda B u (Hermitian G, Hermitian positive definite B):
// R = L^{-H} U with B = L L^H and L^{-1} G L^{-H} = U diag(lambda) U^H.
int small_gep(const std::vector<cd>& G0, const std::vector<cd>& B0, int k, std::vector<double>& lam,
              std::vector<cd>& R) {
  std::vector<cd> G((size_t)k * k), B((size_t)k * k), L((size_t)k * k, cd(0, 0));
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < k; ++i) {  // Hermitian parts
      G[i + (size_t)k * j] = 0.5 * (G0[i + (size_t)k * j] + std::conj(G0[j + (size_t)k * i]));
      B[i + (size_t)k * j] = 0.5 * (B0[i + (size_t)k * j] + std::conj(B0[j + (size_t)k * i]));
    }
  for (int j = 0; j < k; ++j) {  // Cholesky B = L L^H
    double d = std::real(B[j + (size_t)k * j]);
    for (int c = 0; c < j; ++c) d -= std::norm(L[j + (size_t)k * c]);
    if (!(d > 0)) return fail(FAME_ERR_SINGULAR, "Rayleigh-Ritz: the vectors are linearly dependent");
    const double ljj = std::sqrt(d);
    L[j + (size_t)k * j] = ljj;
    for (int i = j + 1; i < k; ++i) {
      cd s = B[i + (size_t)k * j];
      for (int c = 0; c < j; ++c) s -= L[i + (size_t)k * c] * std::conj(L[j + (size_t)k * c]);
      L[i + (size_t)k * j] = s / ljj;
    }
  }
  // Linv = L^{-1} (lower triangular)
  std::vector<cd> Li((size_t)k * k, cd(0, 0));
  for (int c = 0; c < k; ++c) {
    for (int i = 0; i < k; ++i) {
      cd s = (i == c) ? cd(1, 0) : cd(0, 0);
      for (int m = 0; m < i; ++m) s -= L[i + (size_t)k * m] * Li[m + (size_t)k * c];
      Li[i + (size_t)k * c] = s / L[i + (size_t)k * i];
    }
  }
  // Cm = Li G Li^H
  std::vector<cd> T((size_t)k * k, cd(0, 0)), Cm((size_t)k * k, cd(0, 0));
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < k; ++i) {
      cd s = 0;
      for (int m = 0; m < k; ++m) s += Li[i + (size_t)k * m] * G[m + (size_t)k * j];
      T[i + (size_t)k * j] = s;
    }
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < k; ++i) {
      cd s = 0;
      for (int m = 0; m < k; ++m) s += T[i + (size_t)k * m] * std::conj(Li[j + (size_t)k * m]);
      Cm[i + (size_t)k * j] = s;
    }
  std::vector<cd> U;
  herm_jacobi(Cm, k, lam, U);
  R.assign((size_t)k * k, cd(0, 0));  // R = Li^H U
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < k; ++i) {
      cd s = 0;
      for (int m = 0; m < k; ++m) s += std::conj(Li[m + (size_t)k * i]) * U[m + (size_t)k * j];
      R[i + (size_t)k * j] = s;
    }
  return FAME_OK;
}

// Device-to-host copy of a few kilobytes into pageable host memory (stream-ordered, waited on).
int copy_to_host(fame_ctx* ctx, const void* dsrc, void* hdst, size_t bytes) {
  FAME_CUDA_TRY(cudaMemcpyAsync(hdst, dsrc, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  FAME_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return FAME_OK;
}

}  // namespace fame

using namespace fame;

extern "C" int fame_rayleigh_ritz(fame_basis* b, fame_mass* m, void* Y, int k, double* lambda, double* relres) {
  if (!b || !m || !Y || !lambda) return fail(FAME_ERR_INVALID, "fame_rayleigh_ritz arguments");
  if (b->N != m->N) return fail(FAME_ERR_INVALID, "basis and mass have different N");
  if (k < 1 || k > kRRMaxK) return fail(FAME_ERR_INVALID, "Rayleigh-Ritz refines 1..32 vectors");
  fame_ctx* ctx = b->ctx;
  cudaStream_t st = ctx->stream;
  const long long NF = b->NF, nr = 2 * NF;
  const int nblk = std::min<long long>(kGramBlocksMax, std::max<long long>(1, nr / (kGramRows * 8)));
  const int npair = 2 * k * k;
  // workspace: 3 work fields, Z (nr x k), Gram partials and totals, R, lambda, residual partials
  Carve cv;
  cv.take<double2>(3 * NF);
  cv.take<double2>((size_t)nr * k);
  cv.take<double2>((size_t)nr * k);
  cv.take<double2>((size_t)nblk * npair);
  cv.take<double2>(npair);
  cv.take<double2>((size_t)k * k);
  cv.take<double>(k);
  cv.take<double>((size_t)kGramBlocksMax * 2 * k);
  void* ws = nullptr;
  FAME_TRY(ctx_workspace(ctx, cv.used, &ws));
  Carve c2;
  c2.base = (char*)ws;
  double2* work = c2.take<double2>(3 * NF);
  double2* Z = c2.take<double2>((size_t)nr * k);
  double2* Yr = c2.take<double2>((size_t)nr * k);
  double2* part = c2.take<double2>((size_t)nblk * npair);
  double2* gram = c2.take<double2>(npair);
  double2* Rd = c2.take<double2>((size_t)k * k);
  double* lamd = c2.take<double>(k);
  double* resd = c2.take<double>((size_t)kGramBlocksMax * 2 * k);
  double2* Yd = (double2*)Y;
  // Z = K_r Y = V^* M^{-1} V Y, one chain per column on the material 1/eps
  for (int j = 0; j < k; ++j) {
    ProVy pro;
    EpiVHz epi;
    for (int c = 0; c < 6; ++c) pro.V[c] = epi.V[c] = b->V[c];
    pro.y = Yd + (size_t)nr * j;
    pro.NF = epi.NF = NF;
    epi.z = Z + (size_t)nr * j;
    FAME_TRY((run_chain<double, 3>(b->n, pro, epi, work, m->EtInv64, NF, st)));
  }
  k_rr_gram<<<nblk, kGramThreads, 0, st>>>(Yd, Z, nr, k, part);
  k_rr_gram_reduce<<<(npair + 255) / 256, 256, 0, st>>>(part, nblk, npair, gram);
  count_launch(2);
  FAME_CUDA_TRY(cudaGetLastError());
  std::vector<double2> hg(npair);
  FAME_TRY(copy_to_host(ctx, gram, hg.data(), npair * sizeof(double2)));
  FAME_TRY(check_fault(ctx));
  std::vector<cd> G((size_t)k * k), B((size_t)k * k);
  for (int p = 0; p < k * k; ++p) {
    G[p] = cd(hg[p].x, hg[p].y);
    B[p] = cd(hg[k * k + p].x, hg[k * k + p].y);
  }
  for (int p = 0; p < npair; ++p)
    if (!std::isfinite(hg[p].x) || !std::isfinite(hg[p].y)) return fail(FAME_ERR_NONFINITE, "Rayleigh-Ritz: non-finite input");
  std::vector<double> lam;
  std::vector<cd> R;
  FAME_TRY(small_gep(G, B, k, lam, R));
  std::vector<double2> hR((size_t)k * k);
  for (int p = 0; p < k * k; ++p) hR[p] = make_double2(R[p].real(), R[p].imag());
  FAME_CUDA_TRY(cudaMemcpyAsync(Rd, hR.data(), hR.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  FAME_CUDA_TRY(cudaMemcpyAsync(lamd, lam.data(), k * sizeof(double), cudaMemcpyHostToDevice, st));
  const int rblk = (int)std::min<long long>(kGramBlocksMax, (nr + 255) / 256);
  k_rr_rotate<<<rblk, 256, 0, st>>>(Yd, Z, nr, k, Rd, lamd, Yr, resd);
  count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  FAME_CUDA_TRY(cudaMemcpyAsync(Yd, Yr, (size_t)nr * k * sizeof(double2), cudaMemcpyDeviceToDevice, st));
  std::vector<double> hres((size_t)rblk * 2 * k);
  FAME_TRY(copy_to_host(ctx, resd, hres.data(), hres.size() * sizeof(double)));
  for (int j = 0; j < k; ++j) {
    lambda[j] = lam[j];
    if (relres) {
      double rn = 0.0, zn = 0.0;
      for (int bb = 0; bb < rblk; ++bb) {
        rn += hres[(size_t)bb * 2 * k + 2 * j];
        zn += hres[(size_t)bb * 2 * k + 2 * j + 1];
      }
      relres[j] = zn > 0 ? std::sqrt(rn / zn) : 0.0;
    }
  }
  return FAME_OK;
}
