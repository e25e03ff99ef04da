// Null-space-free transverse basis and its block-diagonal maps.
//   assembly: exp1/assemble_K_and_nullspace_free_basis.m:18-105,
//             exp1/build_experiment1_q_system.m:7-24,
//             exp1/build_inner_system_operators.m:10-14
//   maps:     exp1/apply_V_blockdiag.m, exp1/apply_VH_blockdiag.m,
//             exp1/solveV1_blockdiag.m, exp1/solveV1H_blockdiag.m
#include <algorithm>
#include <cmath>
#include <cstring>
#include "internal.cuh"

namespace fame {

struct BasisReduce {
  unsigned long long minQq;     // bit pattern of a non-negative double
  unsigned long long minAbsDet;
  unsigned int nsingular;
};

struct BasisArgs {
  int N, n;
  int piv;  // physical component used as the third block row (V3); V1 = the other two
  long long NF;
  double P[18];  // column-major 6x3
  double k[6];
  double2 *V11, *V21, *V31, *V12, *V22, *V32, *det, *W1, *W2;
  double2 *P11, *P12, *P21, *P22;  // pivoted V1 block (aliases of V when piv == 2)
  double *invC, *Qq, *q1, *q2, *q3;
  float2 *W1f, *W2f;
  float* invCf;
  double2 *W1_l, *W2_l;
  double* invC_l;
  float2 *W1f_l, *W2f_l;
  float* invCf_l;
  BasisReduce* red;
};

__global__ void k_build_basis(BasisArgs a) {
  const double tol = 1e-13;
  // min |q|^2 and min |det V1| as bit patterns of non-negative doubles (their integer
  // order is their numeric order), reduced per thread and per warp: one atomic per warp
  unsigned long long mq = ~0ull, md = ~0ull;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.NF;
       i += (long long)gridDim.x * blockDim.x) {
    double q[3] = {0.0, 0.0, 0.0};
    long long tmp = i;
    for (int ell = 0; ell < 6; ++ell) {
      const int j = (int)(tmp % a.n);
      tmp /= a.n;
      const double xi = (j < a.N) ? (double)j : (double)(j - a.n);  // T = 2*pi
      const double s = xi + a.k[ell];
      q[0] += a.P[ell] * s;
      q[1] += a.P[6 + ell] * s;
      q[2] += a.P[12 + ell] * s;
    }
    const double Qq = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    const double sq = sqrt(Qq);
    const double Qs = q[0] + q[1] + q[2];
    const double denom = 3.0 * Qq - Qs * Qs;
    double u11, u21, u31, u12, u22, u32;
    if (denom > tol) {  // regular branch (:57-68)
      const double s1 = 1.0 / sqrt(Qq * denom), s2 = 1.0 / sqrt(denom);
      u11 = (Qq - q[0] * Qs) * s1;
      u21 = (Qq - q[1] * Qs) * s1;
      u31 = (Qq - q[2] * Qs) * s1;
      u12 = (q[2] - q[1]) * s2;
      u22 = (q[0] - q[2]) * s2;
      u32 = (q[1] - q[0]) * s2;
    } else {  // singular branch (:75-91)
      atomicAdd(&a.red->nsingular, 1u);
      const double qn = sq > 0 ? sq : 1.0;
      const double h[3] = {q[0] / qn, q[1] / qn, q[2] / qn};
      int imin = 0;
      for (int c = 1; c < 3; ++c)
        if (fabs(h[c]) < fabs(h[imin])) imin = c;
      double z1[3] = {0.0, 0.0, 0.0};
      z1[imin] = 1.0;
      const double ha = h[imin];
      for (int c = 0; c < 3; ++c) z1[c] -= h[c] * ha;
      double nz = sqrt(z1[0] * z1[0] + z1[1] * z1[1] + z1[2] * z1[2]);
      for (int c = 0; c < 3; ++c) z1[c] /= nz;
      double z2[3] = {h[1] * z1[2] - h[2] * z1[1], h[2] * z1[0] - h[0] * z1[2],
                      h[0] * z1[1] - h[1] * z1[0]};
      nz = sqrt(z2[0] * z2[0] + z2[1] * z2[1] + z2[2] * z2[2]);
      for (int c = 0; c < 3; ++c) z2[c] /= nz;
      u11 = z1[0]; u21 = z1[1]; u31 = z1[2];
      u12 = z2[0]; u22 = z2[1]; u32 = z2[2];
    }
    const double V11 = u11 * sq, V21 = u21 * sq, V31 = u31 * sq;
    const double V12 = u12 * sq, V22 = u22 * sq, V32 = u32 * sq;
    // pivoted split: rows ra, rb form V1, row piv forms V3
    const double Vr[3][2] = {{V11, V12}, {V21, V22}, {V31, V32}};
    const int ra = a.piv == 0 ? 1 : 0, rb = a.piv == 2 ? 1 : 2;
    const double A11 = Vr[ra][0], A12 = Vr[ra][1], A21 = Vr[rb][0], A22 = Vr[rb][1];
    const double B1 = Vr[a.piv][0], B2 = Vr[a.piv][1];
    const double det = A11 * A22 - A12 * A21;
    // W = V1^{-*} [conj V3_1; conj V3_2] (all real for a real cut matrix)
    const double W1 = (A22 * B1 - A21 * B2) / det;
    const double W2 = (-A12 * B1 + A11 * B2) / det;
    const double invC = 1.0 / sqrt(1.0 + W1 * W1 + W2 * W2);
    a.V11[i] = make_double2(V11, 0.0); a.V21[i] = make_double2(V21, 0.0);
    a.V31[i] = make_double2(V31, 0.0); a.V12[i] = make_double2(V12, 0.0);
    a.V22[i] = make_double2(V22, 0.0); a.V32[i] = make_double2(V32, 0.0);
    a.det[i] = make_double2(det, 0.0);
    if (a.piv != 2) {
      a.P11[i] = make_double2(A11, 0.0); a.P12[i] = make_double2(A12, 0.0);
      a.P21[i] = make_double2(A21, 0.0); a.P22[i] = make_double2(A22, 0.0);
    }
    a.W1[i] = make_double2(W1, 0.0);
    a.W2[i] = make_double2(W2, 0.0);
    a.invC[i] = invC;
    a.Qq[i] = Qq;
    a.q1[i] = q[0]; a.q2[i] = q[1]; a.q3[i] = q[2];
    a.W1f[i] = make_float2((float)W1, 0.f);
    a.W2f[i] = make_float2((float)W2, 0.f);
    a.invCf[i] = (float)invC;
    {  // line-order copies: within a column of n^3 modes, axis 1 slowest
      const long long n3 = (long long)a.n * a.n * a.n;
      const long long cb = i - i % n3;
      const long long g = i - cb;
      const long long il = cb + g / a.n + (long long)a.n * a.n * (g % a.n);
      a.W1_l[il] = make_double2(W1, 0.0);
      a.W2_l[il] = make_double2(W2, 0.0);
      a.invC_l[il] = invC;
      a.W1f_l[il] = make_float2((float)W1, 0.f);
      a.W2f_l[il] = make_float2((float)W2, 0.f);
      a.invCf_l[il] = (float)invC;
    }
    const unsigned long long bq = (unsigned long long)__double_as_longlong(Qq);
    const unsigned long long bd = (unsigned long long)__double_as_longlong(fabs(det));
    mq = bq < mq ? bq : mq;
    md = bd < md ? bd : md;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long oq = __shfl_xor_sync(0xffffffffu, mq, o), od = __shfl_xor_sync(0xffffffffu, md, o);
    mq = oq < mq ? oq : mq;
    md = od < md ? od : md;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&a.red->minQq, mq);
    atomicMin(&a.red->minAbsDet, md);
  }
}

// ------------------------------------------------------------ raw maps
__global__ void k_apply_V(const double2* x, const double2* V11, const double2* V12,
                          const double2* V21, const double2* V22, const double2* V31,
                          const double2* V32, long long n, int nrhs, double2* y) {
  const long long tot = n * nrhs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / n, i = t % n;
    const double2 x1 = x[2 * n * j + i], x2 = x[2 * n * j + n + i];
    double2* yj = y + 3 * n * j;
    yj[i] = cadd<double>(cmul<double>(V11[i], x1), cmul<double>(V12[i], x2));
    yj[n + i] = cadd<double>(cmul<double>(V21[i], x1), cmul<double>(V22[i], x2));
    yj[2 * n + i] = cadd<double>(cmul<double>(V31[i], x1), cmul<double>(V32[i], x2));
  }
}

__global__ void k_apply_VH(const double2* x, const double2* V11, const double2* V12,
                           const double2* V21, const double2* V22, const double2* V31,
                           const double2* V32, long long n, int nrhs, double2* y) {
  const long long tot = n * nrhs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / n, i = t % n;
    const double2* xj = x + 3 * n * j;
    const double2 x1 = xj[i], x2 = xj[n + i], x3 = xj[2 * n + i];
    double2 y1 = cadd<double>(cadd<double>(cmulc<double>(V11[i], x1), cmulc<double>(V21[i], x2)),
                              cmulc<double>(V31[i], x3));
    double2 y2 = cadd<double>(cadd<double>(cmulc<double>(V12[i], x1), cmulc<double>(V22[i], x2)),
                              cmulc<double>(V32[i], x3));
    y[2 * n * j + i] = y1;
    y[2 * n * j + n + i] = y2;
  }
}

template <bool HERM>
__global__ void k_solveV1(const double2* x, const double2* V11, const double2* V12,
                          const double2* V21, const double2* V22, const double2* det, long long n,
                          int nrhs, double2* y) {
  const long long tot = n * nrhs;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const long long j = t / n, i = t % n;
    const double2 x1 = x[2 * n * j + i], x2 = x[2 * n * j + n + i];
    double2 y1, y2;
    if (HERM) {  // y = V1^{-*} x
      const double2 d = cconj<double>(det[i]);
      y1 = cdiv<double>(csub<double>(cmulc<double>(V22[i], x1), cmulc<double>(V21[i], x2)), d);
      y2 = cdiv<double>(csub<double>(cmulc<double>(V11[i], x2), cmulc<double>(V12[i], x1)), d);
    } else {  // y = V1^{-1} x
      const double2 d = det[i];
      y1 = cdiv<double>(csub<double>(cmul<double>(V22[i], x1), cmul<double>(V12[i], x2)), d);
      y2 = cdiv<double>(csub<double>(cmul<double>(V11[i], x2), cmul<double>(V21[i], x1)), d);
    }
    y[2 * n * j + i] = y1;
    y[2 * n * j + n + i] = y2;
  }
}

// exp2/compute_fourier_diagnostics_exp2.m:10-19 for one column: with
// K the modewise curl-curl symbol (exp1/assemble_K_and_nullspace_free_basis.m:110-119)
// accumulate |Kx|^2, |Kx - lam Mx|^2, |Mx|^2, Re x^H Kx, Re x^H Mx, |D0 U0^H Mx|^2.
__global__ void k_fourier_diag(const double2* X, const double2* MX, const double* q1, const double* q2,
                               const double* q3, long long NF, double lam, double* partials,
                               unsigned* counter, double* out) {
  Red<double, 6> acc{};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < NF;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = q1[i], b = q2[i], c = q3[i];
    const double2 x1 = X[i], x2 = X[NF + i], x3 = X[2 * NF + i];
    const double2 m1 = MX[i], m2 = MX[NF + i], m3 = MX[2 * NF + i];
    const double2 k1 = make_double2((b * b + c * c) * x1.x - a * b * x2.x - a * c * x3.x,
                                    (b * b + c * c) * x1.y - a * b * x2.y - a * c * x3.y);
    const double2 k2 = make_double2(-a * b * x1.x + (a * a + c * c) * x2.x - b * c * x3.x,
                                    -a * b * x1.y + (a * a + c * c) * x2.y - b * c * x3.y);
    const double2 k3 = make_double2(-a * c * x1.x - b * c * x2.x + (a * a + b * b) * x3.x,
                                    -a * c * x1.y - b * c * x2.y + (a * a + b * b) * x3.y);
    acc.v[0] += cabs2<double>(k1) + cabs2<double>(k2) + cabs2<double>(k3);
    acc.v[1] += cabs2<double>(csub<double>(k1, cscale<double>(m1, lam))) +
                cabs2<double>(csub<double>(k2, cscale<double>(m2, lam))) +
                cabs2<double>(csub<double>(k3, cscale<double>(m3, lam)));
    acc.v[2] += cabs2<double>(m1) + cabs2<double>(m2) + cabs2<double>(m3);
    acc.v[3] += cmulc<double>(x1, k1).x + cmulc<double>(x2, k2).x + cmulc<double>(x3, k3).x;
    acc.v[4] += cmulc<double>(x1, m1).x + cmulc<double>(x2, m2).x + cmulc<double>(x3, m3).x;
    const double2 g = make_double2(a * m1.x + b * m2.x + c * m3.x, a * m1.y + b * m2.y + c * m3.y);
    acc.v[5] += cabs2<double>(g);
  }
  grid_sum_finalize<double, 6>(acc, partials, counter, [&](const Red<double, 6>& t) {
    for (int k = 0; k < 6; ++k) out[k] = t.v[k];
  });
}

inline int ew_blocks(long long tot) { return (int)std::min<long long>((tot + 255) / 256, 148 * 16); }

int check_map_args(fame_ctx* c, const void* x, const void* y, long long n, int nrhs) {
  if (!c || !x || !y || n <= 0 || nrhs < 0) return fail(FAME_ERR_INVALID, "basis map arguments");
  return FAME_OK;
}

}  // namespace fame

using namespace fame;

extern "C" {

int fame_apply_V_blockdiag(fame_ctx* c, const void* x, const void* V11, const void* V12,
                           const void* V21, const void* V22, const void* V31, const void* V32,
                           long long n, int nrhs, void* y) {
  FAME_TRY(check_map_args(c, x, y, n, nrhs));
  if (nrhs == 0) return FAME_OK;
  k_apply_V<<<ew_blocks(n * nrhs), 256, 0, c->stream>>>(
      (const double2*)x, (const double2*)V11, (const double2*)V12, (const double2*)V21,
      (const double2*)V22, (const double2*)V31, (const double2*)V32, n, nrhs, (double2*)y);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int fame_apply_VH_blockdiag(fame_ctx* c, const void* x, const void* V11, const void* V12,
                            const void* V21, const void* V22, const void* V31, const void* V32,
                            long long n, int nrhs, void* y) {
  FAME_TRY(check_map_args(c, x, y, n, nrhs));
  if (nrhs == 0) return FAME_OK;
  k_apply_VH<<<ew_blocks(n * nrhs), 256, 0, c->stream>>>(
      (const double2*)x, (const double2*)V11, (const double2*)V12, (const double2*)V21,
      (const double2*)V22, (const double2*)V31, (const double2*)V32, n, nrhs, (double2*)y);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int fame_solveV1_blockdiag(fame_ctx* c, const void* x, const void* V11, const void* V12,
                           const void* V21, const void* V22, const void* det, long long n,
                           int nrhs, void* y) {
  FAME_TRY(check_map_args(c, x, y, n, nrhs));
  if (nrhs == 0) return FAME_OK;
  k_solveV1<false><<<ew_blocks(n * nrhs), 256, 0, c->stream>>>(
      (const double2*)x, (const double2*)V11, (const double2*)V12, (const double2*)V21,
      (const double2*)V22, (const double2*)det, n, nrhs, (double2*)y);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int fame_solveV1H_blockdiag(fame_ctx* c, const void* x, const void* V11, const void* V12,
                            const void* V21, const void* V22, const void* det, long long n,
                            int nrhs, void* y) {
  FAME_TRY(check_map_args(c, x, y, n, nrhs));
  if (nrhs == 0) return FAME_OK;
  k_solveV1<true><<<ew_blocks(n * nrhs), 256, 0, c->stream>>>(
      (const double2*)x, (const double2*)V11, (const double2*)V12, (const double2*)V21,
      (const double2*)V22, (const double2*)det, n, nrhs, (double2*)y);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int fame_basis_create(fame_ctx* ctx, int N, const double* P, const double* q, fame_basis** out) {
  if (!ctx || !P || !q || !out) return fail(FAME_ERR_INVALID, "fame_basis_create arguments");
  *out = nullptr;
  if (N < 1 || N > 7) return fail(FAME_ERR_UNSUPPORTED, "N must be in [1,7]");
  // kLift = P (P^T P)^{-1} q  (exp1/build_experiment1_q_system.m:7), 3x3 solve on the host
  double G[9] = {0};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int l = 0; l < 6; ++l) G[a * 3 + b] += P[a * 6 + l] * P[b * 6 + l];
  double A[3][4];
  for (int a = 0; a < 3; ++a) {
    for (int b = 0; b < 3; ++b) A[a][b] = G[a * 3 + b];
    A[a][3] = q[a];
  }
  for (int col = 0; col < 3; ++col) {  // Gaussian elimination, partial pivoting
    int piv = col;
    for (int r = col + 1; r < 3; ++r)
      if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
    for (int cc = 0; cc < 4; ++cc) std::swap(A[col][cc], A[piv][cc]);
    if (std::fabs(A[col][col]) < 1e-300) return fail(FAME_ERR_INVALID, "P^T P is singular");
    for (int r = 0; r < 3; ++r) {
      if (r == col) continue;
      const double f = A[r][col] / A[col][col];
      for (int cc = col; cc < 4; ++cc) A[r][cc] -= f * A[col][cc];
    }
  }
  double w[3];
  for (int a = 0; a < 3; ++a) w[a] = A[a][3] / A[a][a];

  fame_basis* b = new fame_basis();
  b->ctx = ctx;
  std::memcpy(b->P, P, sizeof(b->P));
  b->N = N;
  b->n = 2 * N;
  long long NF = 1;
  for (int d = 0; d < 6; ++d) NF *= b->n;
  b->NF = NF;
  BasisArgs a{};
  a.N = N;
  a.n = b->n;
  a.NF = NF;
  std::memcpy(a.P, P, sizeof(a.P));
  for (int l = 0; l < 6; ++l) a.k[l] = P[l] * w[0] + P[6 + l] * w[1] + P[12 + l] * w[2];
  int s = FAME_OK;
  for (int j = 0; j < 6 && s == FAME_OK; ++j) s = dalloc((void**)&b->V[j], NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&b->det, NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&b->W1, NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&b->W2, NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&b->invC, NF * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&b->Qq, NF * sizeof(double));
  for (int j = 0; j < 3 && s == FAME_OK; ++j) s = dalloc((void**)&b->q[j], NF * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&b->W1f, NF * sizeof(float2));
  if (s == FAME_OK) s = dalloc((void**)&b->W2f, NF * sizeof(float2));
  if (s == FAME_OK) s = dalloc((void**)&b->invCf, NF * sizeof(float));
  if (s == FAME_OK) s = dalloc((void**)&b->W1_l, NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&b->W2_l, NF * sizeof(double2));
  if (s == FAME_OK) s = dalloc((void**)&b->invC_l, NF * sizeof(double));
  if (s == FAME_OK) s = dalloc((void**)&b->W1f_l, NF * sizeof(float2));
  if (s == FAME_OK) s = dalloc((void**)&b->W2f_l, NF * sizeof(float2));
  if (s == FAME_OK) s = dalloc((void**)&b->invCf_l, NF * sizeof(float));
  BasisReduce* red = nullptr;
  if (s == FAME_OK) s = dalloc((void**)&red, sizeof(BasisReduce));
  if (s != FAME_OK) {
    fame_basis_destroy(b);
    return s;
  }
  a.V11 = b->V[0]; a.V21 = b->V[1]; a.V31 = b->V[2];
  a.V12 = b->V[3]; a.V22 = b->V[4]; a.V32 = b->V[5];
  a.det = b->det; a.W1 = b->W1; a.W2 = b->W2;
  a.invC = b->invC; a.Qq = b->Qq; a.q1 = b->q[0]; a.q2 = b->q[1]; a.q3 = b->q[2];
  a.W1f = b->W1f; a.W2f = b->W2f; a.invCf = b->invCf;
  a.W1_l = b->W1_l; a.W2_l = b->W2_l; a.invC_l = b->invC_l;
  a.W1f_l = b->W1f_l; a.W2f_l = b->W2f_l; a.invCf_l = b->invCf_l;
  a.red = red;
  BasisReduce h{};
  // the reference splits components (1,2 | 3); when that V1 block is singular for some
  // mode (q_3 = 0 makes it singular for xi = 0), pivot on the largest |q_c| instead --
  // K_r = V^* diag(M,M,M)^{-1} V does not depend on the order of the components.
  int pivots[2] = {2, 0};
  {
    double qa[3] = {std::fabs(q[0]), std::fabs(q[1]), std::fabs(q[2])};
    pivots[1] = qa[0] >= qa[1] ? (qa[0] >= qa[2] ? 0 : 2) : (qa[1] >= qa[2] ? 1 : 2);
  }
  for (int attempt = 0; attempt < 2 && s == FAME_OK; ++attempt) {
    a.piv = pivots[attempt];
    if (attempt == 1) {
      if (a.piv == 2) break;
      for (int j = 0; j < 4 && s == FAME_OK; ++j) s = dalloc((void**)&b->Vp[j], NF * sizeof(double2));
      if (s != FAME_OK) break;
    }
    a.P11 = b->Vp[0]; a.P12 = b->Vp[1]; a.P21 = b->Vp[2]; a.P22 = b->Vp[3];
    BasisReduce init{0x7FF0000000000000ull, 0x7FF0000000000000ull, 0u};  // +inf
    cudaMemcpyAsync(red, &init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream);
    k_build_basis<<<ew_blocks(NF), 256, 0, ctx->stream>>>(a);
    ::fame::count_launch();
    s = cudaGetLastError() == cudaSuccess ? read_back(ctx, red, &h, sizeof(h)) : fail(FAME_ERR_CUDA, "basis kernel launch");
    double md;
    std::memcpy(&md, &h.minAbsDet, 8);
    if (s != FAME_OK || md >= 1e-10) break;
  }
  b->pivot = a.piv;
  dfree(red);
  if (s != FAME_OK) {
    fame_basis_destroy(b);
    return s;
  }
  double minQq, minDet;
  std::memcpy(&minQq, &h.minQq, 8);
  std::memcpy(&minDet, &h.minAbsDet, 8);
  b->info.NF = NF;
  b->info.N = N;
  b->info.pivot = b->pivot;
  b->info.nsingular = (int)h.nsingular;
  b->info.minQq = minQq;
  b->info.minAbsDetV1 = minDet;
  for (int l = 0; l < 6; ++l) b->info.kLift[l] = a.k[l];
  if (minQq <= 1e-13) {
    fame_basis_destroy(b);
    return fail(FAME_ERR_SINGULAR,
                "zero projected Fourier mode (Gamma point): the null-space-free reduction "
                "requires every |q_xi| > 0");
  }
  *out = b;
  return FAME_OK;
}

int fame_basis_destroy(fame_basis* b) {
  if (!b) return FAME_OK;
  cudaStreamSynchronize(b->ctx->stream);
  for (int j = 0; j < 6; ++j) dfree(b->V[j]);
  dfree(b->det); dfree(b->W1); dfree(b->W2); dfree(b->invC); dfree(b->Qq);
  for (int j = 0; j < 3; ++j) dfree(b->q[j]);
  dfree(b->W1f); dfree(b->W2f); dfree(b->invCf);
  dfree(b->W1_l); dfree(b->W2_l); dfree(b->invC_l);
  dfree(b->W1f_l); dfree(b->W2f_l); dfree(b->invCf_l);
  dfree(b->work);
  for (int j = 0; j < 4; ++j) dfree(b->Vp[j]);
  delete b;
  return FAME_OK;
}

int fame_fourier_diagnostics(fame_basis* b, const void* X, const void* MX, const double* lambda, int k,
                             double* resGEVP, double* divRelative2, double* rayleigh) {
  if (!b || !X || !MX || !lambda || k < 0) return fail(FAME_ERR_INVALID, "fame_fourier_diagnostics arguments");
  const long long NF = b->NF;
  const int blocks = ew_blocks(NF);
  double* buf = nullptr;
  unsigned* counter = nullptr;
  FAME_TRY(dalloc((void**)&buf, (6 * (size_t)blocks + 8) * sizeof(double)));
  int s = dalloc((void**)&counter, sizeof(unsigned));
  if (s != FAME_OK) {
    dfree(buf);
    return s;
  }
  cudaMemsetAsync(counter, 0, sizeof(unsigned), b->ctx->stream);
  const double eps = 2.220446049250313e-16;
  for (int j = 0; j < k && s == FAME_OK; ++j) {
    k_fourier_diag<<<blocks, 256, 0, b->ctx->stream>>>((const double2*)X + 3 * NF * j, (const double2*)MX + 3 * NF * j,
                                                       b->q[0], b->q[1], b->q[2], NF, lambda[j], buf + 8, counter, buf);
    ::fame::count_launch();
    double h[6];
    s = cudaGetLastError() == cudaSuccess ? read_back(b->ctx, buf, h, sizeof(h)) : fail(FAME_ERR_CUDA, "diagnostics launch");
    if (s != FAME_OK) break;
    const double den = std::sqrt(h[0]) + std::fabs(lambda[j]) * std::sqrt(h[2]);
    if (resGEVP) resGEVP[j] = std::sqrt(h[1]) / std::max(den, eps);
    if (divRelative2) divRelative2[j] = std::sqrt(h[5]) / std::max(std::sqrt(h[2]), eps);
    if (rayleigh) rayleigh[j] = h[3] / h[4];
  }
  dfree(buf);
  dfree(counter);
  return s;
}

int fame_basis_info_get(fame_basis* b, fame_basis_info* out) {
  if (!b || !out) return fail(FAME_ERR_INVALID, "fame_basis_info_get arguments");
  *out = b->info;
  return FAME_OK;
}

int fame_basis_get(fame_basis* b, int which, void* dst) {
  if (!b || !dst) return fail(FAME_ERR_INVALID, "fame_basis_get arguments");
  const void* src = nullptr;
  size_t el = sizeof(double2);
  if (which >= 0 && which < 6) src = b->V[which];
  else if (which == 6) src = b->det;
  else if (which == 7) src = b->W1;
  else if (which == 8) src = b->W2;
  else {
    el = sizeof(double);
    if (which == 9) src = b->invC;
    else if (which == 10) src = b->Qq;
    else if (which >= 11 && which <= 13) src = b->q[which - 11];
    else return fail(FAME_ERR_INVALID, "unknown basis diagonal");
  }
  FAME_CUDA_TRY(cudaMemcpyAsync(dst, src, b->NF * el, cudaMemcpyDeviceToDevice, b->ctx->stream));
  return FAME_OK;
}

}  // extern "C"
