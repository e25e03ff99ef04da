// Physical validation of a reconstructed Yee field by the local weighted
// Rayleigh quotient (LWRQ), restating exp3/compute_yee_lwrq_metrics_exp4.m,
// exp3/compute_lwrq_exp4.m, exp3/apply_cropped_A_exp3.m,
// exp3/separable_conv3_same_exp4.m and exp3/sample_scalar_yee_material_exp4.m.
//
// Input: the three components on the plus-grid, m = 2n+3 points per axis,
// column-major with x fastest (the order of the Yee reconstruction).  All work
// is on the (2n+1)^3 interior, q = 2n+1:
//   k_lwrq_ab     curl-curl stencil Au, eps on the Yee edges, Bu = eps u,
//                 a = Re<u,Au>, b = Re<u,Bu> per point, and sum a, sum b,
//                 ||Au||^2, ||Bu||^2;
//   k_lwrq_conv   one axis of the zero-padded separable Gaussian window
//                 (radius 3 cells, sigma 2h) for the a- and b-paths together;
//                 the first axis divides by the column normalisation
//                 den = dx(i) dy(j) dz(k) (separable, computed on the fly);
//   k_lwrq_stat1  sum E, sum M, non-finite count; k_lwrq_max max M;
//   k_lwrq_stat2  count of M <= 1e-14 max M, sum M |E/M - lambda|^2, and the
//                 z = 0 / x = 0 slices of rho = E/M;
//   k_lwrq_resid  ||Au - lambda Bu||^2 for lambda3D and lambda6D (stencil
//                 recomputed instead of stored).
// Reductions are the deterministic fixed-order grid sums used everywhere.
#include <cmath>
#include <vector>
#include "internal.cuh"

namespace fame {

constexpr int kLwrqR = 3;  // window radius in cells (exp3/make_config_experiment4.m:73)

struct YeeMat {
  int kind;          // 0: epsC exp(alpha/6 sum cos), 1: 1 + delta prod (1 + cos)/2
  double p0, p1;     // (epsC, alpha) or (delta, -)
  double P[18];      // cut matrix, column-major 6 x 3: P(l, c) = P[l + 6 c]
};

struct YeeGeom {
  const double2 *u1, *u2, *u3;
  int n, m, q;
  double h;
};

__device__ __forceinline__ double yee_eps(const YeeMat& mt, double x, double y, double z) {
  if (mt.kind == 0) {
    double s = 0.0;
#pragma unroll
    for (int l = 0; l < 6; ++l) s += cos(mt.P[l] * x + mt.P[l + 6] * y + mt.P[l + 12] * z);
    return mt.p0 * exp(mt.p1 / 6.0 * s);
  }
  double prod = 1.0;
#pragma unroll
  for (int l = 0; l < 6; ++l) prod *= 0.5 * (1.0 + cos(mt.P[l] * x + mt.P[l + 6] * y + mt.P[l + 12] * z));
  return 1.0 + mt.p0 * prod;
}

// Au and Bu (three components) at interior point (i, j, k) of the crop.
__device__ __forceinline__ void yee_ab(const YeeGeom& g, const YeeMat& mt, int i, int j, int k, double2* A,
                                       double2* B, double2* U) {
  const long long m = g.m;
  const long long c0 = (i + 1) + m * (j + 1) + m * m * (k + 1);
  auto at = [&](const double2* u, int dx, int dy, int dz) { return u[c0 + dx + m * dy + m * m * dz]; };
  auto second = [&](const double2* u, int ax) {
    const int ex = ax == 0, ey = ax == 1, ez = ax == 2;
    const double2 c = at(u, 0, 0, 0), lo = at(u, -ex, -ey, -ez), hi = at(u, ex, ey, ez);
    return make_double2(2.0 * c.x - lo.x - hi.x, 2.0 * c.y - lo.y - hi.y);
  };
  // backward difference along `bk` of the forward difference along `fw`
  auto mixed = [&](const double2* u, int bk, int fw) {
    const int fx = fw == 0, fy = fw == 1, fz = fw == 2, bx = -(bk == 0), by = -(bk == 1), bz = -(bk == 2);
    const double2 a = at(u, fx + bx, fy + by, fz + bz), b = at(u, bx, by, bz), c = at(u, fx, fy, fz),
                  d = at(u, 0, 0, 0);
    return make_double2(a.x - b.x - c.x + d.x, a.y - b.y - c.y + d.y);
  };
  const double s = 1.0 / (g.h * g.h);
  double2 t1 = cadd<double>(second(g.u1, 1), second(g.u1, 2));
  t1 = csub<double>(csub<double>(t1, mixed(g.u2, 1, 0)), mixed(g.u3, 2, 0));
  double2 t2 = cadd<double>(second(g.u2, 0), second(g.u2, 2));
  t2 = csub<double>(csub<double>(t2, mixed(g.u1, 0, 1)), mixed(g.u3, 2, 1));
  double2 t3 = cadd<double>(second(g.u3, 0), second(g.u3, 1));
  t3 = csub<double>(csub<double>(t3, mixed(g.u1, 0, 2)), mixed(g.u2, 1, 2));
  A[0] = cscale<double>(t1, s);
  A[1] = cscale<double>(t2, s);
  A[2] = cscale<double>(t3, s);
  U[0] = at(g.u1, 0, 0, 0);
  U[1] = at(g.u2, 0, 0, 0);
  U[2] = at(g.u3, 0, 0, 0);
  const double x = (i - g.n) * g.h, y = (j - g.n) * g.h, z = (k - g.n) * g.h, hh = 0.5 * g.h;
  B[0] = cscale<double>(U[0], yee_eps(mt, x + hh, y, z));
  B[1] = cscale<double>(U[1], yee_eps(mt, x, y + hh, z));
  B[2] = cscale<double>(U[2], yee_eps(mt, x, y, z + hh));
}

static inline int lblocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

// sums: [0] sum a, [1] sum b, [2] ||Au||^2, [3] ||Bu||^2
__global__ void __launch_bounds__(256) k_lwrq_ab(YeeGeom g, YeeMat mt, double* a, double* b, double* out,
                                                 double* partials, unsigned* counter) {
  const long long q = g.q, tot = q * q * q;
  Red<double, 4> acc{};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % q), j = (int)((p / q) % q), k = (int)(p / (q * q));
    double2 A[3], B[3], U[3];
    yee_ab(g, mt, i, j, k, A, B, U);
    double av = 0.0, bv = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      av += U[c].x * A[c].x + U[c].y * A[c].y;  // Re(conj(u) Au)
      bv += U[c].x * B[c].x + U[c].y * B[c].y;
      acc.v[2] += cabs2<double>(A[c]);
      acc.v[3] += cabs2<double>(B[c]);
    }
    a[p] = av;
    b[p] = bv;
    acc.v[0] += av;
    acc.v[1] += bv;
  }
  grid_sum_finalize<double, 4>(acc, partials, counter, [&](const Red<double, 4>& t) {
    for (int s = 0; s < 4; ++s) out[s] = t.v[s];
  });
}

struct Window {
  double k[2 * kLwrqR + 1];
};

// sum of the window taps that fall inside [0, q) around index i (the
// normalisation of the zero-padded window along one axis)
__device__ __forceinline__ double window_mass(const Window& w, int i, int q) {
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 2 * kLwrqR + 1; ++t) {
    const int src = i - (t - kLwrqR);
    if (src >= 0 && src < q) s += w.k[t];
  }
  return s;
}

// One axis of the separable window for two arrays: out(i) = sum_t k[t] in(i - (t - R)).
// With normalise, in is divided by den = dx(i) dy(j) dz(k) at the source point.
__global__ void __launch_bounds__(256) k_lwrq_conv(const double* inA, const double* inB, double* outA, double* outB,
                                                   int q, int axis, Window w, int normalise) {
  const long long tot = (long long)q * q * q;
  const long long stride = axis == 0 ? 1 : axis == 1 ? q : (long long)q * q;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % q), j = (int)((p / q) % q), k = (int)(p / ((long long)q * q));
    const int c = axis == 0 ? i : axis == 1 ? j : k;
    double dyz = 1.0;
    if (normalise) dyz = window_mass(w, j, q) * window_mass(w, k, q);
    double sa = 0.0, sb = 0.0;
#pragma unroll
    for (int t = 0; t < 2 * kLwrqR + 1; ++t) {
      const int src = c - (t - kLwrqR);
      if (src >= 0 && src < q) {
        const long long ps = p + (long long)(src - c) * stride;
        double wa = w.k[t], wb = w.k[t];
        if (normalise) {
          const double den = window_mass(w, src, q) * dyz;
          wa /= den;
          wb /= den;
        }
        sa += wa * inA[ps];
        sb += wb * inB[ps];
      }
    }
    outA[p] = sa;
    outB[p] = sb;
  }
}

// [0] sum E, [1] sum M, [2] non-finite count
__global__ void __launch_bounds__(256) k_lwrq_stat1(const double* E, const double* M, long long tot, double* out,
                                                    double* partials, unsigned* counter) {
  Red<double, 3> acc{};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
    const double e = E[p], mm = M[p];
    acc.v[0] += e;
    acc.v[1] += mm;
    acc.v[2] += (isfinite(e) && isfinite(mm)) ? 0.0 : 1.0;
  }
  grid_sum_finalize<double, 3>(acc, partials, counter, [&](const Red<double, 3>& t) {
    for (int s = 0; s < 3; ++s) out[s] = t.v[s];
  });
}

// per-block max of M into bmax[blockIdx.x]
__global__ void __launch_bounds__(256) k_lwrq_max(const double* M, long long tot, double* bmax) {
  __shared__ double red[256];
  double v = -INFINITY;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x)
    v = fmax(v, M[p]);
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) bmax[blockIdx.x] = red[0];
}
__global__ void k_lwrq_max_final(const double* bmax, int nb, double* out) {
  __shared__ double red[256];
  double v = -INFINITY;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v = fmax(v, bmax[i]);
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// [0] count M <= floor, [1] sum M |E/M - lambda|^2; slices of rho at z = 0 and x = 0
__global__ void __launch_bounds__(256) k_lwrq_stat2(const double* E, const double* M, int q, double floor_,
                                                    double lambda, double* z0, double* x0, double* out,
                                                    double* partials, unsigned* counter) {
  const long long tot = (long long)q * q * q;
  const int c = (q - 1) / 2;
  Red<double, 2> acc{};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
    const double mm = M[p], rho = E[p] / mm;
    acc.v[0] += (mm <= floor_) ? 1.0 : 0.0;
    const double d = rho - lambda;
    acc.v[1] += mm * d * d;
    const int i = (int)(p % q), j = (int)((p / q) % q), k = (int)(p / ((long long)q * q));
    if (z0 && k == c) z0[i + (long long)q * j] = rho;
    if (x0 && i == c) x0[j + (long long)q * k] = rho;
  }
  grid_sum_finalize<double, 2>(acc, partials, counter, [&](const Red<double, 2>& t) {
    out[0] = t.v[0];
    out[1] = t.v[1];
  });
}

// [0] ||Au - l3 Bu||^2, [1] ||Au - l6 Bu||^2
__global__ void __launch_bounds__(256) k_lwrq_resid(YeeGeom g, YeeMat mt, double l3, double l6, double* out,
                                                    double* partials, unsigned* counter) {
  const long long q = g.q, tot = q * q * q;
  Red<double, 2> acc{};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < tot; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % q), j = (int)((p / q) % q), k = (int)(p / (q * q));
    double2 A[3], B[3], U[3];
    yee_ab(g, mt, i, j, k, A, B, U);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      acc.v[0] += cabs2<double>(csub<double>(A[c], cscale<double>(B[c], l3)));
      acc.v[1] += cabs2<double>(csub<double>(A[c], cscale<double>(B[c], l6)));
    }
  }
  grid_sum_finalize<double, 2>(acc, partials, counter, [&](const Red<double, 2>& t) {
    out[0] = t.v[0];
    out[1] = t.v[1];
  });
}

}  // namespace fame

using namespace fame;

extern "C" int fame_yee_lwrq_metrics(fame_ctx* ctx, const void* u1, const void* u2, const void* u3, int n, double h,
                                     const double* P, int material_kind, double mp0, double mp1, double lambda6D,
                                     double* metrics, double* slice_z0, double* slice_x0) {
  if (!ctx || !u1 || !u2 || !u3 || !P || !metrics || n < 1 || !(h > 0.0) || (material_kind != 0 && material_kind != 1))
    return fail(FAME_ERR_INVALID, "fame_yee_lwrq_metrics arguments");
  if (!(std::fabs(lambda6D) > 0.0)) return fail(FAME_ERR_INVALID, "lambda6D must be nonzero");
  const int q = 2 * n + 1;
  const long long tot = (long long)q * q * q;
  cudaStream_t s = ctx->stream;
  YeeGeom g{(const double2*)u1, (const double2*)u2, (const double2*)u3, n, 2 * n + 3, q, h};
  YeeMat mt{};
  mt.kind = material_kind;
  mt.p0 = mp0;
  mt.p1 = mp1;
  for (int i = 0; i < 18; ++i) mt.P[i] = P[i];
  Window w{};
  const double sigma = 2.0 * h;
  for (int t = 0; t < 2 * kLwrqR + 1; ++t) {
    const double off = (t - kLwrqR) * h;
    w.k[t] = std::exp(-(off * off) / (sigma * sigma));
  }
  const int nb = lblocks(tot);
  Carve size_only;
  auto carve = [&](Carve& cv, double** a, double** b, double** T, double** U, double** sc, double** part,
                   double** bmax, double** z0, double** x0, unsigned** counter) {
    *a = cv.take<double>(tot);
    *b = cv.take<double>(tot);
    *T = cv.take<double>(tot);
    *U = cv.take<double>(tot);
    *sc = cv.take<double>(16);
    *part = cv.take<double>((size_t)nb * 4);
    *bmax = cv.take<double>(nb);
    *z0 = cv.take<double>((size_t)q * q);
    *x0 = cv.take<double>((size_t)q * q);
    *counter = cv.take<unsigned>(1);
  };
  double *a, *b, *T, *U, *sc, *part, *bmax, *z0, *x0;
  unsigned* counter;
  carve(size_only, &a, &b, &T, &U, &sc, &part, &bmax, &z0, &x0, &counter);
  void* ws = nullptr;
  FAME_TRY(ctx_workspace(ctx, size_only.used, &ws));
  Carve cv;
  cv.base = static_cast<char*>(ws);
  carve(cv, &a, &b, &T, &U, &sc, &part, &bmax, &z0, &x0, &counter);
  FAME_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));

  double h1[4], h2[3], h3[2], h4[2], maxM = 0.0;
  k_lwrq_ab<<<nb, 256, 0, s>>>(g, mt, a, b, sc, part, counter);
  ::fame::count_launch();
  FAME_TRY(read_back(ctx, sc, h1, sizeof(h1)));
  const double sumA = h1[0], sumB = h1[1], nA = std::sqrt(h1[2]), nB = std::sqrt(h1[3]);
  if (!(sumB > 0.0)) return fail(FAME_ERR_INVALID, "Cropped Yee mass is not positive.");
  const double lamCrop = sumA / sumB;
  // E- and M-paths through the separable window: a -> T -> a -> T (E), b -> U -> b -> U (M)
  k_lwrq_conv<<<nb, 256, 0, s>>>(a, b, T, U, q, 0, w, 1);
  k_lwrq_conv<<<nb, 256, 0, s>>>(T, U, a, b, q, 1, w, 0);
  k_lwrq_conv<<<nb, 256, 0, s>>>(a, b, T, U, q, 2, w, 0);
  ::fame::count_launch(3);
  const double* E = T;
  const double* M = U;
  k_lwrq_stat1<<<nb, 256, 0, s>>>(E, M, tot, sc, part, counter);
  k_lwrq_max<<<nb, 256, 0, s>>>(M, tot, bmax);
  k_lwrq_max_final<<<1, 256, 0, s>>>(bmax, nb, sc + 8);
  ::fame::count_launch(3);
  FAME_CUDA_TRY(cudaGetLastError());
  FAME_TRY(read_back(ctx, sc, h2, sizeof(h2)));
  FAME_TRY(read_back(ctx, sc + 8, &maxM, sizeof(double)));
  if (h2[2] != 0.0) return fail(FAME_ERR_NONFINITE, "Invalid LWRQ column-normalization or non-finite window sums.");
  const double sumE = h2[0], sumM = h2[1];
  const double lam = sumE / sumM;
  k_lwrq_stat2<<<nb, 256, 0, s>>>(E, M, q, 1e-14 * maxM, lam, slice_z0 ? z0 : nullptr, slice_x0 ? x0 : nullptr,
                                  sc, part, counter);
  ::fame::count_launch();
  FAME_TRY(read_back(ctx, sc, h3, sizeof(h3)));
  if (h3[0] != 0.0) return fail(FAME_ERR_NONFINITE, "Nonpositive or numerically tiny local LWRQ mass encountered.");
  const double V = h3[1] / (sumM * lam * lam);
  k_lwrq_resid<<<nb, 256, 0, s>>>(g, mt, lam, lambda6D, sc, part, counter);
  ::fame::count_launch();
  FAME_TRY(read_back(ctx, sc, h4, sizeof(h4)));
  const double tiny = 2.220446049250313e-16;
  const double partE = std::fabs(sumE - sumA) / std::max(std::fabs(sumA), tiny);
  const double partM = std::fabs(sumM - sumB) / std::max(std::fabs(sumB), tiny);
  metrics[0] = lamCrop;
  metrics[1] = lam;
  metrics[2] = std::sqrt(h4[0]) / (nA + std::fabs(lam) * nB);
  metrics[3] = std::sqrt(h4[1]) / (nA + std::fabs(lambda6D) * nB);
  metrics[4] = std::fabs(lam - lambda6D) / std::fabs(lambda6D);
  metrics[5] = V;
  metrics[6] = std::sqrt(std::max(V, 0.0));
  metrics[7] = std::max(partE, partM);
  metrics[8] = std::fabs(lam - lamCrop) / std::max(std::fabs(lamCrop), tiny);
  metrics[9] = sumB;
  if (slice_z0 || slice_x0) {
    FAME_CUDA_TRY(cudaStreamSynchronize(s));
    if (slice_z0) FAME_CUDA_TRY(cudaMemcpy(slice_z0, z0, (size_t)q * q * sizeof(double), cudaMemcpyDeviceToHost));
    if (slice_x0) FAME_CUDA_TRY(cudaMemcpy(slice_x0, x0, (size_t)q * q * sizeof(double), cudaMemcpyDeviceToHost));
    // relative deviation |rho - lambda3D| / |lambda3D| (exp3/compute_yee_lwrq_metrics_exp4.m:77-80)
    for (double* sl : {slice_z0, slice_x0})
      if (sl)
        for (long long i = 0; i < (long long)q * q; ++i) sl[i] = std::fabs(sl[i] - lam) / std::fabs(lam);
  }
  return FAME_OK;
}
