// Small-radix 6D FFT building blocks for the Fourier mass operator
//   y = fftn(E .* ifftn(x))          (exp1/applyMij_fft.m:11)
// on the (2N)^6 grid, n = 2N <= 14 points per axis.
//
// The 6D transform is split into three passes over HBM/L2:
//   pass A  inverse DFT along axes 1-3 (contiguous n^3 cubes), fused prologue;
//   pass B  inverse DFT along axes 4-6 (cubes strided by n^3), multiply by
//           E/NF, forward DFT along axes 4-6;
//   pass C  forward DFT along axes 1-3, fused epilogue (+ grid reduction).
// Each CTA stages whole n^3 cubes in shared memory (rows padded to n+1 to
// avoid bank conflicts), one thread transforms one line in registers with a
// fully unrolled mixed-radix (2,3,5,7) DFT whose twiddles are compile-time
// constants.
#pragma once
#include "fame_common.cuh"
#include "twiddles.cuh"

namespace fame {

template <int n> struct SmallestFactor {
  static constexpr int value = (n % 2 == 0) ? 2 : (n % 3 == 0) ? 3 : (n % 5 == 0) ? 5 : (n % 7 == 0) ? 7 : n;
};

// x *= exp(SIGN * 2*pi*i*e/n); quarter-turn rotations are exact.
template <int n, int SIGN, typename T>
__device__ __forceinline__ void rotate(T& xr, T& xi, int e) {
  const double c = tw_cos(n, e), s = SIGN * tw_sin(n, e);
  if (s == 0.0) {
    if (c == 1.0) return;
    if (c == -1.0) { xr = -xr; xi = -xi; return; }
  }
  if (c == 0.0) {
    if (s == 1.0) { T t = xr; xr = -xi; xi = t; return; }
    if (s == -1.0) { T t = xr; xr = xi; xi = -t; return; }
  }
  T tr = xr * (T)c - xi * (T)s;
  xi = xr * (T)s + xi * (T)c;
  xr = tr;
}

// In-place DFT of length n on register arrays.  SIGN=-1: forward (fftn),
// SIGN=+1: inverse without the 1/n factor.
template <int n, int SIGN, typename T, bool PRIME = (SmallestFactor<n>::value == n)>
struct Dft;

template <int SIGN, typename T> struct Dft<1, SIGN, T, true> {
  static __device__ __forceinline__ void run(T*, T*) {}
};

template <int SIGN, typename T> struct Dft<2, SIGN, T, true> {
  static __device__ __forceinline__ void run(T* re, T* im) {
    T ar = re[0], ai = im[0];
    re[0] = ar + re[1]; im[0] = ai + im[1];
    re[1] = ar - re[1]; im[1] = ai - im[1];
  }
};

// Odd prime length: pair j with n-j (real symmetric/antisymmetric parts).
template <int n, int SIGN, typename T> struct Dft<n, SIGN, T, true> {
  static __device__ __forceinline__ void run(T* re, T* im) {
    constexpr int h = (n - 1) / 2;
    T sr[h], si[h], dr[h], di[h];
#pragma unroll
    for (int j = 1; j <= h; ++j) {
      sr[j - 1] = re[j] + re[n - j]; si[j - 1] = im[j] + im[n - j];
      dr[j - 1] = re[j] - re[n - j]; di[j - 1] = im[j] - im[n - j];
    }
    const T x0r = re[0], x0i = im[0];
    T sumr = x0r, sumi = x0i;
#pragma unroll
    for (int j = 0; j < h; ++j) { sumr += sr[j]; sumi += si[j]; }
#pragma unroll
    for (int k = 1; k <= h; ++k) {
      T Ar = x0r, Ai = x0i, Br = 0, Bi = 0;
#pragma unroll
      for (int j = 1; j <= h; ++j) {
        const T c = (T)tw_cos(n, (j * k) % n), s = (T)tw_sin(n, (j * k) % n);
        Ar += sr[j - 1] * c; Ai += si[j - 1] * c;
        Br += dr[j - 1] * s; Bi += di[j - 1] * s;
      }
      re[k] = Ar - SIGN * Bi; im[k] = Ai + SIGN * Br;
      re[n - k] = Ar + SIGN * Bi; im[n - k] = Ai - SIGN * Br;
    }
    re[0] = sumr; im[0] = sumi;
  }
};

// Composite length n = R*M (R smallest prime factor): decimation in time.
template <int n, int SIGN, typename T> struct Dft<n, SIGN, T, false> {
  static __device__ __forceinline__ void run(T* re, T* im) {
    constexpr int R = SmallestFactor<n>::value, M = n / R;
    T ar[R][M], ai[R][M];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int m = 0; m < M; ++m) { ar[r][m] = re[R * m + r]; ai[r][m] = im[R * m + r]; }
#pragma unroll
    for (int r = 0; r < R; ++r) Dft<M, SIGN, T>::run(ar[r], ai[r]);
#pragma unroll
    for (int r = 1; r < R; ++r)
#pragma unroll
      for (int k2 = 1; k2 < M; ++k2) rotate<n, SIGN, T>(ar[r][k2], ai[r][k2], (r * k2) % n);
#pragma unroll
    for (int k2 = 0; k2 < M; ++k2) {
      T br[R], bi[R];
#pragma unroll
      for (int r = 0; r < R; ++r) { br[r] = ar[r][k2]; bi[r] = ai[r][k2]; }
      Dft<R, SIGN, T>::run(br, bi);
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) { re[k2 + M * k1] = br[k1]; im[k2 + M * k1] = bi[k1]; }
    }
  }
};

// ------------------------------------------------------------ cube geometry
// One n^3 cube in shared memory: element (i1,i2,i3) at i1 + (n+1)*(i2 + n*i3).
template <int n> struct Cube {
  static constexpr int n2 = n * n, n3 = n * n * n, pitch = n + 1;
  static constexpr int size = pitch * n2;  // elements incl. padding
  static __device__ __forceinline__ int sidx(int g) { return (g % n) + pitch * (g / n); }
};

template <int n, int SIGN, typename T>
__device__ __forceinline__ void line_dft(C<T>* p, int stride) {
  T re[n], im[n];
#pragma unroll
  for (int j = 0; j < n; ++j) { C<T> v = p[j * stride]; re[j] = v.x; im[j] = v.y; }
  Dft<n, SIGN, T>::run(re, im);
#pragma unroll
  for (int j = 0; j < n; ++j) p[j * stride] = mk<T>(re[j], im[j]);
}

// 3D DFT of `ncubes` consecutive cubes in shared memory (all threads).
template <int n, int SIGN, typename T>
__device__ __forceinline__ void cubes_dft3(C<T>* s, int ncubes) {
  using Q = Cube<n>;
  const int lines = ncubes * Q::n2;
  for (int t = threadIdx.x; t < lines; t += blockDim.x) {  // axis 1 (unit stride)
    const int c = t / Q::n2, l = t % Q::n2;
    line_dft<n, SIGN, T>(s + c * Q::size + Q::pitch * l, 1);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < lines; t += blockDim.x) {  // axis 2 (stride pitch)
    const int c = t / Q::n2, l = t % Q::n2;
    line_dft<n, SIGN, T>(s + c * Q::size + (l % n) + Q::pitch * n * (l / n), Q::pitch);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < lines; t += blockDim.x) {  // axis 3 (stride pitch*n)
    const int c = t / Q::n2, l = t % Q::n2;
    line_dft<n, SIGN, T>(s + c * Q::size + (l % n) + Q::pitch * (l / n), Q::pitch * n);
  }
  __syncthreads();
}

// Device-resident status word used to gate queued iterations: kernels return
// immediately when *gate == 0.
struct Gate {
  const int* active;  // nullptr: always run
  __device__ __forceinline__ bool off() const { return active != nullptr && *((volatile const int*)active) == 0; }
};

// ------------------------------------------------------------------ pass A
// CTA = one column c456 (contiguous cube of n^3 modes) x F fields.
// Pro::load(i, v[F]) produces the F field values at mode i.
template <int n, typename T, int F, class Pro>
__global__ void __launch_bounds__(512) k_passA(Pro pro, C<T>* __restrict__ work, long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  const long long base = (long long)blockIdx.x * Q::n3;
  for (int g = threadIdx.x; g < Q::n3; g += blockDim.x) {
    C<T> v[F];
    pro.load(base + g, v);
#pragma unroll
    for (int f = 0; f < F; ++f) s[f * Q::size + Q::sidx(g)] = v[f];
  }
  __syncthreads();
  cubes_dft3<n, +1, T>(s, F);
  for (int idx = threadIdx.x; idx < F * Q::n3; idx += blockDim.x) {
    const int f = idx / Q::n3, g = idx % Q::n3;
    work[f * NF + base + g] = s[f * Q::size + Q::sidx(g)];
  }
}

// ------------------------------------------------------------------ pass B
// CTA = TT consecutive c123 indices x all n^3 c456 indices of one field
// (blockIdx.y).  Inverse DFT over axes 4-6, multiply by Es = E/NF, forward.
template <int n, typename T, int TT, typename TE>
__global__ void __launch_bounds__(512) k_passB(C<T>* __restrict__ work, const TE* __restrict__ Es, TE escale,
                                              long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  C<T>* w = work + (long long)blockIdx.y * NF;
  const long long c0 = (long long)blockIdx.x * TT;
  for (int idx = threadIdx.x; idx < TT * Q::n3; idx += blockDim.x) {
    const int t = idx % TT, g = idx / TT;
    s[t * Q::size + Q::sidx(g)] = w[c0 + t + (long long)Q::n3 * g];
  }
  __syncthreads();
  cubes_dft3<n, +1, T>(s, TT);
  for (int idx = threadIdx.x; idx < TT * Q::n3; idx += blockDim.x) {
    const int t = idx % TT, g = idx / TT;
    const T e = (T)(Es[c0 + t + (long long)Q::n3 * g] * escale);
    C<T>& v = s[t * Q::size + Q::sidx(g)];
    v = cscale<T>(v, e);
  }
  __syncthreads();
  cubes_dft3<n, -1, T>(s, TT);
  for (int idx = threadIdx.x; idx < TT * Q::n3; idx += blockDim.x) {
    const int t = idx % TT, g = idx / TT;
    w[c0 + t + (long long)Q::n3 * g] = s[t * Q::size + Q::sidx(g)];
  }
}

// ------------------------------------------------------------------ pass C
// CTA = one column c456 x F fields; forward DFT over axes 1-3, then
// Epi::store(i, v[F], acc) per mode, then a grid reduction of acc with
// Epi::finalize (when Epi::K > 0).
template <int n, typename T, int F, class Epi>
__global__ void __launch_bounds__(512) k_passC(Epi epi, const C<T>* __restrict__ work, long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n>;
  using A = typename Epi::Acc;
  constexpr int K = Epi::K;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  const long long base = (long long)blockIdx.x * Q::n3;
  for (int idx = threadIdx.x; idx < F * Q::n3; idx += blockDim.x) {
    const int f = idx / Q::n3, g = idx % Q::n3;
    s[f * Q::size + Q::sidx(g)] = work[f * NF + base + g];
  }
  __syncthreads();
  cubes_dft3<n, -1, T>(s, F);
  Red<A, (K > 0 ? K : 1)> acc;
#pragma unroll
  for (int k = 0; k < (K > 0 ? K : 1); ++k) acc.v[k] = 0;
  for (int g = threadIdx.x; g < Q::n3; g += blockDim.x) {
    C<T> v[F];
#pragma unroll
    for (int f = 0; f < F; ++f) v[f] = s[f * Q::size + Q::sidx(g)];
    epi.store(base + g, v, acc);
  }
  if constexpr (K > 0) {
    grid_sum_finalize<A, K>(acc, epi.partials, epi.counter, [&](const Red<A, K>& tot) { epi.finalize(tot); });
  }
}

}  // namespace fame
