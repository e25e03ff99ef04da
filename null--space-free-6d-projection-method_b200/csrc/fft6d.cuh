// Small-radix 6D FFT building blocks for the Fourier mass operator
//   y = fftn(E .* ifftn(x))          (exp1/applyMij_fft.m:11)
// on the (2N)^6 grid, n = 2N <= 14 points per axis.
//
// The 6D transform is split into three passes over HBM/L2:
//   pass A  inverse DFT along axes 1-3 (contiguous n^3 cubes), fused prologue;
//   pass B  inverse DFT along axes 4-6 (one tile of TT c123 indices x n^3
//           c456 indices at a time, see WorkTile), multiply by E/NF, forward
//           DFT along axes 4-6 (passb.cuh);
//   pass C  forward DFT along axes 1-3, fused epilogue (+ grid reduction).
// Each CTA stages whole n^3 cubes in shared memory (rows padded to n+1 to
// avoid bank conflicts), one thread transforms one line in registers with a
// fully unrolled mixed-radix (2,3,5,7) DFT whose twiddles are compile-time
// constants.
//
// Two orderings of the modes of one column (cube of n^3 modes, column index
// c456) are used:
//   natural  (the reference's column-major order): g = i1 + n*(i2 + n*i3)
//   line     (axis 1 slowest):                     q = (i2 + n*i3) + n^2*i1
// Vectors that stay inside a solve (PCG iterates, W1/W2/invC) use the line
// order, so that pass A reads and pass C writes one axis-1 line per thread
// with consecutive threads on consecutive addresses.  Prologue and epilogue
// functors receive both indices (ia = line order, in = natural order).
#pragma once
#include "fame_common.cuh"
#include "twiddles.cuh"

namespace fame {

// a * b + c (written out so that the DFTs below state their fused multiply-adds)
__host__ __device__ __forceinline__ float fmadd(float a, float b, float c) { return a * b + c; }
__host__ __device__ __forceinline__ double fmadd(double a, double b, double c) { return a * b + c; }

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
  const T tr = fmadd(xr, (T)c, xi * (T)(-s));
  xi = fmadd(xr, (T)s, xi * (T)c);
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
      T Ar = x0r, Ai = x0i;
      const T s1 = (T)tw_sin(n, k % n);
      T Br = dr[0] * s1, Bi = di[0] * s1;
#pragma unroll
      for (int j = 1; j <= h; ++j) {
        const T c = (T)tw_cos(n, (j * k) % n);
        Ar = fmadd(sr[j - 1], c, Ar);
        Ai = fmadd(si[j - 1], c, Ai);
        if (j > 1) {
          const T s = (T)tw_sin(n, (j * k) % n);
          Br = fmadd(dr[j - 1], s, Br);
          Bi = fmadd(di[j - 1], s, Bi);
        }
      }
      if constexpr (SIGN > 0) {
        re[k] = Ar - Bi; im[k] = Ai + Br;
        re[n - k] = Ar + Bi; im[n - k] = Ai - Br;
      } else {
        re[k] = Ar + Bi; im[k] = Ai - Br;
        re[n - k] = Ar - Bi; im[n - k] = Ai + Br;
      }
    }
    re[0] = sumr; im[0] = sumi;
  }
};

// Coprime split n = n1*n2 (n1 the full power of the smallest prime factor),
// n2 == 1 when n is a prime power.
template <int n> struct PfaSplit {
  static constexpr int p = SmallestFactor<n>::value;
  static constexpr int pow_of(int m) { return m % p == 0 ? p * pow_of(m / p) : 1; }
  static constexpr int n1 = pow_of(n), n2 = n / n1;
  static constexpr int inv(int a, int m) {  // a^{-1} mod m (m > 1, gcd(a, m) = 1)
    int r = 1;
    while ((a * r) % m != 1) ++r;
    return r;
  }
};

// Composite length n = R*M (R smallest prime factor): decimation in time for
// prime powers; for n = n1*n2 with coprime n1, n2 > 1 the prime-factor
// (Good-Thomas) algorithm, which needs no twiddle factors: input
// x[(n2*i1 + n1*i2) mod n] -> length-n2 DFTs over i2, length-n1 DFTs over i1
// -> output X[(k1*n2*(n2^-1 mod n1) + k2*n1*(n1^-1 mod n2)) mod n].
template <int n, int SIGN, typename T> struct Dft<n, SIGN, T, false> {
  static __device__ __forceinline__ void run(T* re, T* im) {
    if constexpr (PfaSplit<n>::n2 > 1) {
      constexpr int n1 = PfaSplit<n>::n1, n2 = PfaSplit<n>::n2;
      constexpr int u2 = PfaSplit<n>::inv(n2 % n1, n1), u1 = PfaSplit<n>::inv(n1 % n2, n2);
      T ar[n1][n2], ai[n1][n2];
#pragma unroll
      for (int i1 = 0; i1 < n1; ++i1)
#pragma unroll
        for (int i2 = 0; i2 < n2; ++i2) {
          ar[i1][i2] = re[(n2 * i1 + n1 * i2) % n];
          ai[i1][i2] = im[(n2 * i1 + n1 * i2) % n];
        }
#pragma unroll
      for (int i1 = 0; i1 < n1; ++i1) Dft<n2, SIGN, T>::run(ar[i1], ai[i1]);
#pragma unroll
      for (int k2 = 0; k2 < n2; ++k2) {
        T br[n1], bi[n1];
#pragma unroll
        for (int i1 = 0; i1 < n1; ++i1) { br[i1] = ar[i1][k2]; bi[i1] = ai[i1][k2]; }
        Dft<n1, SIGN, T>::run(br, bi);
#pragma unroll
        for (int k1 = 0; k1 < n1; ++k1) {
          re[(k1 * n2 * u2 + k2 * n1 * u1) % n] = br[k1];
          im[(k1 * n2 * u2 + k2 * n1 * u1) % n] = bi[k1];
        }
      }
    } else {
      run_dit(re, im);
    }
  }
  static __device__ __forceinline__ void run_dit(T* re, T* im) {
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
// One n^3 cube in shared memory: element (i1,i2,i3) at i1 + P1*i2 + P2*i3.
// The row pitch P1, plane pitch P2 and cube stride S were chosen per size and
// element width by minimising shared-memory wavefronts over every access
// pattern of the passes below (32 lanes, 128-byte wavefronts).
template <int n, int ESZ> struct CubePitch;
template <> struct CubePitch<2, 8> { static constexpr int P1 = 3, P2 = 6, S = 12; };
template <> struct CubePitch<2, 16> { static constexpr int P1 = 3, P2 = 6, S = 12; };
template <> struct CubePitch<4, 8> { static constexpr int P1 = 4, P2 = 20, S = 81; };
template <> struct CubePitch<4, 16> { static constexpr int P1 = 5, P2 = 20, S = 84; };
template <> struct CubePitch<6, 8> { static constexpr int P1 = 9, P2 = 54, S = 324; };
template <> struct CubePitch<6, 16> { static constexpr int P1 = 9, P2 = 54, S = 324; };
template <> struct CubePitch<8, 8> { static constexpr int P1 = 9, P2 = 72, S = 580; };
template <> struct CubePitch<8, 16> { static constexpr int P1 = 9, P2 = 72, S = 580; };
template <> struct CubePitch<10, 8> { static constexpr int P1 = 17, P2 = 170, S = 1700; };
template <> struct CubePitch<10, 16> { static constexpr int P1 = 13, P2 = 130, S = 1300; };
template <> struct CubePitch<12, 8> { static constexpr int P1 = 12, P2 = 156, S = 1873; };
template <> struct CubePitch<12, 16> { static constexpr int P1 = 13, P2 = 156, S = 1876; };
template <> struct CubePitch<14, 8> { static constexpr int P1 = 17, P2 = 238, S = 3332; };
template <> struct CubePitch<14, 16> { static constexpr int P1 = 17, P2 = 238, S = 3332; };

template <int n, typename T> struct Cube {
  static constexpr int n2 = n * n, n3 = n * n * n;
  static constexpr int P1 = CubePitch<n, (int)sizeof(C<T>)>::P1;
  static constexpr int P2 = CubePitch<n, (int)sizeof(C<T>)>::P2;
  static constexpr int size = CubePitch<n, (int)sizeof(C<T>)>::S;  // elements per cube incl. padding
  static_assert(P1 >= n && P2 >= P1 * n && size >= P2 * n, "cube pitches");
  static __device__ __forceinline__ int at(int i1, int i2, int i3) { return i1 + P1 * i2 + P2 * i3; }
  // natural in-column index g = i1 + n*i2 + n^2*i3
  static __device__ __forceinline__ int sidx(int g) { return at(g % n, (g / n) % n, g / n2); }
  // start of the axis-1 line l = i2 + n*i3 (stride 1)
  static __device__ __forceinline__ int line1(int l) { return P1 * (l % n) + P2 * (l / n); }
  // start of the axis-2 line l = i1 + n*i3 (stride P1)
  static __device__ __forceinline__ int line2(int l) { return (l % n) + P2 * (l / n); }
  // start of the axis-3 line m = i1 + n*i2 (stride P2)
  static __device__ __forceinline__ int line3(int m) { return (m % n) + P1 * (m / n); }
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

// Device-resident status word used to gate queued iterations: kernels return
// immediately when *gate == 0.
struct Gate {
  const int* active;  // nullptr: always run
  __device__ __forceinline__ bool off() const { return active != nullptr && *((volatile const int*)active) == 0; }
};

// Columns (contiguous n^3 cubes) per CTA of passes A and C: enough lines
// (G*n^2) per CTA to keep ~200-300 threads busy, bounded by shared memory.
template <int n, typename T> struct PassACols {
  static constexpr int n2 = n * n, n3 = n * n * n;
  static constexpr int value = sizeof(T) == 4
      ? (n == 2 ? 8 : n == 4 ? 16 : n == 6 ? 6 : n == 8 ? 4 : n == 10 ? 2 : n == 12 ? 2 : 1)
      : (n == 2 ? 8 : n == 4 ? 8 : n == 6 ? 3 : n == 8 ? 2 : 1);
  static_assert(n3 % value == 0, "columns per CTA must divide n^3");
};

// Fields of one line are kept in registers together (FP32, or a single field);
// FP64 multi-field lines are processed one field at a time.
template <typename T, int F> struct FieldsInRegs {
  static constexpr bool value = sizeof(T) == 4 || F == 1;
};

// Functors whose vectors are mostly in natural order declare
// `static constexpr bool natural = true`; the staged prologue/epilogue loops
// then enumerate modes in natural order.
template <class E, class = void> struct Natural { static constexpr bool value = false; };
template <class E> struct Natural<E, decltype(void(E::natural))> { static constexpr bool value = E::natural; };

// Natural <-> line order of a global mode index (see the header comment).
template <int n> __device__ __forceinline__ long long nat_to_line(long long i) {
  constexpr int n2 = n * n, n3 = n * n * n;
  const long long cb = i - i % n3;
  const int g = (int)(i - cb);
  return cb + g / n + n2 * (g % n);
}
template <int n> __device__ __forceinline__ long long line_to_nat(long long i) {
  constexpr int n2 = n * n, n3 = n * n * n;
  const long long cb = i - i % n3;
  const int q = (int)(i - cb);
  return cb + q / n2 + n * (q % n2);
}

// Layout of the F work fields between the passes ("tile-major"): the n^3
// values of c123 = i1 + n*i2 + n^2*i3 are cut into tiles of TT consecutive
// indices, and tile k of a field is one contiguous block of TT*n^3 elements,
// rows of TT elements ordered by c456 = i4 + n*i5 + n^2*i6:
//   element (c123, c456) at TT*((c123/TT)*n^3 + c456) + c123%TT.
// Pass A writes and pass C reads rows of TT*sizeof(C<T>) >= 16 bytes; pass B
// pulls a tile (or one i6-plane of it) with a single bulk copy.
template <int n, typename T> struct WorkTile {
  static constexpr int TT = sizeof(T) == 4 ? (n <= 6 ? 8 : n <= 10 ? 4 : 2)
                                           : (n <= 6 ? 4 : n <= 12 ? 2 : 1);
  static_assert((n * n * n) % TT == 0, "tile width must divide n^3");
};
template <int n, typename T> __host__ __device__ __forceinline__ long long work_at(long long c123, long long c456) {
  constexpr int TT = WorkTile<n, T>::TT;
  constexpr long long n3 = (long long)n * n * n;
  return TT * ((c123 / TT) * n3 + c456) + c123 % TT;
}

// Element access to field f of the work fields (rows of TT interleaved complex values).
template <int n, typename T> struct WorkIO {
  static __device__ __forceinline__ void store(C<T>* w, long long c123, long long c456, C<T> v) {
    w[work_at<n, T>(c123, c456)] = v;
  }
  static __device__ __forceinline__ C<T> load(const C<T>* w, long long c123, long long c456) {
    return w[work_at<n, T>(c123, c456)];
  }
};

// ------------------------------------------------------------------ pass A
// CTA = G consecutive columns c456 x F fields.
//   phase 1: axis-1 lines through Pro::load(ia, in, v[F]) (thread <-> line
//            l = i2 + n*i3, element j = i1: ia = base + l + n^2 j, coalesced
//            across threads in line order), inverse DFT in registers, to smem;
//   phase 2: axis-2 lines in shared memory;
//   phase 3: axis-3 lines from shared memory, DFT, written to work in natural
//            order (coalesced).
template <int n, typename T, int F, int G, class Pro>
__global__ void __launch_bounds__(512) k_passA(Pro pro, C<T>* __restrict__ work, long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  const long long col0 = (long long)blockIdx.x * G;
  constexpr int items = G * Q::n2;
  if constexpr (FieldsInRegs<T, F>::value) {
    for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 1 from global
      const int cc = it / Q::n2, l = it % Q::n2;
      const long long cb = (col0 + cc) * Q::n3;
      C<T>* sc = s + cc * F * Q::size + Q::line1(l);
      T re[F][n], im[F][n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        C<T> v[F];
        pro.load(cb + l + Q::n2 * j, cb + j + (long long)n * l, v);
#pragma unroll
        for (int f = 0; f < F; ++f) { re[f][j] = v[f].x; im[f][j] = v[f].y; }
      }
#pragma unroll
      for (int f = 0; f < F; ++f) {
        Dft<n, +1, T>::run(re[f], im[f]);
#pragma unroll
        for (int j = 0; j < n; ++j) sc[f * Q::size + j] = mk<T>(re[f][j], im[f][j]);
      }
    }
  } else {
    // FP64 multi-field: prologue staged through shared memory, then axis 1 there;
    // modes enumerated in the functor's order (consecutive threads, consecutive addresses)
    for (int idx = threadIdx.x; idx < G * Q::n3; idx += blockDim.x) {
      const int cc = idx / Q::n3, q = idx % Q::n3;
      const int i1 = Natural<Pro>::value ? q % n : q / Q::n2, l = Natural<Pro>::value ? q / n : q % Q::n2;
      const long long cb = (col0 + cc) * Q::n3;
      C<T> v[F];
      pro.load(cb + l + (long long)Q::n2 * i1, cb + i1 + (long long)n * l, v);
#pragma unroll
      for (int f = 0; f < F; ++f) s[(cc * F + f) * Q::size + i1 + Q::line1(l)] = v[f];
    }
    __syncthreads();
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
      const int cc = it / Q::n2, l = it % Q::n2;
      C<T>* sc = s + cc * F * Q::size + Q::line1(l);
#pragma unroll
      for (int f = 0; f < F; ++f) line_dft<n, +1, T>(sc + f * Q::size, 1);
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 2
    const int cc = it / Q::n2, l = it % Q::n2;
    C<T>* sc = s + cc * F * Q::size + Q::line2(l);
#pragma unroll
    for (int f = 0; f < F; ++f) line_dft<n, +1, T>(sc + f * Q::size, Q::P1);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 3 -> global (natural order)
    const int cc = it / Q::n2, m = it % Q::n2;
    const C<T>* sc = s + cc * F * Q::size + Q::line3(m);
    const long long c456 = col0 + cc;
#pragma unroll
    for (int f = 0; f < F; ++f) {
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = sc[f * Q::size + Q::P2 * j];
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, +1, T>::run(re, im);
#pragma unroll
      for (int j = 0; j < n; ++j) WorkIO<n, T>::store(work + f * NF, m + Q::n2 * j, c456, mk<T>(re[j], im[j]));
    }
  }
}

// ------------------------------------------------------------------ pass C
// CTA = G columns x F fields; forward DFT over axes 3, 2, 1: axis-3 lines
// read from work (natural order, coalesced), axis 2 in shared memory, axis-1
// lines in registers, then Epi::store(ia, in, v[F], acc) per mode (line
// order coalesced across threads) and a grid reduction of acc with
// Epi::finalize (when Epi::K > 0).  FP64 multi-field chains run axis 1 in
// shared memory and feed the epilogue from there.
template <int n, typename T, int F, int G, class Epi>
__global__ void __launch_bounds__(512) k_passC(Epi epi, const C<T>* __restrict__ work, long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n, T>;
  using A = typename Epi::Acc;
  constexpr int K = Epi::K;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  const long long col0 = (long long)blockIdx.x * G;
  constexpr int items = G * Q::n2;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 3 from global
    const int cc = it / Q::n2, m = it % Q::n2;
    const long long c456 = col0 + cc;
    C<T>* sc = s + cc * F * Q::size + Q::line3(m);
#pragma unroll
    for (int f = 0; f < F; ++f) {
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = WorkIO<n, T>::load(work + f * NF, m + Q::n2 * j, c456);
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, -1, T>::run(re, im);
#pragma unroll
      for (int j = 0; j < n; ++j) sc[f * Q::size + Q::P2 * j] = mk<T>(re[j], im[j]);
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 2
    const int cc = it / Q::n2, l = it % Q::n2;
    C<T>* sc = s + cc * F * Q::size + Q::line2(l);
#pragma unroll
    for (int f = 0; f < F; ++f) line_dft<n, -1, T>(sc + f * Q::size, Q::P1);
  }
  __syncthreads();
  Red<A, (K > 0 ? K : 1)> acc;
#pragma unroll
  for (int k = 0; k < (K > 0 ? K : 1); ++k) acc.v[k] = 0;
  if constexpr (FieldsInRegs<T, F>::value) {
    for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 1 + epilogue in registers
      const int cc = it / Q::n2, l = it % Q::n2;
      const C<T>* sc = s + cc * F * Q::size + Q::line1(l);
      const long long cb = (col0 + cc) * Q::n3;
      T re[F][n], im[F][n];
#pragma unroll
      for (int f = 0; f < F; ++f) {
#pragma unroll
        for (int j = 0; j < n; ++j) {
          const C<T> v = sc[f * Q::size + j];
          re[f][j] = v.x;
          im[f][j] = v.y;
        }
        Dft<n, -1, T>::run(re[f], im[f]);
      }
#pragma unroll
      for (int j = 0; j < n; ++j) {
        C<T> v[F];
#pragma unroll
        for (int f = 0; f < F; ++f) v[f] = mk<T>(re[f][j], im[f][j]);
        epi.store(cb + l + Q::n2 * j, cb + j + (long long)n * l, v, acc);
      }
    }
  } else {
    for (int it = threadIdx.x; it < items; it += blockDim.x) {  // axis 1 in shared memory
      const int cc = it / Q::n2, l = it % Q::n2;
      C<T>* sc = s + cc * F * Q::size + Q::line1(l);
#pragma unroll
      for (int f = 0; f < F; ++f) line_dft<n, -1, T>(sc + f * Q::size, 1);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < G * Q::n3; idx += blockDim.x) {  // epilogue, functor's order
      const int cc = idx / Q::n3, q = idx % Q::n3;
      const int i1 = Natural<Epi>::value ? q % n : q / Q::n2, l = Natural<Epi>::value ? q / n : q % Q::n2;
      const long long cb = (col0 + cc) * Q::n3;
      C<T> v[F];
#pragma unroll
      for (int f = 0; f < F; ++f) v[f] = s[(cc * F + f) * Q::size + i1 + Q::line1(l)];
      epi.store(cb + l + (long long)Q::n2 * i1, cb + i1 + (long long)n * l, v, acc);
    }
  }
  if constexpr (K > 0) {
    grid_sum_finalize<A, K>(acc, epi.partials, epi.counter, [&](const Red<A, K>& tot) { epi.finalize(tot); });
  }
}

// ------------------------------------------------- linear-field chains
// Operators whose fields are linear in one vector, field_f(i) = a_f(i) u(i),
// and whose result is out(i) = S(i, sum_f b_f(i) v_f(i)) -- every Mhat chain
// (exp1/apply_Mhat_C_scalar_compact.m:8-21) is of this form.  Passes A and C
// then run the F fields one after another through a single shared-memory cube
// per column, holding one line of u (pass A) or of the running sum (pass C) in
// registers: a third of the shared memory and far fewer registers than the
// general chain.  One line per thread (blockDim >= G*n^2).
//
// LinPro:  C<T> load(ia, in, Ext&)   u(i) (pure loads; stores deferred to commit)
//          void commit(ia, in, const Ext&)
//          C<T> coef(f, ia, in)      a_f(i) (a_0 == 1 when unit0)
// LinEpi:  C<T> coef(f, ia, in)      b_f(i) (b_0 == 1 when unit0)
//          void store(ia, in, C<T> s, Red<Acc,K>& acc), finalize(tot)
template <int n, typename T, int F, int G, class Pro>
__global__ void __launch_bounds__(512) k_passA_lin(Pro pro, C<T>* __restrict__ work, long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  const long long col0 = (long long)blockIdx.x * G;
  constexpr int items = G * Q::n2;
  const int it = threadIdx.x;
  const bool act = it < items;
  const int cc = act ? it / Q::n2 : 0, l = act ? it % Q::n2 : 0;
  const long long cb = (col0 + cc) * Q::n3;
  C<T> u[n];
  if (act) {  // each thread owns the modes of its line: stores may follow each load
#pragma unroll
    for (int j = 0; j < n; ++j) {
      typename Pro::Ext e;
      u[j] = pro.load(cb + l + Q::n2 * j, cb + j + (long long)n * l, e);
      pro.commit(cb + l + Q::n2 * j, cb + j + (long long)n * l, e);
    }
  }
#pragma unroll 1
  for (int f = 0; f < F; ++f) {
    if (act) {  // axis 1 in registers
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        C<T> v = u[j];
        if (!(Pro::unit0 && f == 0)) v = cmul<T>(pro.coef(f, cb + l + Q::n2 * j, cb + j + (long long)n * l), v);
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, +1, T>::run(re, im);
      C<T>* sc = s + cc * Q::size + Q::line1(l);
#pragma unroll
      for (int j = 0; j < n; ++j) sc[j] = mk<T>(re[j], im[j]);
    }
    __syncthreads();
    if (act) line_dft<n, +1, T>(s + cc * Q::size + Q::line2(l), Q::P1);  // axis 2
    __syncthreads();
    if (act) {  // axis 3 -> work (tile-major), thread <-> m = i1 + n*i2
      const C<T>* sc = s + cc * Q::size + Q::line3(l);
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = sc[Q::P2 * j];
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, +1, T>::run(re, im);
      C<T>* wf = work + f * NF;
#pragma unroll
      for (int j = 0; j < n; ++j) WorkIO<n, T>::store(wf, l + Q::n2 * j, col0 + cc, mk<T>(re[j], im[j]));
    }
    __syncthreads();
  }
}

template <int n, typename T, int F, int G, class Epi>
__global__ void __launch_bounds__(512) k_passC_lin(Epi epi, const C<T>* __restrict__ work, long long NF, Gate gate) {
  if (gate.off()) return;
  using Q = Cube<n, T>;
  using A = typename Epi::Acc;
  constexpr int K = Epi::K;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C<T>* s = reinterpret_cast<C<T>*>(smem_raw);
  const long long col0 = (long long)blockIdx.x * G;
  constexpr int items = G * Q::n2;
  const int it = threadIdx.x;
  const bool act = it < items;
  const int cc = act ? it / Q::n2 : 0, l = act ? it % Q::n2 : 0;
  const long long cb = (col0 + cc) * Q::n3;
  C<T> sum[n];
#pragma unroll
  for (int j = 0; j < n; ++j) sum[j] = mk<T>(0, 0);
#pragma unroll 1
  for (int f = 0; f < F; ++f) {
    if (act) {  // axis 3 from work (tile-major), thread <-> m = i1 + n*i2
      const C<T>* wf = work + f * NF;
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = WorkIO<n, T>::load(wf, l + Q::n2 * j, col0 + cc);
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, -1, T>::run(re, im);
      C<T>* sc = s + cc * Q::size + Q::line3(l);
#pragma unroll
      for (int j = 0; j < n; ++j) sc[Q::P2 * j] = mk<T>(re[j], im[j]);
    }
    __syncthreads();
    if (act) line_dft<n, -1, T>(s + cc * Q::size + Q::line2(l), Q::P1);  // axis 2
    __syncthreads();
    if (act) {  // axis 1 in registers, accumulate b_f v_f
      const C<T>* sc = s + cc * Q::size + Q::line1(l);
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = sc[j];
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, -1, T>::run(re, im);
#pragma unroll
      for (int j = 0; j < n; ++j) {
        C<T> v = mk<T>(re[j], im[j]);
        if (!(Epi::unit0 && f == 0)) v = cmul<T>(epi.coef(f, cb + l + Q::n2 * j, cb + j + (long long)n * l), v);
        sum[j] = cadd<T>(sum[j], v);
      }
    }
    __syncthreads();
  }
  Red<A, (K > 0 ? K : 1)> acc;
#pragma unroll
  for (int k = 0; k < (K > 0 ? K : 1); ++k) acc.v[k] = 0;
  if (act) {
#pragma unroll
    for (int j = 0; j < n; ++j) epi.store(cb + l + Q::n2 * j, cb + j + (long long)n * l, sum[j], acc);
  }
  if constexpr (K > 0) {
    grid_sum_finalize<A, K>(acc, epi.partials, epi.counter, [&](const Red<A, K>& tot) { epi.finalize(tot); });
  }
}

}  // namespace fame
