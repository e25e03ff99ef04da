// Pass B of the 6D mass operator: inverse DFT along axes 4-6, multiply by the
// material E/NF, forward DFT along axes 4-6, for every tile of the
// tile-major work fields (WorkTile in fft6d.cuh).
//
// Persistent kernel: each CTA owns a contiguous range of units (tile k,
// field f) and streams them through two shared-memory stages.  One thread
// pulls a unit with n bulk copies (one per i6-plane, completed on the stage's
// mbarrier) plus, at the first unit of a tile, the material tile; the copy of
// unit i+2 is issued as soon as unit i has been read out of its stage, so
// global latency overlaps the transforms of the next unit.  In shared memory
// element (t, i4, i5, i6) of a unit sits at t + TT*i4 + P5*i5 + P6*i6 with
// P5 = TT*n and P6 = TT*n^2 + TT (one padding row per plane); each phase
// transforms one line per thread in place:
//   phase 1  axis 4, lanes (t, i6, i5) -- stride TT
//   phase 2  axis 6, lanes (t, i4, i5) -- stride P6
//   phase 3  axis 5, lanes (t, i4, i6) -- stride P5: inverse, *E/NF, forward
//   phase 4  axis 6 (forward)
//   phase 5  axis 4 (forward), then rows of TT elements stored to global.
// The lane orders and the padding row were chosen by counting shared-memory
// wavefronts of every phase (16-lane halves for 8-byte, 8-lane quarters for
// 16-byte elements); they reach the conflict-free count for n <= 8 and stay
// within 12% of it for the larger sizes.
#pragma once
#include "bulk.cuh"
#include "fft6d.cuh"


namespace fame {

template <int n, typename T> struct PassBGeom {
  static constexpr int TT = WorkTile<n, T>::TT;
  static constexpr int n2 = n * n, n3 = n * n * n;
  static constexpr int L = TT * n2;        // lines per phase (one per working thread)
  static constexpr int P5 = TT * n;        // i5 pitch (elements)
  static constexpr int P6 = TT * n2 + TT;  // i6 plane pitch
  static constexpr int stage = n * P6;     // elements per stage
  static constexpr int tile = TT * n3;     // elements per tile (global)
  static constexpr unsigned plane_bytes = (unsigned)(TT * n2 * sizeof(C<T>));
  static constexpr int threads = (L + 31) / 32 * 32;
  static_assert((P6 * sizeof(C<T>)) % 16 == 0 && (stage * sizeof(C<T>)) % 16 == 0, "bulk-copy alignment");
  static_assert(plane_bytes % 16 == 0, "bulk-copy size");
  template <typename TE> static constexpr size_t smem_bytes() {
    return 2 * stage * sizeof(C<T>) + 2 * (size_t)tile * sizeof(TE) + 2 * sizeof(uint64_t);
  }
};

template <int n, typename T, typename TE>
__global__ void __launch_bounds__(512) k_passB(C<T>* __restrict__ work, const TE* __restrict__ Et, int nfields,
                                              long long NF, Gate gate, unsigned* fault,
                                              unsigned poll_limit = kMbarPollLimit, int arm_only = 0) {
  if (gate.off()) return;
  using G = PassBGeom<n, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C<T>* stg = reinterpret_cast<C<T>*>(smem_raw);
  TE* es = reinterpret_cast<TE*>(smem_raw + 2 * G::stage * sizeof(C<T>));
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * G::stage * sizeof(C<T>) + 2 * G::tile * sizeof(TE));
  constexpr int tiles = G::n3 / G::TT;
  const int U = tiles * nfields;
  const int u0 = (int)((long long)blockIdx.x * U / gridDim.x);
  const int u1 = (int)((long long)(blockIdx.x + 1) * U / gridDim.x);
  if (u0 >= u1) return;
  const int k0 = u0 / nfields;
  const int tid = threadIdx.x;

  auto issue = [&](int u, int s) {
    const int k = u / nfields, f = u - k * nfields;
    const bool needE = (u == u0) || (f == 0);
    mbar_arrive_expect_tx(&bar[s], n * G::plane_bytes + (needE ? (unsigned)(G::tile * sizeof(TE)) : 0u));
    if (arm_only) return;  // fault-path self-test: the bytes never come, nothing is in flight
    const C<T>* src = work + (long long)f * NF + (long long)k * G::tile;
    C<T>* dst = stg + s * G::stage;
#pragma unroll 1
    for (int p = 0; p < n; ++p) bulk_g2s(dst + p * G::P6, src + p * G::TT * G::n2, G::plane_bytes, &bar[s]);
    if (needE)
      bulk_g2s(es + ((k - k0) & 1) * G::tile, Et + (long long)k * G::tile, (unsigned)(G::tile * sizeof(TE)), &bar[s]);
  };

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
    issue(u0, 0);
    if (u0 + 1 < u1) issue(u0 + 1, 1);
  }
  __syncthreads();

  const bool act = tid < G::L;
  const int t = tid % G::TT, r = tid / G::TT, ra = r % n, rb = r / n;
  const int b1 = t + G::P5 * rb + G::P6 * ra;  // axis-4 line (t, i6 = ra, i5 = rb)
  const int b2 = t + G::TT * ra + G::P5 * rb;  // axis-6 line (t, i4 = ra, i5 = rb)
  const int b3 = t + G::TT * ra + G::P6 * rb;  // axis-5 line (t, i4 = ra, i6 = rb)
  const int gout = G::TT * (n * rb + G::n2 * ra) + t;  // (t, i4 = 0, i5 = rb, i6 = ra) within a tile

#pragma unroll 1
  for (int u = u0, i = 0; u < u1; ++u, ++i) {
    const int s = i & 1;
    const bool landed = mbar_wait(&bar[s], (unsigned)((i >> 1) & 1), poll_limit);
    if (!__syncthreads_and(landed)) {  // bounded wait, agreed on by the whole CTA
      if (fault && tid == 0) atomicOr(fault, 1u);
      return;
    }
    C<T>* S = stg + s * G::stage;
    const int k = u / nfields, f = u - k * nfields;
    const TE* E = es + ((k - k0) & 1) * G::tile;
    if (act) line_dft<n, +1, T>(S + b1, G::TT);
    __syncthreads();
    if (act) line_dft<n, +1, T>(S + b2, G::P6);
    __syncthreads();
    if (act) {
      C<T>* p = S + b3;
      T re[n], im[n];
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = p[j * G::P5];
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, +1, T>::run(re, im);
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const T e = (T)E[j * G::L + tid];
        re[j] *= e;
        im[j] *= e;
      }
      Dft<n, -1, T>::run(re, im);
#pragma unroll
      for (int j = 0; j < n; ++j) p[j * G::P5] = mk<T>(re[j], im[j]);
    }
    __syncthreads();
    if (act) line_dft<n, -1, T>(S + b2, G::P6);
    __syncthreads();
    T re[n], im[n];
    if (act) {
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const C<T> v = S[b1 + j * G::TT];
        re[j] = v.x;
        im[j] = v.y;
      }
      Dft<n, -1, T>::run(re, im);
    }
    __syncthreads();  // stage s has been read out: refill it
    if (tid == 0 && u + 2 < u1) {
      fence_proxy_async_smem();
      issue(u + 2, s);
    }
    if (act) {
      C<T>* dst = work + (long long)f * NF + (long long)k * G::tile + gout;
#pragma unroll
      for (int j = 0; j < n; ++j) dst[j * G::TT] = mk<T>(re[j], im[j]);
    }
  }
}

// Inverse-only pass B (axes 4-6, no material) in place on the tile-major
// fields, for the mass adjoint.  One CTA per (tile, field); plain loads.
template <int n, typename T>
__global__ void __launch_bounds__(512) k_passB_inv(C<T>* __restrict__ work, long long NF) {
  using G = PassBGeom<n, T>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C<T>* S = reinterpret_cast<C<T>*>(smem_raw);
  C<T>* w = work + (long long)blockIdx.y * NF + (long long)blockIdx.x * G::tile;
  constexpr int PL = G::TT * G::n2;
  for (int e = threadIdx.x; e < G::tile; e += blockDim.x) S[(e / PL) * G::P6 + e % PL] = w[e];
  __syncthreads();
  const int tid = threadIdx.x;
  const bool act = tid < G::L;
  const int t = tid % G::TT, r = tid / G::TT, ra = r % n, rb = r / n;
  if (act) line_dft<n, +1, T>(S + t + G::P5 * rb + G::P6 * ra, G::TT);
  __syncthreads();
  if (act) line_dft<n, +1, T>(S + t + G::TT * ra + G::P5 * rb, G::P6);
  __syncthreads();
  if (act) line_dft<n, +1, T>(S + t + G::TT * ra + G::P6 * rb, G::P5);
  __syncthreads();
  for (int e = threadIdx.x; e < G::tile; e += blockDim.x) w[e] = S[(e / PL) * G::P6 + e % PL];
}

// Material in the order pass B reads it: tile kt holds, for j = i5 and the
// phase-3 line index kk = t + TT*(i4 + n*i6), the value E(c123, c456)*scale at
// kt*TT*n^3 + j*TT*n^2 + kk, with c123 = kt*TT + t, c456 = i4 + n*j + n^2*i6.
// With invert, the tile holds scale / E (the material of the inverse mass operator).
template <typename TE>
__global__ void k_tile_E(const double* __restrict__ E, int n, int TT, long long NF, double scale, int invert,
                         TE* __restrict__ out) {
  const long long n3 = (long long)n * n * n, L = (long long)TT * n * n, tile = TT * n3;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < NF; o += (long long)gridDim.x * blockDim.x) {
    const long long kt = o / tile, rem = o % tile;
    const long long j = rem / L, kk = rem % L;
    const long long t = kk % TT, rr = kk / TT, i4 = rr % n, i6 = rr / n;
    const long long c123 = kt * TT + t, c456 = i4 + n * j + (long long)n * n * i6;
    const double e = E[c123 + n3 * c456];
    out[o] = (TE)(invert ? scale / e : e * scale);
  }
}

}  // namespace fame
