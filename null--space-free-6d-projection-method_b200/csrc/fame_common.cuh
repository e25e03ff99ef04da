// Common device/host helpers for the FAME B200 library: complex arithmetic,
// status plumbing, deterministic grid reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <string>
#include "../../include/fame.h"

namespace fame {

// ----------------------------------------------------------------- complex
template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };
template <typename T> using C = typename cplx_t<T>::type;

template <typename T> __host__ __device__ __forceinline__ C<T> mk(T re, T im) {
  C<T> z; z.x = re; z.y = im; return z;
}
template <typename T> __host__ __device__ __forceinline__ C<T> cadd(C<T> a, C<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __host__ __device__ __forceinline__ C<T> csub(C<T> a, C<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __host__ __device__ __forceinline__ C<T> cmul(C<T> a, C<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
template <typename T> __host__ __device__ __forceinline__ C<T> cmulc(C<T> a, C<T> b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename T> __host__ __device__ __forceinline__ C<T> cscale(C<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
template <typename T> __host__ __device__ __forceinline__ C<T> cconj(C<T> a) { return mk<T>(a.x, -a.y); }
// a / b (complex), straightforward formula (operands are O(1) here)
template <typename T> __host__ __device__ __forceinline__ C<T> cdiv(C<T> a, C<T> b) {
  T d = b.x * b.x + b.y * b.y;
  return mk<T>((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
template <typename T> __host__ __device__ __forceinline__ T cabs2(C<T> a) { return a.x * a.x + a.y * a.y; }

template <typename To, typename From> __host__ __device__ __forceinline__ C<To> ccast(C<From> a) {
  return mk<To>((To)a.x, (To)a.y);
}

// ------------------------------------------------------------------ status
struct Error {
  int code;
  std::string msg;
};
void set_last_error(int code, const std::string& msg);
#define FAME_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess) {                                                      \
      ::fame::set_last_error(FAME_ERR_CUDA, std::string(#expr) + ": " +           \
                                                cudaGetErrorString(_e));          \
      return FAME_ERR_CUDA;                                                       \
    }                                                                             \
  } while (0)
#define FAME_TRY(expr)                   \
  do {                                   \
    int _s = (expr);                     \
    if (_s != FAME_OK) return _s;        \
  } while (0)
int fail(int code, const std::string& msg);
// Number of kernels this library has launched (all devices, all handles).
void count_launch(long long n = 1);
// Per-device fault word (set by bounded in-kernel waits that gave up; nullptr
// before a context exists on the current device) and SM count of the current device.
unsigned* fault_word();
int num_sms();

// --------------------------------------------------------------- reductions
// Sum of K accumulators.  Each block reduces its threads' values, writes
// them to partials[blockIdx.x*K + k]; the last block to finish sums the
// partials in block order (fixed order => bitwise reproducible) and calls
// fin(sum).  counter must be zero before the launch; the last block resets it.
template <typename A, int K> struct Red {
  A v[K];
};

template <typename A, int K>
__device__ __forceinline__ Red<A, K> warp_sum(Red<A, K> r) {
#pragma unroll
  for (int k = 0; k < K; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r.v[k] += __shfl_xor_sync(0xffffffffu, r.v[k], o);
  }
  return r;
}

// Block-wide sum; result valid in thread 0.  smem must hold 32*K A's.
template <typename A, int K>
__device__ __forceinline__ Red<A, K> block_sum(Red<A, K> r, A* smem) {
  r = warp_sum<A, K>(r);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) smem[wid * K + k] = r.v[k];
  }
  __syncthreads();
  Red<A, K> out;
#pragma unroll
  for (int k = 0; k < K; ++k) out.v[k] = 0;
  if (wid == 0) {
    for (int w = lane; w < nw; w += 32) {
#pragma unroll
      for (int k = 0; k < K; ++k) out.v[k] += smem[w * K + k];
    }
    out = warp_sum<A, K>(out);
  }
  return out;
}

template <typename A, int K, class Fin>
__device__ __forceinline__ void grid_sum_finalize(Red<A, K> r, A* partials, unsigned* counter,
                                                  Fin fin) {
  __shared__ A red_smem[32 * K];
  __shared__ bool am_last;
  Red<A, K> b = block_sum<A, K>(r, red_smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) partials[(size_t)blockIdx.x * K + k] = b.v[k];
    __threadfence();
    unsigned prev = atomicAdd(counter, 1u);
    am_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  Red<A, K> s;
#pragma unroll
  for (int k = 0; k < K; ++k) s.v[k] = 0;
  // fixed assignment of partials to threads, then fixed-order tree
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; ++k) s.v[k] += ((volatile A*)partials)[(size_t)i * K + k];
  }
  Red<A, K> tot = block_sum<A, K>(s, red_smem);
  if (threadIdx.x == 0) {
    fin(tot);
    *counter = 0u;
  }
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace fame
