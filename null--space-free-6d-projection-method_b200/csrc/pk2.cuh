// Two FP32 values of two different lines carried in one 64-bit register pair, so
// that each arithmetic instruction of a DFT advances two lines at once (the
// sm_100 packed FP32 instructions behind __fadd2_rn / __fmul2_rn / __ffma2_rn).
// A line pair's real parts form one F2, its imaginary parts another; the DFT
// templates of fft6d.cuh run on F2 unchanged (their multiply-adds go through
// fmadd, which is one packed fused multiply-add here).
#pragma once
#include <cuda_runtime.h>

namespace fame {

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ explicit F2(float2 a) : v(a) {}
  // broadcast of a real constant (twiddle factors, 0)
  __device__ __forceinline__ F2(double c) : v(make_float2((float)c, (float)c)) {}
  __device__ __forceinline__ F2& operator+=(F2 b) {
    v = __fadd2_rn(v, b.v);
    return *this;
  }
};

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(__fmul2_rn(a.v, make_float2(-1.0f, -1.0f))); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }

// a * b + c: one fused multiply-add (scalars: the contraction nvcc makes of a * b + c)
__device__ __forceinline__ F2 fmadd(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__host__ __device__ __forceinline__ float fmadd(float a, float b, float c) { return a * b + c; }
__host__ __device__ __forceinline__ double fmadd(double a, double b, double c) { return a * b + c; }

}  // namespace fame
