// Batched TF32 GEMM on the sm_100a tensor cores (tcgen05 UMMA, operands
// brought into shared memory by TMA, accumulators in TMEM), built from the
// CUTLASS sm100 collective templates:
//   D[l][m][n] = sum_k A[m][l*K + k] * B[n][l*K + k]     (l = 0 .. L-1)
// A is M x (L*K) row-major and B is N x (L*K) row-major (both K-contiguous,
// leading dimension ldk); D is L packed M x N row-major FP32 blocks.  The
// batch index splits a long K across CTAs (split-K); the caller reduces the L
// partial products.  Used by the 3xTF32 Taylor moments (recon.cu).
#include "internal.cuh"

#ifndef FAME_NO_CUTLASS
#include "cute/tensor.hpp"
#include "cutlass/cutlass.h"
#include "cutlass/epilogue/collective/collective_builder.hpp"
#include "cutlass/gemm/collective/collective_builder.hpp"
#include "cutlass/gemm/device/gemm_universal_adapter.h"
#include "cutlass/gemm/dispatch_policy.hpp"
#include "cutlass/gemm/kernel/gemm_universal.hpp"
#include "cutlass/util/packed_stride.hpp"

namespace fame {
namespace {
using namespace cute;
using ElementA = cutlass::tfloat32_t;
using ElementB = cutlass::tfloat32_t;
using LayoutA = cutlass::layout::RowMajor;     // M x K, K contiguous
using LayoutB = cutlass::layout::ColumnMajor;  // K x N stored N x K, K contiguous
using LayoutD = cutlass::layout::RowMajor;
using MmaTile = Shape<_128, _128, _32>;
using Cluster = Shape<_1, _1, _1>;
using Epilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, MmaTile, Cluster,
    cutlass::epilogue::collective::EpilogueTileAuto, float, float, void, LayoutD, 4, float, LayoutD, 4,
    cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;
using Mainloop = typename cutlass::gemm::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElementA, LayoutA, 4, ElementB, LayoutB, 4, float,
    MmaTile, Cluster,
    cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(typename Epilogue::SharedStorage))>,
    cutlass::gemm::collective::KernelScheduleAuto>::CollectiveOp;
using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Mainloop, Epilogue, void>;
using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;

typename Gemm::Arguments make_args(int M, int N, int K, int L, long long ldk, const float* A, const float* B,
                                   float* D) {
  using SA = typename Gemm::GemmKernel::StrideA;
  using SB = typename Gemm::GemmKernel::StrideB;
  using SD = typename Gemm::GemmKernel::StrideD;
  SA sa = make_stride(int64_t(ldk), Int<1>{}, int64_t(K));
  SB sb = make_stride(int64_t(ldk), Int<1>{}, int64_t(K));
  SD sd = cutlass::make_cute_packed_stride(SD{}, make_shape(M, N, L));
  return typename Gemm::Arguments{cutlass::gemm::GemmUniversalMode::kBatched,
                                  {M, N, K, L},
                                  {reinterpret_cast<const ElementA*>(A), sa, reinterpret_cast<const ElementB*>(B), sb},
                                  {{1.0f, 0.0f}, nullptr, sd, D, sd}};
}
}  // namespace

size_t tf32_gemm_workspace(int M, int N, int K, int L, long long ldk) {
  return Gemm::get_workspace_size(make_args(M, N, K, L, ldk, nullptr, nullptr, nullptr));
}

int tf32_gemm_batched(int M, int N, int K, int L, long long ldk, const float* A, const float* B, float* D,
                      void* workspace, cudaStream_t st) {
  if (M <= 0 || N <= 0 || K <= 0 || L <= 0 || K % 4 != 0 || ldk % 4 != 0 || N % 4 != 0)
    return fail(FAME_ERR_INVALID, "tf32_gemm_batched: K, ldk and N must be positive multiples of 4");
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(D)) % 16)
    return fail(FAME_ERR_INVALID, "tf32_gemm_batched: operands must be 16-byte aligned");
  auto args = make_args(M, N, K, L, ldk, A, B, D);
  Gemm g;
  if (g.can_implement(args) != cutlass::Status::kSuccess) return fail(FAME_ERR_UNSUPPORTED, "TF32 GEMM shape");
  if (g.initialize(args, workspace, st) != cutlass::Status::kSuccess) return fail(FAME_ERR_CUDA, "TF32 GEMM init");
  if (g.run(st) != cutlass::Status::kSuccess) return fail(FAME_ERR_CUDA, "TF32 GEMM launch");
  ::fame::count_launch();
  return FAME_OK;
}

}  // namespace fame

#else  // built without the CUTLASS headers

namespace fame {
size_t tf32_gemm_workspace(int, int, int, int, long long) { return 0; }
int tf32_gemm_batched(int, int, int, int, long long, const float*, const float*, float*, void*, cudaStream_t) {
  return fail(FAME_ERR_UNSUPPORTED, "library built without the CUTLASS headers: no tensor-core GEMM");
}
}  // namespace fame

#endif
