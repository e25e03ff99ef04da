// Mhat action without any device allocation: the three-field scratch of the
// chain is a file-scope static device array instead of cudaMalloc'd memory.
//
// Some callers cannot let a library allocate device memory: hosts that own
// every byte of the GPU through their own pool (a MATLAB gpuArray session that
// hands out preallocated buffers, a serving process that reserves its memory
// up front) and loops that must not pay the implicit device synchronisation a
// cudaMalloc or cudaFree can cause.  For them this entry point takes only the
// caller's input and output buffers and uses a fixed 32 MiB scratch array that
// every GPU which loads this library holds until the process exits.
#include <mutex>
#include "internal.cuh"
#include "krinv_impl.cuh"

namespace fame {

// 32 MiB: three FP32 fields up to N=5 (NF = 10^6), three FP64 fields up to N=4.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with cudaGetSymbolAddress (with that device current) and cached.
static int noalloc_scratch_address(int device, void** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  if (device < 0 || device >= 64) return fail(FAME_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(FAME_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    addr[device] = p;
  }
  *out = addr[device];
  return FAME_OK;
}

}  // namespace fame

using namespace fame;

extern "C" int fame_apply_Mhat_C_scalar_compact_noalloc(fame_basis* b, fame_mass* m, const void* x,
                                                        void* y, int prec) {
  if (!b || !m || !x || !y) return fail(FAME_ERR_INVALID, "apply_Mhat_noalloc arguments");
  if (b->N != m->N) return fail(FAME_ERR_INVALID, "basis and mass have different N");
  if (prec != FAME_F64 && prec != FAME_F32) return fail(FAME_ERR_INVALID, "prec must be FAME_F64 or FAME_F32");
  const size_t el = prec == FAME_F32 ? sizeof(float2) : sizeof(double2);
  const size_t need = 3 * (size_t)b->NF * el;
  if (need > kNoAllocScratchBytes)
    return fail(FAME_ERR_INVALID, "apply_Mhat_noalloc: 3 fields of NF=" + std::to_string(b->NF) +
                                      " need " + std::to_string(need) + " bytes, above the " +
                                      std::to_string(kNoAllocScratchBytes) +
                                      "-byte static scratch (FP32 up to N=5, FP64 up to N=4)");
  int prev = -1;
  FAME_CUDA_TRY(cudaGetDevice(&prev));
  if (prev != b->ctx->device) FAME_CUDA_TRY(cudaSetDevice(b->ctx->device));
  void* work = nullptr;
  int s = noalloc_scratch_address(b->ctx->device, &work);
  if (s == FAME_OK) {
    cudaStream_t st = b->ctx->stream;
    if (prec == FAME_F64) {
      const MhatCoef<double> c = coef_of<double>(b);
      s = run_chain_lin<double, 3>(b->n, ProMhat<double, false>{c, (const double2*)x},
                                   EpiMhat<double, false>{c, (double2*)y}, (double2*)work, m->Et64,
                                   b->NF, st);
    } else {
      const MhatCoef<float> c = coef_of<float>(b);
      s = run_chain_lin<float, 3>(b->n, ProMhat<float, false>{c, (const float2*)x},
                                  EpiMhat<float, false>{c, (float2*)y}, (float2*)work, m->Et32,
                                  b->NF, st);
    }
  }
  if (prev != b->ctx->device) cudaSetDevice(prev);
  return s;
}
