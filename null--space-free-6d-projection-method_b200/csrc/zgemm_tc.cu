// Batched complex GEMM C = A B (FP64 complex operands and result) on the tcgen05
// tensor cores in split FP32 (3xTF32): each operand value v = head + tail, both
// TF32, and the product is head*head + head*tail + tail*head.
//
// The complex product becomes one real GEMM over interleaved (re, im) pairs:
//   A' row 2m   = (Re A[m,k], -Im A[m,k]) for k = 0..K-1,
//   A' row 2m+1 = (Im A[m,k],  Re A[m,k]),
//   B' row n    = (Re B[k,n],  Im B[k,n]),
// so D[2m][n] = Re C[m,n] and D[2m+1][n] = Im C[m,n].  A CTA owns 64 rows m and up
// to 256 columns n; per stage of 16 complex k (32 TF32 values of K', one 128-byte
// swizzle atom) eight generator warps load the FP64 operands, split them and write
// the swizzled K-major UMMA layout, and a ninth warp issues tcgen05.mma kind::tf32.
// head*head accumulates in one TMEM accumulator and the two cross products in a
// second one: the tensor cores round the FP32 accumulation toward zero, and the
// cross products are 2^-11 smaller, so only the head*head sum carries that bias.
// The epilogue adds the two accumulators in FP64.
#include "internal.cuh"
#include "umma.cuh"

namespace fame {
namespace {

constexpr int kZGenWarps = 8;
constexpr int kZGenThreads = kZGenWarps * 32;
constexpr int kZThreads = kZGenThreads + 32;  // + the MMA-issuing warp
constexpr int kZM = 64;                        // complex rows per CTA (128 accumulator lanes)
constexpr int kZKC = 16;                       // complex k per stage
constexpr int kZStages = 2;
constexpr uint32_t kZABytes = 128u * 128u;     // one TF32 part of A' per stage
constexpr int kAPer = kZM * kZKC / kZGenThreads;  // A values per generator thread and stage
constexpr int kBBatch = 8;                        // B values per generator thread and load batch
static_assert(kAPer * kZGenThreads == kZM * kZKC, "A tile divides over the generator threads");

__host__ __device__ inline uint32_t zb_bytes(int nt) { return (uint32_t)nt * 128u; }
__host__ __device__ inline uint32_t zstage_bytes(int nt) { return 2u * (kZABytes + zb_bytes(nt)); }
inline size_t zsmem(int nt) { return 1024 + (size_t)kZStages * zstage_bytes(nt) + 128; }

struct ZgArgs {
  const double2* A;
  const double2* B;
  double2* C;
  int M, N, K, Nt;
  long long sam, sak, sbk, sbn, scm, scn;
  long long bA, bB, bC;
  int bdivB;  // B advances by bB every bdivB batch entries
};

__device__ __forceinline__ void put2(unsigned char* base, int row, int k, float x, float y) {
  *reinterpret_cast<float2*>(base + umma::sw128_offset(row, k)) = make_float2(x, y);
}

__global__ void __launch_bounds__(kZThreads, 1) k_zgemm_3xtf32(ZgArgs g, unsigned* fault) {
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
  const int Nt = g.Nt;
  const uint32_t bB = zb_bytes(Nt), stB = zstage_bytes(Nt);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + (size_t)kZStages * stB);  // [2]
  uint64_t* empty = full + 2;                                                 // [2]
  uint64_t* done = full + 4;
  uint32_t* slot = reinterpret_cast<uint32_t*>(full + 5);
  volatile int* abortf = reinterpret_cast<volatile int*>(slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kZM, n0 = blockIdx.y * Nt;
  const double2* A = g.A + g.bA * blockIdx.z;
  const double2* B = g.B + g.bB * (blockIdx.z / g.bdivB);
  double2* Cm = g.C + g.bC * blockIdx.z;
  const int nch = (g.K + kZKC - 1) / kZKC;
  const uint32_t ncols = 2 * Nt <= 32 ? 32u : 2 * Nt <= 64 ? 64u : 2 * Nt <= 128 ? 128u : 2 * Nt <= 256 ? 256u : 512u;

  if (tid == 0) {
    for (int s = 0; s < kZStages; ++s) {
      mbar_init(&full[s], kZGenThreads);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abortf = 0;
    mbar_init_fence();
  }
  if (warp == 0) {
    umma::tmem_alloc(slot, ncols);
    umma::tmem_relinquish();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = *slot;  // columns [0, Nt): head*head; [Nt, 2 Nt): cross products

  if (warp < kZGenWarps) {
    const bool aMfast = g.sam == 1, bNfast = g.sbn == 1 && g.sbk != 1;
    for (int i = 0; i < nch; ++i) {
      const int s = i % kZStages;
      unsigned char* stg = sm + (size_t)s * stB;
      bool ok = !*abortf;
      if (ok && i >= kZStages) ok = mbar_wait(&empty[s], (unsigned)((i / kZStages - 1) & 1));
      if (!ok) *abortf = 1;
      if (ok) {
        const int kc0 = i * kZKC;
        unsigned char* Ahi = stg;
        unsigned char* Alo = stg + kZABytes;
        unsigned char* Bhi = stg + 2 * kZABytes;
        unsigned char* Blo = Bhi + bB;
        // every load of a batch is issued before the first split: the stage then waits for
        // one global-memory latency per batch instead of one per element
        auto a_at = [&](int idx, int& m, int& k) {
          m = aMfast ? idx % kZM : idx / kZKC;
          k = aMfast ? idx / kZM : idx % kZKC;
        };
        auto b_at = [&](int idx, int& n, int& k) {
          n = bNfast ? idx % Nt : idx / kZKC;
          k = bNfast ? idx / Nt : idx % kZKC;
        };
        // A: 64 x 16 complex (kAPer per thread), with the first batch of B
        double2 va[kAPer], vb[kBBatch];
#pragma unroll
        for (int u = 0; u < kAPer; ++u) {
          int m, k;
          a_at(tid + u * kZGenThreads, m, k);
          va[u] = m0 + m < g.M && kc0 + k < g.K
                      ? __ldg(A + (long long)(m0 + m) * g.sam + (long long)(kc0 + k) * g.sak)
                      : make_double2(0.0, 0.0);
        }
        const int nB = Nt * kZKC;  // B: Nt x 16 complex
#pragma unroll 1
        for (int b0 = 0; b0 < nB; b0 += kBBatch * kZGenThreads) {
#pragma unroll
          for (int u = 0; u < kBBatch; ++u) {
            const int idx = b0 + tid + u * kZGenThreads;
            int n, k;
            b_at(idx, n, k);
            vb[u] = idx < nB && n0 + n < g.N && kc0 + k < g.K
                        ? __ldg(B + (long long)(kc0 + k) * g.sbk + (long long)(n0 + n) * g.sbn)
                        : make_double2(0.0, 0.0);
          }
          if (b0 == 0) {
#pragma unroll
            for (int u = 0; u < kAPer; ++u) {
              int m, k;
              a_at(tid + u * kZGenThreads, m, k);
              float rh, rl, ih, il;
              umma::tf32_split_fast(va[u].x, rh, rl);
              umma::tf32_split_fast(va[u].y, ih, il);
              put2(Ahi, 2 * m, 2 * k, rh, -ih);
              put2(Alo, 2 * m, 2 * k, rl, -il);
              put2(Ahi, 2 * m + 1, 2 * k, ih, rh);
              put2(Alo, 2 * m + 1, 2 * k, il, rl);
            }
          }
#pragma unroll
          for (int u = 0; u < kBBatch; ++u) {
            const int idx = b0 + tid + u * kZGenThreads;
            if (idx < nB) {
              int n, k;
              b_at(idx, n, k);
              float rh, rl, ih, il;
              umma::tf32_split_fast(vb[u].x, rh, rl);
              umma::tf32_split_fast(vb[u].y, ih, il);
              put2(Bhi, n, 2 * k, rh, ih);
              put2(Blo, n, 2 * k, rl, il);
            }
          }
        }
      }
      fence_proxy_async_smem();  // generic-proxy writes -> tensor-core reads
      mbar_arrive(&full[s]);
    }
  } else {
    const uint32_t id = umma::idesc_tf32(128, Nt);
    for (int i = 0; i < nch; ++i) {
      const int s = i % kZStages;
      const bool ok = !*abortf && mbar_wait(&full[s], (unsigned)((i / kZStages) & 1));
      if (!ok) {
        *abortf = 1;
        break;
      }
      umma::fence_after_sync();
      if (lane == 0) {
        const uint32_t sa = smem_u32(sm + (size_t)s * stB);
        for (int kk = 0; kk < 2 * kZKC / 8; ++kk) {
          const uint32_t o = kk * 32u, acc = (i | kk) != 0 ? 1u : 0u;
          const uint64_t ahi = umma::desc_kmajor_sw128(sa + o), alo = umma::desc_kmajor_sw128(sa + kZABytes + o);
          const uint64_t bhi = umma::desc_kmajor_sw128(sa + 2u * kZABytes + o);
          const uint64_t blo = umma::desc_kmajor_sw128(sa + 2u * kZABytes + bB + o);
          umma::mma_tf32(tmem, ahi, bhi, id, acc);
          umma::mma_tf32(tmem + (uint32_t)Nt, ahi, blo, id, acc);
          umma::mma_tf32(tmem + (uint32_t)Nt, alo, bhi, id, 1u);
        }
        umma::commit(&empty[s]);
      }
      __syncwarp();
    }
    if (lane == 0) umma::commit(done);
    __syncwarp();
  }
  const bool fin = mbar_wait(done, 0u);
  const bool ok = __syncthreads_and(fin && !*abortf);
  if (ok && warp < kZGenWarps) {
    umma::fence_after_sync();
    const int q = warp & 3;                       // TMEM lanes 32 q .. 32 q + 31
    const int m = m0 + (q * 32 + lane) / 2;       // lane pair (2j, 2j+1) = (Re, Im) of row m
    const bool odd = lane & 1;
    for (int cc = warp >> 2; cc < Nt / 32; cc += kZGenWarps / 4) {
      uint32_t hh[32], xx[32];
      umma::ld_32x32b_x32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(cc * 32), hh);
      umma::ld_32x32b_x32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(Nt + cc * 32), xx);
      umma::wait_ld(hh);
      umma::wait_ld(xx);
      // the even lane stores columns 0..15 of the chunk, the odd lane 16..31
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        const double lo = (double)__uint_as_float(hh[c]) + (double)__uint_as_float(xx[c]);
        const double hi = (double)__uint_as_float(hh[c + 16]) + (double)__uint_as_float(xx[c + 16]);
        const double other = __shfl_xor_sync(0xffffffffu, odd ? lo : hi, 1);
        const int n = n0 + cc * 32 + c + (odd ? 16 : 0);
        if (m < g.M && n < g.N)
          Cm[(long long)m * g.scm + (long long)n * g.scn] = odd ? make_double2(other, hi) : make_double2(lo, other);
      }
    }
  } else if (!ok && tid == 0 && fault) {
    atomicOr(fault, 1u);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, ncols);
  }
}

}  // namespace

int zgemm_3xtf32(const double2* A, const double2* B, double2* C, int M, int N, int K, long long sam, long long sak,
                 long long sbk, long long sbn, long long scm, long long scn, long long bA, long long bB, long long bC,
                 int batch, cudaStream_t s, int bdivB) {
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return fail(FAME_ERR_INVALID, "zgemm_3xtf32: empty shape");
  const int Nt = std::min(256, (N + 31) / 32 * 32);
  const size_t smem = zsmem(Nt);
  static int attr = [] {
    return cudaFuncSetAttribute(k_zgemm_3xtf32, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) ==
                   cudaSuccess
               ? FAME_OK
               : FAME_ERR_CUDA;
  }();
  if (attr != FAME_OK) return fail(attr, "zgemm_3xtf32: shared-memory limit");
  const long long gy = (N + Nt - 1) / Nt;
  if (gy > 65535 || batch > 65535) return fail(FAME_ERR_UNSUPPORTED, "zgemm_3xtf32: grid too large");
  if (bdivB < 1) return fail(FAME_ERR_INVALID, "zgemm_3xtf32: batch divisor");
  ZgArgs g{A, B, C, M, N, K, Nt, sam, sak, sbk, sbn, scm, scn, bA, bB, bC, bdivB};
  dim3 grid((unsigned)((M + kZM - 1) / kZM), (unsigned)gy, (unsigned)batch);
  k_zgemm_3xtf32<<<grid, kZThreads, smem, s>>>(g, fault_word());
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

}  // namespace fame
