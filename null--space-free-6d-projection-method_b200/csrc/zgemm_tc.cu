// Batched complex GEMM C = A B (FP64 complex operands and result) on the tcgen05
// tensor cores in split FP32 (3xTF32): each operand value v = head + tail, both
// TF32, and the product is head*head + head*tail + tail*head.
//
// The complex product becomes one real GEMM over interleaved (re, im) pairs:
//   A' row 2m   = (Re A[m,k], -Im A[m,k]) for k = 0..K-1,
//   A' row 2m+1 = (Im A[m,k],  Re A[m,k]),
//   B' row n    = (Re B[k,n],  Im B[k,n]),
// so D[2m][n] = Re C[m,n] and D[2m+1][n] = Im C[m,n].
//
// Two kernels.  k_zsplit splits each operand once, in a bandwidth-bound pass, into
// panels already in the shared-memory form of the MMA: per (row tile, stage of 16
// complex k = 32 TF32 values of K', one 128-byte swizzle atom) a head part and a
// tail part, each rows x 128 bytes in the 128-byte swizzled K-major UMMA layout,
// one contiguous block per (tile, stage).  k_zgemm_3xtf32 then streams those blocks:
// one thread issues the A and B bulk copies of each stage (completed on the stage's
// mbarrier), one
// thread issues tcgen05.mma kind::tf32 -- head*head into one TMEM accumulator, the two
// cross products into a second (the tensor cores round the FP32 accumulation toward
// zero, and the cross products are 2^-11 smaller, so only the head*head sum carries
// that bias) -- and commits to the stage's release mbarrier; the epilogue (four warps,
// one per 32 TMEM lanes) adds the two accumulators in FP64.  An A panel tile is 64
// complex rows (128 accumulator lanes); a B panel tile is Nt <= 256 columns.  Operands
// shared by several output tiles (the phase tables of the direct sum) are split once
// instead of once per tile.
#include "internal.cuh"
#include "umma.cuh"

namespace fame {
namespace {

constexpr int kZM = 64;                     // complex rows per A tile (128 accumulator lanes)
constexpr int kZKC = 16;                    // complex k per stage
constexpr int kZThreads = 128;              // producer (thread 0), MMA issuer (thread 32), epilogue (all)
constexpr uint32_t kZABytes = 128u * 128u;  // one TF32 part of an A stage

__host__ __device__ inline uint32_t zb_bytes(int nt) { return (uint32_t)nt * 128u; }
__host__ __device__ inline uint32_t zstage_bytes(int nt) { return 2u * (kZABytes + zb_bytes(nt)); }
inline int zstages(int nt) { return zstage_bytes(nt) * 3u + 2048u <= 227u * 1024u ? 3 : 2; }
inline size_t zsmem(int nt) { return 1024 + (size_t)zstages(nt) * zstage_bytes(nt) + 128; }

// Operand panels: element (real row r, K' index kk) of stage ks of tile t of batch b sits at
// byte ((b * tiles + t) * stages + ks) * 2 * part + half * part + sw128_offset(r, kk),
// part = real rows per tile * 128 bytes (head: half 0, tail: half 1).
struct SplitArgs {
  const double2* src;
  long long s_row, s_k, s_batch;  // element strides of (complex row, k, batch)
  int rows, K, batches;
  int tile_rows;                   // complex rows per tile: 64 (A role) or Nt (B role)
  int a_role;                      // A: two real rows (Re, -Im), (Im, Re); B: one (Re, Im)
  unsigned char* out;
};

// A CTA takes (a share of the rows of) one panel block (batch, tile, stage): the FP64 values
// are read along the operand's contiguous dimension into shared memory, then written as
// whole 128-byte rows, 16 bytes (four TF32 values of K' = two complex k) per thread.
constexpr int kSplitThreads = 256;
constexpr int kSplitMaxRows = 256;  // complex rows of a tile (B role, Nt <= 256)
// several operands in one launch: job j owns blocks [first[j], first[j + 1])
constexpr int kMaxSplitJobs = 4;
struct SplitJobs {
  SplitArgs job[kMaxSplitJobs];
  int first[kMaxSplitJobs + 1];
  int njobs;
  int pitch;  // shared tile row pitch: the largest per-CTA row share of the jobs, plus one
};
// A CTA covers at most kSplitRows complex rows of a panel block (B blocks of Nt = 256 rows
// take two CTAs: the rows of a block are independent), so its shared tile stays within 33 KB.
constexpr int kSplitRows = 128;
__device__ __forceinline__ int split_subs(const SplitArgs& a) { return (a.tile_rows + kSplitRows - 1) / kSplitRows; }
__global__ void __launch_bounds__(kSplitThreads) k_zsplit(SplitJobs jobs) {
  extern __shared__ double2 tile_raw[];  // [kZKC][pitch]: [k][complex row of this CTA's share]
  const int pitch = jobs.pitch;
  int j = 0;
  while (j + 1 < jobs.njobs && (int)blockIdx.x >= jobs.first[j + 1]) ++j;
  const SplitArgs& a = jobs.job[j];
  const int bid = (int)blockIdx.x - jobs.first[j];
  const int tiles = (a.rows + a.tile_rows - 1) / a.tile_rows;
  const int stages = (a.K + kZKC - 1) / kZKC, subs = split_subs(a);
  const int ks = bid % stages, rest = bid / stages, h = rest % subs, t = (rest / subs) % tiles,
            b = rest / (subs * tiles);
  const int rr0 = h * kSplitRows, nr = a.tile_rows - rr0 < kSplitRows ? a.tile_rows - rr0 : kSplitRows;
  const int r0 = t * a.tile_rows + rr0, k0 = ks * kZKC;
  const bool rfast = a.s_row == 1;  // read along the contiguous dimension
  const double2* src = a.src + (long long)b * a.s_batch;
  for (int e = threadIdx.x; e < nr * kZKC; e += kSplitThreads) {
    const int rr = rfast ? e % nr : e / kZKC, kk = rfast ? e / nr : e % kZKC;
    const int r = r0 + rr, k = k0 + kk;
    tile_raw[kk * pitch + rr] = (r < a.rows && k < a.K) ? __ldg(src + (long long)r * a.s_row + (long long)k * a.s_k)
                                                        : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const int per = a.a_role ? 2 : 1;  // real rows per complex row
  const size_t part = (size_t)a.tile_rows * per * 128u;
  unsigned char* blk = a.out + ((size_t)((long long)b * tiles + t) * stages + ks) * 2 * part;
  // 16-byte chunk c of real row R holds K' = 4c .. 4c+3, i.e. complex k = 2c, 2c+1
  for (int e = threadIdx.x; e < nr * per * 8; e += kSplitThreads) {
    const int Rl = e / 8, c = e % 8, R = rr0 * per + Rl;  // Rl: real row within this CTA's share
    float hv[4], lv[4];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const double2 v = tile_raw[(2 * c + q) * pitch + Rl / per];
      float rh, rl, ih, il;
      umma::tf32_split_fast(v.x, rh, rl);
      umma::tf32_split_fast(v.y, ih, il);
      const bool second = a.a_role && (R & 1);  // A rows: (Re, -Im) then (Im, Re)
      hv[2 * q] = second ? ih : rh;
      hv[2 * q + 1] = second ? rh : (a.a_role ? -ih : ih);
      lv[2 * q] = second ? il : rl;
      lv[2 * q + 1] = second ? rl : (a.a_role ? -il : il);
    }
    const uint32_t off = umma::sw128_offset(R, 4 * c);
    *reinterpret_cast<float4*>(blk + off) = make_float4(hv[0], hv[1], hv[2], hv[3]);
    *reinterpret_cast<float4*>(blk + part + off) = make_float4(lv[0], lv[1], lv[2], lv[3]);
  }
}

struct ZgArgs {
  const unsigned char* Ap;  // A panels (64-row tiles), per batch
  const unsigned char* Bp;  // B panels (Nt-row tiles), per B batch
  double2* C;
  int M, N, K, Nt, S;
  long long scm, scn, bC;
  int bdivB;  // B panel batch = blockIdx.z / bdivB
};

__global__ void __launch_bounds__(kZThreads, 1) k_zgemm_3xtf32(ZgArgs g, unsigned* fault) {
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
  const int Nt = g.Nt, S = g.S;
  const uint32_t bB = zb_bytes(Nt), stB = zstage_bytes(Nt);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + (size_t)S * stB);  // [S]: stage landed
  uint64_t* empty = full + S;                                          // [S]: stage read by the MMAs
  uint64_t* done = full + 2 * S;                                       // every MMA complete
  uint32_t* slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abortf = reinterpret_cast<volatile int*>(slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kZM, n0 = blockIdx.y * Nt;
  const int nch = (g.K + kZKC - 1) / kZKC;
  const size_t astride = 2 * (size_t)kZABytes, bstride = 2 * (size_t)bB;  // bytes per stage of a tile
  const unsigned char* Ap = g.Ap + ((size_t)blockIdx.z * gridDim.x + blockIdx.x) * nch * astride;
  const unsigned char* Bp = g.Bp + ((size_t)(blockIdx.z / g.bdivB) * gridDim.y + blockIdx.y) * nch * bstride;
  double2* Cm = g.C + g.bC * blockIdx.z;
  const uint32_t ncols = 2 * Nt <= 32 ? 32u : 2 * Nt <= 64 ? 64u : 2 * Nt <= 128 ? 128u : 2 * Nt <= 256 ? 256u : 512u;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
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

  if (tid == 0) {
    // producer: stage i of the A and B panels into buffer i % S once the MMAs of i - S are done
    int issued = 0;
    for (int i = 0; i < nch; ++i) {
      const int s = i % S;
      if (*abortf) break;
      if (i >= S && !mbar_wait(&empty[s], (unsigned)((i / S - 1) & 1))) {
        *abortf = 1;
        break;
      }
      unsigned char* stg = sm + (size_t)s * stB;
      mbar_arrive_expect_tx(&full[s], (unsigned)(astride + bstride));
      bulk_g2s(stg, Ap + (size_t)i * astride, (unsigned)astride, &full[s]);
      bulk_g2s(stg + astride, Bp + (size_t)i * bstride, (unsigned)bstride, &full[s]);
      issued = i + 1;
    }
    // copies issued for stages the MMAs never consumed still land in this CTA's shared
    // memory: wait for them (bounded) before the CTA may exit
    if (*abortf)
      for (int i = issued - S < 0 ? 0 : issued - S; i < issued; ++i) mbar_wait(&full[i % S], (unsigned)((i / S) & 1));
  } else if (tid == 32) {
    const uint32_t id = umma::idesc_tf32(128, Nt);
    for (int i = 0; i < nch; ++i) {
      const int s = i % S;
      if (*abortf || !mbar_wait(&full[s], (unsigned)((i / S) & 1))) {
        *abortf = 1;
        break;
      }
      umma::fence_after_sync();
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
    umma::commit(done);  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  const bool fin = mbar_wait(done, 0u);
  const bool ok = __syncthreads_and(fin && !*abortf);
  if (ok) {
    umma::fence_after_sync();
    const int m = m0 + (warp * 32 + lane) / 2;  // TMEM lane pair (2j, 2j+1) = (Re, Im) of row m
    const bool odd = lane & 1;
    for (int cc = 0; cc < Nt / 32; ++cc) {
      uint32_t hh[32], xx[32];
      umma::ld_32x32b_x32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc * 32), hh);
      umma::ld_32x32b_x32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(Nt + cc * 32), xx);
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

inline int z_nt(int N) { return std::min(256, (N + 31) / 32 * 32); }
inline size_t panel_bytes(int rows, int K, int batches, int tile_rows, bool a_role) {
  const size_t tiles = (size_t)(rows + tile_rows - 1) / tile_rows, stages = (size_t)(K + kZKC - 1) / kZKC;
  return (size_t)batches * tiles * stages * 2 * (size_t)tile_rows * (a_role ? 2 : 1) * 128u;
}

}  // namespace

size_t zpanel_bytes(const ZPanelJob& j) {
  return panel_bytes(j.rows, j.K, j.batches, j.a_role ? kZM : z_nt(j.cols_for_b), j.a_role);
}

int zsplit_panels(const ZPanelJob* jobs, int njobs, cudaStream_t s) {
  if (njobs < 1 || njobs > kMaxSplitJobs) return fail(FAME_ERR_INVALID, "zsplit_panels: job count");
  SplitJobs sj{};
  long long blocks = 0;
  int share = 1;
  for (int j = 0; j < njobs; ++j) {
    const ZPanelJob& z = jobs[j];
    const int tile_rows = z.a_role ? kZM : z_nt(z.cols_for_b);
    if (!z.src || !z.out || z.rows <= 0 || z.K <= 0 || z.batches <= 0 || tile_rows > kSplitMaxRows ||
        (reinterpret_cast<uintptr_t>(z.out) & 1023u) != 0)
      return fail(FAME_ERR_INVALID, "zsplit_panels: job");
    sj.job[j] = SplitArgs{z.src, z.s_row, z.s_k, z.s_batch, z.rows, z.K, z.batches, tile_rows, z.a_role ? 1 : 0, z.out};
    sj.first[j] = (int)blocks;
    blocks += (long long)z.batches * ((z.rows + tile_rows - 1) / tile_rows) * ((z.K + kZKC - 1) / kZKC) *
              ((tile_rows + kSplitRows - 1) / kSplitRows);
    share = std::max(share, std::min(tile_rows, kSplitRows));
    if (blocks > 0x7fffffffLL) return fail(FAME_ERR_UNSUPPORTED, "zsplit_panels: too many panel blocks");
  }
  sj.first[njobs] = (int)blocks;
  sj.njobs = njobs;
  sj.pitch = share + 1;
  k_zsplit<<<(unsigned)blocks, kSplitThreads, (size_t)kZKC * sj.pitch * sizeof(double2), s>>>(sj);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

int zgemm_3xtf32_panels(const unsigned char* Ap, const unsigned char* Bp, double2* C, int M, int N, int K,
                        long long scm, long long scn, long long bC, int batch, int bdivB, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0 || !Ap || !Bp || !C || bdivB < 1)
    return fail(FAME_ERR_INVALID, "zgemm_3xtf32: arguments");
  if ((reinterpret_cast<uintptr_t>(Ap) & 1023u) != 0 || (reinterpret_cast<uintptr_t>(Bp) & 1023u) != 0)
    return fail(FAME_ERR_INVALID, "zgemm_3xtf32: panels must be 1024-byte aligned");
  const int Nt = z_nt(N), S = zstages(Nt);
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
  ZgArgs g{Ap, Bp, C, M, N, K, Nt, S, scm, scn, bC, bdivB};
  dim3 grid((unsigned)((M + kZM - 1) / kZM), (unsigned)gy, (unsigned)batch);
  k_zgemm_3xtf32<<<grid, kZThreads, smem, s>>>(g, fault_word());
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

}  // namespace fame
