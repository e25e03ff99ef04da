// Taylor block moments on the tcgen05 tensor cores, operands generated on chip.
//
// gamma[b, a] = coef[a] * sum_j c_j exp(i q_j . r_b) q_j^a
// (exp2/taylor_on_blocks_exp3.m:53-54,65-73: the moment GEMM Qalpha^T (c .* phase)).
//
// One CTA owns a slice of Kc modes, a tile of 64 block centers and Nc of the
// monomial columns.  Per stage of 32 modes its threads write into shared memory, in
// the 128-byte swizzled K-major UMMA layout and split into TF32 head + tail (3xTF32):
//   A (128 x 32): rows 2b, 2b+1 = Re, Im of c_j exp(i q_j . r_b)
//   B (Nc x 32):  row col(a) = qx^a1 qy^a2 qz^a3                       (FP64 products)
// When the block centers form a tensor grid (the Yee block partition does), the
// phase factorises per axis, exp(i q.r_b) = ex(bx) ey(by) ez(bz): the generators
// first tabulate the m1 + m2 + m3 axis phases of the stage's 32 modes in shared
// memory (3m sincosf per mode instead of m^3), then combine them with two complex
// products per center; otherwise each center's phase is reduced in FP64 and taken
// by sincosf.  Fifteen generator warps fill a stage and arrive on its "full"
// mbarrier; a sixteenth warp waits for it and issues tcgen05.mma kind::tf32 with
// Ahi*Bhi into one FP32 TMEM accumulator (columns [0, Nc)) and Ahi*Blo + Alo*Bhi of
// the first Csep columns into a second one (columns [Nc, Nc + Csep)): the tensor
// cores round each FP32 accumulation toward zero, and keeping the 2^-11 smaller
// cross products apart leaves the large head*head sum with a third of the
// roundings.  The cross products of columns [Csep, Nc) accumulate into the head*head
// columns.  The host places the monomials of degree p, whose moments weigh least in
// the Taylor sum, in those last columns (col() is a permutation), and splits the
// columns over two CTAs only when even then the degree < p columns would not fit in
// the 512 TMEM columns.  It commits to the stage's "empty" mbarrier while the
// generators fill the other stage.  The epilogue adds the two accumulators and
// writes the slice's partial moments (FP32); a second kernel sums the slices in FP64
// in a fixed order.  Neither Qalpha (L x NF) nor the phase matrix ever exists in
// HBM: the kernel reads 40 bytes per mode.
#include "internal.cuh"
#include "umma.cuh"

namespace fame {
namespace {

constexpr int kGenWarps = 15;                 // operand generators
constexpr int kGenThreads = kGenWarps * 32;
constexpr int kThreads = kGenThreads + 32;    // + the MMA-issuing warp (16 warps: 128 registers)
constexpr int kKC = 32;        // modes per stage (one swizzle atom of TF32)
constexpr int kBT = 64;        // block centers per accumulator tile (128 rows)
constexpr int kBPW = (kBT + kGenWarps - 1) / kGenWarps;  // block centers per generator warp, at most
constexpr int kBlockCost = 3;  // generation cost of one block center (Re, Im rows) in monomial rows
constexpr int kPmax = 12;
constexpr int kLmax = 512;
// Modes per slice accumulated in one FP32 TMEM accumulator at most (the tensor cores'
// toward-zero rounding of that accumulation sets the error of the moments).
constexpr long long kKcMax = 512;
constexpr uint32_t kABytes = 128u * 128u;  // one TF32 part of the phase operand
constexpr int kMaxAxis = kTaylorTcMaxAxis;

__host__ __device__ inline uint32_t b_bytes(int Nc) { return (uint32_t)Nc * 128u; }
__host__ __device__ inline uint32_t stage_bytes(int Nc) { return 2u * (kABytes + b_bytes(Nc)); }
constexpr size_t kTailBytes = kBT * 3 * sizeof(double)                 // centers
                              + kLmax * sizeof(int)                      // packed multi-indices
                              + 2 * kMaxAxis * kKC * sizeof(float2)      // axis phase tables (two stages)
                              + kMaxAxis * sizeof(double)                // axis center values
                              + 5 * sizeof(uint64_t) + 16;               // mbarriers, TMEM slot, abort flag
inline size_t tc_smem(int Nc, int stages) { return 1024 + (size_t)stages * stage_bytes(Nc) + kTailBytes; }

struct TcArgs {
  const double* Q;      // 3 x NF (rows qx, qy, qz)
  const double2* c;     // NF
  long long NF;
  const double* centers;  // nB x 3
  int nB;
  const int* alist;     // L packed multi-indices a1 | a2 << 8 | a3 << 16
  const int* col;       // Npad: output column of monomial a (identity past L)
  int L, p, Npad, Nc, Csep, stages;
  long long Kc;
  float* out;           // [slice][tile][128][Npad]
  const double* ax;     // tensor-grid centers (or nullptr)
  int m1, m2, m3;
};

// head = v rounded to TF32; tail = the exact FP32 remainder, passed as is: the MMA reads
// its TF32 part (measured on the moments of mode 10: the same field error as rounding the
// tail first, 1.4e-6 against the FP64 Taylor form at p = 10, m = 4, and 4 % faster)
__device__ __forceinline__ void split_tc(float v, float& h, float& l) {
  h = umma::tf32_rna(v);
  l = v - h;
}
__device__ __forceinline__ void put(unsigned char* base, int row, int k, float v) {
  *reinterpret_cast<float*>(base + umma::sw128_offset(row, k)) = v;
}

// exp(i th) in FP32 with th reduced to [-pi, pi] in FP64 first
__device__ __forceinline__ float2 cis(double th) {
  const double tr = fma(-rint(th * 0.15915494309189535), 6.283185307179586, th);
  float sf, cf;
  sincosf((float)tr, &sf, &cf);
  return make_float2(cf, sf);
}
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__global__ void __launch_bounds__(kThreads, 1) k_taylor_moments_tc(TcArgs a, unsigned* fault) {
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
  const int Nc = a.Nc, S = a.stages;
  const uint32_t bB = b_bytes(Nc), stB = stage_bytes(Nc);
  double* cen = reinterpret_cast<double*>(sm + (size_t)S * stB);  // [kBT][3]
  int* col = reinterpret_cast<int*>(cen + kBT * 3);                 // [kLmax]: column of monomial c0 + r
  float2* tab = reinterpret_cast<float2*>(col + kLmax);             // [2][kMaxAxis][kKC]
  double* axv = reinterpret_cast<double*>(tab + 2 * kMaxAxis * kKC);  // [kMaxAxis]
  uint64_t* full = reinterpret_cast<uint64_t*>(axv + kMaxAxis);     // [2]: stage written
  uint64_t* empty = full + 2;                                       // [2]: stage read by the MMAs
  uint64_t* done = full + 4;                                        // every MMA complete
  uint32_t* slot = reinterpret_cast<uint32_t*>(full + 5);
  volatile int* abortf = reinterpret_cast<volatile int*>(slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long z = blockIdx.x;
  const int bt = blockIdx.y;
  const int c0 = blockIdx.z * Nc;  // first monomial column of this CTA
  const long long j0 = z * a.Kc, j1 = j0 + a.Kc < a.NF ? j0 + a.Kc : a.NF;
  const int nch = (int)((j1 - j0 + kKC - 1) / kKC);
  const int nbl = a.nB - bt * kBT < kBT ? a.nB - bt * kBT : kBT;
  const bool factored = a.ax != nullptr;
  const int nax = factored ? a.m1 + a.m2 + a.m3 : 0;
  const int Csep = a.Csep;
  const uint32_t need = (uint32_t)(Nc + Csep);
  const uint32_t ncols = need <= 32 ? 32u : need <= 64 ? 64u : need <= 128 ? 128u : need <= 256 ? 256u : 512u;

  for (int t = tid; t < Nc; t += kThreads) col[t] = a.col[c0 + t] - c0;
  for (int t = tid; t < kBT * 3; t += kThreads) cen[t] = t / 3 < nbl ? a.centers[(long long)bt * kBT * 3 + t] : 0.0;
  for (int t = tid; t < nax; t += kThreads) axv[t] = a.ax[t];
  if (tid == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&full[s], kGenThreads);
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
  const uint32_t tmem = *slot;

  if (warp < kGenWarps) {
    // block centers bl = warp + u * kGenWarps are this warp's; monomial rows [r0, r1) of the
    // CTA's Nc columns too, sized so that every warp gets the same share of
    // (kBlockCost * blocks + rows)
    auto row_start = [&](int w) {
      const int total = kBlockCost * kBT + Nc;
      int rs = 0;
      for (int v = 1; v <= w; ++v) {
        const int blocksBefore = v < kBT % kGenWarps ? v * kBPW : (kBT % kGenWarps) * kBPW + (v - kBT % kGenWarps) * (kBPW - 1);
        int t = (v * total + kGenWarps / 2) / kGenWarps - kBlockCost * blocksBefore;
        t = t < rs ? rs : t;
        rs = t < Nc ? t : Nc;
      }
      return w >= kGenWarps ? Nc : rs;
    };
    const int r0 = row_start(warp), r1 = row_start(warp + 1);
    const int e0 = c0 + r0 < a.L ? a.alist[c0 + r0] : 0;
    double cx[kBPW], cy[kBPW], cz[kBPW];
    int tx[kBPW], ty[kBPW], tz[kBPW];  // axis-table rows of the centers (factorised phases)
#pragma unroll
    for (int u = 0; u < kBPW; ++u) {
      const int bl = warp + u * kGenWarps;
      cx[u] = bl < kBT ? cen[3 * bl] : 0.0;
      cy[u] = bl < kBT ? cen[3 * bl + 1] : 0.0;
      cz[u] = bl < kBT ? cen[3 * bl + 2] : 0.0;
      const int b = bt * kBT + bl;
      tx[u] = factored ? b % a.m1 : 0;
      ty[u] = factored ? a.m1 + (b / a.m1) % a.m2 : 0;
      tz[u] = factored ? a.m1 + a.m2 + b / (a.m1 * a.m2) : 0;
      if (!(bl < nbl)) tx[u] = ty[u] = tz[u] = 0;
    }
    // this lane's mode of the next stage, loaded one stage ahead
    double nqx = 0.0, nqy = 0.0, nqz = 0.0;
    double2 ncj = make_double2(0.0, 0.0);
    if (j0 + lane < j1) {
      nqx = a.Q[j0 + lane];
      nqy = a.Q[a.NF + j0 + lane];
      nqz = a.Q[2 * a.NF + j0 + lane];
      ncj = a.c[j0 + lane];
    }
    for (int i = 0; i < nch; ++i) {
      const int s = i % S;
      unsigned char* stg = sm + (size_t)s * stB;
      const long long j = j0 + (long long)i * kKC + lane;
      const bool in = j < j1;
      const double qx = nqx, qy = nqy, qz = nqz;
      const double2 cj = ncj;
      if (j + kKC < j1) {
        nqx = a.Q[j + kKC];
        nqy = a.Q[a.NF + j + kKC];
        nqz = a.Q[2 * a.NF + j + kKC];
        ncj = a.c[j + kKC];
      }
      // the MMAs that read this stage last time are done (bounded wait; a miss aborts)
      bool ok = !*abortf;
      if (ok && i >= S) ok = mbar_wait(&empty[s], (unsigned)((i / S - 1) & 1));
      if (!ok) *abortf = 1;
      float2* tb = tab + (i & 1) * kMaxAxis * kKC;
      if (factored) {
        // axis phases of this stage's modes: entry e (x values, then y, then z) for lane's mode;
        // thread (warp, lane) fills entries warp, warp + 15, ... (every generator warp takes part
        // in the barrier below on every stage, so the tables of stage i are complete before use
        // and the other buffer's readers of stage i - 1 are done before stage i + 1 writes it)
        for (int e = warp; e < nax; e += kGenWarps) {
          const double qc = e < a.m1 ? qx : e < a.m1 + a.m2 ? qy : qz;
          tb[e * kKC + lane] = cis(qc * axv[e]);
        }
        asm volatile("bar.sync 1, %0;" ::"n"(kGenThreads) : "memory");
      }
      if (ok) {
        // A: rows 2 bl, 2 bl + 1 = Re, Im of c_j exp(i q_j . r_bl)
        unsigned char* Ahi = stg;
        unsigned char* Alo = stg + kABytes;
        // c_j e^{i theta} in FP32: the products carry an absolute error ~2^-23 |c_j|, below
        // the 2^-22 of the TF32 split
        const float2 cf = make_float2((float)cj.x, (float)cj.y);
#pragma unroll
        for (int u = 0; u < kBPW; ++u) {
          const int bl = warp + u * kGenWarps;
          if (bl < kBT) {
            float2 w = make_float2(0.0f, 0.0f);
            if (in && bl < nbl) {
              const float2 ph = factored ? cmulf(cmulf(tb[tx[u] * kKC + lane], tb[ty[u] * kKC + lane]),
                                                 tb[tz[u] * kKC + lane])
                                         : cis(qx * cx[u] + qy * cy[u] + qz * cz[u]);
              w = cmulf(cf, ph);
            }
            float h, l;
            split_tc(w.x, h, l);
            put(Ahi, 2 * bl, lane, h);
            put(Alo, 2 * bl, lane, l);
            split_tc(w.y, h, l);
            put(Ahi, 2 * bl + 1, lane, h);
            put(Alo, 2 * bl + 1, lane, l);
          }
        }
        // B: local row r = column c0 + r: qx^a1 qy^a2 qz^a3 for that multi-index (a1 outer,
        // a3 inner), one multiplication per row; zero rows past L and for modes past the slice
        unsigned char* Bhi = stg + 2 * kABytes;
        unsigned char* Blo = Bhi + bB;
        const int a1 = e0 & 255, a2 = (e0 >> 8) & 255, a3 = e0 >> 16;
        double t1 = in ? 1.0 : 0.0;
        for (int k = 0; k < a1; ++k) t1 *= qx;
        double t12 = t1;
        for (int k = 0; k < a2; ++k) t12 *= qy;
        double m = t12;
        for (int k = 0; k < a3; ++k) m *= qz;
        int left1 = a.p - a1, left2 = left1 - a2, left3 = left2 - a3;  // steps left on each axis
        const int rL = r1 < a.L - c0 ? r1 : a.L - c0;
        for (int r = r0; r < rL; ++r) {
          float h, l;
          split_tc((float)m, h, l);
          const int rc = col[r];
          put(Bhi, rc, lane, h);
          put(Blo, rc, lane, l);
          if (left3 > 0) {
            --left3;
            m *= qz;
          } else if (left2 > 0) {
            left3 = --left2;
            t12 *= qy;
            m = t12;
          } else {
            left3 = left2 = --left1;
            t1 *= qx;
            t12 = t1;
            m = t1;
          }
        }
        for (int r = rL > r0 ? rL : r0; r < r1; ++r) {
          put(Bhi, col[r], lane, 0.0f);
          put(Blo, col[r], lane, 0.0f);
        }
      }
      fence_proxy_async_smem();  // generic-proxy writes -> tensor-core reads
      mbar_arrive(&full[s]);
    }
  } else {
    // MMA warp: wait for each stage, issue its 3xTF32 products, release it on completion
    for (int i = 0; i < nch; ++i) {
      const int s = i % S;
      const bool ok = !*abortf && mbar_wait(&full[s], (unsigned)((i / S) & 1));
      if (!ok) {
        *abortf = 1;
        break;
      }
      umma::fence_after_sync();
      if (lane == 0) {
        const uint32_t sa = smem_u32(sm + (size_t)s * stB);
        for (int kk = 0; kk < kKC / 8; ++kk) {
          const uint64_t ahi = umma::desc_kmajor_sw128(sa + kk * 32u);
          const uint64_t alo = umma::desc_kmajor_sw128(sa + kABytes + kk * 32u);
          const uint32_t b0 = sa + 2u * kABytes + kk * 32u;  // B head; the tail follows bB bytes later
          const uint32_t acc = (i | kk) != 0 ? 1u : 0u;
          // head * head over all Nc columns, at most 256 per MMA (B row c starts c * 128 bytes in)
          for (int c = 0; c < Nc; c += 256) {
            const int w = Nc - c < 256 ? Nc - c : 256;
            umma::mma_tf32(tmem + (uint32_t)c, ahi, umma::desc_kmajor_sw128(b0 + c * 128u), umma::idesc_tf32(128, w), acc);
          }
          // cross products of columns [0, Csep) into their own accumulator
          for (int c = 0; c < Csep; c += 256) {
            const int w = Csep - c < 256 ? Csep - c : 256;
            const uint32_t id = umma::idesc_tf32(128, w), d = tmem + (uint32_t)(Nc + c);
            umma::mma_tf32(d, ahi, umma::desc_kmajor_sw128(b0 + bB + c * 128u), id, acc);
            umma::mma_tf32(d, alo, umma::desc_kmajor_sw128(b0 + c * 128u), id, 1u);
          }
          // cross products of columns [Csep, Nc) into the head * head columns (after their
          // head * head product of this step, which initialises them on the first step)
          if (Csep < Nc) {
            const uint32_t id = umma::idesc_tf32(128, Nc - Csep), d = tmem + (uint32_t)Csep;
            umma::mma_tf32(d, ahi, umma::desc_kmajor_sw128(b0 + bB + Csep * 128u), id, 1u);
            umma::mma_tf32(d, alo, umma::desc_kmajor_sw128(b0 + Csep * 128u), id, 1u);
          }
        }
        umma::commit(&empty[s]);
      }
      __syncwarp();
    }
    if (lane == 0) umma::commit(done);  // arrives once every MMA issued above has completed
    __syncwarp();
  }
  // every thread: the accumulators are final (or the pipeline gave up)
  const bool fin = mbar_wait(done, 0u);
  const bool ok = __syncthreads_and(fin && !*abortf);
  if (ok) {  // all 16 warps: warp w reads lanes 32 (w % 4), 16-column blocks w / 4 + 4 t
    umma::fence_after_sync();
    const int q = warp & 3;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    float* orow = a.out + (((long long)z * gridDim.y + bt) * 128 + q * 32 + lane) * (long long)a.Npad + c0;
    for (int cb = warp >> 2; cb < Nc / 16; cb += (kGenWarps + 1) / 4) {
      uint32_t hh[16], cr[16];
      umma::ld_32x32b_x16_wait(tmem + lane_base + (uint32_t)(cb * 16), hh);
      if (cb * 16 < Csep) {
        umma::ld_32x32b_x16_wait(tmem + lane_base + (uint32_t)(Nc + cb * 16), cr);
      } else {
#pragma unroll
        for (int u = 0; u < 16; ++u) cr[u] = 0u;  // +0.0f: these columns hold both sums
      }
      float4* o = reinterpret_cast<float4*>(orow + cb * 16);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        o[u] = make_float4(__uint_as_float(hh[4 * u]) + __uint_as_float(cr[4 * u]),
                           __uint_as_float(hh[4 * u + 1]) + __uint_as_float(cr[4 * u + 1]),
                           __uint_as_float(hh[4 * u + 2]) + __uint_as_float(cr[4 * u + 2]),
                           __uint_as_float(hh[4 * u + 3]) + __uint_as_float(cr[4 * u + 3]));
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

// part[g][e] = sum of the partial moments e (of all tiles) over slice group g (FP64, fixed order)
__global__ void k_taylor_tc_sum_slices(const float* __restrict__ out, long long nslices, long long per, int groups,
                                       double* __restrict__ part) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= per) return;
  const int g = blockIdx.y;
  const long long z0 = nslices * g / groups, z1 = nslices * (g + 1) / groups;
  double acc = 0.0;
  for (long long z = z0; z < z1; ++z) acc += (double)out[z * per + e];
  part[(long long)g * per + e] = acc;
}

// gamma[b L + a] = coef[a] * (Re + i Im) of the group sums, groups in order
__global__ void k_taylor_tc_finish(const double* __restrict__ part, int groups, long long per, int Npad, int L, int nB,
                                   const int* __restrict__ col, const double2* __restrict__ coef,
                                   double2* __restrict__ gamma) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nB * L) return;
  const int b = (int)(t / L), al = (int)(t % L);
  const long long e = ((long long)(b / kBT) * 128 + 2 * (b % kBT)) * Npad + col[al];
  double re = 0.0, im = 0.0;
  for (int g = 0; g < groups; ++g) {
    re += part[(long long)g * per + e];
    im += part[(long long)g * per + e + Npad];
  }
  const double2 cf = coef[al];
  gamma[t] = make_double2(cf.x * re - cf.y * im, cf.x * im + cf.y * re);
}

}  // namespace

TaylorTcPlan taylor_tc_plan(long long NF, int nB, int L, int p) {
  TaylorTcPlan pl{};
  pl.Npad = std::max(32, (L + 31) / 32 * 32);
  // head*head (Nc columns) and cross (Csep columns) accumulators share the 512 TMEM columns
  const int low = p * (p + 1) * (p + 2) / 6;  // monomials of degree < p
  if (2 * pl.Npad <= 512) {                   // every column keeps its cross products apart
    pl.nsplit = 1;
    pl.Nc = pl.Csep = pl.Npad;
  } else if (pl.Npad + (low + 15) / 16 * 16 <= 512) {  // all but the degree-p columns do
    pl.nsplit = 1;
    pl.Nc = pl.Npad;
    pl.Csep = (512 - pl.Npad) / 16 * 16;
    pl.graded = true;
  } else {  // two CTAs per slice, Npad / 2 columns each, all cross products apart
    pl.nsplit = 2;
    pl.Nc = pl.Csep = pl.Npad / 2;  // a multiple of 16
  }
  pl.stages = tc_smem(pl.Nc, 2) <= 227 * 1024 ? 2 : 1;
  pl.smem = tc_smem(pl.Nc, pl.stages);
  pl.ntiles = (nB + kBT - 1) / kBT;
  const long long sms = num_sms() > 0 ? num_sms() : 148;
  const long long per_slice = (long long)pl.ntiles * pl.nsplit;  // CTAs per mode slice
  const long long waves = std::max<long long>(1, (NF * per_slice + sms * kKcMax - 1) / (sms * kKcMax));
  const long long want = std::max<long long>(1, (waves * sms + per_slice - 1) / per_slice);
  pl.Kc = std::max<long long>(kKC, ((NF + want - 1) / want + kKC - 1) / kKC * kKC);
  pl.nslices = (NF + pl.Kc - 1) / pl.Kc;
  const size_t per = (size_t)pl.ntiles * 128 * pl.Npad;
  pl.groups = (int)std::min<long long>(pl.nslices, 32);
  pl.out_floats = (size_t)pl.nslices * per + 2 * (size_t)pl.groups * per;  // FP32 slices + FP64 group sums
  return pl;
}

void taylor_tc_columns(const TaylorTcPlan& pl, const int* alist3, int L, int p, int* col) {
  int lo = 0, hi = pl.graded ? p * (p + 1) * (p + 2) / 6 : 0;
  for (int a = 0; a < pl.Npad; ++a) {
    const bool top = a < L && alist3[3 * a] + alist3[3 * a + 1] + alist3[3 * a + 2] == p;
    col[a] = !pl.graded || a >= L ? a : top ? hi++ : lo++;
  }
}

int taylor_moments_tc(const TaylorTcPlan& pl, cudaStream_t s, const double2* c, const double* Q, long long NF,
                      const double* centers, int nB, const int* alistPacked, const int* col, int L, int p,
                      const double2* coef, float* out, double2* gamma, const TaylorTcGrid& grid) {
  if (L > kLmax || L > pl.Npad || p > kPmax || pl.Nc + pl.Csep > 512 || pl.Nc % 16 != 0 || pl.Csep % 16 != 0 ||
      pl.Csep > pl.Nc || pl.smem > 227 * 1024)
    return fail(FAME_ERR_UNSUPPORTED, "tensor-core Taylor moments: order too high");
  if (grid.ax && (grid.m1 < 1 || grid.m2 < 1 || grid.m3 < 1 || grid.m1 * grid.m2 * grid.m3 != nB ||
                  grid.m1 + grid.m2 + grid.m3 > kMaxAxis))
    return fail(FAME_ERR_INVALID, "tensor-core Taylor moments: bad center grid");
  static int attr = [] {
    return cudaFuncSetAttribute(k_taylor_moments_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) ==
                   cudaSuccess
               ? FAME_OK
               : FAME_ERR_CUDA;
  }();
  if (attr != FAME_OK) return fail(attr, "tensor-core Taylor moments: shared-memory limit");
  TcArgs a{Q, c, NF, centers, nB, alistPacked, col, L, p, pl.Npad, pl.Nc, pl.Csep, pl.stages, pl.Kc, out,
           grid.ax, grid.m1, grid.m2, grid.m3};
  dim3 g3((unsigned)pl.nslices, (unsigned)pl.ntiles, (unsigned)pl.nsplit);
  k_taylor_moments_tc<<<g3, kThreads, pl.smem, s>>>(a, fault_word());
  ::fame::count_launch();
  const long long per = (long long)pl.ntiles * 128 * pl.Npad;
  double* part = reinterpret_cast<double*>(out + pl.nslices * per);
  k_taylor_tc_sum_slices<<<dim3((unsigned)((per + 255) / 256), (unsigned)pl.groups), 256, 0, s>>>(out, pl.nslices, per,
                                                                                                pl.groups, part);
  k_taylor_tc_finish<<<(unsigned)(((long long)nB * L + 255) / 256), 256, 0, s>>>(part, pl.groups, per, pl.Npad, L, nB,
                                                                                 col, coef, gamma);
  ::fame::count_launch(2);
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

}  // namespace fame
