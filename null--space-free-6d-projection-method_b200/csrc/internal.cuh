// Internal handle layouts behind the opaque C ABI types.
#pragma once
#include <vector>
#include "fame_common.cuh"

struct fame_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t capture = nullptr;  // graph-capture stream when `stream` is the context's own
  cudaEvent_t ev = nullptr;
  void* pinned = nullptr;  // small host staging area (4 KB)
  void* ws = nullptr;      // grow-only device workspace (ctx_workspace)
  size_t ws_bytes = 0;
  std::vector<void*> allocs;
};

struct fame_mass {
  fame_ctx* ctx = nullptr;
  int N = 0, n = 0;
  long long NF = 0;
  double* Et64 = nullptr;  // E / NF, FP64, pass-B tile order of the FP64 chains (k_tile_E)
  float* Et32 = nullptr;   // E / NF, FP32, pass-B tile order of the FP32 chains
  void* work = nullptr;    // one NF-field of complex128 scratch for the mass modes
  double* EtInv64 = nullptr;  // NF^-1 / E in the same tile order: the inverse mass operator
  float* EtInv32 = nullptr;
};

struct fame_basis {
  fame_ctx* ctx = nullptr;
  int N = 0, n = 0;
  long long NF = 0;
  double2 *V[6] = {nullptr};  // V11,V21,V31,V12,V22,V32
  double2 *det = nullptr, *W1 = nullptr, *W2 = nullptr;
  double *invC = nullptr, *Qq = nullptr, *q[3] = {nullptr};
  float2 *W1f = nullptr, *W2f = nullptr;
  float* invCf = nullptr;
  // line-order copies used inside solves (axis 1 slowest within each column)
  double2 *W1_l = nullptr, *W2_l = nullptr;
  double* invC_l = nullptr;
  float2 *W1f_l = nullptr, *W2f_l = nullptr;
  float* invCf_l = nullptr;
  void* work = nullptr;  // scratch of fame_apply_Mhat_C_scalar_compact (3 fields)
  size_t work_bytes = 0;
  double P[18] = {0};  // cut matrix, column-major 6 x 3
  int pivot = 2;       // physical component forming the V3 row of the explicit split
  double2* Vp[4] = {nullptr, nullptr, nullptr, nullptr};  // V1 block when pivot != 2
  fame_basis_info info{};
  // (r, c) entry of the V1 block of the explicit split (rows = the components other than pivot)
  const double2* V1(int r, int c) const { return pivot == 2 ? V[r + 3 * c] : Vp[2 * r + c]; }
};

namespace fame {
// device allocation helpers recorded for cleanup by the owner
int dalloc(void** p, size_t bytes);
void dfree(void* p);
// While alive, dalloc/dfree of this host thread allocate from the library's memory
// pool in the order of stream s (all work on the blocks must be queued on s): frees
// then no longer synchronise the whole device.  Used by concurrent solves.
struct StreamOrderedAlloc {
  explicit StreamOrderedAlloc(cudaStream_t s);
  ~StreamOrderedAlloc();
  StreamOrderedAlloc(const StreamOrderedAlloc&) = delete;
  StreamOrderedAlloc& operator=(const StreamOrderedAlloc&) = delete;
  bool prev_on;
  cudaStream_t prev;
};
// copy a small device struct to host (synchronises the stream)
int read_back(fame_ctx* ctx, const void* dsrc, void* hdst, size_t bytes);
// FAME_ERR_CUDA (and clears the word) if a bounded device-side wait gave up on ctx's device
int check_fault(fame_ctx* ctx);
// At least `bytes` of device workspace owned by ctx, reused across calls (grown
// after a stream synchronisation); valid until the next call on the context.
int ctx_workspace(fame_ctx* ctx, size_t bytes, void** out);
// Taylor block moments on the tensor cores (taylor_tc.cu): launch shape and the
// FP32 partial-moment buffer (out_floats) it needs.
struct TaylorTcPlan {
  int Npad = 0, stages = 0, ntiles = 0, groups = 0;
  int nsplit = 1, Nc = 0;  // monomial columns split over nsplit CTAs of Nc columns each
  int Csep = 0;            // columns (of a CTA's Nc) whose cross products accumulate apart
  bool graded = false;     // the degree-p monomials take the last columns (taylor_tc_columns)
  long long Kc = 0, nslices = 0;
  size_t smem = 0, out_floats = 0;
};
TaylorTcPlan taylor_tc_plan(long long NF, int nB, int L, int p);
// col[a] (Npad entries): output column of monomial a (alist3: L triples a1, a2, a3).
void taylor_tc_columns(const TaylorTcPlan& plan, const int* alist3, int L, int p, int* col);
// Centers on a tensor grid: center b = (ax[b % m1], ax[m1 + (b / m1) % m2], ax[m1 + m2 + b / (m1 m2)]).
struct TaylorTcGrid {
  const double* ax = nullptr;  // device, m1 + m2 + m3 values (nullptr: centers are general)
  int m1 = 0, m2 = 0, m3 = 0;
};
constexpr int kTaylorTcMaxAxis = 24;  // m1 + m2 + m3 at most for the factorised phases
// gamma[b L + a] = coef[a] sum_j c_j e^{i q_j.r_b} q_j^a, with alistPacked[a] = a1 | a2 << 8 | a3 << 16.
int taylor_moments_tc(const TaylorTcPlan& plan, cudaStream_t s, const double2* c, const double* Q, long long NF,
                      const double* centers, int nB, const int* alistPacked, const int* col, int L, int p,
                      const double2* coef, float* out, double2* gamma, const TaylorTcGrid& grid);
// Batched complex GEMM C = A B (FP64 complex, element strides) as split-FP32
// (3xTF32) tcgen05 products (zgemm_tc.cu), in two steps: the operands are split into
// head/tail TF32 panels in the UMMA shared-memory layout (up to four operands per launch),
// then the GEMM streams the panels.  A panels: rows = M (complex rows m), batches = the
// GEMM's batch; B panels: rows = N (columns n), cols_for_b = N, batches = the distinct B
// operands (the GEMM uses B panel batch z / bdivB).  Strides are those of the FP64 operand:
// A (s_row, s_k) = (sam, sak), B = (sbn, sbk).  Panel buffers are 1024-byte aligned.
struct ZPanelJob {
  const double2* src;
  long long s_row, s_k, s_batch;
  int rows, K, batches;
  bool a_role;
  int cols_for_b;  // B role: the GEMM's N (sets the panel tile)
  unsigned char* out;
};
size_t zpanel_bytes(const ZPanelJob& job);
int zsplit_panels(const ZPanelJob* jobs, int njobs, cudaStream_t s);
int zgemm_3xtf32_panels(const unsigned char* Ap, const unsigned char* Bp, double2* C, int M, int N, int K,
                        long long scm, long long scn, long long bC, int batch, int bdivB, cudaStream_t s);
// A Hermitian operator on n-vectors of complex128 for the restarted Lanczos
// (lanczos.cu): y = A x on ctx's stream; *ws holds the reusable basis workspace.
struct LanczosOperator {
  fame_ctx* ctx;
  long long n;
  void** ws;
  int (*apply)(void* self, const double2* x, double2* y);
  void* self;
  // optional: reports an error of the last apply that was left for Lanczos to detect
  // (called when the step's Lanczos coefficients come back NaN/Inf)
  int (*check)(void* self) = nullptr;
};
int lanczos_run(const LanczosOperator& op, int nev, double tol, int maxiter, int p, const void* v0, double* theta,
                void* Y, fame_lanczos_info* info);
void lanczos_ws_release(void** ws);
// Consecutive 256-byte aligned pieces of one workspace.
struct Carve {
  size_t used = 0;
  char* base = nullptr;
  template <typename T> T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base ? base + used : nullptr);
    used += (count * sizeof(T) + 255) / 256 * 256;
    return p;
  }
};
}  // namespace fame
