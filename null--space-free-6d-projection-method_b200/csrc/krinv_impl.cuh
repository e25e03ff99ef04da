// fame_krinv layout and helpers shared by krinv.cu, nested.cu and lanczos.cu.
#pragma once
#include "internal.cuh"
#include "krylov.cuh"

namespace fame {

template <typename T> struct PcgBuf {
  C<T>* work = nullptr;  // 3 fields of NF (mass chain)
  C<T>* z = nullptr;     // preconditioned residual (Mhat PCG with the inverse-material preconditioner)
  C<T>* x = nullptr;
  C<T>* r = nullptr;
  C<T>* p = nullptr;
  C<T>* Ap = nullptr;
};

// Outer (K_r) PCG state of the nested realisation.
struct OuterState {
  double rho, rho1, beta, pq_re, pq_im, alpha_re, alpha_im, rr, bnorm2, tolb2;
  int iter, pad;
};

}  // namespace fame

// refinement rounds of the mixed explicit K_r^{-1} that keep their own chunk hint (later
// rounds share the last one)
constexpr int kRoundHints = 4;

struct fame_krinv {
  fame_basis* b = nullptr;
  fame_mass* m = nullptr;
  fame_ctx* ctx = nullptr;
  fame_krinv_opts o{};
  fame_krinv_stats stats{};
  long long NF = 0;
  int n = 0;
  fame::PcgBuf<double> b64;
  fame::PcgBuf<float> b32;
  double2 *mr1 = nullptr, *mr2 = nullptr, *bhat = nullptr;
  double* partials = nullptr;
  unsigned* counter = nullptr;
  fame::PcgState *st64 = nullptr, *st32 = nullptr;
  int lastIt64 = 0, lastIt32 = 0;
  int lastIt32Round[kRoundHints] = {};  // explicit mixed: FP32 iterations of each refinement round
  // nested (method B) outer vectors, 2NF each
  double2 *ox = nullptr, *orr = nullptr, *oz = nullptr, *op = nullptr, *oq = nullptr;
  double* sigma = nullptr;  // |q|^2 (NF), sigma_r = [sigma; sigma]
  fame::OuterState* ost = nullptr;
  void* lanczos_ws = nullptr;  // Lanczos basis workspace reused across solves
  // set while Lanczos applies the explicit operator: the NaN/Inf test of each output is
  // left to Lanczos, whose own read of the step's coefficients would see it, instead of
  // costing a host synchronisation per call (krinv_output_check runs it on demand)
  bool deferOutputCheck = false;
  // CUDA graphs of PCG iterations per (precision, operator): [slot] holds kGraphIters
  // iterations, [6 + slot] one iteration (the remainder of a chunk)
  cudaGraphExec_t graphs[12] = {};
};

namespace fame {
int nested_alloc(fame_krinv* K);
void nested_free(fame_krinv* K);
int krinv_nested_apply_one(fame_krinv* K, const double2* b, double2* x);
int krinv_output_check(fame_krinv* K);
void lanczos_ws_free(fame_krinv* K);
int recover_one(fame_krinv* K, const double2* y, double2* X, double2* MX, int* iters, double* relres);
template <typename T> MhatCoef<T> coef_of(fame_basis* b);       // natural order
template <typename T> MhatCoef<T> coef_line_of(fame_basis* b);  // line order
template <typename T> const T* es_of(fame_mass* m);
}  // namespace fame

namespace fame {

// Operator tags for the generic PCG driver: each launches one PCG matvec
// chain (search-direction update fused in front, p^H A p reduction behind)
// and one true-residual chain r = b - A x.
template <typename T> struct OpMhat {
  MhatCoef<T> c;
  const T* Es;
  static constexpr int nvec = 1;   // vector length in units of NF
  static constexpr int mass_per_matvec = 3;
  static constexpr bool fused_update = true;  // x/r update inside the next matvec's prologue
  static constexpr int launches_per_iter = 3;
  static constexpr int kind = 0;
  int matvec(fame_krinv* K, PcgBuf<T>& B, PcgState* st, cudaStream_t s) const {
    ProPcgMhat<T> pro{c, B.x, B.r, B.p, B.Ap, st};
    EpiPcgMhat<T> epi{c, B.Ap, B.p, B.r, st, K->partials, K->counter};
    return run_chain_lin<T, 3>(K->n, pro, epi, B.work, Es, K->NF, s, Gate{&st->active}, K->o.passColumns);
  }
  int resid(fame_krinv* K, PcgBuf<T>& B, const C<T>* b, double* out, cudaStream_t s) const {
    ProResidMhat<T, T, false> pro{c, B.x, nullptr};
    EpiResidMhat<T> epi{c, b, B.r, out, reinterpret_cast<T*>(K->partials), K->counter};
    return run_chain_lin<T, 3>(K->n, pro, epi, B.work, Es, K->NF, s, Gate{nullptr}, K->o.passColumns);
  }
};

template <typename T> struct OpM3 {
  const T* Es;
  static constexpr int nvec = 3;
  static constexpr int mass_per_matvec = 3;
  static constexpr bool fused_update = false;
  static constexpr int launches_per_iter = 4;
  static constexpr int kind = 1;
  int matvec(fame_krinv* K, PcgBuf<T>& B, PcgState* st, cudaStream_t s) const {
    ProPcgM3<T> pro{B.p, B.r, st, K->NF};
    EpiPcgM3<T> epi{B.Ap, B.p, st, K->NF, reinterpret_cast<T*>(K->partials), K->counter};
    return run_chain<T, 3>(K->n, pro, epi, B.work, Es, K->NF, s, Gate{&st->active});
  }
  int resid(fame_krinv* K, PcgBuf<T>& B, const C<T>* b, double* out, cudaStream_t s) const {
    ProResidM3<T, T, false> pro{B.x, nullptr, K->NF};
    EpiResidM3<T> epi{b, B.r, out, K->NF, reinterpret_cast<T*>(K->partials), K->counter};
    return run_chain<T, 3>(K->n, pro, epi, B.work, Es, K->NF, s);
  }
};

// Mhat with the inverse-material preconditioner (krylov.cuh, ProPcgPre): two
// chains per iteration, the second material 1/E.
template <typename T> struct OpMhatPre {
  MhatCoef<T> c;
  const T* Es;
  const T* EsInv;
  static constexpr int nvec = 1;
  static constexpr int mass_per_matvec = 6;
  static constexpr bool fused_update = true;
  static constexpr int launches_per_iter = 6;
  static constexpr int kind = 2;
  int matvec(fame_krinv* K, PcgBuf<T>& B, PcgState* st, cudaStream_t s) const {
    ProPcgPre<T> pp{c, B.x, B.r, B.p, B.Ap, st};
    EpiPcgPre<T> ep{c, B.z, B.r, st, K->partials, K->counter};
    FAME_TRY((run_chain_lin<T, 3>(K->n, pp, ep, B.work, EsInv, K->NF, s, Gate{&st->active}, K->o.passColumns)));
    ProPcgDir<T> pd{c, B.p, B.z, st};
    EpiPcgMhat<T, true> ea{c, B.Ap, B.p, B.r, st, K->partials, K->counter};
    return run_chain_lin<T, 3>(K->n, pd, ea, B.work, Es, K->NF, s, Gate{&st->active}, K->o.passColumns);
  }
  int resid(fame_krinv* K, PcgBuf<T>& B, const C<T>* b, double* out, cudaStream_t s) const {
    return OpMhat<T>{c, Es}.resid(K, B, b, out, s);
  }
};

// PCG iterations per captured graph.  A chunk of c iterations replays the graph of
// kGraphIters iterations c / kGraphIters times and a one-iteration graph for the rest,
// so it queues exactly the iterations asked for: surplus iterations are gated off on
// the device but still cost their launches (~15 us per iteration at 2N = 10), and
// every graph launch adds a few microseconds on the device.
constexpr int kGraphIters = 4;

template <typename T, class Op> constexpr int graph_slot() {
  return (sizeof(T) == 8 ? 0 : 1) + 2 * Op::kind;
}

template <typename T, class Op>
int enqueue_iterations(fame_krinv* K, const Op& op, PcgBuf<T>& B, PcgState* st, cudaStream_t s, int count) {
  T* partials = reinterpret_cast<T*>(K->partials);
  const long long nlen = (long long)Op::nvec * K->NF;
  for (int it = 0; it < count; ++it) {
    FAME_TRY(op.matvec(K, B, st, s));
    if constexpr (!Op::fused_update) {
      k_pcg_update<T><<<upd_blocks(nlen), 256, 0, s>>>(B.x, B.r, B.p, B.Ap, nlen, st, partials, K->counter);
      ::fame::count_launch();
    }
  }
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

// Capture `iters` PCG iterations as a graph (on a capture stream, so that the work
// already queued on the context stream is not part of it).
template <typename T, class Op>
int capture_iterations(fame_krinv* K, const Op& op, PcgBuf<T>& B, PcgState* st, int iters, cudaGraphExec_t& ge) {
  cudaStream_t cs = K->ctx->own;
  if (cs == K->ctx->stream) {
    if (!K->ctx->capture) FAME_CUDA_TRY(cudaStreamCreateWithFlags(&K->ctx->capture, cudaStreamNonBlocking));
    cs = K->ctx->capture;
  }
  cudaGraph_t g = nullptr;
  FAME_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  const int st_enq = enqueue_iterations<T>(K, op, B, st, cs, iters);
  const cudaError_t e_end = cudaStreamEndCapture(cs, &g);
  if (st_enq != FAME_OK) {
    if (g) cudaGraphDestroy(g);
    return st_enq;
  }
  if (e_end != cudaSuccess) return fail(FAME_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e_end));
  const cudaError_t e_inst = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e_inst != cudaSuccess) {
    ge = nullptr;
    return fail(FAME_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e_inst));
  }
  return FAME_OK;
}

// Queue `count` gated PCG iterations: replays of the captured graphs of kGraphIters
// and of one iteration, or plain launches before the graphs exist (the first
// iterations run eagerly, so that kernel attributes are set and modules loaded
// before the capture).
template <typename T, class Op>
int queue_iterations(fame_krinv* K, const Op& op, PcgBuf<T>& B, PcgState* st, int count) {
  cudaStream_t s = K->ctx->stream;
  if (!K->o.useGraphs) return enqueue_iterations<T>(K, op, B, st, s, count);
  cudaGraphExec_t& ge = K->graphs[graph_slot<T, Op>()];
  cudaGraphExec_t& ge1 = K->graphs[6 + graph_slot<T, Op>()];
  if (!ge) {
    const int eager = std::min(count, kGraphIters);
    FAME_TRY(enqueue_iterations<T>(K, op, B, st, s, eager));
    count -= eager;
    FAME_TRY(capture_iterations<T>(K, op, B, st, kGraphIters, ge));
  }
  for (; count >= kGraphIters; count -= kGraphIters) {
    FAME_CUDA_TRY(cudaGraphLaunch(ge, s));
    ::fame::count_launch((long long)Op::launches_per_iter * kGraphIters);
  }
  if (count > 0 && !ge1) FAME_TRY(capture_iterations<T>(K, op, B, st, 1, ge1));
  for (; count > 0; --count) {
    FAME_CUDA_TRY(cudaGraphLaunch(ge1, s));
    ::fame::count_launch((long long)Op::launches_per_iter);
  }
  return FAME_OK;
}

// Queue PCG iterations until the device state stops them; the host reads the
// state once per chunk (the first chunk is the previous solve's iteration count).  With verify, convergence is confirmed on the true
// residual as MATLAB pcg does, continuing up to three times if it fails.
template <typename T, class Op>
int pcg_iterate(fame_krinv* K, const Op& op, PcgBuf<T>& B, PcgState* st, int& lastIt, PcgState& h,
                bool verify, const C<T>* b, bool keepPending = false) {
  cudaStream_t s = K->ctx->stream;
  const int every = std::max(1, K->o.checkEvery);
  int chunk = lastIt > 0 ? lastIt : every;  // iteration counts repeat from call to call
  int queued = 0, moresteps = 0;
  for (;;) {
    FAME_TRY((queue_iterations<T, Op>(K, op, B, st, chunk)));
    queued += chunk;
    FAME_TRY(read_back(K->ctx, st, &h, sizeof(PcgState)));
    if (h.active) {
      if (queued > h.maxit + 4 * every + kGraphIters) return fail(FAME_ERR_CUDA, "PCG state did not stop at maxit");
      chunk = every;
      continue;
    }
    // apply the last iteration's x/r update (keepPending: the caller's next kernel applies
    // it to x, and r is not needed)
    if (Op::fused_update && h.pend && !keepPending) {
      const long long nlen = (long long)Op::nvec * K->NF;
      k_pcg_finish<T><<<vec_blocks(nlen), 256, 0, s>>>(B.x, B.r, B.p, B.Ap, nlen, st);
      ::fame::count_launch();
      FAME_CUDA_TRY(cudaMemsetAsync(&st->pend, 0, sizeof(int), s));
      h.pend = 0;
    }
    if (verify && h.conv && h.flag == 0) {
      FAME_TRY(op.resid(K, B, b, &st->aux, s));
      K->stats.massApplies += Op::mass_per_matvec;
      FAME_TRY(read_back(K->ctx, st, &h, sizeof(PcgState)));
      if (h.aux > h.tolb2) {
        if (++moresteps < 3 && h.iter < h.maxit) {
          k_pcg_resume<<<1, 1, 0, s>>>(st);
          ::fame::count_launch();
          chunk = every;
          continue;
        }
        h.flag = 3;
      }
      h.rho = h.aux;
    }
    break;
  }
  lastIt = h.iter;
  K->stats.massApplies += (long long)Op::mass_per_matvec * h.iter;
  return FAME_OK;
}

}  // namespace fame
