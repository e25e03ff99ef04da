// Device-resident PCG machinery shared by the K_r^{-1} realisations.
//
// MATLAB pcg (closed builtin; documented semantics restated): x0 = 0,
// stop when ||r|| <= tol*||b||, confirm on the true residual b - A*x (which
// then replaces r), flag 1 at maxit, flag 4 on breakdown.  Here every scalar
// (rho, p'Ap, alpha, beta) lives in a PcgState in device memory; kernels of
// queued iterations read PcgState::active and return at once after
// convergence, so the host checks convergence only every few iterations.
#pragma once
#include <algorithm>
#include "mass_chain.cuh"

namespace fame {

struct PcgState {
  double rho;       // r^H r of the current residual
  double rho_old;
  double pq_re, pq_im;
  double alpha_re, alpha_im;
  double beta;
  double bnorm2;    // ||b||^2
  double tolb2;     // (tol*||b||)^2
  double aux;       // last auxiliary reduction (true residual^2, output check)
  int iter, maxit, active, flag, conv, pad;
  int pend;         // 1: x += alpha p, r -= alpha Ap still to be applied (fused-update PCG)
  int pad2;
  double rz, rz_old;  // preconditioned PCG: r^H z of the current and previous iteration
};

// alpha = rho / p^H A p (complex, as MATLAB pcg); breakdown -> flag 4.
__device__ __forceinline__ void pcg_alpha_finalize(PcgState* st, double pr, double pi) {
  st->pq_re = pr;
  st->pq_im = pi;
  if (!(pr > 0.0) || !isfinite(pr) || !isfinite(pi)) {
    st->flag = 4;
    st->active = 0;
    return;
  }
  const double d = pr * pr + pi * pi;
  st->alpha_re = st->rho * pr / d;
  st->alpha_im = -st->rho * pi / d;
}

// PCG start state with x0 = 0 and ||b||^2 = rho.
__device__ __forceinline__ void pcg_init_state(PcgState* st, double rho, double tol, int maxit) {
  st->rho = rho;
  st->rho_old = rho;
  st->bnorm2 = rho;
  st->tolb2 = tol * tol * rho;
  st->beta = 0.0;
  st->iter = 0;
  st->maxit = maxit;
  st->aux = 0.0;
  st->pend = 0;
  if (!isfinite(rho)) {
    st->flag = -1;
    st->active = 0;
    st->conv = 0;
  } else {
    st->flag = 0;
    st->active = rho > 0.0 ? 1 : 0;
    st->conv = rho > 0.0 ? 0 : 1;
  }
}

// continue after a failed true-residual check (r already replaced by b - A x)
static __global__ void k_pcg_resume(PcgState* st) {
  st->pend = 0;
  st->rho = st->aux;
  st->beta = st->aux / st->rho_old;
  st->conv = 0;
  st->active = 1;
}

// ---------------------------------------------------------------- functors
// Unless stated otherwise, functors index line-order vectors (ia) and the
// line-order copies of W1, W2, invC.
// Mhat x = C^{-1}(M z + W1^* M(W1 z) + W2^* M(W2 z)), z = C^{-1} x
// (exp1/apply_Mhat_C_scalar_compact.m:8-21) as a linear-field chain:
// fields a_f z with a = (1, W1, W2), result C^{-1} sum_f b_f v_f with
// b = (1, conj W1, conj W2).  Read-only arrays go through the read-only path.
template <typename T> __device__ __forceinline__ C<T> ldc(const C<T>* p) { return __ldg(p); }
template <typename T> __device__ __forceinline__ T ldr(const T* p) { return __ldg(p); }

struct NoExt {};

template <typename T> struct MhatLinCoef {
  MhatCoef<T> c;
  __device__ __forceinline__ C<T> a(int f, long long i) const { return ldc<T>((f == 1 ? c.W1 : c.W2) + i); }
  __device__ __forceinline__ C<T> b(int f, long long i) const { return cconj<T>(ldc<T>((f == 1 ? c.W1 : c.W2) + i)); }
};

// Plain Mhat action; LINE selects line-order (ia) or natural-order (in)
// vectors and coefficients.
template <typename T, bool LINE> struct ProMhat {
  using Ext = NoExt;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  const C<T>* x;
  __device__ __forceinline__ C<T> load(long long ia, long long in, Ext&) const {
    const long long i = LINE ? ia : in;
    return cscale<T>(ldc<T>(x + i), ldr<T>(c.invC + i));
  }
  __device__ __forceinline__ void commit(long long, long long, const Ext&) const {}
  __device__ __forceinline__ C<T> coef(int f, long long ia, long long in) const {
    return MhatLinCoef<T>{c}.a(f, LINE ? ia : in);
  }
};
template <typename T, bool LINE> struct EpiMhat {
  using Acc = T;
  static constexpr int K = 0;
  static constexpr bool unit0 = true;
  static constexpr bool natural = !LINE;
  MhatCoef<T> c;
  C<T>* y;
  T* partials = nullptr;
  unsigned* counter = nullptr;
  __device__ __forceinline__ C<T> coef(int f, long long ia, long long in) const {
    return MhatLinCoef<T>{c}.b(f, LINE ? ia : in);
  }
  __device__ __forceinline__ void store(long long ia, long long in, C<T> s, Red<T, 1>&) const {
    const long long i = LINE ? ia : in;
    y[i] = cscale<T>(s, ldr<T>(c.invC + i));
  }
  __device__ __forceinline__ void finalize(const Red<T, 1>&) const {}
};

// One PCG iteration on Mhat in two fused halves (no separate update kernel).
// Prologue (pass A of iteration k): when a previous iteration left its update
// pending, x += alpha p and r -= alpha Ap first; then p = r (first iteration)
// or p = r + beta p, u = C^{-1} p.  x, r, p are stored after all loads.
template <typename T> struct PcgUpd {
  C<T> x, r, p;
};
template <typename T> struct ProPcgMhat {
  using Ext = PcgUpd<T>;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  C<T>* x;
  C<T>* r;
  C<T>* p;
  const C<T>* Ap;
  const PcgState* st;
  __device__ __forceinline__ C<T> load(long long i, long long, Ext& e) const {
    C<T> ri = r[i], pi = p[i];
    if (st->pend) {
      const C<T> a = mk<T>((T)st->alpha_re, (T)st->alpha_im);
      e.x = cadd<T>(x[i], cmul<T>(a, pi));
      ri = csub<T>(ri, cmul<T>(a, ldc<T>(Ap + i)));
    }
    e.r = ri;
    pi = st->iter > 0 ? cadd<T>(ri, cscale<T>(pi, (T)st->beta)) : ri;
    e.p = pi;
    return cscale<T>(pi, ldr<T>(c.invC + i));
  }
  __device__ __forceinline__ void commit(long long i, long long, const Ext& e) const {
    if (st->pend) {
      x[i] = e.x;
      r[i] = e.r;
    }
    p[i] = e.p;
  }
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.a(f, i); }
};
// Epilogue (pass C): Ap = Mhat p with the reductions p^H Ap, r^H Ap, ||Ap||^2
// and ||r||^2 (in FP64).  alpha = ||r||^2 / p^H Ap and the next residual norm
// follow without touching r again: ||r - alpha Ap||^2 = ||r||^2 -
// 2 Re(alpha r^H Ap) + |alpha|^2 ||Ap||^2.  Anchoring each step on ||r||^2 of
// the stored r keeps the rounding error to one step's cancellation (a pure
// recurrence on rho accumulates an absolute error of eps*||b||^2 and stalls
// near sqrt(eps) relative residual).  The update itself is left pending for
// the next prologue (or k_pcg_finish once the iteration stops).
template <typename T, bool PRE = false> struct EpiPcgMhat {
  using Acc = double;
  static constexpr int K = 6;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  C<T>* Ap;
  const C<T>* p;
  const C<T>* r;
  PcgState* st;
  double* partials;
  unsigned* counter;
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.b(f, i); }
  __device__ __forceinline__ void store(long long i, long long, C<T> s, Red<double, 6>& acc) const {
    const C<T> ap = cscale<T>(s, ldr<T>(c.invC + i));
    Ap[i] = ap;
    const C<T> pi = ldc<T>(p + i), ri = ldc<T>(r + i);
    acc.v[0] += (double)pi.x * ap.x + (double)pi.y * ap.y;  // p^H Ap
    acc.v[1] += (double)pi.x * ap.y - (double)pi.y * ap.x;
    acc.v[2] += (double)ri.x * ap.x + (double)ri.y * ap.y;  // r^H Ap
    acc.v[3] += (double)ri.x * ap.y - (double)ri.y * ap.x;
    acc.v[4] += (double)ap.x * ap.x + (double)ap.y * ap.y;  // ||Ap||^2
    acc.v[5] += (double)ri.x * ri.x + (double)ri.y * ri.y;  // ||r||^2
  }
  __device__ __forceinline__ void finalize(const Red<double, 6>& tot) const {
    if (!isfinite(tot.v[5])) {
      st->flag = 4;
      st->active = 0;
      st->pend = 0;
      return;
    }
    const double rr = tot.v[5];
    // alpha = rho / p^H Ap with rho = r^H r (plain) or r^H z (preconditioned)
    st->rho = PRE ? st->rz : rr;
    pcg_alpha_finalize(st, tot.v[0], tot.v[1]);
    if (st->flag == 4) {
      st->pend = 0;
      return;
    }
    const double ar = st->alpha_re, ai = st->alpha_im;
    double rho = rr - 2.0 * (ar * tot.v[2] - ai * tot.v[3]) + (ar * ar + ai * ai) * tot.v[4];
    if (rho < 0.0) rho = 0.0;  // one-step cancellation at convergence; confirmed on the true residual
    st->pend = 1;
    st->rho_old = rr;
    st->rho = rho;  // predicted ||r||^2 after the pending update
    st->iter += 1;
    if (!PRE) st->beta = rho / rr;
    if (!isfinite(rho)) {
      st->flag = 4;
      st->active = 0;
    } else if (rho <= st->tolb2) {
      st->conv = 1;
      st->flag = 0;
      st->active = 0;
    } else if (st->iter >= st->maxit) {
      st->flag = 1;
      st->active = 0;
    }
  }
};

// Preconditioned PCG on Mhat, P = C^{-1}(M^{-1} + W1^* M^{-1} W1 + W2^* M^{-1} W2) C^{-1}:
// Mhat = B^H (I3 (x) M) B with the isometry B = [I; W1; W2] C^{-1}, and since
// M = F diag(E) F^{-1} on the grid, M^{-1} is the same chain with 1/E, so P is
// the compression of M^{-1}.  One iteration is two chains:
//   P-chain  prologue applies the pending x += alpha p, r -= alpha Ap, input r;
//            epilogue z = P r and rz = r^H z (beta = rz / rz_old);
//   A-chain  prologue p = z + beta p, input p; epilogue Ap, alpha = rz / p^H Ap
//            and the predicted ||r||^2 for the convergence test (EpiPcgMhat<T, true>).
// The stopping test is on ||r|| / ||b|| as in MATLAB pcg.
template <typename T> struct ProPcgPre {
  using Ext = PcgUpd<T>;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  C<T>* x;
  C<T>* r;
  const C<T>* p;
  const C<T>* Ap;
  const PcgState* st;
  __device__ __forceinline__ C<T> load(long long i, long long, Ext& e) const {
    C<T> ri = r[i];
    if (st->pend) {
      const C<T> a = mk<T>((T)st->alpha_re, (T)st->alpha_im);
      e.x = cadd<T>(x[i], cmul<T>(a, ldc<T>(p + i)));
      ri = csub<T>(ri, cmul<T>(a, ldc<T>(Ap + i)));
    }
    e.r = ri;
    return cscale<T>(ri, ldr<T>(c.invC + i));
  }
  __device__ __forceinline__ void commit(long long i, long long, const Ext& e) const {
    if (st->pend) {
      x[i] = e.x;
      r[i] = e.r;
    }
  }
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.a(f, i); }
};
template <typename T> struct EpiPcgPre {
  using Acc = double;
  static constexpr int K = 2;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  C<T>* z;
  const C<T>* r;
  PcgState* st;
  double* partials;
  unsigned* counter;
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.b(f, i); }
  __device__ __forceinline__ void store(long long i, long long, C<T> s, Red<double, 2>& acc) const {
    const C<T> zi = cscale<T>(s, ldr<T>(c.invC + i));
    z[i] = zi;
    const C<T> ri = ldc<T>(r + i);
    acc.v[0] += (double)ri.x * zi.x + (double)ri.y * zi.y;  // r^H z (real for Hermitian P)
    acc.v[1] += (double)ri.x * zi.y - (double)ri.y * zi.x;
  }
  __device__ __forceinline__ void finalize(const Red<double, 2>& tot) const {
    st->pend = 0;  // the prologue of this chain has applied it
    const double rz = tot.v[0];
    if (!(rz > 0.0) || !isfinite(rz) || !isfinite(tot.v[1])) {
      st->flag = 4;
      st->active = 0;
      return;
    }
    st->rz_old = st->rz;
    st->rz = rz;
    st->beta = st->iter > 0 ? rz / st->rz_old : 0.0;
  }
};
template <typename T> struct ProPcgDir {
  using Ext = C<T>;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  C<T>* p;
  const C<T>* z;
  const PcgState* st;
  __device__ __forceinline__ C<T> load(long long i, long long, Ext& e) const {
    C<T> pi = ldc<T>(z + i);
    if (st->iter > 0) pi = cadd<T>(pi, cscale<T>(p[i], (T)st->beta));
    e = pi;
    return cscale<T>(pi, ldr<T>(c.invC + i));
  }
  __device__ __forceinline__ void commit(long long i, long long, const Ext& e) const { p[i] = e; }
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.a(f, i); }
};

// r = b - Mhat x with ||r||^2 into *out (true residual / refinement residual).
// With ADDX, the prologue first forms x = x + dx (dx in lower precision); with dst,
// dx is the solution of a PCG whose last update is still pending (dst->pend), and
// dx + alpha p is formed first, in dx's precision as k_pcg_finish would.
template <typename T, typename TD, bool ADDX> struct ProResidMhat {
  using Ext = C<T>;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  C<T>* x;
  const C<TD>* dx;
  const C<TD>* dp = nullptr;
  const PcgState* dst = nullptr;
  __device__ __forceinline__ C<T> load(long long i, long long, Ext& e) const {
    C<T> xi = x[i];
    if (ADDX) {
      C<TD> d = ldc<TD>(dx + i);
      if (dst && dst->pend) d = cadd<TD>(d, cmul<TD>(mk<TD>((TD)dst->alpha_re, (TD)dst->alpha_im), ldc<TD>(dp + i)));
      xi = cadd<T>(xi, ccast<T, TD>(d));
    }
    e = xi;
    return cscale<T>(xi, ldr<T>(c.invC + i));
  }
  __device__ __forceinline__ void commit(long long i, long long, const Ext& e) const {
    if (ADDX) x[i] = e;
  }
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.a(f, i); }
};
template <typename T> struct EpiResidMhat {
  using Acc = T;
  static constexpr int K = 1;
  static constexpr bool unit0 = true;
  MhatCoef<T> c;
  const C<T>* b;
  C<T>* r;
  double* out;
  T* partials;
  unsigned* counter;
  __device__ __forceinline__ C<T> coef(int f, long long i, long long) const { return MhatLinCoef<T>{c}.b(f, i); }
  __device__ __forceinline__ void store(long long i, long long, C<T> s, Red<T, 1>& acc) const {
    const C<T> ri = csub<T>(ldc<T>(b + i), cscale<T>(s, ldr<T>(c.invC + i)));
    r[i] = ri;
    acc.v[0] += cabs2<T>(ri);
  }
  __device__ __forceinline__ void finalize(const Red<T, 1>& tot) const { *out = (double)tot.v[0]; }
};

// Block-diagonal mass M3 = diag(M,M,M) on component-stacked 3NF vectors
// (the Mop handle, exp1/applyM_component_first_rank1_scalar.m:11-19):
// the three components are the three fields of one chain.
template <typename T> struct ProPcgM3 {
  C<T>* p;
  const C<T>* r;
  const PcgState* st;
  long long NF;
  __device__ __forceinline__ void load(long long i, long long, C<T>* v) const {
    const bool upd = st->iter > 0;
    const T beta = (T)st->beta;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      C<T> pi = r[c * NF + i];
      if (upd) pi = cadd<T>(pi, cscale<T>(p[c * NF + i], beta));
      p[c * NF + i] = pi;
      v[c] = pi;
    }
  }
};
template <typename T> struct EpiPcgM3 {
  using Acc = T;
  static constexpr int K = 2;
  C<T>* Ap;
  const C<T>* p;
  PcgState* st;
  long long NF;
  T* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long i, long long, const C<T>* v, Red<T, 2>& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Ap[c * NF + i] = v[c];
      const C<T> d = cmulc<T>(p[c * NF + i], v[c]);
      acc.v[0] += d.x;
      acc.v[1] += d.y;
    }
  }
  __device__ __forceinline__ void finalize(const Red<T, 2>& tot) const {
    pcg_alpha_finalize(st, (double)tot.v[0], (double)tot.v[1]);
  }
};
template <typename T, typename TD, bool ADDX> struct ProResidM3 {
  C<T>* x;
  const C<TD>* dx;
  long long NF;
  __device__ __forceinline__ void load(long long i, long long, C<T>* v) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      C<T> xi = x[c * NF + i];
      if (ADDX) {
        xi = cadd<T>(xi, ccast<T, TD>(dx[c * NF + i]));
        x[c * NF + i] = xi;
      }
      v[c] = xi;
    }
  }
};
template <typename T> struct EpiResidM3 {
  using Acc = T;
  static constexpr int K = 1;
  const C<T>* b;
  C<T>* r;
  double* out;
  long long NF;
  T* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long i, long long, const C<T>* v, Red<T, 1>& acc) const {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const C<T> ri = csub<T>(b[c * NF + i], v[c]);
      r[c * NF + i] = ri;
      acc.v[0] += cabs2<T>(ri);
    }
  }
  __device__ __forceinline__ void finalize(const Red<T, 1>& tot) const { *out = (double)tot.v[0]; }
};

// ------------------------------------------------------------ vector kernels
inline int vec_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 8); }
constexpr int kVecBlocksMax = 148 * 8;

// x += alpha p; r -= alpha Ap; rho = r^H r; convergence bookkeeping.
// Four independent elements per thread, all loads issued before the stores.
constexpr int kUpdUnroll = 4;
inline int upd_blocks(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + 256LL * kUpdUnroll - 1) / (256LL * kUpdUnroll), 148 * 8));
}
template <typename T>
__global__ void __launch_bounds__(256) k_pcg_update(C<T>* x, C<T>* r, const C<T>* __restrict__ p,
                                                   const C<T>* __restrict__ Ap, long long n, PcgState* st,
                                                   T* partials, unsigned* counter) {
  if (*((volatile int*)&st->active) == 0) return;
  const C<T> a = mk<T>((T)st->alpha_re, (T)st->alpha_im);
  Red<T, 1> acc;
  acc.v[0] = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i + (kUpdUnroll - 1) * stride < n; i += kUpdUnroll * stride) {
    C<T> xv[kUpdUnroll], rv[kUpdUnroll], pv[kUpdUnroll], av[kUpdUnroll];
#pragma unroll
    for (int k = 0; k < kUpdUnroll; ++k) {
      const long long ik = i + k * stride;
      xv[k] = x[ik];
      rv[k] = r[ik];
      pv[k] = __ldg(p + ik);
      av[k] = __ldg(Ap + ik);
    }
#pragma unroll
    for (int k = 0; k < kUpdUnroll; ++k) {
      const long long ik = i + k * stride;
      x[ik] = cadd<T>(xv[k], cmul<T>(a, pv[k]));
      const C<T> ri = csub<T>(rv[k], cmul<T>(a, av[k]));
      r[ik] = ri;
      acc.v[0] += cabs2<T>(ri);
    }
  }
  for (; i < n; i += stride) {
    x[i] = cadd<T>(x[i], cmul<T>(a, p[i]));
    const C<T> ri = csub<T>(r[i], cmul<T>(a, Ap[i]));
    r[i] = ri;
    acc.v[0] += cabs2<T>(ri);
  }
  grid_sum_finalize<T, 1>(acc, partials, counter, [&](const Red<T, 1>& tot) {
    const double rho = (double)tot.v[0];
    st->rho_old = st->rho;
    st->rho = rho;
    st->iter += 1;
    st->beta = rho / st->rho_old;
    if (!isfinite(rho)) {
      st->flag = 4;
      st->active = 0;
    } else if (rho <= st->tolb2) {
      st->conv = 1;
      st->flag = 0;
      st->active = 0;
    } else if (st->iter >= st->maxit) {
      st->flag = 1;
      st->active = 0;
    }
  });
}

// The update left pending by the last fused iteration: x += alpha p,
// r -= alpha Ap (queued by the host only when PcgState::pend is set).
template <typename T>
__global__ void __launch_bounds__(256) k_pcg_finish(C<T>* x, C<T>* r, const C<T>* __restrict__ p,
                                                   const C<T>* __restrict__ Ap, long long n, PcgState* st) {
  const C<T> a = mk<T>((T)st->alpha_re, (T)st->alpha_im);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] = cadd<T>(x[i], cmul<T>(a, p[i]));
    r[i] = csub<T>(r[i], cmul<T>(a, Ap[i]));
  }
}

// PCG start with x0 = 0: r = (T) b, x = 0, rho = ||r||^2.  With ref (a correction
// solve of FP64 iterative refinement, b the refinement residual whose squared norm and
// right-hand side norm ref holds): the relative tolerance is half the reduction that
// takes ||b|| to tolIR ||bhat||, at least tol and at most 1e-2, and a residual already at
// the target starts converged (no iterations).
template <typename T, typename TB>
__global__ void __launch_bounds__(256) k_pcg_init(const C<TB>* b, C<T>* r, C<T>* x, long long n,
                                                 PcgState* st, double tol, int maxit, T* partials,
                                                 unsigned* counter, const PcgState* ref = nullptr,
                                                 double tolIR = 0.0) {
  Red<T, 1> acc;
  acc.v[0] = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const C<T> ri = ccast<T, TB>(b[i]);
    r[i] = ri;
    x[i] = mk<T>(0, 0);
    acc.v[0] += cabs2<T>(ri);
  }
  grid_sum_finalize<T, 1>(acc, partials, counter, [&](const Red<T, 1>& tot) {
    double tau = tol;
    bool at_target = false;
    if (ref) {
      const double bn2 = ref->bnorm2, rn2 = ref->rho;
      at_target = rn2 <= tolIR * tolIR * bn2 || !(bn2 > 0.0);
      if (!at_target) tau = fmin(1e-2, fmax(tol, 0.5 * tolIR * sqrt(bn2 / rn2)));
    }
    pcg_init_state(st, (double)tot.v[0], tau, maxit);
    if (at_target && st->flag == 0) {
      st->active = 0;
      st->conv = 1;
    }
  });
}

}  // namespace fame
