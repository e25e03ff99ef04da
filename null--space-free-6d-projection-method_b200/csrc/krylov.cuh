// Device-resident PCG machinery shared by the K_r^{-1} realisations.
//
// MATLAB pcg (closed builtin; documented semantics restated): x0 = 0,
// stop when ||r|| <= tol*||b||, confirm on the true residual b - A*x (which
// then replaces r), flag 1 at maxit, flag 4 on breakdown.  Here every scalar
// (rho, p'Ap, alpha, beta) lives in a PcgState in device memory; kernels of
// queued iterations read PcgState::active and return at once after
// convergence, so the host checks convergence only every few iterations.
#pragma once
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
  st->rho = st->aux;
  st->beta = st->aux / st->rho_old;
  st->conv = 0;
  st->active = 1;
}

// ---------------------------------------------------------------- functors
// Unless stated otherwise, functors index line-order vectors (ia) and the
// line-order copies of W1, W2, invC.
// Mhat x = C^{-1}(M z + W1^* M(W1 z) + W2^* M(W2 z)), z = C^{-1} x
// (exp1/apply_Mhat_C_scalar_compact.m:8-21): three mass fields per vector.
template <typename T>
__device__ __forceinline__ void mhat_fields(const MhatCoef<T>& c, long long i, C<T> x, C<T>* v) {
  const C<T> z = cscale<T>(x, c.invC[i]);
  v[0] = z;
  v[1] = cmul<T>(c.W1[i], z);
  v[2] = cmul<T>(c.W2[i], z);
}
template <typename T>
__device__ __forceinline__ C<T> mhat_combine(const MhatCoef<T>& c, long long i, const C<T>* v) {
  C<T> s = cadd<T>(v[0], cadd<T>(cmulc<T>(c.W1[i], v[1]), cmulc<T>(c.W2[i], v[2])));
  return cscale<T>(s, c.invC[i]);
}

// Plain Mhat action; LINE selects line-order (ia) or natural-order (in)
// vectors and coefficients.
template <typename T, bool LINE> struct ProMhat {
  MhatCoef<T> c;
  const C<T>* x;
  __device__ __forceinline__ void load(long long ia, long long in, C<T>* v) const {
    const long long i = LINE ? ia : in;
    mhat_fields<T>(c, i, x[i], v);
  }
};
template <typename T, bool LINE> struct EpiMhat {
  using Acc = T;
  static constexpr int K = 0;
  MhatCoef<T> c;
  C<T>* y;
  T* partials = nullptr;
  unsigned* counter = nullptr;
  __device__ __forceinline__ void store(long long ia, long long in, const C<T>* v, Red<T, 1>&) const {
    const long long i = LINE ? ia : in;
    y[i] = mhat_combine<T>(c, i, v);
  }
  __device__ __forceinline__ void finalize(const Red<T, 1>&) const {}
};

// PCG search-direction update fused into the matvec prologue:
// p = r (first iteration) or p = r + beta p; then the Mhat fields of p.
template <typename T> struct ProPcgMhat {
  MhatCoef<T> c;
  C<T>* p;
  const C<T>* r;
  const PcgState* st;
  __device__ __forceinline__ void load(long long i, long long, C<T>* v) const {
    C<T> pi = r[i];
    if (st->iter > 0) pi = cadd<T>(pi, cscale<T>(p[i], (T)st->beta));
    p[i] = pi;
    mhat_fields<T>(c, i, pi, v);
  }
};
// Ap = Mhat p and the reduction p^H Ap -> alpha = rho / p^H Ap.
template <typename T> struct EpiPcgMhat {
  using Acc = T;
  static constexpr int K = 2;
  MhatCoef<T> c;
  C<T>* Ap;
  const C<T>* p;
  PcgState* st;
  T* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long i, long long, const C<T>* v, Red<T, 2>& acc) const {
    const C<T> ap = mhat_combine<T>(c, i, v);
    Ap[i] = ap;
    const C<T> d = cmulc<T>(p[i], ap);
    acc.v[0] += d.x;
    acc.v[1] += d.y;
  }
  __device__ __forceinline__ void finalize(const Red<T, 2>& tot) const {
    pcg_alpha_finalize(st, (double)tot.v[0], (double)tot.v[1]);
  }
};

// r = b - Mhat x with ||r||^2 into *out (true residual / refinement residual).
// With ADDX, the prologue first forms x = x + dx (dx in lower precision).
template <typename T, typename TD, bool ADDX> struct ProResidMhat {
  MhatCoef<T> c;
  C<T>* x;
  const C<TD>* dx;
  __device__ __forceinline__ void load(long long i, long long, C<T>* v) const {
    C<T> xi = x[i];
    if (ADDX) {
      xi = cadd<T>(xi, ccast<T, TD>(dx[i]));
      x[i] = xi;
    }
    mhat_fields<T>(c, i, xi, v);
  }
};
template <typename T> struct EpiResidMhat {
  using Acc = T;
  static constexpr int K = 1;
  MhatCoef<T> c;
  const C<T>* b;
  C<T>* r;
  double* out;
  T* partials;
  unsigned* counter;
  __device__ __forceinline__ void store(long long i, long long, const C<T>* v, Red<T, 1>& acc) const {
    const C<T> ri = csub<T>(b[i], mhat_combine<T>(c, i, v));
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
template <typename T>
__global__ void __launch_bounds__(256) k_pcg_update(C<T>* x, C<T>* r, const C<T>* p, const C<T>* Ap,
                                                   long long n, PcgState* st, T* partials,
                                                   unsigned* counter) {
  if (*((volatile int*)&st->active) == 0) return;
  const C<T> a = mk<T>((T)st->alpha_re, (T)st->alpha_im);
  Red<T, 1> acc;
  acc.v[0] = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
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

// PCG start with x0 = 0: r = (T) b, x = 0, rho = ||r||^2.
template <typename T, typename TB>
__global__ void __launch_bounds__(256) k_pcg_init(const C<TB>* b, C<T>* r, C<T>* x, long long n,
                                                 PcgState* st, double tol, int maxit, T* partials,
                                                 unsigned* counter) {
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
    pcg_init_state(st, (double)tot.v[0], tol, maxit);
  });
}

}  // namespace fame
