// Host-side launch of one fused mass-operator chain (pass A -> B -> C) for a
// runtime axis length n = 2N, dispatching to the compile-time kernels.
#pragma once
#include "passb.cuh"

namespace fame {

inline int round32(int x) { return (x + 31) / 32 * 32; }

// Set the dynamic shared-memory limit of a kernel once per process.
template <typename K> int ensure_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return FAME_OK;
  FAME_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return FAME_OK;
}

// Pass B over nfields tile-major fields with the tiled material Et (E/NF in the
// layout of k_tile_E for this n and T): a persistent grid of (resident CTAs per
// SM) x SMs, each CTA owning a contiguous range of (tile, field) units.
// poll_limit / arm_only: fault-path self-test (fame_selftest_bounded_wait).
template <int n, typename T, typename TE>
int launch_passB(C<T>* work, int nfields, const TE* Et, long long NF, cudaStream_t st, Gate gate,
                 unsigned poll_limit = kMbarPollLimit, int arm_only = 0) {
  using G = PassBGeom<n, T>;
  constexpr size_t smem = G::template smem_bytes<TE>();
  static int attr = ensure_smem(k_passB<n, T, TE>, smem);
  if (attr != FAME_OK) return attr;
  static int per_sm = [] {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_passB<n, T, TE>, G::threads, smem) != cudaSuccess) b = 1;
    return b < 1 ? 1 : b;
  }();
  const int units = (G::n3 / G::TT) * nfields;
  const int grid = std::min(units, per_sm * num_sms());
  k_passB<n, T, TE><<<grid, G::threads, smem, st>>>(work, Et, nfields, NF, gate, fault_word(), poll_limit, arm_only);
  ::fame::count_launch();
  return FAME_OK;
}

template <int n, typename T, int F, class Pro>
int launch_passA(const Pro& pro, C<T>* work, long long NF, cudaStream_t st, Gate gate) {
  using Q = Cube<n, T>;
  constexpr int G = PassACols<n, T>::value;
  const size_t smem = (size_t)G * F * Q::size * sizeof(C<T>);
  static int attr = ensure_smem(k_passA<n, T, F, G, Pro>, smem);
  if (attr != FAME_OK) return attr;
  const int threads = std::min(512, std::max(32, round32(G * Q::n2)));
  k_passA<n, T, F, G, Pro><<<Q::n3 / G, threads, smem, st>>>(pro, work, NF, gate);
  ::fame::count_launch();
  return FAME_OK;
}

template <int n, typename T, int F, class Epi>
int launch_passC(const Epi& epi, const C<T>* work, long long NF, cudaStream_t st, Gate gate) {
  using Q = Cube<n, T>;
  constexpr int G = PassACols<n, T>::value;
  const size_t smem = (size_t)G * F * Q::size * sizeof(C<T>);
  static int attr = ensure_smem(k_passC<n, T, F, G, Epi>, smem);
  if (attr != FAME_OK) return attr;
  const int threads = std::min(512, std::max(32, round32(G * Q::n2)));
  k_passC<n, T, F, G, Epi><<<Q::n3 / G, threads, smem, st>>>(epi, work, NF, gate);
  ::fame::count_launch();
  return FAME_OK;
}

// Number of CTAs pass C launches (size of the reduction partials it needs).
inline long long passC_blocks(int n) { return (long long)n * n * n; }

template <int n, typename T, int F, class Pro, class Epi, typename TE>
int chain_n(const Pro& pro, const Epi& epi, C<T>* work, const TE* Et, long long NF,
            cudaStream_t st, Gate gate) {
  FAME_TRY((launch_passA<n, T, F, Pro>(pro, work, NF, st, gate)));
  FAME_TRY((launch_passB<n, T, TE>(work, F, Et, NF, st, gate)));
  FAME_TRY((launch_passC<n, T, F, Epi>(epi, work, NF, st, gate)));
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

// y-chain for axis length n in {2,4,...,14}.  work holds F fields of NF.
template <typename T, int F, class Pro, class Epi, typename TE>
int run_chain(int n, const Pro& pro, const Epi& epi, C<T>* work, const TE* Et, long long NF, cudaStream_t st, Gate gate = Gate{nullptr}) {
  switch (n) {
    case 2: return chain_n<2, T, F>(pro, epi, work, Et, NF, st, gate);
    case 4: return chain_n<4, T, F>(pro, epi, work, Et, NF, st, gate);
    case 6: return chain_n<6, T, F>(pro, epi, work, Et, NF, st, gate);
    case 8: return chain_n<8, T, F>(pro, epi, work, Et, NF, st, gate);
    case 10: return chain_n<10, T, F>(pro, epi, work, Et, NF, st, gate);
    case 12: return chain_n<12, T, F>(pro, epi, work, Et, NF, st, gate);
    case 14: return chain_n<14, T, F>(pro, epi, work, Et, NF, st, gate);
    default: return fail(FAME_ERR_UNSUPPORTED, "mass operator supports 2N in {2,4,...,14}");
  }
}

// Columns per CTA of the linear-field passes (one line per thread).
// n = 10: one column (100 lines) per CTA, several CTAs per SM (measured 1-3 % faster K_r^{-1}
// actions than two columns, in both precision forms).
template <int n, typename T> struct LinCols {
  static constexpr int value = n == 10 ? 1
                               : n == 2 ? 8 : n == 4 ? 16 : n == 6 ? 12 : n == 8 ? 8 : n == 12 ? 2 : 2;
  static_assert((n * n * n) % value == 0 && value * n * n <= 512, "linear chain tiling");
};

template <int n, typename T, int F, int G, class Pro, class Epi, typename TE>
int chain_lin_g(const Pro& pro, const Epi& epi, C<T>* work, const TE* Et, long long NF,
                cudaStream_t st, Gate gate) {
  using Q = Cube<n, T>;
  const size_t smem = (size_t)G * Q::size * sizeof(C<T>);
  const int threads = round32(G * Q::n2);
  static int attrA = ensure_smem(k_passA_lin<n, T, F, G, Pro>, smem);
  static int attrC = ensure_smem(k_passC_lin<n, T, F, G, Epi>, smem);
  if (attrA != FAME_OK) return attrA;
  if (attrC != FAME_OK) return attrC;
  k_passA_lin<n, T, F, G, Pro><<<Q::n3 / G, threads, smem, st>>>(pro, work, NF, gate);
  ::fame::count_launch();
  FAME_TRY((launch_passB<n, T, TE>(work, F, Et, NF, st, gate)));
  k_passC_lin<n, T, F, G, Epi><<<Q::n3 / G, threads, smem, st>>>(epi, work, NF, gate);
  ::fame::count_launch();
  FAME_CUDA_TRY(cudaGetLastError());
  return FAME_OK;
}

// Columns per CTA of the linear passes: LinCols by default; `cols` selects one of the
// alternatives compiled for the Bloch-path sizes (n = 6, 8, 10), any other value the default.
// The choice changes the CTA grouping (and so the order of the grid reductions), not the
// arithmetic of a mode.
template <int n, typename T, int F, class Pro, class Epi, typename TE>
int chain_lin_n(const Pro& pro, const Epi& epi, C<T>* work, const TE* Et, long long NF, cudaStream_t st, Gate gate,
                int cols) {
  if constexpr (n == 10) {
    if (cols == 2) return chain_lin_g<n, T, F, 2>(pro, epi, work, Et, NF, st, gate);
    if (cols == 4) return chain_lin_g<n, T, F, 4>(pro, epi, work, Et, NF, st, gate);
  } else if constexpr (n == 8) {
    if (cols == 2) return chain_lin_g<n, T, F, 2>(pro, epi, work, Et, NF, st, gate);
    if (cols == 4) return chain_lin_g<n, T, F, 4>(pro, epi, work, Et, NF, st, gate);
  } else if constexpr (n == 6) {
    if (cols == 4) return chain_lin_g<n, T, F, 4>(pro, epi, work, Et, NF, st, gate);
    if (cols == 6) return chain_lin_g<n, T, F, 6>(pro, epi, work, Et, NF, st, gate);
  }
  return chain_lin_g<n, T, F, LinCols<n, T>::value>(pro, epi, work, Et, NF, st, gate);
}

// Linear-field chain (see k_passA_lin) for axis length n in {2,4,...,14}.
template <typename T, int F, class Pro, class Epi, typename TE>
int run_chain_lin(int n, const Pro& pro, const Epi& epi, C<T>* work, const TE* Et, long long NF, cudaStream_t st,
                  Gate gate = Gate{nullptr}, int cols = 0) {
  switch (n) {
    case 2: return chain_lin_n<2, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    case 4: return chain_lin_n<4, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    case 6: return chain_lin_n<6, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    case 8: return chain_lin_n<8, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    case 10: return chain_lin_n<10, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    case 12: return chain_lin_n<12, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    case 14: return chain_lin_n<14, T, F>(pro, epi, work, Et, NF, st, gate, cols);
    default: return fail(FAME_ERR_UNSUPPORTED, "mass operator supports 2N in {2,4,...,14}");
  }
}

// ------------------------------------------------------------ functors
// Identity prologue/epilogue (plain mass action, natural order): F columns.
template <typename T, int F> struct ProCols {
  static constexpr bool natural = true;
  const C<T>* x[F];
  __device__ __forceinline__ void load(long long, long long i, C<T>* v) const {
#pragma unroll
    for (int f = 0; f < F; ++f) v[f] = x[f][i];
  }
};
template <typename T, int F> struct EpiCols {
  using Acc = T;
  static constexpr int K = 0;
  static constexpr bool natural = true;
  C<T>* y[F];
  T* partials = nullptr;
  unsigned* counter = nullptr;
  __device__ __forceinline__ void store(long long, long long i, const C<T>* v, Red<T, 1>&) const {
#pragma unroll
    for (int f = 0; f < F; ++f) y[f][i] = v[f];
  }
  __device__ __forceinline__ void finalize(const Red<T, 1>&) const {}
};

// Coefficients of the orthogonalised inner operator
// (exp1/build_experiment1_q_system_C_compact.m:21-31).
template <typename T> struct MhatCoef {
  const T* invC;
  const C<T>* W1;
  const C<T>* W2;
};

}  // namespace fame
