// fft_kernels.cuh -- row-pass and column-pass kernel templates built on fft_core.
//
// A 2-D transform of an nx-by-ny plane (row-major, idx = x + y*nx) is a row pass
// (contiguous vectors of length nx) and a column pass (vectors of length ny with
// element stride nx). Both kernels are batched over planes and take an operator
// `Op` that supplies
//   kStages            1 (one transform) or 2 (two chained transforms)
//   kInv1, kInv2       direction of each transform
//   State init(plane, line)                         per-thread invariants of a line
//   load(State&, e)                 -> float2        input element e of the line
//   mid(State&, e, float2&, Acc&)                    pointwise op between stages
//   store(State&, e, float2, Acc&)                   consume output element e
//   finish(plane, block_in_plane, blocks_per_plane, Acc&)   block epilogue
// `line` is the row index y for the row kernel and the column index x for the
// column kernel; `e` is the element position along the transformed axis. init()
// is called for inactive lines too (with a clamped line index) and must not fault.
#pragma once
#include <tuple>
#include <type_traits>
#include <utility>

#include "fft_core.cuh"

namespace doe {

struct NoAcc {};

// CTA shapes. A row shape processes V vectors of a plane per CTA (one vector =
// one row), a column shape C adjacent columns (element-major tile in shared
// memory, the C columns of an element adjacent; padded per the plan's PSHIFT).
template <class P, int V_, int MINB_ = 1>
struct RowShape {
  using Plan = P;
  static constexpr int N = P::N;
  static constexpr int V = V_;
  static constexpr int MINB = MINB_;  // CTAs per SM the register budget is sized for
  static constexpr int T = P::T;
  static constexpr int THREADS = V * T;
  static constexpr int SMEM = P::NP > 1 ? V * padded_len<P::N>() * (int)sizeof(float2) : 0;
};

template <class P, int C_, int MINB_ = 1>
struct ColShape {
  using Plan = P;
  static constexpr int N = P::N;
  static constexpr int C = C_;
  static constexpr int MINB = MINB_;  // CTAs per SM the register budget is sized for
  static constexpr int T = P::T;
  static constexpr int THREADS = C * T;
  static constexpr int SMEM = P::NP > 1 ? padded_col<P>(P::N * C) * (int)sizeof(float2) : 0;
};

// Default shapes: ~256 threads per CTA (512 for the longest vectors).
template <int N>
struct DefRow {
  using P = typename DefaultPlan<N>::type;
  using type = RowShape<P, ((256 / P::T) > 0 ? (256 / P::T) : 1)>;
};
template <int N>
struct DefCol {
  using P = typename DefaultPlan<N>::type;
  static constexpr int C = P::NP == 1 ? 128
                           : (P::T >= 128 ? (512 / P::T > 0 ? 512 / P::T : 1)
                                          : ((256 / P::T) < 4 ? 4 : ((256 / P::T) > 32 ? 32 : (256 / P::T))));
  using type = ColShape<P, C>;
};

// 2048-point rows: the default plan, with registers capped for three 256-thread
// CTAs per SM (the design loops' fused row operators otherwise take ~100-128
// registers, two CTAs per SM, and stall on memory latency).
template <>
struct DefRow<2048> {
  using type = RowShape<typename DefaultPlan<2048>::type, 2, 3>;
};

// 2048-point columns: radix 32-2-32 with 4 columns per CTA (256 threads; the
// design loops' two-transform column operators use ~254 registers, one CTA per
// SM, no spills) beats the default 16-8-16 plan with 512-thread CTAs in those
// column passes on B200 (~12 % less time per pass; capping the 16-8-16 plan at
// three 256-thread CTAs per SM spills and is ~45 % slower); rows keep the default
// plan (their fused operators spill at RMAX 32).
template <>
struct DefCol<2048> {
  using type = ColShape<FftPlan<2048, 3, 32, 2, 32>, 4>;
};

// 256-point columns: registers capped for two CTAs of 16 columns per SM.
template <>
struct DefCol<256> {
  using type = ColShape<typename DefaultPlan<256>::type, 16, 2>;
};

// Tunable shape lists (index 0 is the default). Only the large lengths, where
// register pressure and occupancy trade against shared-memory passes, carry
// alternatives; the autotuner measures them on the device.
template <int N>
struct RowVariants {
  using list = std::tuple<typename DefRow<N>::type>;
};
template <int N>
struct ColVariants {
  using list = std::tuple<typename DefCol<N>::type>;
};
template <>
struct RowVariants<1024> {
  using list = std::tuple<RowShape<FftPlan<1024, 2, 32, 32>, 8>, RowShape<FftPlan<1024, 3, 16, 4, 16>, 4>,
                          RowShape<FftPlan<1024, 3, 16, 4, 16>, 2>, RowShape<FftPlan<1024, 2, 32, 32>, 4>>;
};
template <>
struct ColVariants<1024> {
  using list = std::tuple<ColShape<FftPlan<1024, 2, 32, 32>, 8>, ColShape<FftPlan<1024, 3, 16, 4, 16>, 4>,
                          ColShape<FftPlan<1024, 3, 16, 4, 16>, 8>, ColShape<FftPlan<1024, 2, 32, 32>, 4>,
                          ColShape<FftPlan<1024, 3, 16, 4, 16>, 4, 4>, ColShape<FftPlan<1024, 3, 16, 4, 16>, 2, 6>>;
};  // the last two cap registers for 4 x 256 and 6 x 128 threads per SM (the sweep column pass picks the first)
template <>
struct RowVariants<2048> {
  using list = std::tuple<RowShape<FftPlan<2048, 3, 16, 8, 16>, 2>, RowShape<FftPlan<2048, 3, 32, 2, 32>, 4>,
                          RowShape<FftPlan<2048, 3, 8, 32, 8>, 1>, RowShape<FftPlan<2048, 3, 16, 8, 16>, 1>>;
};
template <>
struct ColVariants<2048> {
  using list = std::tuple<ColShape<FftPlan<2048, 3, 16, 8, 16>, 4>, ColShape<FftPlan<2048, 3, 32, 2, 32>, 4>,
                          ColShape<FftPlan<2048, 3, 16, 8, 16>, 2>, ColShape<FftPlan<2048, 3, 32, 2, 32>, 8>>;
};
// Shape variants of the design-loop passes: the default plan of length N in every
// variant (so a variant changes how lines are grouped into CTAs and the register
// cap, never the transform's arithmetic), for the lengths the benchmarked design
// loops use. Index 0 is the default; 1 toggles the register cap between one and
// two resident CTAs; 2 halves the lines per CTA with a cap for four CTAs per SM.
template <int N>
struct DesignRowVariants {
  using D = typename DefRow<N>::type;
  using P = typename D::Plan;
  using list = std::conditional_t<
      (N >= 64 && N <= 2048),
      std::tuple<D, RowShape<P, D::V, (D::MINB == 2 ? 1 : 2)>, RowShape<P, (D::V > 1 ? D::V / 2 : 1), 4>>,
      std::tuple<D>>;
};
template <int N>
struct DesignColVariants {
  using D = typename DefCol<N>::type;
  using P = typename D::Plan;
  using list = std::conditional_t<
      (N >= 64 && N <= 2048),
      std::tuple<D, ColShape<P, D::C, (D::MINB == 2 ? 1 : 2)>, ColShape<P, (D::C > 2 ? D::C / 2 : 1), 4>>,
      std::tuple<D>>;
};

template <>
struct RowVariants<512> {
  using list = std::tuple<RowShape<FftPlan<512, 3, 8, 8, 8>, 4>, RowShape<FftPlan<512, 2, 16, 32>, 16>,
                          RowShape<FftPlan<512, 2, 32, 16>, 16>>;
};
template <>
struct ColVariants<512> {
  using list = std::tuple<ColShape<FftPlan<512, 3, 8, 8, 8>, 4>, ColShape<FftPlan<512, 2, 16, 32>, 16>,
                          ColShape<FftPlan<512, 2, 32, 16>, 16>>;
};

struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Operators may expose `bool skip(int plane)`: a CTA whose plane is skipped
// returns before its first barrier (the plane is uniform per CTA).
template <class Op, class = void>
struct HasSkip : std::false_type {};
template <class Op>
struct HasSkip<Op, std::void_t<decltype(std::declval<const Op&>().skip(0))>> : std::true_type {};
// Operators may split their load: `load` issues the global reads only and
// `finish_load(state, e, raw)` applies the pointwise factor afterwards, so that
// every read of a thread is in flight before the first factor is evaluated (a
// factor with a rarely taken out-of-line branch would otherwise keep the compiler
// from hoisting the next element's read above it).
template <class Op, class = void>
struct HasFinishLoad : std::false_type {};
template <class Op>
struct HasFinishLoad<Op, std::void_t<decltype(std::declval<const Op&>().finish_load(
                             std::declval<const typename Op::State&>(), 0, float2{}))>> : std::true_type {};

// Operators may expose `prefetch(state, e)`: it touches the lines of side planes
// that a later stage of the pass reads for element e, and runs just before the
// element's load. Column passes use it up to 1024 points only: the 2048-point
// design column operators need ~250 registers without it and the extra addresses
// cost them more than the hidden latency saves.
template <class Op, class = void>
struct HasPrefetch : std::false_type {};
template <class Op>
struct HasPrefetch<Op, std::void_t<decltype(std::declval<const Op&>().prefetch(
                           std::declval<const typename Op::State&>(), 0))>> : std::true_type {};

template <class Op>
__device__ __forceinline__ bool op_skip(const Op& op, int plane) {
  if constexpr (HasSkip<Op>::value) {
    return op.skip(plane);
  } else {
    return false;
  }
}

// Row pass. Grid: nplanes * ceil(nlines / V) CTAs; rows beyond nlines idle.
template <class S, class Op>
__device__ __forceinline__ void row_pass(const Op& op, const float2* __restrict__ tw, int nlines) {
  using P = typename S::Plan;
  constexpr int T = P::T;
  constexpr int V = S::V;
  constexpr int RMAX = P::RMAX;
  extern __shared__ float2 smem[];
  const int lv = threadIdx.x / T;
  const int t = threadIdx.x % T;
  const int bpp = (nlines + V - 1) / V;  // blocks per plane
  const int plane = blockIdx.x / bpp;
  const int bip = blockIdx.x % bpp;
  const int line = bip * V + lv;
  const bool active = line < nlines;
  if (op_skip(op, plane)) return;
  SmemVec<> s{smem + lv * padded_len<P::N>(), 1, 0};
  auto st = op.init(plane, active ? line : 0);
  typename Op::Acc acc{};
  float2 v[RMAX];
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) {
      if constexpr (HasPrefetch<Op>::value) op.prefetch(st, in_elem<P>(t, q));
      v[q] = op.load(st, in_elem<P>(t, q));
    }
    if constexpr (HasFinishLoad<Op>::value) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) v[q] = op.finish_load(st, in_elem<P>(t, q), v[q]);
    }
  } else {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) v[q] = make_float2(0.f, 0.f);
  }
  if constexpr (Op::kStages >= 1) fft_run<P, Op::kInv1>(v, t, s, tw, BlockSync{});
  if constexpr (Op::kStages == 2) {
    if (active) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) op.mid(st, out_elem<P>(t, q), v[q], acc);
    }
    relayout_out_to_in<P>(v, t, s, BlockSync{});
    fft_run<P, Op::kInv2>(v, t, s, tw, BlockSync{});
  }
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) op.store(st, out_elem<P>(t, q), v[q], acc);
  }
  op.finish(plane, bip, bpp, acc);
}

// Column pass. Grid: (ceil(ncols / C), nplanes); columns beyond ncols idle.
template <class S, class Op>
__device__ __forceinline__ void col_pass(const Op& op, const float2* __restrict__ tw, int ncols) {
  using P = typename S::Plan;
  constexpr int C = S::C;
  constexpr int RMAX = P::RMAX;
  extern __shared__ float2 smem[];
  const int c = threadIdx.x % C;
  const int t = threadIdx.x / C;
  const int plane = blockIdx.y;
  const int line = blockIdx.x * C + c;
  const bool active = line < ncols;
  if (op_skip(op, plane)) return;
  SmemVec<P::PSHIFT> s{smem, C, c};
  auto st = op.init(plane, active ? line : 0);
  typename Op::Acc acc{};
  float2 v[RMAX];
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) {
      if constexpr (HasPrefetch<Op>::value && S::N <= 1024) op.prefetch(st, in_elem<P>(t, q));
      v[q] = op.load(st, in_elem<P>(t, q));
    }
    if constexpr (HasFinishLoad<Op>::value) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) v[q] = op.finish_load(st, in_elem<P>(t, q), v[q]);
    }
  } else {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) v[q] = make_float2(0.f, 0.f);
  }
  if constexpr (Op::kStages >= 1) fft_run<P, Op::kInv1>(v, t, s, tw, BlockSync{});
  if constexpr (Op::kStages == 2) {
    if (active) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) op.mid(st, out_elem<P>(t, q), v[q], acc);
    }
    relayout_out_to_in<P>(v, t, s, BlockSync{});
    fft_run<P, Op::kInv2>(v, t, s, tw, BlockSync{});
  }
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) op.store(st, out_elem<P>(t, q), v[q], acc);
  }
  op.finish(plane, blockIdx.x, gridDim.x, acc);
}

// The kernels. Shapes with MINB > 1 get the register cap of MINB resident CTAs
// per SM; the others leave the register budget to the compiler (an explicit
// minimum of one CTA per SM lets it use all 255 registers, which costs occupancy).
template <class S, class Op>
__global__ void __launch_bounds__(S::THREADS) row_kernel(Op op, const float2* __restrict__ tw, int nlines) {
  row_pass<S, Op>(op, tw, nlines);
}
template <class S, class Op>
__global__ void __launch_bounds__(S::THREADS, S::MINB) row_kernel_capped(Op op, const float2* __restrict__ tw,
                                                                         int nlines) {
  row_pass<S, Op>(op, tw, nlines);
}
template <class S, class Op>
__global__ void __launch_bounds__(S::THREADS) col_kernel(Op op, const float2* __restrict__ tw, int ncols) {
  col_pass<S, Op>(op, tw, ncols);
}
template <class S, class Op>
__global__ void __launch_bounds__(S::THREADS, S::MINB) col_kernel_capped(Op op, const float2* __restrict__ tw,
                                                                         int ncols) {
  col_pass<S, Op>(op, tw, ncols);
}

// ---------------------------------------------------------------- FP64 reductions
// K running sums per thread, reduced per block in a fixed order, written as a
// per-block partial; the last block of each group (plane) folds the partials in
// block order and stores the group total. Deterministic run to run.
template <int K>
struct DAcc {
  double v[K];
};

template <int K>
__device__ __forceinline__ void block_sum(DAcc<K>& a) {
  __shared__ double red[32][K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = a.v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    a.v[k] = x;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) red[warp][k] = a.v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double x = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      a.v[k] = x;
    }
  }
}

// partials: [ngroups][blocks_per_group][K]; counters: [ngroups]; totals: [ngroups][K].
// Returns true (in every thread) for the last block of the group; totals are
// valid for that block once this returns.
template <int K>
__device__ __forceinline__ bool group_reduce(DAcc<K>& a, int group, int block_in_group, int blocks_per_group,
                                             double* __restrict__ partials, unsigned* __restrict__ counters,
                                             double* __restrict__ totals) {
  __shared__ bool s_last;
  block_sum<K>(a);
  if (threadIdx.x == 0) {
    double* p = partials + ((long)group * blocks_per_group + block_in_group) * K;
#pragma unroll
    for (int k = 0; k < K; ++k) p[k] = a.v[k];
    __threadfence();
    const unsigned ticket = atomicAdd(&counters[group], 1u);
    s_last = (ticket == (unsigned)blocks_per_group - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  // last block: fold partials in block order (fixed-order tree over threads)
  DAcc<K> b;
#pragma unroll
  for (int k = 0; k < K; ++k) b.v[k] = 0.0;
  const volatile double* p = partials + (long)group * blocks_per_group * K;
  for (int i = threadIdx.x; i < blocks_per_group; i += blockDim.x) {
#pragma unroll
    for (int k = 0; k < K; ++k) b.v[k] += p[(long)i * K + k];
  }
  block_sum<K>(b);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) totals[(long)group * K + k] = b.v[k];
    counters[group] = 0u;  // re-arm for the next launch
  }
  __syncthreads();
  return true;
}

}  // namespace doe
