// fft_kernels.cuh -- row-pass and column-pass kernel templates built on fft_core.
//
// A 2-D transform of an nx-by-ny plane (row-major, idx = x + y*nx) is a row pass
// (contiguous vectors of length nx) and a column pass (vectors of length ny with
// element stride nx). Both kernels are batched over planes and take an operator
// `Op` that supplies
//   kStages            1 (one transform) or 2 (two chained transforms)
//   kInv1, kInv2       direction of each transform
//   load(plane, line, e)                 -> float2   input element e of the line
//   mid(plane, line, e, float2&)                      pointwise op between stages
//   store(plane, line, e, float2, Acc&)               consume output element e
//   finish(plane, block_in_plane, blocks_per_plane, Acc&)   block epilogue
// `line` is the row index y for the row kernel and the column index x for the
// column kernel; `e` is the element position along the transformed axis.
#pragma once
#include "fft_core.cuh"

namespace doe {

struct NoAcc {};

// Threads per CTA and vectors per CTA chosen per transform length.
template <int N>
struct RowCfg {
  static constexpr int T = Plan<N>::T;
  static constexpr int V = (256 / T) > 0 ? (256 / T) : 1;  // vectors per CTA
  static constexpr int THREADS = V * T;
  static constexpr int SMEM = Plan<N>::NP > 1 ? V * padded_len<N>() * (int)sizeof(float2) : 0;
};

template <int N>
struct ColCfg {
  static constexpr int T = Plan<N>::T;
  // columns per CTA: 256-512 threads, enough registers for RMAX = 32 per thread
  static constexpr int C = Plan<N>::NP == 1 ? 128
                           : (T >= 128 ? (512 / T > 0 ? 512 / T : 1)
                                       : ((256 / T) < 4 ? 4 : ((256 / T) > 32 ? 32 : (256 / T))));
  static constexpr int THREADS = C * T;
  static constexpr int SMEM = Plan<N>::NP > 1 ? (N * C + (N * C) / 32 + 1) * (int)sizeof(float2) : 0;
};

struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Row pass. Grid: nplanes * ceil(nlines / V) CTAs; rows beyond nlines idle.
template <int N, class Op>
__global__ void __launch_bounds__(RowCfg<N>::THREADS) row_kernel(Op op, const float2* __restrict__ tw,
                                                                 int nlines) {
  constexpr int T = Plan<N>::T;
  constexpr int V = RowCfg<N>::V;
  constexpr int RMAX = Plan<N>::RMAX;
  extern __shared__ float2 smem[];
  const int lv = threadIdx.x / T;
  const int t = threadIdx.x % T;
  const int bpp = (nlines + V - 1) / V;  // blocks per plane
  const int plane = blockIdx.x / bpp;
  const int bip = blockIdx.x % bpp;
  const int line = bip * V + lv;
  const bool active = line < nlines;
  SmemVec s{smem + lv * padded_len<N>(), 1, 0};
  float2 v[RMAX];
#pragma unroll
  for (int q = 0; q < RMAX; ++q)
    v[q] = active ? op.load(plane, line, in_elem<N, 0>(t, q)) : make_float2(0.f, 0.f);
  if constexpr (Op::kStages >= 1) fft_run<N, Op::kInv1>(v, t, s, tw, BlockSync{});
  if constexpr (Op::kStages == 2) {
    if (active) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) op.mid(plane, line, out_elem<N>(t, q), v[q]);
    }
    relayout_out_to_in<N>(v, t, s, BlockSync{});
    fft_run<N, Op::kInv2>(v, t, s, tw, BlockSync{});
  }
  typename Op::Acc acc{};
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) op.store(plane, line, out_elem<N>(t, q), v[q], acc);
  }
  op.finish(plane, bip, bpp, acc);
}

// Column pass. Grid: (ceil(ncols / C), nplanes); columns beyond ncols idle.
template <int N, class Op>
__global__ void __launch_bounds__(ColCfg<N>::THREADS) col_kernel(Op op, const float2* __restrict__ tw,
                                                                 int ncols) {
  constexpr int C = ColCfg<N>::C;
  constexpr int RMAX = Plan<N>::RMAX;
  extern __shared__ float2 smem[];
  const int c = threadIdx.x % C;
  const int t = threadIdx.x / C;
  const int plane = blockIdx.y;
  const int line = blockIdx.x * C + c;
  const bool active = line < ncols;
  SmemVec s{smem, C, c};
  float2 v[RMAX];
#pragma unroll
  for (int q = 0; q < RMAX; ++q)
    v[q] = active ? op.load(plane, line, in_elem<N, 0>(t, q)) : make_float2(0.f, 0.f);
  if constexpr (Op::kStages >= 1) fft_run<N, Op::kInv1>(v, t, s, tw, BlockSync{});
  if constexpr (Op::kStages == 2) {
    if (active) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) op.mid(plane, line, out_elem<N>(t, q), v[q]);
    }
    relayout_out_to_in<N>(v, t, s, BlockSync{});
    fft_run<N, Op::kInv2>(v, t, s, tw, BlockSync{});
  }
  typename Op::Acc acc{};
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) op.store(plane, line, out_elem<N>(t, q), v[q], acc);
  }
  op.finish(plane, blockIdx.x, gridDim.x, acc);
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
