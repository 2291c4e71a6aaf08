// sweep_sym.cuh -- focus-sweep column pass (src/propagate.js:427-434 over
// :57-133) with the transfer function shared between mirrored rows.
//
// H(kx, ky) depends on fy only through fy^2 (the propagation phase, the band limit
// and its raised-cosine edge are all even in fy), and the FFT bins ky and N - ky
// carry opposite frequencies, so H(kx, ky) = H(kx, N - ky). A CTA of this pass owns
// C whole columns; it evaluates H once for rows 0..N/2 of each of its columns into
// shared memory (half the per-pixel transfer-function work of the plain column
// pass) and every element reads its factor there. The spectrum reads go first, so
// that their latency overlaps the table evaluation; the inverse column FFT and the
// intermediate's layout are those of the plain pass (ColSweepBase).
#pragma once
#include <atomic>

#include "ops_propagate.cuh"
#include "tcgen05.cuh"

namespace doe {

template <class S>
constexpr int sweep_sym_smem() {
  return S::SMEM + (S::N / 2 + 1) * S::C * (int)sizeof(float2);
}

template <class S>
__global__ void __launch_bounds__(S::THREADS, S::MINB)
    sweep_col_sym_kernel(ColSweepBase op, const float2* __restrict__ tw, int ncols) {
  using P = typename S::Plan;
  constexpr int C = S::C, RMAX = P::RMAX, N = P::N, NH = N / 2 + 1;
  extern __shared__ float2 smem[];
  float2* hs = smem + S::SMEM / (int)sizeof(float2);  // [NH][C]: H of row k of column c at k * C + c
  const int c = threadIdx.x % C;
  const int t = threadIdx.x / C;
  const int plane = blockIdx.y;
  const int line = blockIdx.x * C + c;
  const bool active = line < ncols;
  SmemVec<P::PSHIFT> s{smem, C, c};
  const auto st = op.init(plane, active ? line : 0);
  float2 v[RMAX];
#pragma unroll
  for (int q = 0; q < RMAX; ++q)
    v[q] = active ? __ldg(&st.spec[(long)in_elem<P>(t, q) * op.nx]) : make_float2(0.f, 0.f);
  for (int ky = t; ky < NH; ky += P::T) hs[ky * C + c] = asm_h_col(st.h, op.tab, ky);
  __syncthreads();
#pragma unroll
  for (int q = 0; q < RMAX; ++q) {
    const int ky = in_elem<P>(t, q);
    v[q] = cmul(v[q], hs[(ky <= N / 2 ? ky : N - ky) * C + c]);
  }
  fft_run<P, true>(v, t, s, tw, BlockSync{});
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) st.out[(long)out_elem<P>(t, q) * op.nx] = v[q];
  }
}

// Launch over `nplanes` planes (grid y) and the ncols columns (grid x, C per CTA).
template <class S>
inline int launch_sweep_sym(doe_ctx* c, const ColSweepBase& op, int nplanes, int ncols) {
  constexpr int smem = sweep_sym_smem<S>();
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  DOE_TRY(prepare_kernel(c, sweep_col_sym_kernel<S>, smem, attr_set, false));
  if (nplanes <= 0) return DOE_OK;
  if (nplanes > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "column pass: at most 65535 planes per launch");
  dim3 grid((ncols + S::C - 1) / S::C, nplanes);
  LaunchScope ls(c, ColSweepBase::kName);
  sweep_col_sym_kernel<S><<<grid, S::THREADS, smem, c->stream>>>(op, c->tw + S::N, ncols);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

// TMA-staged form of the mirrored-row pass: one thread has the tensor memory
// accelerator copy the CTA's whole spectrum tile (C columns x N rows, boxes of 256
// rows, no multicast) into the FFT exchange buffer while every thread evaluates the
// transfer-function table; the elements are then read from shared memory, so the
// pass issues no per-element global loads. The wait on the copy is bounded (1 s;
// code 4 in the context's error word, after a second bounded wait for the copy).
template <class S>
constexpr int sweep_tma_smem() {
  return 128 + S::SMEM + (S::N / 2 + 1) * S::C * (int)sizeof(float2) + 16;
}

template <class S>
__global__ void __launch_bounds__(S::THREADS, S::MINB)
    sweep_col_tma_kernel(const __grid_constant__ CUtensorMap spec_map, ColSweepBase op,
                         const float2* __restrict__ tw, int ncols, int* __restrict__ err) {
  using P = typename S::Plan;
  constexpr int C = S::C, RMAX = P::RMAX, N = P::N, NH = N / 2 + 1, BOX = N < 256 ? N : 256;
  extern __shared__ unsigned char smraw[];
  float2* smem = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
  float2* hs = smem + S::SMEM / (int)sizeof(float2);            // [NH][C] transfer-function table
  uint64_t* bar = reinterpret_cast<uint64_t*>(hs + NH * C);     // 8-byte aligned (NH * C * 8 bytes before)
  const int c = threadIdx.x % C;
  const int t = threadIdx.x / C;
  const int plane = blockIdx.y;
  const int x0 = blockIdx.x * C;
  const int line = x0 + c;
  const bool active = line < ncols;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
                 "r"((uint32_t)(N * C * sizeof(float2)))
                 : "memory");
#pragma unroll 1
    for (int r0 = 0; r0 < N; r0 += BOX)
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
              tc::smem_u32(smem + r0 * C)),
          "l"(reinterpret_cast<uint64_t>(&spec_map)), "r"(2 * x0), "r"(r0), "r"(tc::smem_u32(bar))
          : "memory");
  }
  const auto st = op.init(plane, active ? line : 0);
  for (int ky = t; ky < NH; ky += P::T) hs[ky * C + c] = asm_h_col(st.h, op.tab, ky);
  __syncthreads();  // the table, and the barrier's initialisation, are visible
  bool ok = tc::mbar_wait_bounded(bar, 0, 1000000000ull);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) {
      atomicExch(err, 4);
      (void)tc::mbar_wait_bounded(bar, 0, 1000000000ull);  // the copy lands before the CTA leaves
    }
    __syncthreads();
    return;
  }
  float2 v[RMAX];
#pragma unroll
  for (int q = 0; q < RMAX; ++q) {
    const int ky = in_elem<P>(t, q);
    v[q] = cmul(smem[ky * C + c], hs[(ky <= N / 2 ? ky : N - ky) * C + c]);
  }
  SmemVec<P::PSHIFT> s{smem, C, c};  // the transform's exchanges reuse the tile's buffer (its first step is in registers)
  fft_run<P, true>(v, t, s, tw, BlockSync{});
  if (active) {
#pragma unroll
    for (int q = 0; q < RMAX; ++q) st.out[(long)out_elem<P>(t, q) * op.nx] = v[q];
  }
}

template <class S>
inline int launch_sweep_tma(doe_ctx* c, const ColSweepBase& op, int nplanes, int ncols) {
  constexpr int smem = sweep_tma_smem<S>();
  if (S::N * S::C * (int)sizeof(float2) > S::SMEM || (ncols % S::C) || (S::C * 8) % 16) return DOE_ERR_UNSUPPORTED;
  const auto enc = tmap_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(op.spec) & 15)) return DOE_ERR_UNSUPPORTED;
  // the spectrum plane as a 2-D float tensor: 2 nx floats per row, ny rows
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)2 * op.nx, (cuuint64_t)op.ny};
  const cuuint64_t strides[1] = {(cuuint64_t)op.nx * sizeof(float2)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * S::C), (cuuint32_t)(S::N < 256 ? S::N : 256)}, es[2] = {1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2*>(op.spec), dims, strides, box, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return DOE_ERR_UNSUPPORTED;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  DOE_TRY(prepare_kernel(c, sweep_col_tma_kernel<S>, smem, attr_set, false));
  if (nplanes <= 0) return DOE_OK;
  if (nplanes > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "column pass: at most 65535 planes per launch");
  int* err;
  DOE_TRY(design_error_word(c, &err));
  dim3 grid(ncols / S::C, nplanes);
  LaunchScope ls(c, ColSweepBase::kName);
  sweep_col_tma_kernel<S><<<grid, S::THREADS, smem, c->stream>>>(map, op, c->tw + S::N, ncols, err);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

// Spectrum tile resident across planes: all planes of a field share one spectrum,
// so a CTA has the TMA copy its C-column tile into shared memory once (32 KB at
// 1024 x 4) and then runs K planes over it -- x H of plane k, inverse column FFT,
// store -- reading the spectrum from shared memory each time. The spectrum then
// crosses L2 once per K planes instead of once per plane, and no plane's transform
// waits on global loads of it. Same bounded wait as the TMA-staged form.
template <class S>
constexpr int sweep_res_smem() {
  return 128 + S::N * S::C * (int)sizeof(float2) + S::SMEM + 16;
}

template <class S>
__global__ void __launch_bounds__(S::THREADS, S::MINB)
    sweep_col_res_kernel(const __grid_constant__ CUtensorMap spec_map, ColSweepBase op,
                         const float2* __restrict__ tw, int ncols, int nplanes, int K, int* __restrict__ err) {
  using P = typename S::Plan;
  constexpr int C = S::C, RMAX = P::RMAX, N = P::N, BOX = N < 256 ? N : 256;
  extern __shared__ unsigned char smraw[];
  float2* tile = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
  float2* scratch = tile + N * C;
  uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(scratch) + S::SMEM);
  const int c = threadIdx.x % C;
  const int t = threadIdx.x / C;
  const int x0 = blockIdx.x * C;
  const int line = x0 + c;
  const bool active = line < ncols;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
                 "r"((uint32_t)(N * C * sizeof(float2)))
                 : "memory");
#pragma unroll 1
    for (int r0 = 0; r0 < N; r0 += BOX)
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
              tc::smem_u32(tile + r0 * C)),
          "l"(reinterpret_cast<uint64_t>(&spec_map)), "r"(2 * x0), "r"(r0), "r"(tc::smem_u32(bar))
          : "memory");
  }
  __syncthreads();
  bool ok = tc::mbar_wait_bounded(bar, 0, 1000000000ull);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) {
      atomicExch(err, 4);
      (void)tc::mbar_wait_bounded(bar, 0, 1000000000ull);
    }
    __syncthreads();
    return;
  }
  SmemVec<P::PSHIFT> s{scratch, C, c};
  const int p0 = blockIdx.y * K;
#pragma unroll 1
  for (int k = 0; k < K && p0 + k < nplanes; ++k) {
    const auto st = op.init(p0 + k, active ? line : 0);
    float2 v[RMAX];
#pragma unroll
    for (int q = 0; q < RMAX; ++q) {
      const int ky = in_elem<P>(t, q);
      v[q] = cmul(tile[ky * C + c], asm_h_col(st.h, op.tab, ky));
    }
    fft_run<P, true>(v, t, s, tw, BlockSync{});
    if (active) {
#pragma unroll
      for (int q = 0; q < RMAX; ++q) st.out[(long)out_elem<P>(t, q) * op.nx] = v[q];
    }
    __syncthreads();  // the scratch is reused by the next plane
  }
}

template <class S>
inline int launch_sweep_res(doe_ctx* c, const ColSweepBase& op, int nplanes, int ncols, int K) {
  constexpr int smem = sweep_res_smem<S>();
  if (smem > 200 * 1024 || (ncols % S::C) || (S::C * 8) % 16 || K < 1) return DOE_ERR_UNSUPPORTED;
  const auto enc = tmap_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(op.spec) & 15)) return DOE_ERR_UNSUPPORTED;
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)2 * op.nx, (cuuint64_t)op.ny};
  const cuuint64_t strides[1] = {(cuuint64_t)op.nx * sizeof(float2)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * S::C), (cuuint32_t)(S::N < 256 ? S::N : 256)}, es[2] = {1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2*>(op.spec), dims, strides, box, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return DOE_ERR_UNSUPPORTED;
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  DOE_TRY(prepare_kernel(c, sweep_col_res_kernel<S>, smem, attr_set, false));
  if (nplanes <= 0) return DOE_OK;
  const int gy = (nplanes + K - 1) / K;
  if (gy > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "column pass: too many plane groups per launch");
  int* err;
  DOE_TRY(design_error_word(c, &err));
  LaunchScope ls(c, ColSweepBase::kName);
  sweep_col_res_kernel<S><<<dim3(ncols / S::C, gy), S::THREADS, smem, c->stream>>>(map, op, c->tw + S::N, ncols,
                                                                                     nplanes, K, err);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

// The mirrored-row forms where they fit one SM's shared memory with room to spare
// (lengths 16..4096): 2 with per-element spectrum reads, 3 with the TMA-staged
// tile; else, and when a form does not apply, the plain per-element form.
template <class S>
inline int launch_sweep_col(doe_ctx* c, const ColSweepBase& op, int nplanes, int ncols, int form) {
  if constexpr (S::N >= 16 && S::N <= 4096 && sweep_res_smem<S>() <= 200 * 1024) {
    if (c->tune_sweep_res > 1) {
      const int rc = launch_sweep_res<S>(c, op, nplanes, ncols, c->tune_sweep_res);
      if (rc != DOE_ERR_UNSUPPORTED) return rc;
    }
  }
  if constexpr (S::N >= 16 && S::N <= 4096 && sweep_tma_smem<S>() <= 200 * 1024) {
    if (form == 3) {
      const int rc = launch_sweep_tma<S>(c, op, nplanes, ncols);
      if (rc != DOE_ERR_UNSUPPORTED) return rc;
      form = 2;
    }
    if (form == 2) return launch_sweep_sym<S>(c, op, nplanes, ncols);
  }
  if (form == 1) return launch_col<S>(c, ColSweepFused{op}, nplanes, ncols);
  return launch_col<S>(c, ColSweep{op}, nplanes, ncols);
}

}  // namespace doe
