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
  SmemVec s{smem, C, c};
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

// The symmetric form where it fits one SM's shared memory with room to spare
// (lengths 16..4096), else the plain per-element form.
template <class S>
inline int launch_sweep_col(doe_ctx* c, const ColSweepBase& op, int nplanes, int ncols, int form) {
  if constexpr (S::N >= 16 && S::N <= 4096 && sweep_sym_smem<S>() <= 200 * 1024) {
    if (form == 2) return launch_sweep_sym<S>(c, op, nplanes, ncols);
  }
  if (form == 1) return launch_col<S>(c, ColSweepFused{op}, nplanes, ncols);
  return launch_col<S>(c, ColSweep{op}, nplanes, ncols);
}

}  // namespace doe
