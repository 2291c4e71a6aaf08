// engine.cuh -- context, scratch memory, size dispatch and launch helpers shared
// by the propagation and design translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/doe_b200.h"
#include "fft_kernels.cuh"

namespace doe {

constexpr int kMaxLog2 = 13;  // axes up to 8192
constexpr int kMaxN = 1 << kMaxLog2;

// Scratch slots owned by a context (grown on demand, never shrunk).
enum Slot {
  kSlotW0 = 0,   // complex64 work plane(s)
  kSlotW1,       // second complex64 work area
  kSlotIn,       // FP64 host-mirror planes (re|im)
  kSlotOut,      // FP64 output planes
  kSlotTab,      // per-plane angular-spectrum axis tables
  kSlotParams,   // per-plane parameters
  kSlotRed,      // reduction partials / counters / totals
  kSlotDesign0,  // design-loop state
  kSlotDesign1,
  kSlotDesign2,
  kSlotCount
};

}  // namespace doe

struct doe_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  float2* tw = nullptr;  // twiddle tables: table for length N starts at tw + N
  void* slot[doe::kSlotCount] = {};
  size_t slot_bytes[doe::kSlotCount] = {};
  void* pinned = nullptr;  // host staging for parameter uploads
  size_t pinned_bytes = 0;
};

namespace doe {

inline int set_err(doe_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define DOE_CUDA(ctx, call)                                                                    \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return ::doe::set_err((ctx), DOE_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

#define DOE_TRY(expr)      \
  do {                     \
    int rc_ = (expr);      \
    if (rc_) return rc_;   \
  } while (0)

inline bool is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

inline int check_grid(doe_ctx* c, int nx, int ny, const char* who) {
  if (!is_pow2(nx) || !is_pow2(ny))
    return set_err(c, DOE_ERR_NOT_POW2, "%s: grid must be power-of-two, got %dx%d", who, nx, ny);
  if (nx > kMaxN || ny > kMaxN)
    return set_err(c, DOE_ERR_UNSUPPORTED, "%s: axis length above %d is not supported, got %dx%d", who,
                   kMaxN, nx, ny);
  return DOE_OK;
}

// Ensure scratch slot s holds at least `bytes` bytes of device memory.
inline int ensure_slot(doe_ctx* c, int s, size_t bytes, void** out) {
  if (c->slot_bytes[s] < bytes) {
    if (c->slot[s]) cudaFree(c->slot[s]);
    c->slot[s] = nullptr;
    c->slot_bytes[s] = 0;
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&c->slot[s], want);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return set_err(c, DOE_ERR_CUDA, "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
    }
    c->slot_bytes[s] = want;
  }
  *out = c->slot[s];
  return DOE_OK;
}

inline int ensure_pinned(doe_ctx* c, size_t bytes, void** out) {
  if (c->pinned_bytes < bytes) {
    if (c->pinned) {
      cudaStreamSynchronize(c->stream);
      cudaFreeHost(c->pinned);
    }
    c->pinned = nullptr;
    c->pinned_bytes = 0;
    size_t want = bytes + bytes / 4 + 4096;
    DOE_CUDA(c, cudaMallocHost(&c->pinned, want));
    c->pinned_bytes = want;
  }
  *out = c->pinned;
  return DOE_OK;
}

// Run f(std::integral_constant<int, N>) for the power-of-two n in [1, kMaxN].
template <class F>
inline int with_n(int n, F&& f) {
  switch (n) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 16: return f(std::integral_constant<int, 16>{});
    case 32: return f(std::integral_constant<int, 32>{});
    case 64: return f(std::integral_constant<int, 64>{});
    case 128: return f(std::integral_constant<int, 128>{});
    case 256: return f(std::integral_constant<int, 256>{});
    case 512: return f(std::integral_constant<int, 512>{});
    case 1024: return f(std::integral_constant<int, 1024>{});
    case 2048: return f(std::integral_constant<int, 2048>{});
    case 4096: return f(std::integral_constant<int, 4096>{});
    case 8192: return f(std::integral_constant<int, 8192>{});
    default: return DOE_ERR_UNSUPPORTED;
  }
}

template <int N, class Op>
inline int launch_row(doe_ctx* c, const Op& op, int nplanes, int nlines) {
  using Cfg = RowCfg<N>;
  auto kern = row_kernel<N, Op>;
  static bool attr_set = false;
  if (!attr_set && Cfg::SMEM > 48 * 1024) {
    DOE_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    attr_set = true;
  }
  const long bpp = (nlines + Cfg::V - 1) / Cfg::V;
  const long grid = bpp * (long)nplanes;
  if (grid <= 0) return DOE_OK;
  if (grid > 0x7fffffffL) return set_err(c, DOE_ERR_UNSUPPORTED, "row pass grid too large");
  kern<<<(unsigned)grid, Cfg::THREADS, Cfg::SMEM, c->stream>>>(op, c->tw + N, nlines);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

template <int N, class Op>
inline int launch_col(doe_ctx* c, const Op& op, int nplanes, int ncols) {
  using Cfg = ColCfg<N>;
  auto kern = col_kernel<N, Op>;
  static bool attr_set = false;
  if (!attr_set && Cfg::SMEM > 48 * 1024) {
    DOE_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
    attr_set = true;
  }
  if (nplanes <= 0) return DOE_OK;
  if (nplanes > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "column pass: at most 65535 planes per launch");
  dim3 grid((ncols + Cfg::C - 1) / Cfg::C, nplanes);
  kern<<<grid, Cfg::THREADS, Cfg::SMEM, c->stream>>>(op, c->tw + N, ncols);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

// Blocks per plane of each pass (needed to size reduction partials).
template <int N>
inline int row_blocks_per_plane(int nlines) {
  return (nlines + RowCfg<N>::V - 1) / RowCfg<N>::V;
}
template <int N>
inline int col_blocks_per_plane(int ncols) {
  return (ncols + ColCfg<N>::C - 1) / ColCfg<N>::C;
}
inline int row_bpp(int n, int nlines) {
  int r = 0;
  with_n(n, [&](auto NC) { r = row_blocks_per_plane<decltype(NC)::value>(nlines); return 0; });
  return r;
}
inline int col_bpp(int n, int ncols) {
  int r = 0;
  with_n(n, [&](auto NC) { r = col_blocks_per_plane<decltype(NC)::value>(ncols); return 0; });
  return r;
}

// Centred index of FFT bin k (fftshift position) and its signed frequency index,
// exactly as the reference samples the centred grid: f = (i - n/2) * df.
inline int centred_index(int k, int n) { return (k + (n >> 1)) % n; }
inline double centred_freq_index(int k, int n) { return (double)centred_index(k, n) - n / 2.0; }

// ------------------------------------------------------------ plain-op helpers
struct NoReduce {
  using Acc = NoAcc;
  __device__ __forceinline__ void finish(int, int, int, Acc&) const {}
};

}  // namespace doe
