// engine.cuh -- context, scratch memory, size dispatch and launch helpers shared
// by the propagation and design translation units.
#pragma once
#include <cuda_runtime.h>

#include <cudaTypedefs.h>

#include <atomic>
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
  kSlotTc,       // tensor-core FFT tables and error flag
  kSlotTcMax,    // per-field spectrum maxima (tensor-core input scale)
  kSlotErr,      // error word of the cluster-resident design loop
  kSlotCount
};

}  // namespace doe

struct doe_prof_rec {
  const char* name;
  cudaEvent_t a, b;
};

namespace doe {
struct CopyPool;
}

struct doe_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t aux = nullptr;          // second stream for pipelined passes
  std::vector<cudaEvent_t> sync_ev;    // events ordering the two streams
  long tune_sweep_group = 0;           // planes per sweep launch pair (0 = from L2 size)
  int tune_sweep_graph = 1;            // replay repeated device sweeps from a captured CUDA graph
  cudaGraphExec_t sweep_exec = nullptr;  // graph of the last repeated device sweep
  unsigned long long sweep_key = 0, sweep_pending = 0, sweep_launches = 0;
  int tune_sweep_fused = 0;            // 1: sweep column pass reads and multiplies per element
  int tune_sweep_hsym = 0;             // 1: sweep column pass shares H between mirrored rows
  int tune_sweep_res = 1;              // > 1: planes per CTA over a spectrum tile staged once by TMA
  int tune_sweep_tc = 1;               // 1: 1024^2 sweeps run the tcgen05 tensor-core passes
  unsigned tune_design_cluster = 0;    // bit log2(n): square n^2 image-plane WGS runs cluster-resident
  int tune_surrogate_tc = 2;           // surrogate convolutions with cin % 64 == 0: 0 mma.sync, 1 tcgen05
                                       // with cp.async operands, 2 / 3 tcgen05 with TMA operands (4 / 3 stages)
  void* tc_tables = nullptr;           // tensor-core tables built in this slot allocation
  int num_sms = 0;
  unsigned long long slot_gen = 0;     // bumped whenever a scratch slot is reallocated
  unsigned char tune_row[4][16] = {};  // chosen row-shape variant per [kind][log2 N]
  unsigned char tune_col[4][16] = {};  // chosen column-shape variant per [kind][log2 N]
  std::string err;
  unsigned long long launches = 0;     // kernels launched by this context
  int prof_on = 0;                     // time every launch with CUDA events
  std::vector<doe_prof_rec> prof;      // pending event pairs
  std::vector<cudaEvent_t> ev_pool;    // recycled events
  float2* tw = nullptr;  // twiddle tables: table for length N starts at tw + N
  void* slot[doe::kSlotCount] = {};
  size_t slot_bytes[doe::kSlotCount] = {};
  void* pinned = nullptr;  // host staging for parameter uploads
  size_t pinned_bytes = 0;
  // staging of pageable caller planes (host_copy.cu): two pinned chunks, the
  // events of their last DMA, the host threads that fill and drain them
  void* stage[2] = {nullptr, nullptr};
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  doe::CopyPool* copy_pool = nullptr;
  int host_copy_threads = 1;  // set from the host's threads at creation; 0: straight through the driver
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

// Reads and clears the device error flag of the tensor-core passes (prop_sweep.cu);
// the context's streams must be synchronised.
int tc_check(doe_ctx* c);

// Error word of the cluster-resident design loop (design_cluster.cu): a kernel whose
// bounded cluster-barrier wait ran out stores a nonzero code there. design_error_word
// gives its address (allocated and zeroed on first use, outside any capture);
// design_error_check reads and clears it once the context's streams are synchronised.
int design_error_word(doe_ctx* c, int** out);
int design_error_check(doe_ctx* c);

// cuTensorMapEncodeTiled (the TMA descriptor encoder), fetched once through the
// runtime's driver entry point so that the library needs no link to libcuda;
// null when the driver does not provide it.
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder();

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
    ++c->slot_gen;  // every captured graph that baked the old address is now stale
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

// Host <-> device copies of caller planes: pageable planes of 1 MB or more are
// staged through pinned chunks by host threads (host_copy.cu). Uploads are
// stream-ordered; downloads have completed when the call returns.
int host_upload(doe_ctx* c, void* d, const void* h, size_t bytes);
int host_download(doe_ctx* c, void* h, const void* d, size_t bytes);
void destroy_copy_pool(CopyPool* p);

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

// Kernel label used by the launch profiler: Op::kName when present.
template <class Op, class = void>
struct OpName {
  static const char* get() { return "kernel"; }
};
template <class Op>
struct OpName<Op, std::void_t<decltype(Op::kName)>> {
  static const char* get() { return Op::kName; }
};

inline cudaEvent_t prof_event(doe_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Bracket a launch with events when profiling is on; count every launch.
struct LaunchScope {
  doe_ctx* c;
  const char* name;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  LaunchScope(doe_ctx* c_, const char* n, cudaStream_t s = nullptr) : c(c_), name(n), st(s ? s : c_->stream) {
    ++c->launches;
    if (c->prof_on) {
      a = prof_event(c);
      cudaEventRecord(a, st);
    }
  }
  ~LaunchScope() {
    if (a) {
      cudaEvent_t b = prof_event(c);
      cudaEventRecord(b, st);
      c->prof.push_back({name, a, b});
    }
  }
};

// Tuning kinds: each family of fused operators keeps its own shape choice.
enum TuneKind { kTuneFft = 0, kTuneSweep = 1, kTuneDesign = 2, kTuneKinds = 4 };

inline int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

// The kernel a row / column shape launches (register-capped when MINB > 1).
template <class S, class Op>
inline auto row_kernel_of() {
  if constexpr (S::MINB > 1) return row_kernel_capped<S, Op>;
  else return row_kernel<S, Op>;
}
template <class S, class Op>
inline auto col_kernel_of() {
  if constexpr (S::MINB > 1) return col_kernel_capped<S, Op>;
  else return col_kernel<S, Op>;
}

// One-time per-device preparation of a pass kernel: the dynamic shared-memory
// opt-in above 48 KB. With `load` it also queries the kernel's attributes, which
// makes a lazily loading CUDA runtime load the kernel now rather than at its
// first launch.
template <class K>
inline int prepare_kernel(doe_ctx* c, K kern, int smem, std::atomic<unsigned long long>& done, bool load) {
  const unsigned long long bit = 1ull << (c->device & 63);
  if (smem > 48 * 1024 && !(done.load() & bit)) {
    DOE_CUDA(c, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    done.fetch_or(bit);
  }
  if (load) {
    cudaFuncAttributes fa;
    DOE_CUDA(c, cudaFuncGetAttributes(&fa, kern));
  }
  return DOE_OK;
}
template <class S, class Op>
inline int prepare_row(doe_ctx* c, bool load) {
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  return prepare_kernel(c, row_kernel_of<S, Op>(), S::SMEM, attr_set, load);
}
template <class S, class Op>
inline int prepare_col(doe_ctx* c, bool load) {
  static std::atomic<unsigned long long> attr_set{0};  // one bit per device
  return prepare_kernel(c, col_kernel_of<S, Op>(), S::SMEM, attr_set, load);
}

template <class S, class Op>
inline int launch_row(doe_ctx* c, const Op& op, int nplanes, int nlines, cudaStream_t stream = nullptr) {
  DOE_TRY((prepare_row<S, Op>(c, false)));
  const long bpp = (nlines + S::V - 1) / S::V;
  const long grid = bpp * (long)nplanes;
  if (grid <= 0) return DOE_OK;
  if (grid > 0x7fffffffL) return set_err(c, DOE_ERR_UNSUPPORTED, "row pass grid too large");
  cudaStream_t st = stream ? stream : c->stream;
  LaunchScope ls(c, OpName<Op>::get(), st);
  row_kernel_of<S, Op>()<<<(unsigned)grid, S::THREADS, S::SMEM, st>>>(op, c->tw + S::N, nlines);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

template <class S, class Op>
inline int launch_col(doe_ctx* c, const Op& op, int nplanes, int ncols, cudaStream_t stream = nullptr) {
  DOE_TRY((prepare_col<S, Op>(c, false)));
  if (nplanes <= 0) return DOE_OK;
  if (nplanes > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "column pass: at most 65535 planes per launch");
  dim3 grid((ncols + S::C - 1) / S::C, nplanes);
  cudaStream_t st = stream ? stream : c->stream;
  LaunchScope ls(c, OpName<Op>::get(), st);
  col_kernel_of<S, Op>()<<<grid, S::THREADS, S::SMEM, st>>>(op, c->tw + S::N, ncols);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

// Pick element I of a shape list by runtime index (index 0 when out of range).
template <class L, int I = 0, class F>
inline int select_shape(int idx, F& f) {
  if constexpr (I < (int)std::tuple_size<L>::value) {
    if (idx == I) return f(std::tuple_element_t<I, L>{});
    return select_shape<L, I + 1>(idx, f);
  } else {
    return f(std::tuple_element_t<0, L>{});
  }
}

// f(Shape{}) with the row shape the context selected for length n and `kind`.
template <class F>
inline int with_row(doe_ctx* c, int n, int kind, F&& f) {
  return with_n(n, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return select_shape<typename RowVariants<N>::list>(c->tune_row[kind][ilog2i(N)], f);
  });
}
template <class F>
inline int with_col(doe_ctx* c, int n, int kind, F&& f) {
  return with_n(n, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return select_shape<typename ColVariants<N>::list>(c->tune_col[kind][ilog2i(N)], f);
  });
}
// Default shapes only (operators that are not tuned).
template <class F>
inline int with_row0(int n, F&& f) {
  return with_n(n, [&](auto NC) { return f(typename DefRow<decltype(NC)::value>::type{}); });
}
template <class F>
inline int with_col0(int n, F&& f) {
  return with_n(n, [&](auto NC) { return f(typename DefCol<decltype(NC)::value>::type{}); });
}

// Number of variants for length n (for the autotuner).
inline int row_variant_count(int n) {
  return with_n(n, [&](auto NC) { return (int)std::tuple_size<typename RowVariants<decltype(NC)::value>::list>::value; });
}
inline int col_variant_count(int n) {
  return with_n(n, [&](auto NC) { return (int)std::tuple_size<typename ColVariants<decltype(NC)::value>::list>::value; });
}

// Event k of the context's ordering pool (grown on demand).
inline cudaEvent_t sync_event(doe_ctx* c, size_t k) {
  while (c->sync_ev.size() <= k) {
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    c->sync_ev.push_back(e);
  }
  return c->sync_ev[k];
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
