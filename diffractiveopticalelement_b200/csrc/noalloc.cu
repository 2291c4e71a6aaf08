// noalloc.cu -- angular-spectrum propagation of one device-resident complex64
// plane that performs no device memory allocation.
//
// Who needs this: code that runs where cudaMalloc is not an option -- a caller
// inside a memory-pool-managed runtime that forbids foreign allocations, a
// real-time loop that must not hit the allocator's implicit synchronisation, or a
// plugin host that hands out device buffers but not the right to allocate more.
// Such a caller owns the input and output planes; everything else this routine
// needs (FFT twiddle tables, the per-plane transfer-function tables and one
// complex64 work plane) lives in the fixed array below, which the CUDA module
// reserves on every device that loads this library, for the life of the process.
//
// Limits and sharing: at most kMaxPixels samples per plane (512 x 512, or any
// power-of-two nx-by-ny with nx*ny <= 262144 and each axis <= 8192). Every call
// uses the same array, so two calls whose work overlaps on the GPU (different
// streams, or different host threads on one device) race and corrupt each other;
// serialise them. The array keeps the previous call's contents; nothing in this
// path reads scratch it has not written first in the same call.
//
// Set-up: the first call on a device resolves the array's device address with
// cudaGetSymbolAddress (the host-side name of a __device__ array is only a
// stand-in, not a device pointer), fills the twiddle tables, synchronising the
// caller's stream once, and loads every kernel this path can launch (for every
// grid it accepts), so that a lazily loading CUDA runtime does its module loading
// then and not inside a later call. Make that first call before any stream
// capture. A CUDA error already pending when a call starts is reported as such
// and left pending for its owner.
#include <mutex>

#include "ops_propagate.cuh"

namespace {

using namespace doe;

constexpr long kMaxPixels = 1L << 18;
constexpr size_t kAlign = 256;
constexpr size_t round_up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
// twiddles: table for length N at element N, N <= kMaxN (same layout as a context's)
constexpr size_t kTwBytes = round_up(2 * (size_t)kMaxN * sizeof(float2));
// transfer-function tables of one plane with axes up to kMaxN (asm_tables_carve layout)
constexpr size_t kTabBytes =
    round_up(kAlign + 2 * (size_t)kMaxN * (sizeof(double) + sizeof(AxisBin) + sizeof(float)) + kAlign);
constexpr size_t kWorkBytes = round_up((size_t)kMaxPixels * sizeof(float2));
constexpr size_t kScratchBytes = kTwBytes + kTabBytes + kWorkBytes;  // ~2.6 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_dev[64] = {};  // device address of g_noalloc_scratch, per device

// e^{-2 pi i m / N} for every N <= kMaxN at index N + m; index 0 unused.
__global__ void noalloc_twiddles_kernel(float2* tw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * kMaxN; i += gridDim.x * blockDim.x) {
    if (i == 0) {
      tw[0] = make_float2(1.f, 0.f);
      continue;
    }
    int N = 1;
    while (2 * N <= i) N *= 2;
    const int m = i - N;
    double s, c;
    sincospi(-2.0 * (double)m / (double)N, &s, &c);
    tw[i] = make_float2((float)c, (float)s);
  }
}

int fail(char* err, int err_len, int code, const std::string& msg) {
  if (err && err_len > 0) snprintf(err, (size_t)err_len, "%s", msg.c_str());
  return code;
}

// Device address of the scratch array on the current device (set-up on first use).
int scratch_for_current_device(cudaStream_t stream, unsigned char** out, std::string* msg) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    *msg = "doe_asm_c64_noalloc: no usable current CUDA device";
    return DOE_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      *msg = std::string("doe_asm_c64_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return DOE_ERR_CUDA;
    }
    noalloc_twiddles_kernel<<<64, 256, 0, stream>>>((float2*)p);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      *msg = std::string("doe_asm_c64_noalloc: twiddle set-up failed: ") + cudaGetErrorString(e);
      return DOE_ERR_CUDA;
    }
    // load (and opt in to large shared memory) every pass kernel of every axis length
    doe_ctx lc;
    lc.device = dev;
    cudaFuncAttributes fa;
    int rc = cudaFuncGetAttributes(&fa, asm_tables_kernel) == cudaSuccess ? DOE_OK : DOE_ERR_CUDA;
    for (int n = 1; n <= kMaxN && !rc; n <<= 1) {
      rc = with_row0(n, [&](auto S) {
        DOE_TRY((prepare_row<decltype(S), RowC64<false>>(&lc, true)));
        return prepare_row<decltype(S), RowC64<true>>(&lc, true);
      });
      if (!rc) rc = with_col0(n, [&](auto S) { return prepare_col<decltype(S), ColAsm>(&lc, true); });
    }
    if (rc) {
      *msg = "doe_asm_c64_noalloc: kernel set-up failed: " + (lc.err.empty() ? std::string("cudaFuncGetAttributes")
                                                                          : lc.err);
      return DOE_ERR_CUDA;
    }
    g_scratch_dev[dev] = (unsigned char*)p;
  }
  *out = g_scratch_dev[dev];
  return DOE_OK;
}

}  // namespace

extern "C" int doe_asm_c64_noalloc(const void* d_in, void* d_out, int nx, int ny, double dx, double dy,
                                   double lambda, double z, int band_limit, int evanescent, double soft_edge,
                                   void* stream_handle, char* err, int err_len) {
  if (err && err_len > 0) err[0] = '\0';
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return fail(err, err_len, DOE_ERR_CUDA,
                std::string("doe_asm_c64_noalloc: a CUDA error was pending before this call: ") +
                    cudaGetErrorString(pending));
  if (!d_in || !d_out) return fail(err, err_len, DOE_ERR_BAD_ARG, "doe_asm_c64_noalloc: null plane");
  if (!is_pow2(nx) || !is_pow2(ny))
    return fail(err, err_len, DOE_ERR_NOT_POW2,
                "doe_asm_c64_noalloc: grid must be power-of-two, got " + std::to_string(nx) + "x" + std::to_string(ny));
  if (nx > kMaxN || ny > kMaxN || (long)nx * ny > kMaxPixels)
    return fail(err, err_len, DOE_ERR_UNSUPPORTED,
                "doe_asm_c64_noalloc: " + std::to_string(nx) + "x" + std::to_string(ny) +
                    " exceeds the fixed scratch limit of " + std::to_string(kMaxPixels) +
                    " samples per plane (each axis <= " + std::to_string(kMaxN) + ")");
  cudaStream_t stream = (cudaStream_t)stream_handle;
  const long n = (long)nx * ny;
  if (z == 0) {  // src/propagate.js:113 leaves the field untouched
    if (d_in != d_out) {
      const cudaError_t e = cudaMemcpyAsync(d_out, d_in, n * sizeof(float2), cudaMemcpyDeviceToDevice, stream);
      if (e != cudaSuccess)
        return fail(err, err_len, DOE_ERR_CUDA, std::string("doe_asm_c64_noalloc: ") + cudaGetErrorString(e));
    }
    return DOE_OK;
  }
  unsigned char* scratch = nullptr;
  std::string msg;
  int rc = scratch_for_current_device(stream, &scratch, &msg);
  if (rc) return fail(err, err_len, rc, msg);
  float2* tw = (float2*)scratch;
  void* tab_base = scratch + kTwBytes;
  float2* work = (float2*)(scratch + kTwBytes + kTabBytes);

  // A stack context carrying the stream and twiddles for the shared launch helpers;
  // it owns no device memory.
  doe_ctx lc;
  cudaGetDevice(&lc.device);
  lc.stream = stream;
  lc.tw = tw;

  AsmGroupArgs a;
  memset(&a, 0, sizeof(a));
  a.nplanes = 1;
  a.nx = nx;
  a.ny = ny;
  a.dx = dx;
  a.dy = dy;
  a.band_limit = band_limit;
  a.evanescent = evanescent;
  a.soft_edge = soft_edge;
  a.lam[0] = lambda;
  a.z[0] = z;
  const AsmTables tab = asm_tables_carve(tab_base, 1, nx, ny);
  asm_tables_kernel<<<dim3((nx + ny + 255) / 256, 1), 256, 0, stream>>>(a, tab);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(err, err_len, DOE_ERR_CUDA, std::string("doe_asm_c64_noalloc: ") + cudaGetErrorString(e));

  const float2* in = (const float2*)d_in;
  float2* out = (float2*)d_out;
  rc = with_row0(nx, [&](auto S) {
    return launch_row<decltype(S)>(&lc, RowC64<false>{{}, in, work, nx, ny, n, n, 1.f}, 1, ny);
  });
  if (!rc) rc = with_col0(ny, [&](auto S) {
    return launch_col<decltype(S)>(&lc, ColAsm{{}, work, work, tab, nx, ny}, 1, nx);
  });
  if (!rc) rc = with_row0(nx, [&](auto S) {
    return launch_row<decltype(S)>(&lc, RowC64<true>{{}, work, out, nx, ny, n, n, 1.f / (float)n}, 1, ny);
  });
  if (rc) return fail(err, err_len, rc, lc.err.empty() ? "doe_asm_c64_noalloc: launch failed" : lc.err);
  return DOE_OK;
}
