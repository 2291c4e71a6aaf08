// quantize.cu -- Floyd-Steinberg error-diffusion phase quantisation
// (reference: src/doe.js:185-226 errorDiffusionQuantize, used by designDOE's
// `levels` option at :878-884; wrapPhase is src/propagate.js:410-420).
//
// The scan is serpentine, so every pixel depends on the one before it in scan
// order and every row on the whole previous row: one element is inherently
// sequential. The device runs one element per thread (a batch in parallel) and
// keeps the dependency chain in registers: the error carried to the next pixel
// and the three next-row accumulators roll along the row, and each next-row value
// is written once when it is final. The inputs the chain will need (this row's
// pixels ahead, the next row's pixels two ahead) are read in chunks of kChunk
// scan positions, one chunk ahead of the chain, so that a step waits on
// arithmetic rather than on a global load. The final wrap of the output is a
// separate, fully parallel kernel. FP64 throughout, every product and sum rounded
// separately (no fused multiply-add) in the reference's order, so results are
// bitwise those of the FP64 restatement.
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.cuh"

namespace doe {
namespace {

__device__ __forceinline__ double wrap_pi(double p) {
  // (-pi, pi] as src/propagate.js:410-420: fmod, then one correction
  const double two_pi = 6.283185307179586;  // 2 * Math.PI
  const double pi = 3.141592653589793;      // Math.PI
  p = fmod(p, two_pi);
  if (p > pi) p = __dsub_rn(p, two_pi);
  else if (p <= -pi) p = __dadd_rn(p, two_pi);
  return p;
}

// JavaScript Math.round: nearest integer, ties toward +infinity
__device__ __forceinline__ double js_round(double x) {
  const double f = floor(x);
  return (__dsub_rn(x, f) >= 0.5) ? f + 1.0 : f;
}

constexpr int kChunk = 8;

// Reads of one chunk: this row's pixel at scan position s + 1 (the next carry's
// input) and the next row's at s + 2 (the below-ahead accumulator's start), for
// s = s0 .. s0 + kChunk - 1; positions past the row read as 0. Neither is written
// before the chain consumes it: this row is final, and the next row is written
// only behind the scan position.
struct Chunk {
  double r[kChunk], d[kChunk];
};
__device__ __forceinline__ void load_chunk(Chunk& c, const double* row, const double* nxt, bool below, int s0, int nx,
                                           int i0, int di) {
#pragma unroll
  for (int k = 0; k < kChunk; ++k) {
    const int s = s0 + k;
    c.r[k] = (s + 1 < nx) ? row[i0 + (s + 1) * di] : 0.0;
    c.d[k] = (below && s + 2 < nx) ? nxt[i0 + (s + 2) * di] : 0.0;
  }
}

// buf: [B][n] working copy (the wrapped input), out: [B][n] (unwrapped levels)
__global__ void error_diffusion_kernel(double* buf, double* out, int B, int nx, int ny, int levels, int snake) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const long n = (long)nx * ny;
  double* u = buf + b * n;
  double* o = out + b * n;
  const double two_pi = 6.283185307179586, pi = 3.141592653589793;
  const double step = two_pi / levels;
  const double w7 = 7.0 / 16, w3 = 3.0 / 16, w5 = 5.0 / 16, w1 = 1.0 / 16;
  for (int j = 0; j < ny; ++j) {
    const bool ltr = snake ? (j % 2 == 0) : true;
    const int di = ltr ? 1 : -1;
    const int i0 = ltr ? 0 : nx - 1;
    const bool below = j + 1 < ny;
    const double* row = u + (long)j * nx;
    double* nxt = u + (long)(j + 1) * nx;
    // next-row accumulators for scan positions s-1, s, s+1 (in scan direction)
    double am1 = 0, a0 = 0, ap1 = 0;
    if (below) {
      a0 = nxt[i0];
      ap1 = (nx > 1) ? nxt[i0 + di] : 0.0;
    }
    double carry_v = row[i0];
    Chunk cur, ahead{};
    load_chunk(cur, row, nxt, below, 0, nx, i0, di);
#pragma unroll 1
    for (int s0 = 0; s0 < nx; s0 += kChunk) {
      if (s0 + kChunk < nx) load_chunk(ahead, row, nxt, below, s0 + kChunk, nx, i0, di);
#pragma unroll
      for (int k = 0; k < kChunk; ++k) {
        const int s = s0 + k;
        if (s < nx) {
          const int i = i0 + s * di;
          const double v = carry_v;
          const double q = __dmul_rn(js_round(v / step), step);
          o[(long)j * nx + i] = q;
          double e = __dsub_rn(v, q);
          if (e > pi) e = __dsub_rn(e, two_pi);
          else if (e <= -pi) e = __dadd_rn(e, two_pi);
          // right neighbour in the same row (7/16)
          if (s + 1 < nx) carry_v = __dadd_rn(cur.r[k], __dmul_rn(e, w7));
          if (below) {
            // below-behind (3/16), below (5/16), below-ahead (1/16), in the reference's order
            if (s > 0) am1 = __dadd_rn(am1, __dmul_rn(e, w3));
            a0 = __dadd_rn(a0, __dmul_rn(e, w5));
            if (s + 1 < nx) ap1 = __dadd_rn(ap1, __dmul_rn(e, w1));
            if (s > 0) nxt[i - di] = am1;  // scan position s-1 of the next row is final
            am1 = a0;
            a0 = ap1;
            ap1 = cur.d[k];
          }
        }
      }
      cur = ahead;
    }
    if (below) nxt[i0 + (nx - 1) * di] = am1;
  }
}

__global__ void wrap_kernel(double* p, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    p[i] = wrap_pi(p[i]);
}

}  // namespace
}  // namespace doe

using namespace doe;

// errorDiffusionQuantize of `batch` phase planes of n samples each (host FP64
// arrays, [batch][n]); the grid is inferred as the reference does (square:
// nx = round(sqrt(n))). snake / wrap_first as the reference's options.
extern "C" int doe_error_diffusion(doe_ctx* c, int batch, long long n, int levels, int snake, int wrap_first,
                                   const double* phase, double* out) {
  if (!c) return DOE_ERR_BAD_ARG;
  if (!phase || !out || batch < 1 || n < 1 || levels < 1)
    return set_err(c, DOE_ERR_BAD_ARG, "errorDiffusionQuantize: bad argument");
  const long nx = std::lround(std::sqrt((double)n));
  const long ny = nx > 0 ? n / nx : 0;
  if (nx * ny != n) return set_err(c, DOE_ERR_BAD_ARG, "errorDiffusionQuantize: expected a square grid");
  const size_t total = (size_t)batch * n;
  void* p;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * total * sizeof(double), &p));
  double* buf = (double*)p;
  double* o = buf + total;
  DOE_TRY(host_upload(c, buf, phase, total * sizeof(double)));
  if (wrap_first) {
    LaunchScope ls(c, "wrap_phase");
    wrap_kernel<<<(unsigned)std::min<size_t>((total + 255) / 256, 148 * 16), 256, 0, c->stream>>>(buf, (long)total);
    DOE_CUDA(c, cudaGetLastError());
  }
  {
    LaunchScope ls(c, "error_diffusion");
    // one chain per thread; 32-thread blocks spread the chains over the SMs
    error_diffusion_kernel<<<(batch + 31) / 32, 32, 0, c->stream>>>(buf, o, batch, (int)nx, (int)ny, levels,
                                                                  snake ? 1 : 0);
    DOE_CUDA(c, cudaGetLastError());
  }
  {
    LaunchScope ls(c, "wrap_phase");  // the output into (-pi, pi], every sample in parallel
    wrap_kernel<<<(unsigned)std::min<size_t>((total + 255) / 256, 148 * 16), 256, 0, c->stream>>>(o, (long)total);
    DOE_CUDA(c, cudaGetLastError());
  }
  DOE_TRY(host_download(c, out, o, total * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}
