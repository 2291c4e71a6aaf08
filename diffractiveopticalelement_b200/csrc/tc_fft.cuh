// tc_fft.cuh -- 1024-point FFT passes of the focus sweep on the tcgen05 tensor
// cores (reference transform: src/fft.js:86-139; sweep: src/propagate.js:427-434).
//
// A 1024-point DFT is two radix-32 stages (n = n1 + 32 n2, k = k2 + 32 k1):
//   Y[n1][k2] = sum_n2 x[n1 + 32 n2] w32^(n2 k2)       stage 1 (32-point DFT)
//   Y'        = Y[n1][k2] w1024^(n1 k2)                  twiddle
//   X[k2 + 32 k1] = sum_n1 Y'[n1][k2] w32^(n1 k1)       stage 2 (32-point DFT)
// Each stage is one real GEMM per 128-row tile: a row holds the 32 complex inputs
// of one 32-point DFT as 64 interleaved (re, im) f16 values, and the B operand is
// the 64x64 real form of the 32-point DFT matrix. FP32-class accuracy comes from
// splitting both operands into f16 hi + lo parts: A = [A_hi | A_lo] along K and
// B = [F_hi ; F_lo] along N, so one accumulator tile of 128 rows x 128 FP32
// columns (in TMEM) holds A*F_hi in columns 0-63 and A*F_lo in 64-127; their sum
// is the product to ~2^-22 relative (all four hi/lo cross terms are included).
// The twiddles (FP32 rounded from FP64) are applied on the CUDA cores between
// the stages, with a power-of-two scale that keeps every f16 operand below 2^15:
// the field's spectrum maximum sets the input scale sigma (a power of two), so
// every scale is exact and is removed in the last store.
//
// A CTA (4 warps = the 4 TMEM lane quarters, one 128-row M tile) transforms a
// tile of 4 vectors: 8 MMAs (M128 N128 K16) per stage into 128 TMEM columns. Tiles
// are independent, so the 3-4 CTAs that fit on an SM overlap one another's tensor
// and CUDA-core phases. A CTA takes a contiguous range of tiles (a persistent
// grid), which keeps it on one plane for many tiles. Column tiles are 4 adjacent
// columns (32-byte row segments), row tiles 4 rows.
// Every wait on the tensor core is bounded; on a timeout the kernel records an
// error code, waits once more (bounded), releases its TMEM and returns.
#pragma once
#include "asm.cuh"
#include "tcgen05.cuh"

namespace doe {
namespace tcfft {

constexpr int kN = 1024;
constexpr int kThreads = 128;
constexpr int kVec = 4;                          // vectors per tile
constexpr int kTmemCols = 128;
constexpr int kOffF = 0;                         // [F_hi ; F_lo]: 128 rows x 128 B
constexpr int kOffAhi = 16384;                   // stage operand, hi part (16 KB)
constexpr int kOffAlo = 32768;                   // lo part (16 KB)
constexpr int kOffMisc = 49152;                  // mbarrier + TMEM address slot
constexpr int kOffYt = 49168;                    // column pass: the plane's y bins {cycles, u, w, 0} (16 KB)
constexpr int kSmemRow = kOffMisc + 16 + 1024;   // + alignment slack: 4 CTAs per SM
constexpr int kSmemCol = kOffYt + kN * 16 + 1024;  // 3 CTAs per SM
constexpr int kTwTables = 4;                     // inverse x 2^-10, inverse x 2^-5, forward x 2^-5, forward x 2^-10
constexpr size_t kTableBytes = 2 * 16384 + (size_t)kTwTables * kN * sizeof(float2);
constexpr uint64_t kWaitNs = 1000000000ull;      // 1 s bound on every tensor-core wait

// Builds the B tiles of both directions (dir 0 forward e^{-i}, 1 inverse e^{+i})
// in their swizzled shared-memory image, and the scaled twiddle tables
// tw[sel][k2 * 32 + n1] = w1024^(+-n1 k2) * scale, from FP64.
static __global__ void tc_tables_kernel(uint4* __restrict__ F, float2* __restrict__ tw) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 2 * 128 * 64) {
    const int dir = t >> 13, r = t & 8191, n = r >> 6, k = r & 63;
    const int p = n >> 6, k2 = (n & 63) >> 1, c = n & 1, n2 = k >> 1, cp = k & 1;
    const int e = (n2 * k2) & 31;
    double s, co;
    sincospi((dir ? 2.0 : -2.0) * (double)e / 32.0, &s, &co);
    const double v = c == 0 ? (cp == 0 ? co : -s) : (cp == 0 ? s : co);
    const __half hi = __double2half(v);
    const __half lo = __double2half(v - (double)__half2float(hi));
    unsigned char* base = reinterpret_cast<unsigned char*>(F + dir * 1024);
    *reinterpret_cast<__half*>(base + tc::sw128_off(n, k >> 3) + (k & 7) * 2) = p == 0 ? hi : lo;
  }
  if (t < kTwTables * kN) {
    const int sel = t / kN, j = t % kN;
    const int k2 = j >> 5, n1 = j & 31;
    const bool inv = sel < 2;
    const double scale = (sel == 0 || sel == 3) ? 1.0 / 1024.0 : 1.0 / 32.0;
    double s, co;
    sincospi((inv ? 2.0 : -2.0) * (double)(n1 * k2) / (double)kN, &s, &co);
    tw[sel * kN + j] = make_float2((float)(co * scale), (float)(s * scale));
  }
}

// Largest |re|, |im| of a plane, as FP32 bits (non-negative, so integer max works).
static __global__ void absmax_kernel(const float2* __restrict__ s, long n, unsigned* __restrict__ maxbits) {
  float m = 0.f;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float2 v = s[i];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(m));
}

// Power-of-two input scale: the largest component times sigma lies in [2^13, 2^14)
// (sigma = 2^14 for an all-zero or non-finite plane).
__device__ __forceinline__ float sigma_of(unsigned bits) {
  int e = (int)((bits >> 23) & 0xffu) - 126;  // bits' value < 2^e
  if (bits == 0u || ((bits >> 23) & 0xffu) == 0xffu) e = 0;
  e = max(-100, min(100, e));
  return __uint_as_float((unsigned)(14 - e + 127) << 23);
}

// ------------------------------------------------------------------ CTA machinery
struct Smem {
  unsigned char* base;
  uint32_t sbase;
  uint64_t* mbar;
  uint32_t* tslot;
};

__device__ __forceinline__ Smem smem_setup(unsigned char* raw) {
  Smem s;
  s.base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~(uintptr_t)1023);
  s.sbase = tc::smem_u32(s.base);
  s.mbar = reinterpret_cast<uint64_t*>(s.base + kOffMisc);
  s.tslot = reinterpret_cast<uint32_t*>(s.base + kOffMisc + 8);
  return s;
}

// Copy the B tile of direction `dir` into shared memory, initialise the mbarrier
// and allocate the accumulator columns.
__device__ __forceinline__ uint32_t cta_begin(const Smem& s, const uint4* __restrict__ F, int dir) {
  const int tid = threadIdx.x;
  const uint4* fsrc = F + dir * 1024;
  uint4* fdst = reinterpret_cast<uint4*>(s.base + kOffF);
#pragma unroll
  for (int i = 0; i < 1024 / kThreads; ++i) fdst[tid + i * kThreads] = __ldg(&fsrc[tid + i * kThreads]);
  tc::fence_proxy_async();
  if (tid == 0) {
    tc::mbar_init(s.mbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((tid >> 5) == 0) tc::tmem_alloc(s.tslot, kTmemCols);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  return *s.tslot;
}

__device__ __forceinline__ void cta_end(uint32_t tbase) {
  tc::fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) tc::tmem_dealloc(tbase, kTmemCols);
}

// The 8 MMAs of one stage: A_hi then A_lo against [F_hi ; F_lo].
__device__ __forceinline__ void issue_stage(uint32_t sbase, uint32_t tbase) {
  constexpr uint32_t idesc = tc::idesc_f16_f32(128, 128);
  const uint32_t f = sbase + kOffF, ahi = sbase + kOffAhi, alo = sbase + kOffAlo;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    tc::mma_f16_ss(tbase, tc::desc_k_sw128(ahi + 32 * k), tc::desc_k_sw128(f + 32 * k), idesc, k > 0 ? 1u : 0u);
#pragma unroll
  for (int k = 0; k < 4; ++k) tc::mma_f16_ss(tbase, tc::desc_k_sw128(alo + 32 * k), tc::desc_k_sw128(f + 32 * k), idesc, 1u);
}

// Hand the operand tile to the tensor core, run one stage and wait for it.
// Returns false (uniformly over the CTA) when the wait ran out.
__device__ __forceinline__ bool run_stage(const Smem& s, uint32_t tbase, uint32_t& phase) {
  tc::fence_proxy_async();
  tc::fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after();
    issue_stage(s.sbase, tbase);
    tc::commit(s.mbar);
  }
  const bool ok = tc::mbar_wait_bounded(s.mbar, phase, kWaitNs);
  const bool all_ok = __syncthreads_and(ok);
  if (!all_ok) {  // let anything still in flight finish before the TMEM is released
    (void)tc::mbar_wait_bounded(s.mbar, phase, kWaitNs);
    return false;
  }
  phase ^= 1u;
  tc::fence_after();
  return true;
}

__device__ __forceinline__ float2 cmul(float2 v, float2 w) {
  return make_float2(fmaf(v.x, w.x, -v.y * w.y), fmaf(v.x, w.y, v.y * w.x));
}

// Split 32 complex values (this thread's stage-1 row m: K positions 0..31) into
// f16 hi / lo and store them as the 8 swizzled 16-byte chunks of the row.
__device__ __forceinline__ void put_row(unsigned char* base, int m, const float2 (&v)[32]) {
  unsigned char* hi = base + kOffAhi + (m >> 3) * 1024 + (m & 7) * 128;
  unsigned char* lo = base + kOffAlo + (m >> 3) * 1024 + (m & 7) * 128;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) tc::split_f16x2(v[4 * j + q].x, v[4 * j + q].y, h[q], l[q]);
    const int off = (j ^ (m & 7)) << 4;
    *reinterpret_cast<uint4*>(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// Read 16 complex results (outputs 16h .. 16h+15) of this thread's TMEM lane:
// hi-part columns plus lo-part columns.
__device__ __forceinline__ void read16(uint32_t tbase, int h, float2 (&y)[16]) {
  const uint32_t lane = (uint32_t)((threadIdx.x >> 5) * 32) << 16;
  float a[32], b[32];
  tc::tmem_ld32x2(tbase + lane + (uint32_t)(h * 32), tbase + lane + (uint32_t)(64 + h * 32), a, b);
#pragma unroll
  for (int q = 0; q < 16; ++q) y[q] = make_float2(a[2 * q] + b[2 * q], a[2 * q + 1] + b[2 * q + 1]);
}

// Stage-1 results of this thread's row (index n1 of the first stage) times the
// twiddles tw[k2 * 32 + n1] (a warp reads 32 consecutive entries: one L1 line
// pair), split and stored at K position n1 of stage-2 rows row_of(k2). Stage-2
// row r lives at (r >> 3) * 1024 + (r & 7) * 128 + ((n1 / 4) ^ (r & 7)) * 16
// + (n1 % 4) * 4 in both parts.
template <class RowOf>
__device__ __forceinline__ void twiddle_scatter(const Smem& s, uint32_t tbase, const float2* __restrict__ twt, int n1,
                                                RowOf row_of) {
  const float2* tw = twt + n1;
  const int chunk = n1 >> 2, slot = (n1 & 3) * 4;
#pragma unroll
  for (int hh = 0; hh < 2; ++hh) {
    float2 y[16];
    read16(tbase, hh, y);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int k2 = 16 * hh + q;
      const float2 v = cmul(y[q], __ldg(&tw[k2 * 32]));
      uint32_t h, l;
      tc::split_f16x2(v.x, v.y, h, l);
      const int r = row_of(k2);
      const int off = (r >> 3) * 1024 + (r & 7) * 128 + ((chunk ^ (r & 7)) << 4) + slot;
      *reinterpret_cast<uint32_t*>(s.base + kOffAhi + off) = h;
      *reinterpret_cast<uint32_t*>(s.base + kOffAlo + off) = l;
    }
  }
}

// Contiguous share [t0, t1) of `ntiles` tiles for this CTA.
__device__ __forceinline__ void tile_range(int ntiles, int& t0, int& t1) {
  t0 = (int)(((long)ntiles * blockIdx.x) / gridDim.x);
  t1 = (int)(((long)ntiles * (blockIdx.x + 1)) / gridDim.x);
}

// ------------------------------------------------------------------ operators
// Column pass of the sweep: spectrum column x H (times sigma), inverse
// 1024-point column transform, into the intermediate plane (scaled by
// sigma * 2^-10, which the row pass removes). Tile = (plane, 4 columns).
struct ColSweepTc {
  const float2* spec;      // one spectrum plane (unshifted), 1024 x 1024
  float2* w;               // [planes][1024][1024]
  AsmTables tab;
  const unsigned* maxbits; // spectrum max (FP32 bits)
  int tp0;                 // table plane of the launch's first plane
  static constexpr int kDir = 1, kTw = 0;
};

// Row pass: inverse 1024-point row transform of the intermediate, times
// 2^-5 / sigma (which also applies 1/(nx ny)), to complex64 or FP64 planes.
struct RowOutTc {
  const float2* w;         // [planes][1024][1024]
  float2* out_c64;         // or null
  double* out_re;          // FP64 split output when out_c64 is null
  double* out_im;
  const unsigned* maxbits;
  long out_plane_stride;
  static constexpr int kDir = 1, kTw = 1;
};

// Transfer function of the sweep at one bin, from the per-axis phases in cycles:
// z sqrt(1/l^2 - f^2) = Z - (Z/2)(ux + uy) - q(u), with the first two terms
// reduced per axis in FP64 (cx, cy) and q = (Z/2) u^2 / (1 + sqrt(1 - u))^2. For
// u <= 0.0125 the last factor is its Taylor series 1/4 + u/8 + 5u^2/64 + 7u^3/128
// (relative truncation error <= 4e-9, i.e. <= 8e-9 cycles on the fast path where
// |q| <= 2 cycles); above that it is evaluated directly in FP32. Bins beyond the
// fast-path limit take the FP64 path of the CUDA-core passes (asm_h_slow).
__device__ __forceinline__ float2 sweep_h(float cx, float ux, float wx, float hz, float ucut, float4 yb,
                                          const AsmTables& tab, int p, int kx, int ky) {
  const float u = ux + yb.y;
  const float w = wx * yb.z;
  float poly = fmaf(u, fmaf(u, fmaf(u, 0.0546875f, 0.078125f), 0.125f), 0.25f);
  if (u > 0.0125f) {
    const float om = fmaxf(1.f - u, 1e-3f);
    const float sq = 1.f + om * rsqrtf(om);  // 1 + sqrt(1 - u)
    poly = __fdividef(1.f, sq * sq);
  }
  float ph = (cx + yb.x) - hz * (u * u) * poly;
  ph -= rintf(ph);
  float sn, cs;
  __sincosf(6.283185307179586f * ph, &sn, &cs);
  float2 h = make_float2(w * cs, w * sn);
  if (u > ucut && w != 0.f) h = asm_h_slow(tab.pl + p, tab.xf2 + kx, tab.yf2, ky, w);
  return h;
}

static __global__ void __launch_bounds__(kThreads, 3)
    tc_col_sweep_kernel(ColSweepTc op, const uint4* __restrict__ F, const float2* __restrict__ twg, int ntiles,
                        int* __restrict__ err) {
  extern __shared__ unsigned char smraw[];
  const Smem s = smem_setup(smraw);
  const uint32_t tbase = cta_begin(s, F, ColSweepTc::kDir);
  const float2* twt = twg + ColSweepTc::kTw * kN;
  const int m = threadIdx.x;
  const int c = m & 3;          // column within the tile
  const int n1 = m >> 2;        // stage-1 row (c, n1) = 4 n1 + c; stage-2 row (c, k2) = 4 k2 + c
  const float sigma = sigma_of(__ldg(op.maxbits));
  const float4* yt = reinterpret_cast<const float4*>(s.base + kOffYt);
  constexpr int tpp = kN / kVec;  // tiles per plane
  int t0, t1;
  tile_range(ntiles, t0, t1);
  int cur_plane = -1;
  uint32_t phase = 0;
  for (int tile = t0; tile < t1; ++tile) {
    const int p = tile / tpp;
    const int x = (tile % tpp) * kVec + c;
    const int tp = op.tp0 + p;
    if (p != cur_plane) {  // stage this plane's y bins: {cycles, u, w, 0}
      __syncthreads();     // nobody still reads the previous plane's bins
      float4* dst = reinterpret_cast<float4*>(s.base + kOffYt);
#pragma unroll
      for (int i = 0; i < kN / kThreads; ++i) {
        const int k = m + i * kThreads;
        const AxisBin b = op.tab.yt[(long)tp * kN + k];
        dst[k] = make_float4(__ldg(&op.tab.yc[(long)tp * kN + k]), b.u, b.w, 0.f);
      }
      cur_plane = p;
      __syncthreads();
    }
    const AxisBin bx = op.tab.xt[(long)tp * kN + x];
    const float cx = __ldg(&op.tab.xc[(long)tp * kN + x]);
    const float hz = op.tab.pl[tp].hz, ucut = op.tab.pl[tp].ucut;
    const float wx = bx.w * sigma;
    // stage 1 operand: inputs spec[n1 + 32 n2][x] * H
    {
      const float2* src = op.spec + (long)n1 * kN + x;
      float2 v[32];
#pragma unroll
      for (int n2 = 0; n2 < 32; ++n2) v[n2] = __ldg(&src[(long)n2 * 32 * kN]);
#pragma unroll
      for (int n2 = 0; n2 < 32; ++n2) {
        const int ky = n1 + 32 * n2;
        v[n2] = cmul(v[n2], sweep_h(cx, bx.u, wx, hz, ucut, yt[ky], op.tab, tp, x, ky));
      }
      put_row(s.base, m, v);
    }
    if (!run_stage(s, tbase, phase)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    twiddle_scatter(s, tbase, twt, n1, [c](int k2) { return 4 * k2 + c; });
    if (!run_stage(s, tbase, phase)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    // stage 2 results: row m = (c, k2 = m / 4) holds outputs y = k2 + 32 k1
    {
      float2* dst = op.w + (long)p * kN * kN + (long)n1 * kN + x;  // n1 == m / 4 == k2 here
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        float2 y[16];
        read16(tbase, hh, y);
#pragma unroll
        for (int q = 0; q < 16; ++q) dst[(long)(16 * hh + q) * 32 * kN] = y[q];
      }
    }
  }
  cta_end(tbase);
}

static __global__ void __launch_bounds__(kThreads, 4)
    tc_row_out_kernel(RowOutTc op, const uint4* __restrict__ F, const float2* __restrict__ twg, int ntiles,
                      int* __restrict__ err) {
  extern __shared__ unsigned char smraw[];
  const Smem s = smem_setup(smraw);
  const uint32_t tbase = cta_begin(s, F, RowOutTc::kDir);
  const float2* twt = twg + RowOutTc::kTw * kN;
  const int m = threadIdx.x;
  const int v = m >> 5, lane = m & 31;  // stage-1 row (v, n1 = lane); stage-2 row (v, k2 = lane)
  const float oscale = 1.f / (32.f * sigma_of(__ldg(op.maxbits)));
  constexpr int tpp = kN / kVec;
  int t0, t1;
  tile_range(ntiles, t0, t1);
  uint32_t phase = 0;
  for (int tile = t0; tile < t1; ++tile) {
    const int p = tile / tpp;
    const long row = (long)(tile % tpp) * kVec + v;
    {
      const float2* src = op.w + ((long)p * kN + row) * kN + lane;
      float2 x[32];
#pragma unroll
      for (int n2 = 0; n2 < 32; ++n2) x[n2] = src[32 * n2];
      put_row(s.base, m, x);
    }
    if (!run_stage(s, tbase, phase)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    twiddle_scatter(s, tbase, twt, lane, [v](int k2) { return 32 * v + k2; });
    if (!run_stage(s, tbase, phase)) {
      if (threadIdx.x == 0) atomicExch(err, 1);
      break;
    }
    const long o = (long)p * op.out_plane_stride + row * kN + lane;
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      float2 y[16];
      read16(tbase, hh, y);
      if (op.out_c64) {
#pragma unroll
        for (int q = 0; q < 16; ++q)
          op.out_c64[o + 32 * (16 * hh + q)] = make_float2(y[q].x * oscale, y[q].y * oscale);
      } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          op.out_re[o + 32 * (16 * hh + q)] = (double)(y[q].x * oscale);
          op.out_im[o + 32 * (16 * hh + q)] = (double)(y[q].y * oscale);
        }
      }
    }
  }
  cta_end(tbase);
}

}  // namespace tcfft
}  // namespace doe
