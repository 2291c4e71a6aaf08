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
// Data movement is laid out for shared-memory bandwidth, which the MMAs share
// with the CUDA cores (an M128 N128 K16 MMA with both operands in shared memory
// reads 128 B per cycle, the whole port): inputs go from global memory straight
// to registers; the stage-1 operand goes from registers to TMEM (tcgen05.st) and
// the MMA reads it there, so only the DFT matrix comes from shared memory; the
// stage-1 results come back from TMEM and are written once, transposed, as the
// MN-major stage-2 operand in shared memory (16-byte stores); the stage-2 results
// go from TMEM to global memory. The intermediate plane between the two passes is
// stored transposed, so both passes gather their inputs in 32-byte row segments
// and write their outputs in contiguous 256-byte runs.
//
// A CTA (8 warps: two per TMEM lane quarter, each taking half of every row)
// transforms a tile of 4 vectors: 8 MMAs (M128 N128 K16) per stage, accumulator
// in TMEM columns 0-127, stage-1 operand in columns 128-191; two CTAs per SM. A
// CTA takes a contiguous range of tiles (a persistent grid), which keeps it on
// one plane for many tiles. Every wait on the tensor core is bounded; on a
// timeout the kernel records an error code, waits once more (bounded), releases
// its TMEM and returns.
#pragma once
#include "asm.cuh"
#include "tcgen05.cuh"

namespace doe {
namespace tcfft {

constexpr int kN = 1024;
constexpr int kThreads = 256;
constexpr int kVec = 4;                          // vectors per tile
constexpr int kTmemCols = 256;                   // accumulator 0-127, stage-1 operand hi 128-159, lo 160-191
constexpr int kColAhi = 128, kColAlo = 160;
constexpr int kOffF = 0;                         // [F_hi ; F_lo]: 128 rows x 128 B, K-major
constexpr int kOffA2hi = 16384;                  // stage-2 operand, MN-major, hi part (16 KB)
constexpr int kOffA2lo = 32768;                  // lo part (16 KB)
constexpr int kOffStage = 49152;                 // the next tile's input, raw[e][vec] float2 (32 KB)
constexpr int kOffMisc = 81920;                  // mbarrier + TMEM address slot
constexpr int kOffYt = 81936;                    // column pass: the plane's y bins {cycles, u, w, 0} (16 KB)
// At most two CTAs fit on an SM (shared memory and registers), so the TMEM they
// allocate (2 x 256 columns) never exceeds the SM's 512 and no allocation waits.
constexpr int kSmemBytes = kOffYt + kN * 16 + 1024;
static_assert(3 * (kSmemBytes + 1024) > 228 * 1024, "three CTAs must not fit on an SM");
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
// and allocate the TMEM columns.
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

// Stage 1: A (hi, then lo) from TMEM against [F_hi ; F_lo]. Stage 2: A (hi, then
// lo) MN-major from shared memory (64-row M blocks 1024 B apart, 8-row K blocks
// 2048 B apart; one K step of 16 spans two K blocks).
__device__ __forceinline__ void issue_stage(uint32_t sbase, uint32_t tbase, int stage) {
  constexpr uint32_t idk = tc::idesc_f16_f32(128, 128);
  constexpr uint32_t idmn = idk | (1u << 15);
  const uint32_t f = sbase + kOffF;
  if (stage == 1) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      tc::mma_f16_ts(tbase, tbase + kColAhi + 8 * k, tc::desc_k_sw128(f + 32 * k), idk, k > 0 ? 1u : 0u);
#pragma unroll
    for (int k = 0; k < 4; ++k) tc::mma_f16_ts(tbase, tbase + kColAlo + 8 * k, tc::desc_k_sw128(f + 32 * k), idk, 1u);
  } else {
    const uint32_t ahi = sbase + kOffA2hi, alo = sbase + kOffA2lo;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      tc::mma_f16_ss(tbase, tc::desc_mn_sw128(ahi + 4096 * k, 1024, 2048), tc::desc_k_sw128(f + 32 * k), idmn,
                     k > 0 ? 1u : 0u);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      tc::mma_f16_ss(tbase, tc::desc_mn_sw128(alo + 4096 * k, 1024, 2048), tc::desc_k_sw128(f + 32 * k), idmn, 1u);
  }
}

// Hand the operands to the tensor core, run one stage and wait for it.
// Returns false (uniformly over the CTA) when the wait ran out.
__device__ __forceinline__ bool run_stage(const Smem& s, uint32_t tbase, uint32_t& phase, int stage) {
  tc::fence_proxy_async();
  tc::fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after();
    issue_stage(s.sbase, tbase, stage);
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

// Read 16 complex results (outputs 16h .. 16h+15) of this thread's TMEM lane:
// hi-part columns plus lo-part columns.
__device__ __forceinline__ void read16(uint32_t tbase, uint32_t lane_bits, int h, float2 (&y)[16]) {
  float a[32], b[32];
  tc::tmem_ld32x2(tbase + lane_bits + (uint32_t)(h * 32), tbase + lane_bits + (uint32_t)(64 + h * 32), a, b);
#pragma unroll
  for (int q = 0; q < 16; ++q) y[q] = make_float2(a[2 * q] + b[2 * q], a[2 * q + 1] + b[2 * q + 1]);
}

// 16-byte asynchronous global -> shared copies.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// A tile's input -- 1024 elements x 4 vectors, element e of vector vec at
// src[e * 1024 + vec] -- into the staging buffer as raw[e][vec]: 2048 16-byte
// chunks (8 per thread), 32-byte row segments in global memory.
__device__ __forceinline__ void stage_tile(unsigned char* base, const float2* __restrict__ src) {
  float2* raw = reinterpret_cast<float2*>(base + kOffStage);
#pragma unroll
  for (int i = 0; i < 2048 / kThreads; ++i) {
    const int q = threadIdx.x + i * kThreads;  // element q / 2, vectors 2 (q % 2) .. +1
    cp_async16(raw + 2 * q, src + (long)(q >> 1) * kN + 2 * (q & 1));
  }
  cp_async_commit();
}

// f16 hi / lo parts of (a, b), packed.
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) { tc::split_f16x2(a, b, hi, lo); }

// Contiguous share [t0, t1) of `ntiles` tiles for this CTA.
__device__ __forceinline__ void tile_range(int ntiles, int& t0, int& t1) {
  t0 = (int)(((long)ntiles * blockIdx.x) / gridDim.x);
  t1 = (int)(((long)ntiles * (blockIdx.x + 1)) / gridDim.x);
}

// ------------------------------------------------------------------ operators
// Column pass of the sweep: spectrum column x H (times sigma), inverse
// 1024-point column transform, into the intermediate plane stored transposed
// (wt[x][y]) and scaled by sigma * 2^-10, which the row pass removes.
struct ColSweepTc {
  const float2* spec;      // one spectrum plane (unshifted), 1024 x 1024
  float2* wt;              // [planes][1024 (x)][1024 (y)]
  AsmTables tab;
  const unsigned* maxbits; // spectrum max (FP32 bits)
  int tp0;                 // table plane of the launch's first plane
};

// Row pass: inverse 1024-point row transform of the (transposed) intermediate,
// times 2^-5 / sigma (which also applies 1/(nx ny)), to complex64 or FP64 planes.
struct RowOutTc {
  const float2* wt;        // [planes][1024 (x)][1024 (y)]
  float2* out_c64;         // or null
  double* out_re;          // FP64 split output when out_c64 is null
  double* out_im;
  const unsigned* maxbits;
  long out_plane_stride;
};

// Transfer function of the sweep at one bin, from the per-axis phases in cycles:
// z sqrt(1/l^2 - f^2) = Z - (Z/2)(ux + uy) - q(u), with the first two terms
// reduced per axis in FP64 (cx, cy) and q = (Z/2) u^2 / (1 + sqrt(1 - u))^2. For
// u <= 0.0125 the last factor is its Taylor series 1/4 + u/8 + 5u^2/64 + 7u^3/128
// (relative truncation error <= 4e-9, i.e. <= 8e-9 cycles on the fast path where
// |q| <= 2 cycles); above that it is evaluated directly in FP32. Bins beyond the
// fast-path limit take the FP64 path of the CUDA-core passes (asm_h_slow).
static __device__ __noinline__ float2 sweep_h_slow(const AsmPlane* pl, const double* xf2, const double* yf2, int ky,
                                                   float w) {
  return asm_h_slow(pl, xf2, yf2, ky, w);
}

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
  if (u > ucut && w != 0.f) h = sweep_h_slow(tab.pl + p, tab.xf2 + kx, tab.yf2, ky, w);
  return h;
}

// One kernel for both passes. A tile is 4 vectors (columns of the spectrum in the
// column pass, rows of the output in the row pass) whose element e sits at
// src[e * 1024 + vec]: the spectrum (column pass) or the transposed intermediate
// (row pass). Thread t: half h = t / 128 of row m = t % 128; stage-1 row
// m = 4 n1 + vec holds elements n1 + 32 n2 of vector vec (this thread: n2 in
// 16h .. 16h+15); stage-2 row m = 32 vec + k2 (TMEM lane quarter = vec).
template <bool COL, class Op>
__device__ __forceinline__ void sweep_pass(const Op& op, const uint4* __restrict__ F, const float2* __restrict__ twt,
                                           int ntiles, int* __restrict__ err) {
  extern __shared__ unsigned char smraw[];
  const Smem s = smem_setup(smraw);
  const uint32_t tbase = cta_begin(s, F, 1);
  const int t = threadIdx.x, h = t >> 7, m = t & 127;
  const int vec = m & 3, n1 = m >> 2;            // stage-1 row
  const int qv = m >> 5, lane = m & 31;          // stage-2 row: vector qv, k2 = lane
  const uint32_t lane_bits = (uint32_t)(qv * 32) << 16;
  const float sigma = sigma_of(__ldg(op.maxbits));
  // stage-2 operand (MN-major) address of this thread's values: K row 2 n1 + c in
  // K block n1 / 4, M = 32 vec + 16 h + 8 u + i in M block vec / 2
  const int kpar = (n1 >> 2) & 1;                // the component written first (spreads banks)
  const uint32_t a2base = (uint32_t)((n1 >> 2) * 2048 + (vec >> 1) * 1024);
  const int jb = (vec & 1) * 4 + 2 * h;
  const float4* yt = reinterpret_cast<const float4*>(s.base + kOffYt);
  constexpr int tpp = kN / kVec;
  int t0, t1;
  tile_range(ntiles, t0, t1);
  int cur_plane = -1;
  uint32_t phase = 0;
  // input of tile `tl`: element e of vector vec at src[e * 1024 + vec]
  auto tile_src = [&](int tl) -> const float2* {
    const int pl = tl / tpp, c0 = (tl % tpp) * kVec;
    if constexpr (COL) {
      return ((const ColSweepTc&)op).spec + c0;
    } else {
      return ((const RowOutTc&)op).wt + (long)pl * kN * kN + c0;
    }
  };
  if (t0 < t1) stage_tile(s.base, tile_src(t0));
  const float2* raw = reinterpret_cast<const float2*>(s.base + kOffStage);
  for (int tile = t0; tile < t1; ++tile) {
    const int p = tile / tpp;
    const int b0 = (tile % tpp) * kVec;          // first column (column pass) or row (row pass) of the tile
    // ---- stage 1 operand: 16 elements of this thread's row, through TMEM
    {
      cp_async_wait_all();
      __syncthreads();  // the tile's input is in the staging buffer
      float2 v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = raw[(n1 + 32 * (16 * h + i)) * kVec + vec];
      __syncthreads();  // every thread has its inputs: the buffer takes the next tile
      if (tile + 1 < t1) stage_tile(s.base, tile_src(tile + 1));
      if constexpr (COL) {
        const ColSweepTc& o = (const ColSweepTc&)op;
        const int tp = o.tp0 + p;
        if (p != cur_plane) {  // stage this plane's y bins: {cycles, u, w, 0}
          float4* dst = reinterpret_cast<float4*>(s.base + kOffYt);
#pragma unroll
          for (int i = 0; i < kN / kThreads; ++i) {
            const int k = t + i * kThreads;
            const AxisBin b = o.tab.yt[(long)tp * kN + k];
            dst[k] = make_float4(__ldg(&o.tab.yc[(long)tp * kN + k]), b.u, b.w, 0.f);
          }
          cur_plane = p;
          __syncthreads();
        }
        const int kx = b0 + vec;
        const AxisBin bx = o.tab.xt[(long)tp * kN + kx];
        const float cx = __ldg(&o.tab.xc[(long)tp * kN + kx]);
        const float hz = o.tab.pl[tp].hz, ucut = o.tab.pl[tp].ucut;
        const float wx = bx.w * sigma;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int ky = n1 + 32 * (16 * h + i);
          v[i] = cmul(v[i], sweep_h(cx, bx.u, wx, hz, ucut, yt[ky], o.tab, tp, kx, ky));
        }
      }
      uint32_t hi[16], lo[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) split2(v[i].x, v[i].y, hi[i], lo[i]);
      tc::tmem_st16(tbase + lane_bits + kColAhi + 16 * h, hi);
      tc::tmem_st16(tbase + lane_bits + kColAlo + 16 * h, lo);
      tc::tmem_wait_st();
    }
    if (!run_stage(s, tbase, phase, 1)) {
      if (t == 0) atomicExch(err, 1);
      break;
    }
    // ---- stage 1 results (k2 = 16h + i of row (vec, n1)) x twiddle -> stage-2 operand
    {
      float2 y[16];
      read16(tbase, lane_bits, h, y);
#pragma unroll
      for (int i = 0; i < 16; ++i) y[i] = cmul(y[i], __ldg(&twt[(16 * h + i) * 32 + n1]));
      uint32_t rh[8], rl[8], ih[8], il[8];  // pairs of consecutive k2, per component
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        split2(y[2 * i].x, y[2 * i + 1].x, rh[i], rl[i]);
        split2(y[2 * i].y, y[2 * i + 1].y, ih[i], il[i]);
      }
#pragma unroll
      for (int st = 0; st < 2; ++st) {
        const int c = st ^ kpar;
        const int r = 2 * (n1 & 3) + c;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const uint32_t off = a2base + r * 128 + (((jb + u) ^ r) << 4);
          const uint4 vh = c ? make_uint4(ih[4 * u], ih[4 * u + 1], ih[4 * u + 2], ih[4 * u + 3])
                             : make_uint4(rh[4 * u], rh[4 * u + 1], rh[4 * u + 2], rh[4 * u + 3]);
          const uint4 vl = c ? make_uint4(il[4 * u], il[4 * u + 1], il[4 * u + 2], il[4 * u + 3])
                             : make_uint4(rl[4 * u], rl[4 * u + 1], rl[4 * u + 2], rl[4 * u + 3]);
          *reinterpret_cast<uint4*>(s.base + kOffA2hi + off) = vh;
          *reinterpret_cast<uint4*>(s.base + kOffA2lo + off) = vl;
        }
      }
    }
    if (!run_stage(s, tbase, phase, 2)) {
      if (t == 0) atomicExch(err, 1);
      break;
    }
    // ---- stage 2 results: row (qv, k2 = lane) holds outputs k2 + 32 k1, k1 = 16h + i
    {
      float2 y[16];
      read16(tbase, lane_bits, h, y);
      if constexpr (COL) {
        const ColSweepTc& o = (const ColSweepTc&)op;
        float2* dst = o.wt + ((long)p * kN + b0 + qv) * kN + lane + 32 * 16 * h;
#pragma unroll
        for (int i = 0; i < 16; ++i) dst[32 * i] = y[i];
      } else {
        const RowOutTc& o = (const RowOutTc&)op;
        const float oscale = 1.f / (32.f * sigma);
        const long off = (long)p * o.out_plane_stride + (long)(b0 + qv) * kN + lane + 32 * 16 * h;
        if (o.out_c64) {
#pragma unroll
          for (int i = 0; i < 16; ++i) o.out_c64[off + 32 * i] = make_float2(y[i].x * oscale, y[i].y * oscale);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            o.out_re[off + 32 * i] = (double)(y[i].x * oscale);
            o.out_im[off + 32 * i] = (double)(y[i].y * oscale);
          }
        }
      }
    }
  }
  cp_async_wait_all();
  cta_end(tbase);
}

static __global__ void __launch_bounds__(kThreads, 2)
    tc_col_sweep_kernel(ColSweepTc op, const uint4* __restrict__ F, const float2* __restrict__ twg, int ntiles,
                        int* __restrict__ err) {
  sweep_pass<true>(op, F, twg + 0 * kN, ntiles, err);  // twiddles x 2^-10
}

static __global__ void __launch_bounds__(kThreads, 2)
    tc_row_out_kernel(RowOutTc op, const uint4* __restrict__ F, const float2* __restrict__ twg, int ntiles,
                      int* __restrict__ err) {
  sweep_pass<false>(op, F, twg + 1 * kN, ntiles, err);  // twiddles x 2^-5
}

}  // namespace tcfft
}  // namespace doe
