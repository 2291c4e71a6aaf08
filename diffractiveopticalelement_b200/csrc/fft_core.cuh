// fft_core.cuh -- shared-memory Stockham FFT for sm_100a with fusable operators.
//
// One CTA transforms V independent vectors of compile-time power-of-two length N.
// Each vector is handled by T = N / RMAX threads that keep RMAX complex values in
// registers; passes exchange data through shared memory (Stockham autosort, so
// no bit reversal is ever materialised). The first pass reads straight from
// global memory through a caller-supplied load operator and the last pass hands
// its values to a store operator, so pointwise work (shifts, transfer functions,
// amplitude constraints, reductions, FP64<->FP32 conversion) is fused into the
// transform instead of costing extra HBM round trips.
//
// Numerical contract: FP32 arithmetic with twiddles rounded once from FP64
// (table `tw`, e^{-2 pi i m/N}), inner radix constants evaluated at compile time
// from a Taylor series in double precision. Forward transform is unscaled and the
// inverse carries no scale here; callers fold 1/(nx*ny) into a store, matching
// the reference's fft2d (src/fft.js:148-154) up to FP32 rounding.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace doe {

// ---------------------------------------------------------------- complex helpers
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// ---------------------------------------------------------------- compile-time trig
// Maclaurin series for sin/cos on |x| <= pi/4 in double precision; only ever
// evaluated by the compiler to produce the inner radix constants.
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double ct_sin_small(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int i = 1; i < 14; ++i) {
    term *= -x2 / double((2 * i) * (2 * i + 1));
    sum += term;
  }
  return sum;
}
constexpr double ct_cos_small(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int i = 1; i < 14; ++i) {
    term *= -x2 / double((2 * i - 1) * (2 * i));
    sum += term;
  }
  return sum;
}
// cos(2 pi k / L) and sin(2 pi k / L) for integers, by octant symmetry.
constexpr double ct_cos2pi(long k, long L) {
  k %= L;
  if (k < 0) k += L;
  // reduce to [0, L/2]: cos is even around L/2 mirror
  if (2 * k > L) k = L - k;                     // cos(2pi - a) = cos a
  if (4 * k > L) return -ct_cos2pi(L / 2 - k, L);  // cos(pi - a) = -cos a  (k in (L/4, L/2])
  // now a = 2 pi k / L in [0, pi/2]
  if (8 * k > L) return ct_sin_small(2.0 * kPi * double(L / 4 - k) / double(L)) ;
  return ct_cos_small(2.0 * kPi * double(k) / double(L));
}
constexpr double ct_sin2pi(long k, long L) { return ct_cos2pi(k - L / 4, L); }  // sin a = cos(a - pi/2)

// ---------------------------------------------------------------- twiddled multiply
// v * W_L^k with W_L = e^{-2 pi i / L} (forward) or its conjugate (inverse).
// Exact special cases avoid multiplications by 0/1 that IEEE rules keep alive.
template <int K, int L, bool INV>
__device__ __forceinline__ float2 twiddle_const(float2 v) {
  constexpr int k = ((K % L) + L) % L;
  if constexpr (k == 0) {
    return v;
  } else if constexpr (2 * k == L) {
    return make_float2(-v.x, -v.y);
  } else if constexpr (4 * k == L) {  // -i (fwd) / +i (inv)
    return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  } else if constexpr (4 * k == 3 * L) {  // +i (fwd) / -i (inv)
    return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  } else {
    constexpr float c = (float)ct_cos2pi(k, L);
    constexpr float s = (float)(INV ? ct_sin2pi(k, L) : -ct_sin2pi(k, L));
    if constexpr (8 * k == L || 8 * k == 3 * L || 8 * k == 5 * L || 8 * k == 7 * L) {
      // |c| == |s| == sqrt(1/2): 2 multiplies instead of 4
      constexpr float a = c;
      constexpr float b = s;
      if constexpr ((a > 0) == (b > 0)) {  // (a, a)
        return make_float2(a * (v.x - v.y), a * (v.x + v.y));
      } else {  // (a, -a)
        return make_float2(a * (v.x + v.y), a * (v.y - v.x));
      }
    } else {
      return make_float2(fmaf(v.x, c, -v.y * s), fmaf(v.x, s, v.y * c));
    }
  }
}

// ---------------------------------------------------------------- register DFT
// In-register radix-2 decimation-in-frequency DFT of R points stored in v[OFF..OFF+R),
// natural order in and out (the bit reversal is a compile-time register rename).
template <int R>
struct Log2 {
  static constexpr int value = (R <= 1) ? 0 : 1 + Log2<R / 2>::value;
};
template <>
struct Log2<1> {
  static constexpr int value = 0;
};

template <int R>
__device__ __forceinline__ constexpr int bitrev(int i) {
  int r = 0;
  for (int b = 0; b < Log2<R>::value; ++b)
    if (i & (1 << b)) r |= 1 << (Log2<R>::value - 1 - b);
  return r;
}

template <int L, int HALF, int K, bool INV, int NBLK, int B, int OFF, int RA>
struct DifStage {
  // butterfly k of block b within a stage whose sub-length is L
  static __device__ __forceinline__ void run(float2 (&v)[RA]) {
    constexpr int i0 = OFF + B * L + K;
    constexpr int i1 = i0 + HALF;
    float2 a = v[i0], c = v[i1];
    v[i0] = cadd(a, c);
    v[i1] = twiddle_const<K, L, INV>(csub(a, c));
    if constexpr (K + 1 < HALF) {
      DifStage<L, HALF, K + 1, INV, NBLK, B, OFF, RA>::run(v);
    } else if constexpr (B + 1 < NBLK) {
      DifStage<L, HALF, 0, INV, NBLK, B + 1, OFF, RA>::run(v);
    }
  }
};

template <int R, int L, bool INV, int OFF, int RA>
__device__ __forceinline__ void dif_stages(float2 (&v)[RA]) {
  if constexpr (L >= 2) {
    DifStage<L, L / 2, 0, INV, R / L, 0, OFF, RA>::run(v);
    dif_stages<R, L / 2, INV, OFF, RA>(v);
  }
}

template <int R, bool INV, int OFF, int RA>
__device__ __forceinline__ void dft_reg(float2 (&v)[RA]) {
  if constexpr (R >= 2) {
    dif_stages<R, R, INV, OFF, RA>(v);
    // undo bit reversal by renaming registers
    float2 t[R];
#pragma unroll
    for (int i = 0; i < R; ++i) t[i] = v[OFF + i];
#pragma unroll
    for (int i = 0; i < R; ++i) v[OFF + bitrev<R>(i)] = t[i];
  }
}

// ---------------------------------------------------------------- plans
// A plan is a radix sequence for one length. RMAX registers per thread,
// T = N / RMAX threads per vector; in pass p each thread runs RMAX / R_p
// butterflies. Symmetric plans (first radix == last radix) let two transforms
// chain in registers without a shared-memory re-layout.
template <int N_, int NP_, int R0, int R1 = 1, int R2 = 1>
struct FftPlan {
  static constexpr int N = N_;
  static constexpr int NP = NP_;
  static constexpr int RMAX = (R0 > R1 ? (R0 > R2 ? R0 : R2) : (R1 > R2 ? R1 : R2));
  static constexpr int T = N_ / RMAX;
  static constexpr __host__ __device__ int radix(int p) { return p == 0 ? R0 : (p == 1 ? R1 : R2); }
  static constexpr int last() { return radix(NP_ - 1); }
  static constexpr bool symmetric() { return R0 == radix(NP_ - 1); }
  // Padding of the column kernels' exchanges (C vectors interleaved element by
  // element): one spare slot every 2^PSHIFT complex values. The first pass stores
  // with stride R0 per thread; a 64-bit access is served 16 lanes at a time by 16
  // eight-byte banks, and one spare slot per 16 values keeps radix-8 and radix-16
  // first passes conflict-free in that layout, where one per 32 left them 2-way
  // conflicted on half of their stores; radix-32 first passes need one per 32.
  // (Row kernels keep one per 32: with one per 16 the compiler's register
  // allocation of the fused row operators grew, 64 -> 98 registers for the
  // 256-point DOE update, and the occupancy lost outweighed the conflicts saved.)
  static constexpr int PSHIFT = R0 >= 32 ? 5 : 4;
  static_assert(NP_ == 1 ? R0 == N_ : (NP_ == 2 ? R0 * R1 == N_ : R0 * R1 * R2 == N_), "radices must multiply to N");
};

// Default plan per length.
template <int N>
struct DefaultPlan;
template <> struct DefaultPlan<1> { using type = FftPlan<1, 1, 1>; };
template <> struct DefaultPlan<2> { using type = FftPlan<2, 1, 2>; };
template <> struct DefaultPlan<4> { using type = FftPlan<4, 1, 4>; };
template <> struct DefaultPlan<8> { using type = FftPlan<8, 1, 8>; };
template <> struct DefaultPlan<16> { using type = FftPlan<16, 1, 16>; };
template <> struct DefaultPlan<32> { using type = FftPlan<32, 1, 32>; };
template <> struct DefaultPlan<64> { using type = FftPlan<64, 2, 8, 8>; };
template <> struct DefaultPlan<128> { using type = FftPlan<128, 2, 16, 8>; };
template <> struct DefaultPlan<256> { using type = FftPlan<256, 2, 16, 16>; };
template <> struct DefaultPlan<512> { using type = FftPlan<512, 3, 8, 8, 8>; };
template <> struct DefaultPlan<1024> { using type = FftPlan<1024, 2, 32, 32>; };
template <> struct DefaultPlan<2048> { using type = FftPlan<2048, 3, 16, 8, 16>; };
template <> struct DefaultPlan<4096> { using type = FftPlan<4096, 3, 16, 16, 16>; };
template <> struct DefaultPlan<8192> { using type = FftPlan<8192, 3, 32, 8, 32>; };

template <class P, int PI>
struct PassNs {  // product of the radices before pass PI
  static constexpr int value = PassNs<P, PI - 1>::value * P::radix(PI - 1);
};
template <class P>
struct PassNs<P, 0> {
  static constexpr int value = 1;
};

// Padded shared-memory index: one spare slot every 2^SH complex values keeps the
// stride-R Stockham writes of the early passes free of bank conflicts (SH = 5 for
// row kernels, the plan's PSHIFT for column kernels).
template <int SH>
__device__ __forceinline__ int spad(int x) {
  return x + (x >> SH);
}
// Shared-memory length (complex values) of one row kernel's padded vector.
template <int N>
constexpr int padded_len() {
  return N + N / 32 + 1;
}
// Shared-memory length of a column kernel's padded tile of len values.
template <class P>
constexpr int padded_col(int len) {
  return len + (len >> P::PSHIFT) + 1;
}

// Vector accessor used for the shared-memory exchanges. Row kernels place each
// vector contiguously (stride 1, vector pitch NPAD); column kernels interleave C
// vectors (element-major, element stride C).
template <int SH = 5>
struct SmemVec {
  float2* base;
  int estride;  // distance between consecutive elements (1 or C)
  int off;      // vector offset inside an interleaved tile (column kernels)
  __device__ __forceinline__ float2& at(int e) const { return base[spad<SH>(e * estride + off)]; }
};

// ---------------------------------------------------------------- one pass
// Apply twiddles W_{Ns R}^{r k} and the radix-R DFT for butterfly slot BI of pass PI.
template <class P, int PI, bool INV, int BI>
__device__ __forceinline__ void pass_bfly(float2 (&v)[P::RMAX], int t, const float2* __restrict__ tw) {
  constexpr int N = P::N;
  constexpr int R = P::radix(PI);
  constexpr int RMAX = P::RMAX;
  constexpr int T = P::T;
  constexpr int NS = PassNs<P, PI>::value;
  if constexpr (BI < RMAX / R) {
    if constexpr (NS > 1) {
      const int j = t + BI * T;
      const int k = j % NS;
      constexpr int STEP = N / (NS * R);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 w = __ldg(&tw[r * k * STEP]);
        v[BI * R + r] = INV ? cmulc(v[BI * R + r], w) : cmul(v[BI * R + r], w);
      }
    }
    dft_reg<R, INV, BI * R>(v);
    pass_bfly<P, PI, INV, BI + 1>(v, t, tw);
  }
}

// Write pass-PI outputs to shared memory at their Stockham positions.
template <class P, int PI, class SV>
__device__ __forceinline__ void pass_store(const float2 (&v)[P::RMAX], int t, const SV& s) {
  constexpr int R = P::radix(PI);
  constexpr int NS = PassNs<P, PI>::value;
#pragma unroll
  for (int b = 0; b < P::RMAX / R; ++b) {
    const int j = t + b * P::T;
    const int d = (j / NS) * NS * R + (j % NS);
#pragma unroll
    for (int r = 0; r < R; ++r) s.at(d + r * NS) = v[b * R + r];
  }
}

// Read pass-PI inputs from shared memory (element j + r N/R for butterfly j).
template <class P, int PI, class SV>
__device__ __forceinline__ void pass_load(float2 (&v)[P::RMAX], int t, const SV& s) {
  constexpr int R = P::radix(PI);
#pragma unroll
  for (int b = 0; b < P::RMAX / R; ++b) {
    const int j = t + b * P::T;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = s.at(j + r * (P::N / R));
  }
}

// Element index held by register slot (b, r) before pass 0 (input layout).
template <class P>
__device__ __forceinline__ int in_elem(int t, int slot) {
  constexpr int R = P::radix(0);
  const int b = slot / R, r = slot % R;
  return t + b * P::T + r * (P::N / R);
}
// Element index held by slot after the last pass (natural-order output layout).
template <class P>
__device__ __forceinline__ int out_elem(int t, int slot) {
  constexpr int R = P::last();
  const int b = slot / R, r = slot % R;
  return t + b * P::T + r * (P::N / R);
}

// Full transform: registers hold the pass-0 input layout on entry and the
// natural-order output layout on return. `sync` is a block barrier.
template <class P, bool INV, int PI = 0, class SV, class Sync>
__device__ __forceinline__ void fft_run(float2 (&v)[P::RMAX], int t, const SV& s, const float2* __restrict__ tw,
                                        Sync sync) {
  pass_bfly<P, PI, INV, 0>(v, t, tw);
  if constexpr (PI + 1 < P::NP) {
    sync();  // everyone finished reading the previous contents of s
    pass_store<P, PI>(v, t, s);
    sync();
    pass_load<P, PI + 1>(v, t, s);
    fft_run<P, INV, PI + 1>(v, t, s, tw, sync);
  }
}

// Re-layout registers from the output layout to the pass-0 input layout (only
// needed for asymmetric plans when two transforms are chained).
template <class P, class SV, class Sync>
__device__ __forceinline__ void relayout_out_to_in(float2 (&v)[P::RMAX], int t, const SV& s, Sync sync) {
  if constexpr (!P::symmetric()) {
    sync();
#pragma unroll
    for (int q = 0; q < P::RMAX; ++q) s.at(out_elem<P>(t, q)) = v[q];
    sync();
#pragma unroll
    for (int q = 0; q < P::RMAX; ++q) v[q] = s.at(in_elem<P>(t, q));
  }
}

}  // namespace doe
