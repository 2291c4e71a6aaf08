// design_ops.cuh -- fused operators of the Gerchberg-Saxton family
// (reference: src/doe.js:327-437 gerchbergSaxton, :455-546 weightedGerchbergSaxton,
// :557-626 gerchbergSaxtonMultiPlane, :639-730 fourierCgh).
//
// A batch of B designs of one grid size runs as one launch per pass: the plane
// index of the row/column kernels is the design index. Per-pixel arrays are FP32
// ([B][nx*ny], centred layout idx = x + y*nx exactly as the reference's planes);
// every reduction (error, efficiency, power, RMSE, weight normalisation)
// accumulates in FP64 and is folded per design by the last CTA of that design
// (fixed order, deterministic), which also updates the design's scalar state.
#pragma once
#include "ops_propagate.cuh"

namespace doe {

// Per-design scalars carried across passes (device memory).
struct DesignState {
  double norm;      // WGS: weights = w_raw * norm
  double best;      // WGS: best unweighted ROI RMSE so far
  double eff_cur;   // image-plane WGS: efficiency of the current forward field
  int stop;         // -1 running; else the iteration whose field met the screen goal
  int best_it;      // image-plane WGS (passes): the iteration of the best iterate (-2: none yet)
  double sT, sTT;   // screen goal: sum T over the plane, sum T^2 over the ROI (fixed)
};

enum RedSlot { kErrNum = 0, kErrDen, kInRoi, kTotal, kRmseNum, kRmseDen, kWsum, kTsum, kRedK };
// Screen-RMSE sums of the stopping goal (src/projector.js:554-595): per iteration
// sum I m over the plane and sum I^2, I T over the ROI; the target's sum T (plane)
// and sum T^2 (ROI) are fixed and summed once, by the first pass, in the first two.
enum GoalSlot { kSIM = kRedK, kSII, kSIT, kRedKGoal };
constexpr int kST = kSIM, kSTT = kSII;
using DesignAcc = DAcc<kRedK>;

struct DesignBufs {
  int nx, ny, iters;
  double dx, dy;
  float feedback;   // HIO feedback (0 = plain GS)
  int escape;       // iterations before the feedback applies
  float beta;       // WGS exponent
  const float* illum;   // [B][n] amplitude A
  const float* tgt;     // [B][n] target amplitude t (plane 0 of a multi-plane set)
  const float* roi;     // [B][n] soft ROI m, or null (1 everywhere)
  long tgt_stride;      // elements between designs in tgt / roi
  float* wraw;          // [B][n] WGS weights before normalisation, or null
  float* phase;         // [B][n] DOE phase
  float* best_phase;    // [B][n] WGS best iterate
  float* amp;           // [B][n] amplitude of the current forward field
  float* best_amp;      // [B][n]
  float2* U;            // [B][n] target-plane field (image-plane WGS)
  float2* U2;           // [B][n] image-plane WGS passes: second field buffer (even / odd iterations)
  float* phase2;        // [B][n] image-plane WGS passes: second phase buffer
  float2* W;            // [B][n] work
  const float2* htab;   // transfer function in FFT bin order
  long htab_stride;     // elements between designs (0: shared geometry)
  DesignState* st;      // [B]
  double* err_hist;     // [B][iters]
  double* eff_hist;     // [B][iters]
  double* pp_err;       // multi-plane: [B][nplanes][iters]
  int mp_plane, mp_nplanes;
  unsigned char* improved;  // [B][iters]
  double* partials;     // [B][max blocks][kRedKGoal]
  unsigned* counters;   // [B]
  double* totals;       // [B][kRedKGoal]
  double rmse_goal;     // > 0: image-plane WGS stops a design at this screen RMSE
  const float* screen_irr;  // [B][n] target irradiance of the goal, or null (t^2)
  __device__ __forceinline__ long pe() const { return (long)nx * ny; }
};

__device__ __forceinline__ int rotn(int i, int n) { return (i + (n >> 1)) & (n - 1); }

// Pull the line holding *p into L1. The design passes read their side planes
// (targets, masks, weights, illumination, transfer tables) only after a transform
// stage; touching them in the load step, before that stage, turns those later
// reads from DRAM-latency misses into L1 hits.
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Designs that met the screen goal drop out of every later pass (whole CTAs
// return before any barrier: the plane index is uniform per CTA).
__device__ __forceinline__ bool design_stopped(const DesignState* st, int p) { return st && st[p].stop >= 0; }

__device__ __forceinline__ float2 unit_phasor(float2 v) {
  const float r2 = v.x * v.x + v.y * v.y;
  if (r2 > 0.f) {
    const float inv = rsqrtf(r2);
    return make_float2(v.x * inv, v.y * inv);
  }
  return make_float2(1.f, 0.f);  // atan2(0, 0) = 0
}

// Fold one design's block sums; returns true in the last block (totals valid).
__device__ __forceinline__ bool design_reduce(const DesignBufs& b, int p, int bip, int bpp, DesignAcc& acc) {
  return group_reduce<kRedK>(acc, p, bip, bpp, b.partials, b.counters, b.totals);
}

// ------------------------------------------------------------------ column passes
// Image-plane propagation column pass with a tabulated transfer function:
// forward column FFT, x H (+z) or conj(H) (-z), inverse column FFT, in place.
template <bool CONJ>
struct ColAsmTab : NoReduce {
  static constexpr const char* kName = CONJ ? "design_col_back" : "design_col_fwd";
  static constexpr int kStages = 2;
  static constexpr bool kInv1 = false, kInv2 = true;
  float2* w;
  const float2* htab;
  long htab_stride;
  int nx, ny;
  const DesignState* st;  // null: every design runs
  __device__ __forceinline__ bool skip(int p) const { return design_stopped(st, p); }
  struct State {
    float2* w;
    const float2* h;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    return {w + p * (long)nx * ny + x, htab + p * htab_stride + x};
  }
  __device__ __forceinline__ void prefetch(const State& s, int y) const { prefetch_l1(&s.h[(long)y * nx]); }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.w[(long)y * nx]; }
  __device__ __forceinline__ void mid(const State& s, int y, float2& v, Acc&) const {
    const float2 h = __ldg(&s.h[(long)y * nx]);
    v = CONJ ? cmulc(v, h) : cmul(v, h);
  }
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const { s.w[(long)y * nx] = v; }
};

// Fourier-domain column pass (src/doe.js:666-717): forward column FFT, unitary
// scale, measurement, WGS weight update, amplitude constraint, inverse column
// FFT. Bin (kx, ky) holds the centred sample (rot(kx), rot(ky)).
template <bool WGS>
struct ColFourier {
  static constexpr const char* kName = WGS ? "design_col_fourier_wgs" : "design_col_fourier";
  static constexpr int kStages = 2;
  static constexpr bool kInv1 = false, kInv2 = true;
  using Acc = DesignAcc;
  DesignBufs b;
  int it;
  float norm;  // 1/sqrt(nx ny)
  struct State {
    const float* t;
    const float* m;
    float* w;
    float* amp;
    float2* W;
    float wn;   // weight normalisation of this pass
  };
  __device__ __forceinline__ State init(int p, int x) const {
    const long o = p * b.pe() + rotn(x, b.nx);
    const long ot = p * b.tgt_stride + rotn(x, b.nx);
    return {b.tgt + ot, b.roi ? b.roi + ot : nullptr, WGS ? b.wraw + o : nullptr, b.amp + o,
            b.W + p * b.pe() + x, WGS ? (float)b.st[p].norm : 1.f};
  }
  __device__ __forceinline__ void prefetch(const State& s, int y) const {
    const long j = (long)rotn(y, b.ny) * b.nx;
    prefetch_l1(&s.t[j]);
    if (s.m) prefetch_l1(&s.m[j]);
    if constexpr (WGS) prefetch_l1(&s.w[j]);
  }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.W[(long)y * b.nx]; }
  __device__ __forceinline__ void mid(const State& s, int y, float2& v, Acc& acc) const {
    const long j = (long)rotn(y, b.ny) * b.nx;
    const float m = s.m ? __ldg(&s.m[j]) : 1.f;
    const float t0 = __ldg(&s.t[j]);
    float w = 1.f;
    if constexpr (WGS) w = s.w[j] * s.wn;
    v = cscale(v, norm);
    const float a = sqrtf(v.x * v.x + v.y * v.y);
    const double ad = a;
    s.amp[j] = a;
    const float tw = t0 * w;
    acc.v[kTotal] += ad * ad;
    if (m > 0.f) {
      acc.v[kInRoi] += ad * ad * m;
      const double d = (ad - (double)tw) * m;
      acc.v[kErrNum] += d * d;
      acc.v[kErrDen] += (double)tw * tw;
    }
    if constexpr (WGS) {
      if (m > 0.f) {  // src/doe.js:489-524 on the amplitude of this forward pass
        const double d = ad - (double)t0;
        acc.v[kRmseNum] += d * d;
        acc.v[kRmseDen] += (double)t0 * t0;
        const float ratio = a > 1e-30f ? t0 / a : 2.f;
        float wn = w * powf(fminf(fmaxf(ratio, 0.25f), 4.f), b.beta);
        wn = fminf(fmaxf(wn, 1e-4f), 1e4f);
        s.w[j] = wn;  // stored before normalisation
        acc.v[kWsum] += (double)wn * wn * t0 * t0;
        acc.v[kTsum] += (double)t0 * t0;
      }
    }
    // constraint: target inside the ROI, measured modulus outside
    const float tc = m > 0.f ? tw : a;
    if (a > 0.f) {
      v = cscale(v, tc / a);
    } else {
      v = make_float2(tc, 0.f);
    }
  }
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const { s.W[(long)y * b.nx] = v; }
  __device__ __forceinline__ void finish(int p, int bip, int bpp, Acc& acc) const {
    if (!design_reduce(b, p, bip, bpp, acc) || threadIdx.x != 0) return;
    const double* T = b.totals + (long)p * kRedK;
    const double err = T[kErrDen] > 0 ? sqrt(T[kErrNum] / T[kErrDen]) : 0.0;
    const double eff = T[kTotal] > 0 ? T[kInRoi] / T[kTotal] : 0.0;
    const long h = (long)p * b.iters + it;
    b.eff_hist[h] = eff;
    if constexpr (WGS) {
      DesignState& S = b.st[p];
      const double rmse = T[kRmseDen] > 0 ? sqrt(T[kRmseNum] / T[kRmseDen]) : 0.0;
      const bool imp = rmse < S.best;
      if (imp) S.best = rmse;
      b.improved[h] = imp ? 1 : 0;
      b.err_hist[h] = S.best;
      S.norm = T[kWsum] > 0 ? sqrt(T[kTsum] / T[kWsum]) : 1.0;
    } else {
      b.err_hist[h] = err;
    }
  }
};

// ------------------------------------------------------------------ row passes
// Forward row pass from the DOE phase: A exp(i phi) -> forward row FFT -> W.
// ROT reads the centred phase at the rotated index (ifftshift of the Fourier loop).
template <bool ROT>
struct RowDoeFwd : NoReduce {
  static constexpr const char* kName = "design_row_doe_fwd";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = false, kInv2 = false;
  DesignBufs b;
  struct State {
    const float* A;
    const float* ph;
    float2* w;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long pe = b.pe();
    const int ys = ROT ? rotn(y, b.ny) : y;
    return {b.illum + p * pe + (long)ys * b.nx, b.phase + p * pe + (long)ys * b.nx, b.W + p * pe + (long)y * b.nx};
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const {
    const int xs = ROT ? rotn(x, b.nx) : x;
    const float a = __ldg(&s.A[xs]);
    float sn, cs;
    sincosf(__ldg(&s.ph[xs]), &sn, &cs);
    return make_float2(a * cs, a * sn);
  }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const { s.w[x] = v; }
};

// End of a back-propagation (or inverse Fourier transform) and start of the next
// forward one: inverse row FFT of W gives the DOE-plane field, its argument
// becomes the new DOE phase (src/doe.js:401-410, :718-722), the illumination
// amplitude is re-imposed (A v/|v| = A exp(i atan2(v))) and, when FWD, the
// forward row FFT of the next propagation is taken. ROT stores at the rotated
// (fftshift) index. SNAP copies the phase and the forward amplitude into the
// best-iterate buffers when the last reduction flagged an improvement.
template <bool FWD, bool ROT, bool SNAP>
struct RowDoeUpdate : NoReduce {
  static constexpr const char* kName = FWD ? "design_row_doe_update" : "design_row_doe_last";
  static constexpr int kStages = FWD ? 2 : 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  DesignBufs b;
  int snap_it;  // iteration whose improvement flag is consulted (SNAP)
  __device__ __forceinline__ bool skip(int p) const { return design_stopped(b.st, p); }
  struct State {
    const float* A;
    float* ph;
    float* bph;
    const float* amp;
    float* bamp;
    float2* w;
    bool snap;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long pe = b.pe();
    const long o = p * pe + (long)(ROT ? rotn(y, b.ny) : y) * b.nx;
    bool snap = false;
    if constexpr (SNAP) snap = b.improved[(long)p * b.iters + snap_it] != 0;
    return {b.illum + o, b.phase + o, SNAP ? b.best_phase + o : nullptr, SNAP ? b.amp + o : nullptr,
            SNAP ? b.best_amp + o : nullptr, b.W + p * pe + (long)y * b.nx, snap};
  }
  __device__ __forceinline__ void prefetch(const State& s, int x) const {
    const int xi = ROT ? rotn(x, b.nx) : x;
    prefetch_l1(&s.A[xi]);
    if constexpr (SNAP) {
      if (s.snap) prefetch_l1(&s.amp[xi]);
    }
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.w[x]; }
  __device__ __forceinline__ float2 doe(const State& s, int x, float2 v) const {
    const int xi = ROT ? rotn(x, b.nx) : x;
    const float a = __ldg(&s.A[xi]);
    const float ph = atan2f(v.y, v.x);
    if constexpr (SNAP) {
      if (s.snap) {
        const float am = s.amp[xi];
        s.bph[xi] = ph;
        s.bamp[xi] = am;
      }
    }
    s.ph[xi] = ph;
    const float2 u = unit_phasor(v);
    return make_float2(a * u.x, a * u.y);
  }
  __device__ __forceinline__ void mid(const State& s, int x, float2& v, Acc&) const { v = doe(s, x, v); }
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const {
    if constexpr (FWD) {
      s.w[x] = v;
    } else {
      (void)doe(s, x, v);
    }
  }
};

// Target plane of plain GS / HIO and of one multi-plane step (src/doe.js:355-397,
// :579-611): the inverse row FFT gives the forward field U of the current phase;
// its error and efficiency are measured (FP64), the amplitude constraint is applied
// and the forward row FFT of the back-propagation is taken. FINAL only measures the
// field and stores its amplitude (the reference's final forward pass, :418-426).
// MP selects the multi-plane error definition and per-plane history.
template <bool FINAL, bool MP>
struct RowGsTarget {
  static constexpr const char* kName = FINAL ? "design_row_gs_final" : "design_row_gs_target";
  static constexpr int kStages = FINAL ? 1 : 2;
  static constexpr bool kInv1 = true, kInv2 = false;
  using Acc = DesignAcc;
  DesignBufs b;
  int it;
  float scale;  // 1/(nx ny)
  struct State {
    const float* t;
    const float* m;
    float* amp;
    float2* w;
    float fb;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * b.pe() + (long)y * b.nx;
    const long ot = p * b.tgt_stride + (long)y * b.nx;
    const float fb = (!MP && it >= b.escape) ? b.feedback : 0.f;
    return {b.tgt + ot, b.roi ? b.roi + ot : nullptr, b.amp + o, b.W + o, fb};
  }
  __device__ __forceinline__ void prefetch(const State& s, int x) const {
    prefetch_l1(&s.t[x]);
    if (s.m) prefetch_l1(&s.m[x]);
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.w[x]; }
  __device__ __forceinline__ float measure(const State& s, int x, float2 u, Acc& acc) const {
    const float a = sqrtf(u.x * u.x + u.y * u.y);
    const double ad = a, i2 = ad * ad;
    const float m = s.m ? __ldg(&s.m[x]) : 1.f;
    const double t = __ldg(&s.t[x]);
    acc.v[kTotal] += i2;
    if (m > 0.f) {
      acc.v[kInRoi] += i2 * m;
      if constexpr (MP) {
        const double d = (ad - t) * m;
        acc.v[kErrNum] += d * d;
        acc.v[kErrDen] += t * t;
      } else if (t > 0.0 || i2 > 0.0) {
        const double d = ad * m - t * m;
        acc.v[kErrNum] += d * d;
        acc.v[kErrDen] += t * t;
      }
    }
    return a;
  }
  __device__ __forceinline__ void mid(const State& s, int x, float2& v, Acc& acc) const {
    const float2 u = cscale(v, scale);
    const float a = measure(s, x, u, acc);
    const float m = s.m ? __ldg(&s.m[x]) : 1.f;
    const float t = __ldg(&s.t[x]);
    float na;
    if (m > 0.f) {
      na = t;
      if (s.fb > 0.f && a > 0.f) na = t + s.fb * (a - t);
    } else {
      na = a * (1.f - s.fb) + s.fb * a;
    }
    v = a > 0.f ? cscale(u, na / a) : u;
  }
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc& acc) const {
    if constexpr (FINAL) {
      const float2 u = cscale(v, scale);
      s.amp[x] = measure(s, x, u, acc);
    } else {
      s.w[x] = v;
    }
  }
  __device__ __forceinline__ void finish(int p, int bip, int bpp, Acc& acc) const {
    if constexpr (FINAL) return;  // the final pass only delivers the amplitude
    if (!design_reduce(b, p, bip, bpp, acc) || threadIdx.x != 0) return;
    const double* T = b.totals + (long)p * kRedK;
    const double err = T[kErrDen] > 0 ? sqrt(T[kErrNum] / T[kErrDen]) : 0.0;
    if constexpr (MP) {
      b.pp_err[((long)p * b.mp_nplanes + b.mp_plane) * b.iters + it] = err;
    } else {
      const long h = (long)p * b.iters + it;
      b.err_hist[h] = err;
      b.eff_hist[h] = T[kTotal] > 0 ? (T[kInRoi] * b.dx * b.dy) / (T[kTotal] * b.dx * b.dy) : 0.0;
    }
  }
};

// Image-plane WGS, end of an iteration (src/doe.js:417-426 then :489-529): the
// inverse row FFT gives the forward field U of the new phase, stored for the next
// constraint; FP64 sums of the unweighted ROI RMSE, of the efficiency of U and of
// the weight update (w <- clamp(w clamp(t/a, 1/4, 4)^beta, 1e-4, 1e4), stored
// before normalisation). The last CTA of a design records the histories, the best
// RMSE and the new normalisation sqrt(sum t^2 / sum w^2 t^2). INITIAL only
// measures the efficiency of the first forward field. GOAL also sums the screen
// RMSE of the field (same definition as screen_metrics_kernel) and stops the
// design when it reaches b.rmse_goal; that iterate is forced into the snapshot.
template <bool INITIAL, bool GOAL = false>
struct RowWgsTarget {
  static constexpr const char* kName = INITIAL ? "design_row_wgs_first" : "design_row_wgs_target";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  static constexpr int K = GOAL ? kRedKGoal : kRedK;
  using Acc = DAcc<K>;
  DesignBufs b;
  int it;
  float scale;
  __device__ __forceinline__ bool skip(int p) const { return design_stopped(b.st, p); }
  struct State {
    const float* t;
    const float* m;
    float* w;
    float2* U;
    const float2* W;
    const float* T;
    float wn;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * b.pe() + (long)y * b.nx;
    const long ot = p * b.tgt_stride + (long)y * b.nx;
    return {b.tgt + ot, b.roi ? b.roi + ot : nullptr, b.wraw + o, b.U + o, b.W + o,
            (GOAL && b.screen_irr) ? b.screen_irr + o : nullptr, (float)b.st[p].norm};
  }
  __device__ __forceinline__ void prefetch(const State& s, int x) const {
    prefetch_l1(&s.t[x]);
    if (s.m) prefetch_l1(&s.m[x]);
    if constexpr (!INITIAL) prefetch_l1(&s.w[x]);
    if constexpr (GOAL) {
      if (s.T) prefetch_l1(&s.T[x]);
    }
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.W[x]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc& acc) const {
    const float m = s.m ? __ldg(&s.m[x]) : 1.f;
    const float t = __ldg(&s.t[x]);
    float wold = 0.f;
    if constexpr (!INITIAL) wold = s.w[x];
    const float2 u = cscale(v, scale);
    s.U[x] = u;
    const float a = sqrtf(u.x * u.x + u.y * u.y);
    const double ad = a, i2 = ad * ad;
    acc.v[kTotal] += i2;
    if (m > 0.f) acc.v[kInRoi] += i2 * m;
    if constexpr (!INITIAL) {
      if (m > 0.f) {
        const double d = ad - (double)t;
        acc.v[kRmseNum] += d * d;
        acc.v[kRmseDen] += (double)t * t;
        const float ratio = a > 1e-30f ? t / a : 2.f;
        float w = wold * s.wn * powf(fminf(fmaxf(ratio, 0.25f), 4.f), b.beta);
        w = fminf(fmaxf(w, 1e-4f), 1e4f);
        s.w[x] = w;
        acc.v[kWsum] += (double)w * w * t * t;
        acc.v[kTsum] += (double)t * t;
      }
    }
    if constexpr (GOAL) {
      const double T = s.T ? (double)__ldg(&s.T[x]) : (double)t * t;
      if constexpr (INITIAL) {
        acc.v[kST] += T;
        if (m > 0.f) acc.v[kSTT] += T * T;
      } else {
        acc.v[kSIM] += i2 * m;
        if (m > 0.f) {
          acc.v[kSII] += i2 * i2;
          acc.v[kSIT] += i2 * T;
        }
      }
    }
  }
  __device__ __forceinline__ void finish(int p, int bip, int bpp, Acc& acc) const {
    if (!group_reduce<K>(acc, p, bip, bpp, b.partials, b.counters, b.totals) || threadIdx.x != 0) return;
    const double* T = b.totals + (long)p * K;
    DesignState& S = b.st[p];
    const double eff = T[kTotal] > 0 ? (T[kInRoi] * b.dx * b.dy) / (T[kTotal] * b.dx * b.dy) : 0.0;
    if constexpr (INITIAL) {
      S.eff_cur = eff;
      if constexpr (GOAL) {
        S.sT = T[kST];
        S.sTT = T[kSTT];
      }
    } else {
      const long h = (long)p * b.iters + it;
      const double rmse = T[kRmseDen] > 0 ? sqrt(T[kRmseNum] / T[kRmseDen]) : 0.0;
      bool imp = rmse < S.best;
      if constexpr (GOAL) {
        // screen RMSE exactly as screen_metrics_kernel (the pitch cancels)
        const double sc = S.sT > 0 ? T[kSIM] / S.sT : 0.0;
        const double den = sc * sc * S.sTT;
        const double num = fmax(0.0, T[kSII] - 2.0 * sc * T[kSIT] + sc * sc * S.sTT);
        const double srm = den > 0 ? sqrt(num / den) : 0.0;
        if (srm <= b.rmse_goal) {
          S.stop = it;
          imp = true;  // return the iterate that met the goal
        }
      }
      if (imp) {
        S.best = rmse;
        S.best_it = it;
      }
      b.improved[h] = imp ? 1 : 0;
      b.err_hist[h] = S.best;
      b.eff_hist[h] = S.eff_cur;
      S.eff_cur = eff;
      S.norm = T[kWsum] > 0 ? sqrt(T[kTsum] / T[kWsum]) : 1.0;
    }
  }
};

// Image-plane WGS, start of iteration `it` (src/doe.js:380-397 with weights): load
// the forward field U of iteration it - 1, apply the constraint with
// t * w_raw * norm inside the ROI (outside: unchanged), forward row FFT of the
// back-propagation.
//
// Best iterate, kept lazily: the phase and field of iteration k live in one of two
// alternating buffers each (phase produced by iteration k in buffer (k + 1) mod 2,
// field in buffer k mod 2) until iteration k + 2 overwrites them. So the best
// iterate needs no copy while later iterations keep improving on it; only when
// the design's best is still iteration it - 2 when iteration it starts (it did not
// improve since) does this pass copy that iterate's phase and amplitude into the
// best-iterate buffers, from the buffers iteration it is about to overwrite. The
// loop's last pass resolves where each design's best iterate ended up.
struct RowWgsConstrain : NoReduce {
  static constexpr const char* kName = "design_row_wgs_constrain";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = false, kInv2 = false;
  DesignBufs b;             // b.U: the field of iteration it - 1
  int it;
  const float* ph_old;      // phase produced by iteration it - 2
  const float2* u_old;      // field of iteration it - 2
  __device__ __forceinline__ bool skip(int p) const { return design_stopped(b.st, p); }
  struct State {
    const float* t;
    const float* m;
    const float* w;
    const float2* U;
    float2* W;
    const float* ph;
    const float2* uo;
    float* bph;
    float* bamp;
    float wn;
    bool snap;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * b.pe() + (long)y * b.nx;
    const long ot = p * b.tgt_stride + (long)y * b.nx;
    const bool snap = it >= 2 && b.st[p].best_it == it - 2;
    return {b.tgt + ot, b.roi ? b.roi + ot : nullptr, b.wraw + o, b.U + o, b.W + o, ph_old + o, u_old + o,
            b.best_phase + o, b.best_amp + o, (float)b.st[p].norm, snap};
  }
  // every field read and side-plane prefetch of the thread first, then the
  // constraint (whose snapshot stores would otherwise keep later reads waiting)
  __device__ __forceinline__ float2 load(const State& s, int x) const {
    prefetch_l1(&s.t[x]);
    prefetch_l1(&s.w[x]);
    if (s.m) prefetch_l1(&s.m[x]);
    if (s.snap) {
      prefetch_l1(&s.ph[x]);
      prefetch_l1(&s.uo[x]);
    }
    return __ldg(&s.U[x]);
  }
  __device__ __forceinline__ float2 finish_load(const State& s, int x, float2 u) const {
    const float m = s.m ? __ldg(&s.m[x]) : 1.f;
    const float t = __ldg(&s.t[x]);
    const float w = __ldg(&s.w[x]);
    const float a = sqrtf(u.x * u.x + u.y * u.y);
    if (s.snap) {
      const float2 uo = __ldg(&s.uo[x]);
      s.bph[x] = __ldg(&s.ph[x]);
      s.bamp[x] = sqrtf(uo.x * uo.x + uo.y * uo.y);
    }
    if (m > 0.f && a > 0.f) return cscale(u, (t * (w * s.wn)) / a);
    return u;
  }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const { s.W[x] = v; }
};

// ------------------------------------------------------------------ phase gradient
// Intensity loss of a DOE phase and its gradient (no reference counterpart; the
// training signal of the warm-start surrogate). With U0 = A exp(i phi), U = P U0
// (P the image-plane propagation of the design loops) and I = |U|^2:
//   L = sum m (I - T)^2 / sum m T^2,   T = t^2,
//   dL/dU* = 2 m (I - T) U / D,  dL/dphi = 2 Im(conj(U0) P^H(dL/dU*)),  D = sum m T^2.
// Pass 3 of 5: inverse row FFT gives U; FP64 sums of the numerator and D; the
// unnormalised G = 2 m (I - T) U goes through the forward row FFT of P^H.
struct RowLossField {
  static constexpr const char* kName = "design_row_loss";
  static constexpr int kStages = 2;
  static constexpr bool kInv1 = true, kInv2 = false;
  using Acc = DesignAcc;
  DesignBufs b;
  float scale;
  struct State {
    const float* t;
    const float* m;
    float2* w;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * b.pe() + (long)y * b.nx;
    const long ot = p * b.tgt_stride + (long)y * b.nx;
    return {b.tgt + ot, b.roi ? b.roi + ot : nullptr, b.W + o};
  }
  __device__ __forceinline__ void prefetch(const State& s, int x) const {
    prefetch_l1(&s.t[x]);
    if (s.m) prefetch_l1(&s.m[x]);
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.w[x]; }
  __device__ __forceinline__ void mid(const State& s, int x, float2& v, Acc& acc) const {
    const float m = s.m ? __ldg(&s.m[x]) : 1.f;
    const float t = __ldg(&s.t[x]);
    const float2 u = cscale(v, scale);
    const float I = u.x * u.x + u.y * u.y, T = t * t;
    const float r = I - T;
    acc.v[kErrNum] += (double)m * r * r;
    acc.v[kErrDen] += (double)m * T * T;
    v = cscale(u, 2.f * m * r);
  }
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const { s.w[x] = v; }
  __device__ __forceinline__ void finish(int p, int bip, int bpp, Acc& acc) const {
    design_reduce(b, p, bip, bpp, acc);
  }
};

// Pass 5 of 5: inverse row FFT gives g0 = P^H G; dphi = 2 Im(conj(U0) g0) / D.
struct RowPhaseGrad : NoReduce {
  static constexpr const char* kName = "design_row_phase_grad";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  DesignBufs b;
  float scale;
  float* grad;   // [B][n]
  double* loss;  // [B] or null
  struct State {
    const float* A;
    const float* ph;
    float* g;
    float2* w;
    float inv_d;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * b.pe() + (long)y * b.nx;
    const double* T = b.totals + (long)p * kRedK;  // written by RowLossField's reduction
    const float inv = T[kErrDen] > 0 ? (float)(1.0 / T[kErrDen]) : 0.f;
    if (loss && y == 0 && threadIdx.x == 0) loss[p] = T[kErrDen] > 0 ? T[kErrNum] / T[kErrDen] : 0.0;
    return {b.illum + o, b.phase + o, grad + o, b.W + o, inv};
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.w[x]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const {
    const float2 g0 = cscale(v, scale);
    float sn, cs;
    sincosf(__ldg(&s.ph[x]), &sn, &cs);
    const float a = __ldg(&s.A[x]);
    // Im(conj(a e^{i phi}) g0) = a (cos phi g0.y - sin phi g0.x)
    s.g[x] = 2.f * a * (cs * g0.y - sn * g0.x) * s.inv_d;
  }
};

// Design loops are compiled for every power-of-two axis the transforms take,
// 1..8192, with the default CTA shapes (each operator is instantiated once per size).
constexpr int kDesignMinN = 1, kDesignMaxN = kMaxN;

template <class F>
inline int with_design_n(int n, F&& f) {
  return with_n(n, static_cast<F&&>(f));
}
// Row / column pass of a design loop with the shape variant the context selected
// for that length (tuning kind "design"; doe_autotune_design picks it). Each
// operator's passes, for every length and shape variant, are instantiated once,
// in one of the design_inst_*.cu units (which define DOE_DESIGN_INSTANTIATE), so
// that those heavy kernel instantiations compile in parallel; the pass sequences
// only see the declarations.
template <class Op>
int design_row(doe_ctx* c, const Op& op, int B, int nx, int ny);
template <class Op>
int design_col(doe_ctx* c, const Op& op, int B, int nx, int ny);

#ifdef DOE_DESIGN_INSTANTIATE
template <class Op>
int design_row(doe_ctx* c, const Op& op, int B, int nx, int ny) {
  return with_design_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    auto f = [&](auto S) { return launch_row<decltype(S)>(c, op, B, ny); };
    return select_shape<typename DesignRowVariants<N>::list>(c->tune_row[kTuneDesign][ilog2i(N)], f);
  });
}
template <class Op>
int design_col(doe_ctx* c, const Op& op, int B, int nx, int ny) {
  return with_design_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    auto f = [&](auto S) { return launch_col<decltype(S)>(c, op, B, nx); };
    return select_shape<typename DesignColVariants<N>::list>(c->tune_col[kTuneDesign][ilog2i(N)], f);
  });
}
#define DOE_DESIGN_ROW_INST(...) template int design_row<__VA_ARGS__>(doe_ctx*, const __VA_ARGS__&, int, int, int);
#define DOE_DESIGN_COL_INST(...) template int design_col<__VA_ARGS__>(doe_ctx*, const __VA_ARGS__&, int, int, int);
#endif

// CTAs per design of the widest pass over every shape variant (sizes the
// per-block reduction partials whatever variant a later call selects).
inline int design_bpp(int nx, int ny) {
  int bpp = 1;
  with_design_n(nx, [&](auto NC) {
    auto f = [&](auto S) {
      bpp = std::max(bpp, (ny + decltype(S)::V - 1) / decltype(S)::V);
      return 0;
    };
    using L = typename DesignRowVariants<decltype(NC)::value>::list;
    for (int v = 0; v < (int)std::tuple_size<L>::value; ++v) select_shape<L>(v, f);
    return 0;
  });
  with_design_n(ny, [&](auto NC) {
    auto f = [&](auto S) {
      bpp = std::max(bpp, (nx + decltype(S)::C - 1) / decltype(S)::C);
      return 0;
    };
    using L = typename DesignColVariants<decltype(NC)::value>::list;
    for (int v = 0; v < (int)std::tuple_size<L>::value; ++v) select_shape<L>(v, f);
    return 0;
  });
  return bpp;
}
// Number of design-pass shape variants for length n (for the autotuner).
inline int design_row_variants(int n) {
  return with_design_n(n, [](auto NC) {
    return (int)std::tuple_size<typename DesignRowVariants<decltype(NC)::value>::list>::value;
  });
}
inline int design_col_variants(int n) {
  return with_design_n(n, [](auto NC) {
    return (int)std::tuple_size<typename DesignColVariants<decltype(NC)::value>::list>::value;
  });
}

// Pass sequences, one translation unit each (design_gs.cu, design_wgs.cu,
// design_fourier.cu); the state in `b` is initialised by the caller.
int design_run_gs(doe_ctx* c, const DesignBufs& b, int B, int iterations);
int design_run_wgs(doe_ctx* c, const DesignBufs& b, int B, int iterations);
// Image-plane WGS with the whole loop resident in one thread-block cluster per
// design (square 64^2, 128^2, 256^2); DOE_ERR_UNSUPPORTED for other grids.
int design_run_wgs_cluster(doe_ctx* c, const DesignBufs& b, int B, int iterations);
int design_run_fourier(doe_ctx* c, const DesignBufs& b, int B, int iterations, bool wgs);
// Multi-plane (B designs): plane p uses transfer table htab + p*n and target /
// ROI planes tgt0 + d*nplanes*n + p*n (roi0 may be null).
int design_run_multiplane(doe_ctx* c, DesignBufs b, int B, int iterations, int nplanes, const float2* htab,
                          const float* tgt0, const float* roi0);

}  // namespace doe
