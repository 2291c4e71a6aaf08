// asm.cuh -- angular-spectrum transfer function evaluated on the fly.
//
// Reference: src/propagate.js:57-102 builds, on the centred frequency grid,
//   H = w_x w_y exp(i 2 pi z sqrt(1/lambda^2 - fx^2 - fy^2))   (0 if evanescent)
// with a raised-cosine band-limit window (src/propagate.js:38-51). The phase
// reaches ~1e5 cycles at z = 30-50 mm, so a plain FP32 product loses ~1e-2 rad.
// Here the phase in cycles is split exactly as
//   z sqrt(1/l^2 - f^2) = Z - (Z/2) u - Z u^2 / (2 (1 + sqrt(1-u))^2),
//   Z = z / lambda,  u = lambda^2 (fx^2 + fy^2) = ux + uy,
// The first two terms are separable: per axis bin the table holds the unit
// complex factor exp(i 2 pi (frac(Z) - frac((Z/2) u_x))) (x bins) or
// exp(-i 2 pi frac((Z/2) u_y)) (y bins), reduced and evaluated in FP64 once per
// plane. Per pixel only the small last term q (|q| <= 2 cycles) is evaluated in
// FP32 and reduced to [-1/2, 1/2] cycles, so its sincos argument stays in
// [-pi, pi] where the SFU sin/cos error is below 4e-7; H is the product of the
// three factors and the band-limit window. Pixels with q above 2 cycles (u > ucut),
// which includes every pixel near the evanescent boundary, take an FP64 path that
// mirrors the reference's `invL2 - fx*fx - fy*fy` test exactly.
#pragma once
#include "engine.cuh"

namespace doe {

constexpr int kMaxGroup = 64;  // planes per table-building launch

// Per-plane scalars, built on the device by asm_tables_kernel.
struct AsmPlane {
  double z;       // signed distance
  double invL2;   // 1/lambda^2
  float c0;       // frac(z / lambda) in [-0.5, 0.5)
  float hz;       // z / (2 lambda)
  float ucut;     // fast path valid for u <= ucut
  int evanescent; // 1: zero the evanescent band (reference default)
};

// Per-bin axis entry: separable unit phase factor (er, ei), u = (lambda f)^2 and
// the band-limit window w.
struct __align__(16) AxisBin {
  float er, ei, u, w;
};

struct AsmGroupArgs {
  int nplanes;
  int nx, ny;
  double dx, dy;
  int band_limit, evanescent;
  double soft_edge;
  double lam[kMaxGroup];
  double z[kMaxGroup];
};

struct AsmTables {
  AxisBin* xt;    // [nplanes][nx]
  AxisBin* yt;    // [nplanes][ny]
  double* xf2;    // [nx]   fx*fx (FP64, same rounding as the reference)
  double* yf2;    // [ny]
  AsmPlane* pl;   // [nplanes]
  float* xc;      // [nplanes][nx] the x-bin phase of xt in cycles, in [-1/2, 1/2]
  float* yc;      // [nplanes][ny] the y-bin phase of yt in cycles
};

__device__ __forceinline__ double d_frac(double x) { return x - rint(x); }

// src/propagate.js:38-42
__device__ __forceinline__ double d_soft_window(double v, double lim, double inner) {
  if (v <= inner) return 1.0;
  if (v >= lim) return 0.0;
  return 0.5 * (1.0 + cos((kPi * (v - inner)) / (lim - inner)));
}

// src/propagate.js:48-51
__device__ __forceinline__ double d_local_frequency_limit(int n, double d, double lambda, double z) {
  const double df = 1.0 / (n * d);
  const double a = 2.0 * df * z;
  return 1.0 / (lambda * sqrt(a * a + 1.0));
}

// One thread per (plane, axis bin); thread 0 of each plane also fills AsmPlane.
static __global__ void asm_tables_kernel(AsmGroupArgs a, AsmTables t) {
  const int p = blockIdx.y;
  const double lam = a.lam[p], z = a.z[p];
  const int total = a.nx + a.ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const bool isx = i < a.nx;
    const int n = isx ? a.nx : a.ny;
    const int k = isx ? i : i - a.nx;
    const double d = isx ? a.dx : a.dy;
    const double df = 1.0 / (n * d);
    const int ic = (k + (n >> 1)) % n;
    const double f = (ic - n / 2.0) * df;
    const double f2 = f * f;
    const double u = lam * lam * f2;
    AxisBin b;
    b.u = (float)u;
    // x bins carry frac(Z) - frac((Z/2) u_x), y bins -frac((Z/2) u_y) (cycles)
    const double Z = z / lam;
    const double cyc = isx ? d_frac(d_frac(Z) - d_frac(0.5 * Z * u)) : -d_frac(0.5 * Z * u);
    double sn, cs;
    sincospi(2.0 * cyc, &sn, &cs);
    b.er = (float)cs;
    b.ei = (float)sn;
    (isx ? t.xc[(long)p * a.nx + k] : t.yc[(long)p * a.ny + k]) = (float)cyc;
    double w = 1.0;
    if (a.band_limit) {
      const double lim0 = d_local_frequency_limit(n, d, lam, z);
      const double nyq = 1.0 / (2.0 * d);
      const double lim = fmin(lim0, nyq);
      w = d_soft_window(fabs(f), lim, lim * (1.0 - a.soft_edge));
    }
    b.w = (float)w;
    if (isx) {
      t.xt[(long)p * a.nx + k] = b;
      if (p == 0) t.xf2[k] = f2;
    } else {
      t.yt[(long)p * a.ny + k] = b;
      if (p == 0) t.yf2[k] = f2;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    AsmPlane P;
    P.z = z;
    P.invL2 = 1.0 / (lam * lam);
    const double Z = z / lam;
    P.c0 = (float)d_frac(Z);
    P.hz = (float)(0.5 * Z);
    // largest u in [0, 0.999] with |Z/2| u^2 / (1 + sqrt(1-u))^2 <= 2 (bisection)
    const double hz = fabs(0.5 * Z);
    double lo = 0.0, hi = 0.999;
    const auto g = [&](double u) { const double s = 1.0 + sqrt(1.0 - u); return hz * u * u / (s * s); };
    if (g(hi) <= 2.0) {
      lo = hi;
    } else {
      for (int it = 0; it < 60; ++it) {
        const double m = 0.5 * (lo + hi);
        if (g(m) <= 2.0) lo = m; else hi = m;
      }
    }
    P.ucut = (float)lo;
    P.evanescent = a.evanescent;
    t.pl[p] = P;
  }
}

// FP64 evaluation for pixels beyond the FP32 fast-path range (u > ucut):
// exact reference classification (src/propagate.js:80-98) and FP64 phase.
static __device__ __forceinline__ float2 asm_h_slow(const AsmPlane* __restrict__ pl, const double* __restrict__ xf2,
                                          const double* __restrict__ yf2, int ky, float w) {
  const AsmPlane& P = *pl;
  const double arg = (P.invL2 - *xf2) - yf2[ky];
  double cyc;
  if (arg >= 0.0) {
    cyc = P.z * sqrt(arg);
  } else if (P.evanescent) {
    return make_float2(0.f, 0.f);
  } else {
    cyc = P.z * sqrt(-arg);
  }
  float c = (float)d_frac(cyc);
  c -= rintf(c);
  float sn, cs;
  sincospif(2.f * c, &sn, &cs);
  return make_float2(w * cs, w * sn);
}

// Invariants of one column (fixed bin kx) of plane p, loaded once per thread.
struct AsmCol {
  float er, ei, u, w;   // x-bin factor, u_x, window
  const AxisBin* yt;    // y-bins of plane p
  float hz, ucut;
  int p, kx;
};

__device__ __forceinline__ AsmCol asm_col(const AsmTables& t, int nx, int ny, int p, int kx) {
  const AxisBin bx = t.xt[(long)p * nx + kx];
  AsmCol c;
  c.er = bx.er;
  c.ei = bx.ei;
  c.u = bx.u;
  c.w = bx.w;
  c.yt = t.yt + (long)p * ny;
  c.hz = t.pl[p].hz;
  c.ucut = t.pl[p].ucut;
  c.p = p;
  c.kx = kx;
  return c;
}

// Transfer function at bin (c.kx, ky).
__device__ __forceinline__ float2 asm_h_col(const AsmCol& c, const AsmTables& t, int ky) {
  const float4 b4 = __ldg(reinterpret_cast<const float4*>(c.yt + ky));  // {er, ei, u, w}
  const AxisBin by{b4.x, b4.y, b4.z, b4.w};
  const float w = c.w * by.w;
  const float u = c.u + by.u;
  const float om = fmaxf(1.f - u, 1e-3f);
  const float s = 1.f + om * rsqrtf(om);          // 1 + sqrt(1 - u)
  float q = __fdividef(c.hz * (u * u), s * s);      // Z u^2 / (2 (1 + sqrt(1-u))^2)
  q -= rintf(q);
  float sn, cs;
  __sincosf(-6.283185307179586f * q, &sn, &cs);     // |arg| <= pi
  const float2 e = cmul(cmul(make_float2(c.er, c.ei), make_float2(by.er, by.ei)), make_float2(cs, sn));
  float2 h = make_float2(w * e.x, w * e.y);
  if (u > c.ucut && w != 0.f) h = asm_h_slow(t.pl + c.p, t.xf2 + c.kx, t.yf2, ky, w);
  return h;
}

// Transfer function at unshifted FFT bin (kx, ky) of plane p.
__device__ __forceinline__ float2 asm_h(const AsmTables& t, int nx, int ny, int p, int kx, int ky) {
  return asm_h_col(asm_col(t, nx, ny, p, kx), t, ky);
}

inline int asm_tables_bytes(int nplanes, int nx, int ny, size_t* bytes) {
  size_t b = 0;
  b += sizeof(AxisBin) * (size_t)nplanes * nx;
  b += sizeof(AxisBin) * (size_t)nplanes * ny;
  b += sizeof(double) * (size_t)(nx + ny);
  b += sizeof(float) * (size_t)nplanes * (nx + ny);
  b += sizeof(AsmPlane) * (size_t)nplanes + 256;
  *bytes = b;
  return 0;
}

// Layout from a 256-byte-aligned base: plane scalars (rounded to 256 B), then the
// 16-byte AxisBin arrays, then the FP64 arrays, then the FP32 cycle arrays, so
// every array keeps its natural alignment whatever nx and ny are (including axes
// of length 1).
inline AsmTables asm_tables_carve(void* base, int nplanes, int nx, int ny) {
  char* p = (char*)base;
  AsmTables t;
  t.pl = (AsmPlane*)p;
  p += ((sizeof(AsmPlane) * nplanes + 255) / 256) * 256;
  t.xt = (AxisBin*)p;
  p += sizeof(AxisBin) * (size_t)nplanes * nx;
  t.yt = (AxisBin*)p;
  p += sizeof(AxisBin) * (size_t)nplanes * ny;
  t.xf2 = (double*)p;
  p += sizeof(double) * nx;
  t.yf2 = (double*)p;
  p += sizeof(double) * ny;
  t.xc = (float*)p;
  p += sizeof(float) * (size_t)nplanes * nx;
  t.yc = (float*)p;
  return t;
}

// Build tables for `a.nplanes` planes into scratch slot kSlotTab (offset `slot_off`).
inline int asm_build_tables(doe_ctx* c, const AsmGroupArgs& a, AsmTables* out, int slot = kSlotTab) {
  size_t bytes;
  asm_tables_bytes(a.nplanes, a.nx, a.ny, &bytes);
  void* base;
  DOE_TRY(ensure_slot(c, slot, bytes, &base));
  *out = asm_tables_carve(base, a.nplanes, a.nx, a.ny);
  const int total = a.nx + a.ny;
  dim3 grid((total + 255) / 256, a.nplanes);
  LaunchScope ls(c, "asm_tables");
  asm_tables_kernel<<<grid, 256, 0, c->stream>>>(a, *out);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

}  // namespace doe
