// asm.cuh -- angular-spectrum transfer function evaluated on the fly.
//
// Reference: src/propagate.js:57-102 builds, on the centred frequency grid,
//   H = w_x w_y exp(i 2 pi z sqrt(1/lambda^2 - fx^2 - fy^2))   (0 if evanescent)
// with a raised-cosine band-limit window (src/propagate.js:38-51). The phase
// reaches ~1e5 cycles at z = 30-50 mm, so a plain FP32 product loses ~1e-2 rad.
// Here the phase in cycles is split exactly as
//   z sqrt(1/l^2 - f^2) = Z - (Z/2) u - Z u^2 / (2 (1 + sqrt(1-u))^2),
//   Z = z / lambda,  u = lambda^2 (fx^2 + fy^2) = ux + uy,
// where frac(Z) and frac((Z/2) u_axis) are reduced mod 1 in FP64 per plane / per
// axis bin (tables below) and only the small last term is evaluated in FP32 per
// pixel. Pixels whose last term would exceed 2 cycles (u > ucut), including every
// pixel near the evanescent boundary, take an FP64 path that mirrors the
// reference's `invL2 - fx*fx - fy*fy` test exactly. The reduced cycle count goes
// through FP32 sincospif.
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

// Per-bin axis entry: u = (lambda f)^2, p = frac((Z/2) u), w = band-limit window.
struct AxisBin {
  float u, p, w, pad;
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
__global__ void asm_tables_kernel(AsmGroupArgs a, AsmTables t) {
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
    b.p = (float)d_frac(0.5 * (z / lam) * u);
    double w = 1.0;
    if (a.band_limit) {
      const double lim0 = d_local_frequency_limit(n, d, lam, z);
      const double nyq = 1.0 / (2.0 * d);
      const double lim = fmin(lim0, nyq);
      w = d_soft_window(fabs(f), lim, lim * (1.0 - a.soft_edge));
    }
    b.w = (float)w;
    b.pad = 0.f;
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

// Transfer function at unshifted FFT bin (kx, ky) of plane p.
__device__ __forceinline__ float2 asm_h(const AsmTables& t, int nx, int ny, int p, int kx, int ky) {
  const AxisBin bx = t.xt[(long)p * nx + kx];
  const AxisBin by = t.yt[(long)p * ny + ky];
  const float w = bx.w * by.w;
  const AsmPlane& P = t.pl[p];
  const float u = bx.u + by.u;
  float c;
  if (u <= P.ucut) {
    const float s = 1.f + sqrtf(1.f - u);
    const float q = P.hz * (u * u) / (s * s);
    c = P.c0 - bx.p - by.p - q;
  } else {
    // exact reference classification and FP64 phase (src/propagate.js:80-98)
    const double arg = (P.invL2 - t.xf2[kx]) - t.yf2[ky];
    double cyc;
    if (arg >= 0.0) {
      cyc = P.z * sqrt(arg);
    } else if (P.evanescent) {
      return make_float2(0.f, 0.f);
    } else {
      cyc = P.z * sqrt(-arg);
    }
    c = (float)d_frac(cyc);
  }
  c -= rintf(c);
  float sn, cs;
  sincospif(2.f * c, &sn, &cs);
  return make_float2(w * cs, w * sn);
}

inline int asm_tables_bytes(int nplanes, int nx, int ny, size_t* bytes) {
  size_t b = 0;
  b += sizeof(AxisBin) * (size_t)nplanes * nx;
  b += sizeof(AxisBin) * (size_t)nplanes * ny;
  b += sizeof(double) * (size_t)(nx + ny);
  b += sizeof(AsmPlane) * (size_t)nplanes + 256;
  *bytes = b;
  return 0;
}

inline AsmTables asm_tables_carve(void* base, int nplanes, int nx, int ny) {
  char* p = (char*)base;
  AsmTables t;
  t.pl = (AsmPlane*)p;
  p += ((sizeof(AsmPlane) * nplanes + 255) / 256) * 256;
  t.xf2 = (double*)p;
  p += sizeof(double) * nx;
  t.yf2 = (double*)p;
  p += sizeof(double) * ny;
  t.xt = (AxisBin*)p;
  p += sizeof(AxisBin) * (size_t)nplanes * nx;
  t.yt = (AxisBin*)p;
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
  asm_tables_kernel<<<grid, 256, 0, c->stream>>>(a, *out);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

}  // namespace doe
