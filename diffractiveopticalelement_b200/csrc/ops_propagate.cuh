// ops_propagate.cuh -- fused operators of the transform and propagation passes
// (reference: src/fft.js, src/propagate.js).
//
// Every propagation is three fused passes over the plane:
//   row pass     : load (FP64 host mirror or complex64), forward row FFT
//   column pass  : forward column FFT -> x H(fx, fy) -> inverse column FFT
//   row pass     : inverse row FFT, scale 1/(nx ny), store
// The reference's ifftshift/fftshift pairs around the FFTs cancel for even
// lengths because propagation is a convolution; H is therefore sampled directly
// at each unshifted bin's centred frequency (same values as src/propagate.js:73-77).
#pragma once
#include <cmath>
#include <functional>

#include "asm.cuh"

namespace doe {

// ------------------------------------------------------------------ operators
// Each operator's init() resolves the line's base pointers once per thread;
// load/mid/store then index by element position only.

// FP64 split planes -> complex64 work (rows), with optional quadrant rotation.
template <bool INV>
struct RowF64In : NoReduce {
  static constexpr const char* kName = INV ? "row_f64_in_inv" : "row_f64_in_fwd";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const double* re;
  const double* im;
  float2* w;
  int nx, ny, rx, ry;  // rx/ry: rotation of the source index (0 or n/2)
  struct State {
    const double* re;
    const double* im;
    float2* w;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long pe = (long)nx * ny;
    const long src = p * pe + (long)((y + ry) & (ny - 1)) * nx;
    return {re + src, im + src, w + p * pe + (long)y * nx};
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const {
    const int xs = (x + rx) & (nx - 1);
    return make_float2((float)s.re[xs], (float)s.im[xs]);
  }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const { s.w[x] = v; }
};

// complex64 -> complex64 rows (optionally scaled).
template <bool INV>
struct RowC64 : NoReduce {
  static constexpr const char* kName = INV ? "fft_row_inv" : "fft_row_fwd";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* in;
  float2* out;
  int nx, ny;
  long in_plane_stride, out_plane_stride;
  float scale;
  struct State {
    const float2* in;
    float2* out;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    return {in + p * in_plane_stride + (long)y * nx, out + p * out_plane_stride + (long)y * nx};
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.in[x]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const { s.out[x] = cscale(v, scale); }
};

// complex64 -> complex64 columns (optionally scaled).
template <bool INV>
struct ColC64 : NoReduce {
  static constexpr const char* kName = INV ? "fft_col_inv" : "fft_col_fwd";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* in;
  float2* out;
  int nx, ny;
  long in_plane_stride, out_plane_stride;
  float scale;
  struct State {
    const float2* in;
    float2* out;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    return {in + p * in_plane_stride + x, out + p * out_plane_stride + x};
  }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.in[(long)y * nx]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const {
    s.out[(long)y * nx] = cscale(v, scale);
  }
};

// complex64 work -> FP64 split planes (columns), scaled.
template <bool INV>
struct ColToF64 : NoReduce {
  static constexpr const char* kName = "col_to_f64";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  int nx, ny;
  float scale;
  struct State {
    const float2* w;
    double* re;
    double* im;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    const long o = p * (long)nx * ny + x;
    return {w + o, re + o, im + o};
  }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.w[(long)y * nx]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const {
    s.re[(long)y * nx] = (double)(v.x * scale);
    s.im[(long)y * nx] = (double)(v.y * scale);
  }
};

// Column pass of a propagation: forward column FFT, x H, inverse column FFT.
struct ColAsm : NoReduce {
  static constexpr const char* kName = "asm_col";
  static constexpr int kStages = 2;
  static constexpr bool kInv1 = false, kInv2 = true;
  const float2* in;
  float2* out;
  AsmTables tab;
  int nx, ny;
  struct State {
    const float2* in;
    float2* out;
    AsmCol h;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    const long o = p * (long)nx * ny + x;
    return {in + o, out + o, asm_col(tab, nx, ny, p, x)};
  }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.in[(long)y * nx]; }
  __device__ __forceinline__ void mid(const State& s, int y, float2& v, Acc&) const { v = cmul(v, asm_h_col(s.h, tab, y)); }
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const { s.out[(long)y * nx] = v; }
};

// Column pass of a focus sweep from a resident spectrum: x H then inverse FFT.
// Output plane p of the launch uses transfer-function table plane tp0 + p.
struct ColSweepBase : NoReduce {
  static constexpr const char* kName = "asm_sweep_col";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  const float2* spec;  // one spectrum plane (unshifted)
  float2* out;
  AsmTables tab;
  int nx, ny, tp0;
  struct State {
    const float2* spec;
    float2* out;
    AsmCol h;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    return {spec + x, out + p * (long)nx * ny + x, asm_col(tab, nx, ny, tp0 + p, x)};
  }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const { s.out[(long)y * nx] = v; }
};
// Every spectrum read of the thread first, then the transfer function.
struct ColSweep : ColSweepBase {
  __device__ __forceinline__ float2 load(const State& s, int y) const { return __ldg(&s.spec[(long)y * nx]); }
  __device__ __forceinline__ float2 finish_load(const State& s, int y, float2 v) const {
    return cmul(v, asm_h_col(s.h, tab, y));
  }
};
// Read and factor in one step per element. The autotuner keeps whichever of the
// two formulations is faster on the device.
struct ColSweepFused : ColSweepBase {
  __device__ __forceinline__ float2 load(const State& s, int y) const {
    return cmul(__ldg(&s.spec[(long)y * nx]), asm_h_col(s.h, tab, y));
  }
};

// Inverse row pass -> FP64 split planes with 1/(nx ny).
struct RowInvToF64 : NoReduce {
  static constexpr const char* kName = "row_inv_f64";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  int nx, ny;
  long out_plane_stride;
  float scale;
  struct State {
    const float2* w;
    double* re;
    double* im;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * out_plane_stride + (long)y * nx;
    return {w + p * (long)nx * ny + (long)y * nx, re + o, im + o};
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const { return s.w[x]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const {
    s.re[x] = (double)(v.x * scale);
    s.im[x] = (double)(v.y * scale);
  }
};

// Focal-plane column pass: forward column FFT, then fftshift + chirp + amp0
// (src/propagate.js:346-369); the chirp phase is (u^2+v^2)/(2 lambda f) - 1/4
// cycles, separable, with per-axis parts reduced mod 1 in FP64 (cx, cy).
struct ColFocal : NoReduce {
  static constexpr const char* kName = "focal_col";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = false, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  const float* cx;  // [nx] indexed by centred output column
  const float* cy;  // [ny]
  int nx, ny;
  float amp0;
  struct State {
    const float2* w;
    double* re;
    double* im;
    float cxi;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    const int i = (x + (nx >> 1)) & (nx - 1);
    const long o = p * (long)nx * ny;
    return {w + o + x, re + o + i, im + o + i, cx[i]};
  }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.w[(long)y * nx]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const {
    const int j = (y + (ny >> 1)) & (ny - 1);
    float c = s.cxi + cy[j] - 0.25f;
    c -= rintf(c);
    float sn, cs;
    sincospif(2.f * c, &sn, &cs);
    const float2 z = cmul(v, make_float2(amp0 * cs, amp0 * sn));
    s.re[(long)j * nx] = (double)z.x;
    s.im[(long)j * nx] = (double)z.y;
  }
};

// Single-FFT Fresnel transforms (src/propagate.js:155-316). Both quadratic
// factors are separable: cycles(x, y) = cx[x] + cy[y], each axis term reduced
// mod 1 in FP64 on the host with the checkerboard (-1)^(i+j) folded in as half a
// cycle on odd indices and the sign of the chirp (forward +, inverse -) applied.
// Row pass: FP64 split planes x chirp, row FFT.
template <bool INV>
struct RowChirpIn : NoReduce {
  static constexpr const char* kName = INV ? "fresnel_row_inv" : "fresnel_row_fwd";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const double* re;
  const double* im;
  float2* w;
  const float* cx;  // [nx] cycles
  const float* cy;  // [ny]
  int nx, ny;
  struct State {
    const double* re;
    const double* im;
    float2* w;
    float cyj;
  };
  __device__ __forceinline__ State init(int p, int y) const {
    const long o = p * (long)nx * ny + (long)y * nx;
    return {re + o, im + o, w + o, cy[y]};
  }
  __device__ __forceinline__ float2 load(const State& s, int x) const {
    const float2 u = make_float2((float)s.re[x], (float)s.im[x]);
    float c = __ldg(&cx[x]) + s.cyj;
    c -= rintf(c);
    float sn, cs;
    sincospif(2.f * c, &sn, &cs);
    return cmul(u, make_float2(cs, sn));
  }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int x, float2 v, Acc&) const { s.w[x] = v; }
};

// Column pass: column FFT, x pre (prefactor incl. any 1/N) x output chirp, FP64 out.
template <bool INV>
struct ColChirpOut : NoReduce {
  static constexpr const char* kName = INV ? "fresnel_col_inv" : "fresnel_col_fwd";
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  const float* cu;  // [nx] cycles
  const float* cv;  // [ny]
  int nx, ny;
  float2 pre;
  struct State {
    const float2* w;
    double* re;
    double* im;
    float cux;
  };
  __device__ __forceinline__ State init(int p, int x) const {
    const long o = p * (long)nx * ny + x;
    return {w + o, re + o, im + o, cu[x]};
  }
  __device__ __forceinline__ float2 load(const State& s, int y) const { return s.w[(long)y * nx]; }
  __device__ __forceinline__ void mid(const State&, int, float2&, Acc&) const {}
  __device__ __forceinline__ void store(const State& s, int y, float2 v, Acc&) const {
    float c = s.cux + __ldg(&cv[y]);
    c -= rintf(c);
    float sn, cs;
    sincospif(2.f * c, &sn, &cs);
    const float2 z = cmul(cmul(v, pre), make_float2(cs, sn));
    s.re[(long)y * nx] = (double)z.x;
    s.im[(long)y * nx] = (double)z.y;
  }
};

// Shared entry points implemented in prop_*.cu.
int fft2d_c64(doe_ctx* c, float2* d, int nx, int ny, int nplanes, bool inverse);
int asm_c64_inplace(doe_ctx* c, float2* d, int nplanes, const AsmTables& tab, int nx, int ny, float2* work);
AsmGroupArgs group_args(int nx, int ny, double dx, double dy, int band_limit, int evanescent, double soft_edge);
int upload_f64(doe_ctx* c, double* d, const double* h, size_t n);
int download_f64(doe_ctx* c, double* h, const double* d, size_t n);

}  // namespace doe
