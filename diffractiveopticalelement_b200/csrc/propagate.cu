// propagate.cu -- fft2d, angular-spectrum propagation, focus sweep and the lens
// focal-plane transform (reference: src/fft.js, src/propagate.js).
//
// Every propagation is three fused passes over the plane:
//   row pass     : load (FP64 host mirror or complex64), forward row FFT
//   column pass  : forward column FFT -> x H(fx, fy) -> inverse column FFT
//   row pass     : inverse row FFT, scale 1/(nx ny), store
// The reference's ifftshift/fftshift pairs around the FFTs cancel for even
// lengths because propagation is a convolution; H is therefore sampled directly
// at each unshifted bin's centred frequency (same values as src/propagate.js:73-77).
#include <cmath>

#include "asm.cuh"

namespace doe {

// ------------------------------------------------------------------ operators
// FP64 split planes -> complex64 work, with optional quadrant rotation (shift).
template <bool INV>
struct RowF64In : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const double* re;
  const double* im;
  float2* w;
  int nx, ny, rx, ry;  // rx/ry: rotation of the source index (0 or n/2)
  __device__ __forceinline__ float2 load(int p, int y, int x) const {
    const long pe = (long)nx * ny;
    const long s = p * pe + (long)((y + ry) & (ny - 1)) * nx + ((x + rx) & (nx - 1));
    return make_float2((float)re[s], (float)im[s]);
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int y, int x, float2 v, Acc&) const {
    w[p * (long)nx * ny + (long)y * nx + x] = v;
  }
};

// complex64 planes -> complex64 work (forward or inverse rows).
template <bool INV>
struct RowC64 : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* in;
  float2* out;
  int nx, ny;
  long in_plane_stride, out_plane_stride;
  float scale;
  __device__ __forceinline__ float2 load(int p, int y, int x) const {
    return in[p * in_plane_stride + (long)y * nx + x];
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int y, int x, float2 v, Acc&) const {
    out[p * out_plane_stride + (long)y * nx + x] = cscale(v, scale);
  }
};

// complex64 work -> complex64 (columns), single transform.
template <bool INV>
struct ColC64 : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* in;
  float2* out;
  int nx, ny;
  long in_plane_stride, out_plane_stride;
  float scale;
  __device__ __forceinline__ float2 load(int p, int x, int y) const {
    return in[p * in_plane_stride + (long)y * nx + x];
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int x, int y, float2 v, Acc&) const {
    out[p * out_plane_stride + (long)y * nx + x] = cscale(v, scale);
  }
};

// complex64 work -> FP64 split planes (columns), single transform, scaled.
template <bool INV>
struct ColToF64 : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = INV, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  int nx, ny;
  float scale;
  __device__ __forceinline__ float2 load(int p, int x, int y) const {
    return w[p * (long)nx * ny + (long)y * nx + x];
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int x, int y, float2 v, Acc&) const {
    const long i = p * (long)nx * ny + (long)y * nx + x;
    re[i] = (double)(v.x * scale);
    im[i] = (double)(v.y * scale);
  }
};

// Column pass of a propagation: forward column FFT, x H, inverse column FFT.
// Source plane of output plane p is p / src_div (focus sweeps share one spectrum).
struct ColAsm : NoReduce {
  static constexpr int kStages = 2;
  static constexpr bool kInv1 = false, kInv2 = true;
  const float2* in;
  float2* out;
  AsmTables tab;
  int nx, ny, src_div;
  __device__ __forceinline__ float2 load(int p, int x, int y) const {
    return in[(long)(p / src_div) * nx * ny + (long)y * nx + x];
  }
  __device__ __forceinline__ void mid(int p, int x, int y, float2& v) const {
    v = cmul(v, asm_h(tab, nx, ny, p, x, y));
  }
  __device__ __forceinline__ void store(int p, int x, int y, float2 v, Acc&) const {
    out[p * (long)nx * ny + (long)y * nx + x] = v;
  }
};

// Column pass of a focus sweep from a precomputed spectrum: x H then inverse.
struct ColSweep : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  const float2* spec;  // spectrum planes (unshifted)
  float2* out;
  AsmTables tab;
  int nx, ny, nz, plane0;  // output plane p of this launch is global plane plane0 + p
  __device__ __forceinline__ float2 load(int p, int x, int y) const {
    const int g = plane0 + p;
    const float2 s = spec[(long)(g / nz) * nx * ny + (long)y * nx + x];
    return cmul(s, asm_h(tab, nx, ny, p, x, y));
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int x, int y, float2 v, Acc&) const {
    out[p * (long)nx * ny + (long)y * nx + x] = v;
  }
};

// Inverse row pass -> FP64 split planes with 1/(nx ny).
struct RowInvToF64 : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = true, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  int nx, ny;
  long out_plane_stride;
  float scale;
  __device__ __forceinline__ float2 load(int p, int y, int x) const {
    return w[p * (long)nx * ny + (long)y * nx + x];
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int y, int x, float2 v, Acc&) const {
    const long i = p * out_plane_stride + (long)y * nx + x;
    re[i] = (double)(v.x * scale);
    im[i] = (double)(v.y * scale);
  }
};

// Focal-plane column pass: forward column FFT, then fftshift + chirp + amp0
// (src/propagate.js:346-369); the chirp phase is (u^2+v^2)/(2 lambda f) - 1/4
// cycles, separable, with per-axis parts reduced mod 1 in FP64 (cx, cy).
struct ColFocal : NoReduce {
  static constexpr int kStages = 1;
  static constexpr bool kInv1 = false, kInv2 = false;
  const float2* w;
  double* re;
  double* im;
  const float* cx;  // [nx] indexed by centred output column
  const float* cy;  // [ny]
  int nx, ny;
  float amp0;
  __device__ __forceinline__ float2 load(int p, int x, int y) const {
    return w[p * (long)nx * ny + (long)y * nx + x];
  }
  __device__ __forceinline__ void mid(int, int, int, float2&) const {}
  __device__ __forceinline__ void store(int p, int x, int y, float2 v, Acc&) const {
    const int i = (x + (nx >> 1)) & (nx - 1);
    const int j = (y + (ny >> 1)) & (ny - 1);
    float c = cx[i] + cy[j] - 0.25f;
    c -= rintf(c);
    float sn, cs;
    sincospif(2.f * c, &sn, &cs);
    const float2 z = cmul(v, make_float2(amp0 * cs, amp0 * sn));
    const long o = p * (long)nx * ny + (long)j * nx + i;
    re[o] = (double)z.x;
    im[o] = (double)z.y;
  }
};

// Centred transfer function as FP64 planes (angularSpectrumTransferFunction) and
// the propagating count (w > 0.5, or any non-evanescent bin when evanescent=0).
__global__ void asm_transfer_kernel(AsmTables t, int nx, int ny, double* hre, double* him,
                                    unsigned long long* count) {
  const long n = (long)nx * ny;
  unsigned long long local = 0;
  for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
    const int i = (int)(idx % nx), j = (int)(idx / nx);  // centred indices
    const int kx = (i + (nx - (nx >> 1))) % nx;        // unshifted bin whose centred index is i
    const int ky = (j + (ny - (ny >> 1))) % ny;
    const float2 h = asm_h(t, nx, ny, 0, kx, ky);
    hre[idx] = (double)h.x;
    him[idx] = (double)h.y;
    const double arg = (t.pl[0].invL2 - t.xf2[kx]) - t.yf2[ky];
    const double w = (double)t.xt[kx].w * (double)t.yt[ky].w;
    if (arg >= 0.0) {
      if (w > 0.5) ++local;
    } else if (!t.pl[0].evanescent) {
      ++local;
    }
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// ------------------------------------------------------------------ helpers
static int upload_f64(doe_ctx* c, double* d, const double* h, size_t n) {
  DOE_CUDA(c, cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  return DOE_OK;
}
static int download_f64(doe_ctx* c, double* h, const double* d, size_t n) {
  DOE_CUDA(c, cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  return DOE_OK;
}

static AsmGroupArgs group_args(int nx, int ny, double dx, double dy, int band_limit, int evanescent,
                               double soft_edge) {
  AsmGroupArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = nx;
  a.ny = ny;
  a.dx = dx;
  a.dy = dy;
  a.band_limit = band_limit;
  a.evanescent = evanescent;
  a.soft_edge = soft_edge;
  return a;
}

// 2-D FFT of nplanes complex64 planes: rows then columns.
int fft2d_c64(doe_ctx* c, float2* d, int nx, int ny, int nplanes, bool inverse) {
  const long pe = (long)nx * ny;
  const float scale = inverse ? 1.f / (float)pe : 1.f;
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if (inverse) {
      RowC64<true> op{{}, d, d, nx, ny, pe, pe, 1.f};
      return launch_row<N>(c, op, nplanes, ny);
    }
    RowC64<false> op{{}, d, d, nx, ny, pe, pe, 1.f};
    return launch_row<N>(c, op, nplanes, ny);
  }));
  return with_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if (inverse) {
      ColC64<true> op{{}, d, d, nx, ny, pe, pe, scale};
      return launch_col<N>(c, op, nplanes, nx);
    }
    ColC64<false> op{{}, d, d, nx, ny, pe, pe, scale};
    return launch_col<N>(c, op, nplanes, nx);
  });
}

// Propagate nplanes complex64 planes in place (used by the design loops too).
int asm_c64_inplace(doe_ctx* c, float2* d, int nplanes, const AsmTables& tab, int nx, int ny, float2* work) {
  const long pe = (long)nx * ny;
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    RowC64<false> op{{}, d, work, nx, ny, pe, pe, 1.f};
    return launch_row<N>(c, op, nplanes, ny);
  }));
  DOE_TRY(with_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    ColAsm op{{}, work, work, tab, nx, ny, 1};
    return launch_col<N>(c, op, nplanes, nx);
  }));
  return with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    RowC64<true> op{{}, work, d, nx, ny, pe, pe, 1.f / (float)pe};
    return launch_row<N>(c, op, nplanes, ny);
  });
}

}  // namespace doe

using namespace doe;

// ====================================================================== C ABI
extern "C" int doe_fft2d(doe_ctx* c, double* re, double* im, int nx, int ny, int inverse) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "fft2d"));
  if (!re || !im) return set_err(c, DOE_ERR_BAD_ARG, "fft2d: null plane");
  const size_t n = (size_t)nx * ny;
  void *din, *dw;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &din));
  DOE_TRY(ensure_slot(c, kSlotW0, n * sizeof(float2), &dw));
  double* dre = (double*)din;
  double* dim = dre + n;
  float2* w = (float2*)dw;
  DOE_TRY(upload_f64(c, dre, re, n));
  DOE_TRY(upload_f64(c, dim, im, n));
  const float scale = inverse ? 1.f / (float)n : 1.f;
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if (inverse) return launch_row<N>(c, RowF64In<true>{{}, dre, dim, w, nx, ny, 0, 0}, 1, ny);
    return launch_row<N>(c, RowF64In<false>{{}, dre, dim, w, nx, ny, 0, 0}, 1, ny);
  }));
  DOE_TRY(with_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    if (inverse) return launch_col<N>(c, ColToF64<true>{{}, w, dre, dim, nx, ny, scale}, 1, nx);
    return launch_col<N>(c, ColToF64<false>{{}, w, dre, dim, nx, ny, scale}, 1, nx);
  }));
  DOE_TRY(download_f64(c, re, dre, n));
  DOE_TRY(download_f64(c, im, dim, n));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

extern "C" int doe_asm_transfer(doe_ctx* c, int nx, int ny, double dx, double dy, double lambda, double z,
                                int band_limit, int evanescent, double soft_edge, double* h_re, double* h_im,
                                double* propagating_fraction) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "angularSpectrumTransferFunction"));
  if (!h_re || !h_im) return set_err(c, DOE_ERR_BAD_ARG, "angularSpectrumTransferFunction: null output");
  AsmGroupArgs a = group_args(nx, ny, dx, dy, band_limit, evanescent, soft_edge);
  a.nplanes = 1;
  a.lam[0] = lambda;
  a.z[0] = z;
  AsmTables tab;
  DOE_TRY(asm_build_tables(c, a, &tab));
  const size_t n = (size_t)nx * ny;
  void* dout;
  DOE_TRY(ensure_slot(c, kSlotOut, 2 * n * sizeof(double) + 64, &dout));
  double* hre = (double*)dout;
  double* him = hre + n;
  unsigned long long* cnt = (unsigned long long*)(him + n);
  DOE_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), c->stream));
  asm_transfer_kernel<<<296, 256, 0, c->stream>>>(tab, nx, ny, hre, him, cnt);
  DOE_CUDA(c, cudaGetLastError());
  unsigned long long hcnt = 0;
  DOE_TRY(download_f64(c, h_re, hre, n));
  DOE_TRY(download_f64(c, h_im, him, n));
  DOE_CUDA(c, cudaMemcpyAsync(&hcnt, cnt, sizeof(hcnt), cudaMemcpyDeviceToHost, c->stream));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (propagating_fraction) *propagating_fraction = (double)hcnt / (double)n;
  return DOE_OK;
}

extern "C" int doe_asm(doe_ctx* c, double* re, double* im, int nx, int ny, double dx, double dy, double lambda,
                       double z, int band_limit, int evanescent, double soft_edge) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "propagateAngularSpectrum"));
  if (!re || !im) return set_err(c, DOE_ERR_BAD_ARG, "propagateAngularSpectrum: null plane");
  if (z == 0) return DOE_OK;  // src/propagate.js:113
  const size_t n = (size_t)nx * ny;
  AsmGroupArgs a = group_args(nx, ny, dx, dy, band_limit, evanescent, soft_edge);
  a.nplanes = 1;
  a.lam[0] = lambda;
  a.z[0] = z;
  AsmTables tab;
  DOE_TRY(asm_build_tables(c, a, &tab));
  void *din, *dw;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &din));
  DOE_TRY(ensure_slot(c, kSlotW0, n * sizeof(float2), &dw));
  double* dre = (double*)din;
  double* dim = dre + n;
  float2* w = (float2*)dw;
  DOE_TRY(upload_f64(c, dre, re, n));
  DOE_TRY(upload_f64(c, dim, im, n));
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_row<N>(c, RowF64In<false>{{}, dre, dim, w, nx, ny, 0, 0}, 1, ny);
  }));
  DOE_TRY(with_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_col<N>(c, ColAsm{{}, w, w, tab, nx, ny, 1}, 1, nx);
  }));
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_row<N>(c, RowInvToF64{{}, w, dre, dim, nx, ny, (long)n, 1.f / (float)n}, 1, ny);
  }));
  DOE_TRY(download_f64(c, re, dre, n));
  DOE_TRY(download_f64(c, im, dim, n));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

// Focus sweep of one field whose forward spectrum `spec` (unshifted, complex64)
// is resident: planes k < nz at distances z[k], written either as complex64
// (out_c64, plane stride pe) or as FP64 split planes (out_re/out_im). Planes with
// z == 0 are the input field itself (src/propagate.js:113): copied from `src_c64`
// or from the FP64 input planes.
static int sweep_one_field(doe_ctx* c, const float2* spec, int nx, int ny, double dx, double dy, double lambda,
                           const double* z, int nz, int band_limit, int evanescent, double soft_edge,
                           float2* out_c64, const float2* src_c64, double* out_re, double* out_im,
                           const double* src_re, const double* src_im) {
  const long pe = (long)nx * ny;
  // Planes per launch: keep a group's intermediate planes L2-resident.
  const int G = (int)std::max<long>(1, std::min<long>(kMaxGroup, (32L << 20) / (pe * 8)));
  void* dw;
  DOE_TRY(ensure_slot(c, kSlotW1, (size_t)std::min(G, nz) * pe * sizeof(float2), &dw));
  float2* w = (float2*)dw;
  for (int g0 = 0; g0 < nz; g0 += G) {
    const int gn = std::min(G, nz - g0);
    AsmGroupArgs a = group_args(nx, ny, dx, dy, band_limit, evanescent, soft_edge);
    a.nplanes = gn;
    for (int i = 0; i < gn; ++i) {
      a.lam[i] = lambda;
      a.z[i] = z[g0 + i];
    }
    AsmTables tab;
    DOE_TRY(asm_build_tables(c, a, &tab));
    DOE_TRY(with_n(ny, [&](auto NC) {
      constexpr int N = decltype(NC)::value;
      return launch_col<N>(c, ColSweep{{}, spec, w, tab, nx, ny, 1 << 30, 0}, gn, nx);
    }));
    if (out_c64) {
      DOE_TRY(with_n(nx, [&](auto NC) {
        constexpr int N = decltype(NC)::value;
        return launch_row<N>(c, RowC64<true>{{}, w, out_c64 + (long)g0 * pe, nx, ny, pe, pe, 1.f / (float)pe}, gn,
                             ny);
      }));
    } else {
      DOE_TRY(with_n(nx, [&](auto NC) {
        constexpr int N = decltype(NC)::value;
        return launch_row<N>(
            c, RowInvToF64{{}, w, out_re + (long)g0 * pe, out_im + (long)g0 * pe, nx, ny, pe, 1.f / (float)pe}, gn,
            ny);
      }));
    }
    for (int i = 0; i < gn; ++i) {
      if (a.z[i] != 0.0) continue;
      const long o = (long)(g0 + i) * pe;
      if (out_c64) {
        DOE_CUDA(c, cudaMemcpyAsync(out_c64 + o, src_c64, pe * sizeof(float2), cudaMemcpyDeviceToDevice, c->stream));
      } else {
        DOE_CUDA(c, cudaMemcpyAsync(out_re + o, src_re, pe * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        DOE_CUDA(c, cudaMemcpyAsync(out_im + o, src_im, pe * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      }
    }
  }
  return DOE_OK;
}

extern "C" int doe_asm_sweep(doe_ctx* c, const double* re, const double* im, int nx, int ny, double dx, double dy,
                             double lambda, const double* z, int nz, int band_limit, int evanescent, double soft_edge,
                             double* out_re, double* out_im) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "focusSweep"));
  if (!re || !im || !z || !out_re || !out_im || nz < 0) return set_err(c, DOE_ERR_BAD_ARG, "focusSweep: bad argument");
  if (nz == 0) return DOE_OK;
  const size_t n = (size_t)nx * ny;
  void *din, *dspec, *dout;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &din));
  DOE_TRY(ensure_slot(c, kSlotW0, n * sizeof(float2), &dspec));
  DOE_TRY(ensure_slot(c, kSlotOut, 2 * n * (size_t)nz * sizeof(double), &dout));
  double* dre = (double*)din;
  double* dim = dre + n;
  float2* spec = (float2*)dspec;
  double* ore = (double*)dout;
  double* oim = ore + n * nz;
  DOE_TRY(upload_f64(c, dre, re, n));
  DOE_TRY(upload_f64(c, dim, im, n));
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_row<N>(c, RowF64In<false>{{}, dre, dim, spec, nx, ny, 0, 0}, 1, ny);
  }));
  DOE_TRY(with_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_col<N>(c, ColC64<false>{{}, spec, spec, nx, ny, (long)n, (long)n, 1.f}, 1, nx);
  }));
  DOE_TRY(sweep_one_field(c, spec, nx, ny, dx, dy, lambda, z, nz, band_limit, evanescent, soft_edge, nullptr,
                          nullptr, ore, oim, dre, dim));
  DOE_TRY(download_f64(c, out_re, ore, n * nz));
  DOE_TRY(download_f64(c, out_im, oim, n * nz));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

extern "C" int doe_asm_sweep_dev(doe_ctx* c, const void* d_fields, int nfields, int nx, int ny, double dx, double dy,
                                 const double* lambda, const double* z, int nz, int band_limit, int evanescent,
                                 double soft_edge, void* d_out) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "focusSweep"));
  if (!d_fields || !lambda || !z || !d_out || nfields < 0 || nz < 0)
    return set_err(c, DOE_ERR_BAD_ARG, "focusSweep: bad argument");
  const long pe = (long)nx * ny;
  void* dspec;
  DOE_TRY(ensure_slot(c, kSlotW0, pe * sizeof(float2), &dspec));
  float2* spec = (float2*)dspec;
  const float2* in = (const float2*)d_fields;
  float2* out = (float2*)d_out;
  for (int f = 0; f < nfields; ++f) {
    DOE_TRY(with_n(nx, [&](auto NC) {
      constexpr int N = decltype(NC)::value;
      return launch_row<N>(c, RowC64<false>{{}, in + f * pe, spec, nx, ny, pe, pe, 1.f}, 1, ny);
    }));
    DOE_TRY(with_n(ny, [&](auto NC) {
      constexpr int N = decltype(NC)::value;
      return launch_col<N>(c, ColC64<false>{{}, spec, spec, nx, ny, pe, pe, 1.f}, 1, nx);
    }));
    DOE_TRY(sweep_one_field(c, spec, nx, ny, dx, dy, lambda[f], z + (long)f * nz, nz, band_limit, evanescent,
                            soft_edge, out + (long)f * nz * pe, in + f * pe, nullptr, nullptr, nullptr, nullptr));
  }
  return DOE_OK;
}

extern "C" int doe_fft2d_dev(doe_ctx* c, void* d_planes, int nx, int ny, int nplanes, int inverse) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "fft2d"));
  if (!d_planes || nplanes < 0) return set_err(c, DOE_ERR_BAD_ARG, "fft2d: bad argument");
  return fft2d_c64(c, (float2*)d_planes, nx, ny, nplanes, inverse != 0);
}

extern "C" int doe_focal_plane(doe_ctx* c, const double* re, const double* im, int nx, int ny, double dx, double dy,
                               double lambda, double f, double* out_re, double* out_im, double* out_d) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "focalPlaneSpectrum"));
  if (!re || !im || !out_re || !out_im) return set_err(c, DOE_ERR_BAD_ARG, "focalPlaneSpectrum: null plane");
  const size_t n = (size_t)nx * ny;
  const double dux = (lambda * f) / (nx * dx);
  const double duy = (lambda * f) / (ny * dy);
  const double amp0 = (dx * dy) / (lambda * f);
  // chirp phase per axis in cycles, reduced mod 1 in FP64: u^2 / (2 lambda f)
  std::vector<float> hc(nx + ny);
  for (int i = 0; i < nx; ++i) {
    const double u = (i - nx / 2.0) * dux;
    const double cyc = (u * u) / (2.0 * lambda * f);
    hc[i] = (float)(cyc - std::nearbyint(cyc));
  }
  for (int j = 0; j < ny; ++j) {
    const double v = (j - ny / 2.0) * duy;
    const double cyc = (v * v) / (2.0 * lambda * f);
    hc[nx + j] = (float)(cyc - std::nearbyint(cyc));
  }
  void *din, *dw, *dtab;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &din));
  DOE_TRY(ensure_slot(c, kSlotW0, n * sizeof(float2), &dw));
  DOE_TRY(ensure_slot(c, kSlotTab, (nx + ny) * sizeof(float), &dtab));
  double* dre = (double*)din;
  double* dim = dre + n;
  float2* w = (float2*)dw;
  float* cxy = (float*)dtab;
  DOE_CUDA(c, cudaMemcpyAsync(cxy, hc.data(), (nx + ny) * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  DOE_TRY(upload_f64(c, dre, re, n));
  DOE_TRY(upload_f64(c, dim, im, n));
  // ifftshift on load (rotation by n/2), forward rows
  DOE_TRY(with_n(nx, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_row<N>(c, RowF64In<false>{{}, dre, dim, w, nx, ny, nx >> 1, ny >> 1}, 1, ny);
  }));
  DOE_TRY(with_n(ny, [&](auto NC) {
    constexpr int N = decltype(NC)::value;
    return launch_col<N>(c, ColFocal{{}, w, dre, dim, cxy, cxy + nx, nx, ny, (float)amp0}, 1, nx);
  }));
  DOE_TRY(download_f64(c, out_re, dre, n));
  DOE_TRY(download_f64(c, out_im, dim, n));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  if (out_d) {
    out_d[0] = dux;
    out_d[1] = duy;
  }
  return DOE_OK;
}
