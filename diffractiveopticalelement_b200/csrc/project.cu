// project.cu -- projector simulation and screen metrics
// (reference: src/projector.js:475-498 simulate, :554-595 screenMetrics subset,
// src/metrics.js:10-18 maskedSum, :73-84 rmsError).
//
// simulate: the element field A exp(i phi) is formed on the device inside the
// first row pass, optionally zero-padded (src/field.js:443-461 integer resample),
// propagated (angular spectrum) or lens-transformed, and cropped back.
// screen metrics: one pass of FP64 sums per design; the RMSE uses the expansion
// sum (I - sT)^2 = sum I^2 - 2 s sum I T + s^2 sum T^2 over the ROI, which costs
// ~1e-12 relative in FP64 at the 1e-2 RMSE level it is used for.
#include <cstring>
#include <vector>

#include "ops_propagate.cuh"

namespace doe {

// A exp(i phi) of an nx-by-ny element, centred inside an (nx*pad)-by-(ny*pad)
// zero grid (offset floor((N*pad - N)/2), src/field.js:446-447). ROT (pad 1)
// writes the ifftshifted element: out[X, Y] = element[(X + nx/2) % nx, ...].
__global__ void element_field_kernel(const double* __restrict__ A, const double* __restrict__ ph, int nx, int ny,
                                     int pad, int rot, float2* __restrict__ out) {
  const int NX = nx * pad, NY = ny * pad;
  const int ox = (NX - nx) / 2, oy = (NY - ny) / 2;
  const long total = (long)NX * NY;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int X = (int)(i % NX), Y = (int)(i / NX);
    const int x = rot ? ((X + (nx >> 1)) & (nx - 1)) : X - ox;
    const int y = rot ? ((Y + (ny >> 1)) & (ny - 1)) : Y - oy;
    float2 v = make_float2(0.f, 0.f);
    if (x >= 0 && x < nx && y >= 0 && y < ny) {
      const long k = x + (long)y * nx;
      double s, c;
      sincos(ph[k], &s, &c);
      v = make_float2((float)(A[k] * c), (float)(A[k] * s));
    }
    out[i] = v;
  }
}

// Centre crop of an (nx*pad)-by-(ny*pad) complex64 plane into FP64 planes.
__global__ void crop_to_f64_kernel(const float2* __restrict__ in, int nx, int ny, int pad, double* __restrict__ re,
                                   double* __restrict__ im) {
  const int NX = nx * pad, NY = ny * pad;
  const int ox = (NX - nx) / 2, oy = (NY - ny) / 2;
  const long total = (long)nx * ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)(i / nx);
    const float2 v = in[(x + ox) + (long)(y + oy) * NX];
    re[i] = v.x;
    im[i] = v.y;
  }
}

// Screen-metric sums of design p: intensity from FP32 amplitudes or complex64.
enum { kMIrrM = 0, kMT, kMIll, kMIrr, kMII, kMIT, kMTT, kMK };
struct MetricsArgs {
  int nx, ny;
  const float* amp;      // [B][n] amplitude (or null)
  const float* re;       // [B][n] field real part (when amp is null)
  const float* im;       // [B][n] field imaginary part
  const float* tgt_irr;  // [B][n] target irradiance
  const float* roi;      // [B][n] mask, or null
  const float* illum;    // [B][n] illumination amplitude
  long tgt_stride, ill_stride;
  double sdx, sdy, dx, dy;
  double* partials;
  unsigned* counters;
  double* totals;
  double* out;  // [B][6]: rmse, efficiency, fluxFraction, powerInSignal, powerAtScreen, powerIncident
};

__global__ void screen_metrics_kernel(MetricsArgs a) {
  const int p = blockIdx.y;
  const long n = (long)a.nx * a.ny;
  DAcc<kMK> acc;
#pragma unroll
  for (int k = 0; k < kMK; ++k) acc.v[k] = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double irr;
    if (a.amp) {
      const double am = a.amp[p * n + i];
      irr = am * am;
    } else {
      const double r = a.re[p * n + i], m = a.im[p * n + i];
      irr = r * r + m * m;
    }
    const double m = a.roi ? (double)a.roi[p * a.tgt_stride + i] : 1.0;
    const double T = a.tgt_irr[p * a.tgt_stride + i];
    acc.v[kMIrrM] += irr * m;
    acc.v[kMT] += T;
    acc.v[kMIll] += a.illum[p * a.ill_stride + i];
    acc.v[kMIrr] += irr;
    if (m > 0) {
      acc.v[kMII] += irr * irr;
      acc.v[kMIT] += irr * T;
      acc.v[kMTT] += T * T;
    }
  }
  if (!group_reduce<kMK>(acc, p, blockIdx.x, gridDim.x, a.partials, a.counters, a.totals) || threadIdx.x != 0) return;
  const double* S = a.totals + (long)p * kMK;
  const double cell = a.sdx * a.sdy;
  const double pt = S[kMIrrM] * cell, tt = S[kMT] * cell;
  const double s = tt > 0 ? pt / tt : 0.0;
  const double den = s * s * S[kMTT];
  const double num = fmax(0.0, S[kMII] - 2.0 * s * S[kMIT] + s * s * S[kMTT]);
  const double incident = S[kMIll] * a.dx * a.dy;
  const double total = S[kMIrr] * cell, inSignal = pt;
  double* o = a.out + (long)p * 6;
  o[0] = den > 0 ? sqrt(num / den) : 0.0;
  o[1] = incident > 0 ? inSignal / incident : 0.0;
  o[2] = total > 0 ? inSignal / total : 0.0;
  o[3] = inSignal;
  o[4] = total;
  o[5] = incident;
}

static unsigned grid_n(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

int screen_metrics_launch(doe_ctx* c, int B, MetricsArgs a, int slot) {
  const int blocks = (int)std::max<long>(1, std::min<long>(64, ((long)a.nx * a.ny + 255) / 256));
  void* p;
  DOE_TRY(ensure_slot(c, slot, sizeof(double) * ((size_t)B * blocks * kMK + (size_t)B * kMK) + 4 * B + 512, &p));
  a.partials = (double*)p;
  a.totals = a.partials + (size_t)B * blocks * kMK;
  a.counters = (unsigned*)(a.totals + (size_t)B * kMK);
  DOE_CUDA(c, cudaMemsetAsync(a.counters, 0, sizeof(unsigned) * B, c->stream));
  LaunchScope ls(c, "screen_metrics");
  screen_metrics_kernel<<<dim3(blocks, B), 256, 0, c->stream>>>(a);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

__global__ void f64_to_f32_kernel2(const double* __restrict__ in, float* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

}  // namespace doe

using namespace doe;

extern "C" int doe_simulate(doe_ctx* c, const double* illumination, const double* phase, int nx, int ny, double dx,
                            double dy, double lambda, double z, int band_limit, int far_field, int pad,
                            double* out_re, double* out_im, double* out_d) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "ProjectorSystem.simulate"));
  if (!illumination || !phase || !out_re || !out_im) return set_err(c, DOE_ERR_BAD_ARG, "simulate: null plane");
  if (pad < 1 || (pad & (pad - 1))) return set_err(c, DOE_ERR_BAD_ARG, "simulate: pad must be a power of two");
  if (far_field && !(z > 0)) return set_err(c, DOE_ERR_BAD_ARG, "ProjectorSystem.simulate: far-field mode needs a positive throw");
  if (far_field) pad = 1;  // src/projector.js:481-490 (no padding in the lens geometry)
  DOE_TRY(check_grid(c, nx * pad, ny * pad, "ProjectorSystem.simulate"));
  const long n = (long)nx * ny, NX = (long)nx * pad, NY = (long)ny * pad, N = NX * NY;
  void *pin, *pw, *pw2;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &pin));
  DOE_TRY(ensure_slot(c, kSlotW0, N * sizeof(float2), &pw));
  DOE_TRY(ensure_slot(c, kSlotW1, N * sizeof(float2), &pw2));
  double* dA = (double*)pin;
  double* dP = dA + n;
  float2* w = (float2*)pw;
  float2* w2 = (float2*)pw2;
  DOE_TRY(host_upload(c, dA, illumination, n * sizeof(double)));
  DOE_TRY(host_upload(c, dP, phase, n * sizeof(double)));
  {
    LaunchScope ls(c, "element_field");
    element_field_kernel<<<grid_n(N), 256, 0, c->stream>>>(dA, dP, nx, ny, pad, far_field ? 1 : 0, w);
    DOE_CUDA(c, cudaGetLastError());
  }
  void* pout;
  DOE_TRY(ensure_slot(c, kSlotOut, 2 * n * sizeof(double), &pout));
  double* ore = (double*)pout;
  double* oim = ore + n;
  if (far_field) {
    // focalPlaneSpectrum (src/propagate.js:342-374): rotate on load, forward FFT,
    // rotate + chirp on store
    const double dux = (lambda * z) / (nx * dx), duy = (lambda * z) / (ny * dy);
    const double amp0 = (dx * dy) / (lambda * z);
    std::vector<float> hc(nx + ny);
    for (int i = 0; i < nx; ++i) {
      const double u = (i - nx / 2.0) * dux, cyc = (u * u) / (2.0 * lambda * z);
      hc[i] = (float)(cyc - std::nearbyint(cyc));
    }
    for (int j = 0; j < ny; ++j) {
      const double v = (j - ny / 2.0) * duy, cyc = (v * v) / (2.0 * lambda * z);
      hc[nx + j] = (float)(cyc - std::nearbyint(cyc));
    }
    void* pt;
    DOE_TRY(ensure_slot(c, kSlotTab, (nx + ny) * sizeof(float), &pt));
    float* cxy = (float*)pt;
    DOE_TRY(host_upload(c, cxy, hc.data(), (nx + ny) * sizeof(float)));
    // the element was written ifftshifted; forward rows, then columns with the
    // fftshift + chirp on store
    DOE_TRY(with_row0(nx, [&](auto S) {
      return launch_row<decltype(S)>(c, RowC64<false>{{}, w, w2, nx, ny, n, n, 1.f}, 1, ny);
    }));
    DOE_TRY(with_col0(ny, [&](auto S) {
      return launch_col<decltype(S)>(c, ColFocal{{}, w2, ore, oim, cxy, cxy + nx, nx, ny, (float)amp0}, 1, nx);
    }));
    if (out_d) {
      out_d[0] = dux;
      out_d[1] = duy;
    }
  } else {
    if (z != 0) {
      AsmGroupArgs a = group_args((int)NX, (int)NY, dx, dy, band_limit, 1, 0.02);
      a.nplanes = 1;
      a.lam[0] = lambda;
      a.z[0] = z;
      AsmTables tab;
      DOE_TRY(asm_build_tables(c, a, &tab));
      DOE_TRY(asm_c64_inplace(c, w, 1, tab, (int)NX, (int)NY, w2));
    }
    LaunchScope ls(c, "crop");
    crop_to_f64_kernel<<<grid_n(n), 256, 0, c->stream>>>(w, nx, ny, pad, ore, oim);
    DOE_CUDA(c, cudaGetLastError());
    if (out_d) {
      out_d[0] = dx;
      out_d[1] = dy;
    }
  }
  DOE_TRY(host_download(c, out_re, ore, n * sizeof(double)));
  DOE_TRY(host_download(c, out_im, oim, n * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

extern "C" int doe_screen_metrics(doe_ctx* c, const double* re, const double* im, int nx, int ny, double sdx,
                                  double sdy, const double* target_irr, const double* roi, const double* illumination,
                                  double dx, double dy, double* out) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "screenMetrics"));
  if (!re || !im || !target_irr || !illumination || !out)
    return set_err(c, DOE_ERR_BAD_ARG, "screenMetrics: null plane");
  const long n = (long)nx * ny;
  const int nf = roi ? 5 : 4;
  void *pin, *pf;
  DOE_TRY(ensure_slot(c, kSlotIn, (size_t)n * nf * sizeof(double), &pin));
  DOE_TRY(ensure_slot(c, kSlotOut, (size_t)n * (nf + 1) * sizeof(float) + 64 * sizeof(double), &pf));
  double* din = (double*)pin;
  // each plane straight from the caller's array (no host-side gather)
  const double* planes[5] = {re, im, target_irr, illumination, roi};
  for (int k = 0; k < nf; ++k)
    DOE_TRY(host_upload(c, din + (size_t)k * n, planes[k], n * sizeof(double)));
  float* f = (float*)pf;
  // complex64 field (interleaved) from the FP64 planes, FP32 copies of the rest
  {
    LaunchScope ls(c, "f64_to_f32");
    f64_to_f32_kernel2<<<grid_n(n * nf), 256, 0, c->stream>>>(din, f, n * nf);
    DOE_CUDA(c, cudaGetLastError());
  }
  double* dout = (double*)(f + (size_t)n * (nf + 1));
  dout = (double*)(((uintptr_t)dout + 255) & ~(uintptr_t)255);
  MetricsArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = nx;
  a.ny = ny;
  a.re = f;
  a.im = f + n;
  a.tgt_irr = f + 2 * n;
  a.illum = f + 3 * n;
  a.roi = roi ? f + 4 * n : nullptr;
  a.tgt_stride = n;
  a.ill_stride = n;
  a.sdx = sdx;
  a.sdy = sdy;
  a.dx = dx;
  a.dy = dy;
  a.out = dout;
  DOE_TRY(screen_metrics_launch(c, 1, a, kSlotParams));
  DOE_TRY(host_download(c, out, dout, 6 * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

// Batched screen metrics of device-resident designs from their screen amplitudes
// (image-plane designs: the returned amplitude is the screen field's modulus).
extern "C" int doe_screen_metrics_dev(doe_ctx* c, int B, int nx, int ny, const float* amp, const float* target_irr,
                                      long long target_stride, const float* roi, const float* illumination,
                                      long long illumination_stride, double sdx, double sdy, double dx, double dy,
                                      double* out) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "screenMetrics"));
  if (B <= 0 || B > 65535 || !amp || !target_irr || !illumination || !out)
    return set_err(c, DOE_ERR_BAD_ARG, "screenMetrics: bad argument");
  MetricsArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = nx;
  a.ny = ny;
  a.amp = amp;
  a.tgt_irr = target_irr;
  a.roi = roi;
  a.illum = illumination;
  a.tgt_stride = (long)target_stride;
  a.ill_stride = (long)illumination_stride;
  a.sdx = sdx;
  a.sdy = sdy;
  a.dx = dx;
  a.dy = dy;
  a.out = out;
  return screen_metrics_launch(c, B, a, kSlotParams);
}
