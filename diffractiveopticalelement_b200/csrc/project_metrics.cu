// project_metrics.cu -- every field of ProjectorSystem.screenMetrics on the device
// (reference: src/projector.js:554-614 with src/metrics.js:37-67 regionStats,
// :73-84 rmsError, :87-118 correlation, :145-157 zeroOrderFraction, :164-185
// rmsRadius, :198-259 ssim (window 8, target-weighted), :284-321 spotUniformity).
//
// Three FP64 passes over the screen: (1) the power, ROI, target, zero-order and
// radius sums and the peaks; (2) the thresholded region statistics, the centred
// correlation sums and the spot cells; (3) one thread per 8x8 SSIM window. Sums
// are folded per block in a fixed order (deterministic); maxima and minima of the
// non-negative intensities are exact (integer atomics on the FP64 bit patterns);
// the spot cells are FP64 atomic sums.
#include <cmath>
#include <cstring>
#include <vector>

#include "ops_propagate.cuh"

namespace doe {
namespace {

enum P1 { kIM = 0, kT, kIrr, kIll, kII, kIT, kTT, kCnt, kSP, kST, kZr, kZi, kZp, kRx, kRy, kP1 };
enum P2 { kRn = 0, kRs, kRss, kCov, kVp, kVt, kP2 };
enum PX { kMaxRoi = 0, kMaxAll, kMaxT, kMinR, kMaxR, kPX };

struct FullArgs {
  const double *re, *im, *tgt, *roi, *ill, *ph;
  int nx, ny;
  double sdx, sdy;
  // pass-2 inputs (from pass 1)
  double thr, s, mp, mt, cut;
  int cols, rows;
  double* partials;
  unsigned* counters;
  double* totals;
  unsigned long long* ext;  // kPX bit patterns
  double* cells;            // [cols*rows]
  // ssim
  double C1, C2;
};

// Maxima / minima of non-negative values: folded over the warp first, then one
// integer atomic per warp on the FP64 bit pattern (one atomic per thread on a
// single address serialises every thread of the grid at that address).
__device__ __forceinline__ void amax(unsigned long long* a, double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(a, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void amin(unsigned long long* a, double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMin(a, (unsigned long long)__double_as_longlong(v));
}

__global__ void metrics_pass1(FullArgs a) {
  const long n = (long)a.nx * a.ny;
  DAcc<kP1> acc;
#pragma unroll
  for (int k = 0; k < kP1; ++k) acc.v[k] = 0.0;
  double mroi = 0.0, mall = 0.0, mt = 0.0;
  // pixel coordinates advance with the grid stride (no division per pixel)
  const long i0 = blockIdx.x * (long)blockDim.x + threadIdx.x, stride = (long)gridDim.x * blockDim.x;
  const int sx = (int)(stride % a.nx), sy = (int)(stride / a.nx);
  int xi = (int)(i0 % a.nx), yi = (int)(i0 / a.nx);
  for (long i = i0; i < n; i += stride) {
    const double irr = a.re[i] * a.re[i] + a.im[i] * a.im[i];
    const double m = a.roi ? a.roi[i] : 1.0;
    const double T = a.tgt[i];
    acc.v[kIM] += irr * m;
    acc.v[kT] += T;
    acc.v[kIrr] += irr;
    acc.v[kIll] += a.ill[i];
    if (m > 0) {
      acc.v[kII] += irr * irr;
      acc.v[kIT] += irr * T;
      acc.v[kTT] += T * T;
      acc.v[kCnt] += 1.0;
      acc.v[kSP] += irr;
      acc.v[kST] += T;
      if (irr > 0) mroi = fmax(mroi, irr);
    }
    mall = fmax(mall, irr);
    mt = fmax(mt, T);
    double sn, cs;
    sincos(a.ph[i], &sn, &cs);
    const double zr = a.ill[i] * cs, zi = a.ill[i] * sn;
    acc.v[kZr] += zr;
    acc.v[kZi] += zi;
    acc.v[kZp] += zr * zr + zi * zi;
    const double x = (xi - a.nx / 2.0) * a.sdx, y = (yi - a.ny / 2.0) * a.sdy;
    acc.v[kRx] += irr * x * x;
    acc.v[kRy] += irr * y * y;
    xi += sx;
    yi += sy;
    if (xi >= a.nx) {
      xi -= a.nx;
      ++yi;
    }
  }
  amax(&a.ext[kMaxRoi], mroi);
  amax(&a.ext[kMaxAll], mall);
  amax(&a.ext[kMaxT], mt);
  group_reduce<kP1>(acc, 0, blockIdx.x, gridDim.x, a.partials, a.counters, a.totals);
}

__global__ void metrics_pass2(FullArgs a) {
  const long n = (long)a.nx * a.ny;
  DAcc<kP2> acc;
#pragma unroll
  for (int k = 0; k < kP2; ++k) acc.v[k] = 0.0;
  double mn = __longlong_as_double(0x7ff0000000000000LL), mx = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double irr = a.re[i] * a.re[i] + a.im[i] * a.im[i];
    const double m = a.roi ? a.roi[i] : 1.0;
    if (m > 0) {
      if (irr > a.thr) {
        acc.v[kRn] += 1.0;
        acc.v[kRs] += irr;
        acc.v[kRss] += irr * irr;
        mn = fmin(mn, irr);
        mx = fmax(mx, irr);
      }
      const double dp = irr - a.mp, dt = a.tgt[i] * a.s - a.mt;
      acc.v[kCov] += dp * dt;
      acc.v[kVp] += dp * dp;
      acc.v[kVt] += dt * dt;
    }
    if (a.cols > 0 && irr >= a.cut) {
      const int xi = (int)(i % a.nx), yi = (int)(i / a.nx);
      const int cj = min(a.rows - 1, (int)floor(((double)yi / a.ny) * a.rows));
      const int ci = min(a.cols - 1, (int)floor(((double)xi / a.nx) * a.cols));
      atomicAdd(&a.cells[ci + cj * a.cols], irr);
    }
  }
  amin(&a.ext[kMinR], mn);
  amax(&a.ext[kMaxR], mx);
  group_reduce<kP2>(acc, 1, blockIdx.x, gridDim.x, a.partials, a.counters, a.totals);
}

// one thread per 8x8 window: sum (ssim * w), sum w with w = mean target of the window
__global__ void metrics_ssim(FullArgs a, int wxn, int wyn) {
  DAcc<2> acc;
  acc.v[0] = acc.v[1] = 0.0;
  const long nw = (long)wxn * wyn;
  for (long w = blockIdx.x * (long)blockDim.x + threadIdx.x; w < nw; w += (long)gridDim.x * blockDim.x) {
    const int wx = (int)(w % wxn) * 8, wy = (int)(w / wxn) * 8;
    double sp = 0, st = 0, spp = 0, stt = 0, spt = 0;
    for (int j = 0; j < 8; ++j) {
      for (int i = 0; i < 8; ++i) {
        const long k = wx + i + (long)(wy + j) * a.nx;
        const double p = a.re[k] * a.re[k] + a.im[k] * a.im[k];
        const double t = a.tgt[k] * a.s;
        sp += p;
        st += t;
        spp += p * p;
        stt += t * t;
        spt += p * t;
      }
    }
    const double mp = sp / 64.0, mt = st / 64.0;
    const double vp = fabs(spp / 64.0 - mp * mp), vt = fabs(stt / 64.0 - mt * mt);
    const double cpt = spt / 64.0 - mp * mt;
    const double num = (2 * mp * mt + a.C1) * (2 * cpt + a.C2);
    const double den = (mp * mp + mt * mt + a.C1) * (vp + vt + a.C2);
    const double wt = st / 64.0;
    acc.v[0] += (den != 0 ? num / den : 0.0) * wt;
    acc.v[1] += wt;
  }
  group_reduce<2>(acc, 2, blockIdx.x, gridDim.x, a.partials, a.counters, a.totals);
}

unsigned blocks_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 4)); }

}  // namespace
}  // namespace doe

using namespace doe;

// out[18]: efficiency, fluxFraction, uniformity, spotUniformity (NaN without a
// grid), flatness, contrast, rmse, fidelity, correlation, ssim, snr, zeroOrder,
// rmsRadius, meanIntensity, peakIntensity, powerInSignal, powerAtScreen, powerIncident.
extern "C" int doe_screen_metrics_full(doe_ctx* c, const double* re, const double* im, int nx, int ny, double sdx,
                                       double sdy, const double* target_irr, const double* roi,
                                       const double* illumination, const double* phase, double dx, double dy,
                                       int grid_cols, int grid_rows, double* out) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "screenMetrics"));
  if (!re || !im || !target_irr || !illumination || !phase || !out)
    return set_err(c, DOE_ERR_BAD_ARG, "screenMetrics: null plane");
  if (grid_cols < 0 || grid_rows < 0 || (grid_cols > 0) != (grid_rows > 0) || grid_cols * (long)grid_rows > 65536)
    return set_err(c, DOE_ERR_BAD_ARG, "screenMetrics: bad spot grid %dx%d", grid_cols, grid_rows);
  const long n = (long)nx * ny;
  const int nf = roi ? 6 : 5;
  const unsigned G = blocks_for(n);
  const int cells = grid_cols * grid_rows;
  const size_t red = sizeof(double) * ((size_t)G * kP1 + 16 * 3) + 64 + sizeof(unsigned long long) * kPX +
                     sizeof(double) * (cells + 1) + 1024;
  void *pin, *pr;
  DOE_TRY(ensure_slot(c, kSlotIn, (size_t)n * nf * sizeof(double), &pin));
  DOE_TRY(ensure_slot(c, kSlotRed, red, &pr));
  double* d = (double*)pin;
  // each plane straight from the caller's array (no host-side gather)
  const double* planes[6] = {re, im, target_irr, illumination, phase, roi};
  for (int k = 0; k < nf; ++k) DOE_TRY(upload_f64(c, d + (size_t)k * n, planes[k], (size_t)n));
  char* q = (char*)pr;
  FullArgs a;
  memset(&a, 0, sizeof(a));
  a.re = d;
  a.im = d + n;
  a.tgt = d + 2 * n;
  a.ill = d + 3 * n;
  a.ph = d + 4 * n;
  a.roi = roi ? d + 5 * n : nullptr;
  a.nx = nx;
  a.ny = ny;
  a.sdx = sdx;
  a.sdy = sdy;
  a.partials = (double*)q;                                  // [G][kP1] (largest pass)
  a.totals = a.partials + (size_t)G * kP1;                  // 3 groups x 16
  a.counters = (unsigned*)(a.totals + 48);                  // 3 groups
  a.ext = (unsigned long long*)(((uintptr_t)(a.counters + 16) + 15) & ~(uintptr_t)15);
  a.cells = (double*)(a.ext + kPX + 1);
  a.cols = grid_cols;
  a.rows = grid_rows;
  // group g of pass p uses totals[g * K]: pass 1 group 0 (K=kP1 <= 16), pass 2 group 1 (K=kP2), ssim group 2 (K=2)
  unsigned long long ext0[kPX] = {0ull, 0ull, 0ull, 0x7ff0000000000000ull, 0ull};
  DOE_CUDA(c, cudaMemsetAsync(a.counters, 0, sizeof(unsigned) * 16, c->stream));
  DOE_TRY(host_upload(c, a.ext, ext0, sizeof(ext0)));
  if (cells) DOE_CUDA(c, cudaMemsetAsync(a.cells, 0, sizeof(double) * cells, c->stream));
  {
    LaunchScope ls(c, "screen_metrics_pass1");
    metrics_pass1<<<G, 256, 0, c->stream>>>(a);
    DOE_CUDA(c, cudaGetLastError());
  }
  double t1[kP1];
  unsigned long long e1[kPX];
  DOE_TRY(host_download(c, t1, a.totals, sizeof(t1)));
  DOE_TRY(host_download(c, e1, a.ext, sizeof(e1)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  double maxRoi, maxAll, maxT;
  memcpy(&maxRoi, &e1[kMaxRoi], 8);
  memcpy(&maxAll, &e1[kMaxAll], 8);
  memcpy(&maxT, &e1[kMaxT], 8);
  const double cell = sdx * sdy;
  const double pt = t1[kIM] * cell, tt = t1[kT] * cell;
  const double s = tt > 0 ? pt / tt : 0.0;
  a.thr = 0.1 * maxRoi;  // regionStats(irr, mask, {threshold: 0.1 * provisional max})
  a.s = s;
  a.mp = t1[kCnt] > 0 ? t1[kSP] / t1[kCnt] : 0.0;
  a.mt = t1[kCnt] > 0 ? (t1[kST] * s) / t1[kCnt] : 0.0;
  a.cut = 0.05 * maxAll;  // spotUniformity minPeak
  const double tmax = s >= 0 ? maxT * s : 0.0;
  const double L0 = fmax(maxAll, tmax);
  const double L = L0 > 0 ? L0 : 1.0;
  a.C1 = 0.01 * L * (0.01 * L);
  a.C2 = 0.03 * L * (0.03 * L);
  {
    LaunchScope ls(c, "screen_metrics_pass2");
    metrics_pass2<<<G, 256, 0, c->stream>>>(a);
    DOE_CUDA(c, cudaGetLastError());
  }
  const int wxn = nx / 8, wyn = ny / 8;
  if ((long)wxn * wyn > 0) {
    LaunchScope ls(c, "screen_metrics_ssim");
    metrics_ssim<<<blocks_for((long)wxn * wyn), 256, 0, c->stream>>>(a, wxn, wyn);
    DOE_CUDA(c, cudaGetLastError());
  }
  double tot[48];
  unsigned long long e2[kPX];
  std::vector<double> hc(cells);
  DOE_TRY(host_download(c, tot, a.totals, sizeof(tot)));
  DOE_TRY(host_download(c, e2, a.ext, sizeof(e2)));
  if (cells) DOE_TRY(host_download(c, hc.data(), a.cells, sizeof(double) * cells));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  const double* t2 = tot + kP2;       // group 1 of K = kP2
  const double* t3 = tot + 2 * 2;     // group 2 of K = 2
  double minR, maxR;
  memcpy(&minR, &e2[kMinR], 8);
  memcpy(&maxR, &e2[kMaxR], 8);
  // regionStats over the ROI above the threshold (src/metrics.js:37-67)
  double mean = 0, sd = 0, uni = 0, flat = 0, cv = 0, peak = 0;
  if (t2[kRn] > 0) {
    mean = t2[kRs] / t2[kRn];
    sd = std::sqrt(std::fmax(0.0, t2[kRss] / t2[kRn] - mean * mean));
    uni = maxR + minR > 0 ? 1 - (maxR - minR) / (maxR + minR) : 1;
    flat = mean > 0 ? 1 - sd / mean : 1;
    cv = mean > 0 ? sd / mean : 0;
    peak = maxR;
  }
  // spotUniformity (src/metrics.js:284-321)
  double spots = NAN;
  if (cells) {
    double mn = INFINITY, mx = 0;
    int cnt = 0;
    for (double v : hc) {
      if (v <= 0) continue;
      mn = std::fmin(mn, v);
      mx = std::fmax(mx, v);
      ++cnt;
    }
    spots = cnt == 0 ? 0.0 : (mx + mn > 0 ? (2 * mn) / (mx + mn) : 1.0);
  }
  // rmsError against s * target over the ROI (src/metrics.js:73-84)
  const double num = std::fmax(0.0, t1[kII] - 2 * s * t1[kIT] + s * s * t1[kTT]);
  const double den = s * s * t1[kTT];
  const double rms = den > 0 ? std::sqrt(num / den) : 0.0;
  const double corr = (t2[kVp] > 0 && t2[kVt] > 0) ? t2[kCov] / std::sqrt(t2[kVp] * t2[kVt]) : 0.0;
  const double ss = t3[1] > 0 ? t3[0] / t3[1] : 0.0;
  const double p = t1[kIrr];
  const double rr = p == 0 ? 0.0 : std::hypot(std::sqrt(t1[kRx] / p), std::sqrt(t1[kRy] / p));
  const double zero = t1[kZp] == 0 ? 0.0 : (t1[kZr] * t1[kZr] + t1[kZi] * t1[kZi]) / ((double)n * t1[kZp]);
  const double incident = t1[kIll] * dx * dy, total = t1[kIrr] * cell, inSignal = pt;
  out[0] = incident > 0 ? inSignal / incident : 0;
  out[1] = total > 0 ? inSignal / total : 0;
  out[2] = cells ? spots : uni;
  out[3] = spots;
  out[4] = flat;
  out[5] = cv;
  out[6] = rms;
  out[7] = (corr + 1) / 2;
  out[8] = corr;
  out[9] = ss;
  out[10] = rms > 0 ? 20 * std::log10(1 / rms) : INFINITY;
  out[11] = zero;
  out[12] = rr;
  out[13] = mean;
  out[14] = peak;
  out[15] = inSignal;
  out[16] = total;
  out[17] = incident;
  return DOE_OK;
}
