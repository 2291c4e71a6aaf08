// interference.cu -- hologram recording / reconstruction and modal (partially
// coherent) intensity on the device (reference: src/interference.js:57-69
// modalIntensity, :347-388 recordHologram, :397-411 reconstructHologram).
//
// Reconstruction and the propagated modal sum are batches of angular-spectrum
// propagations: the planes go through the same three fused passes as
// propagateAngularSpectrum (FP64 planes in and out, FP32 transforms, FP64-reduced
// transfer-function phase), one plane per distance or mode in one launch each.
// The elementwise steps run in FP64 with every product and sum rounded
// separately, in the reference's order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ops_propagate.cuh"

namespace doe {
namespace {

unsigned grid_n(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

// illumination = plate * reference, written to planes [copies][n] (re, im)
__global__ void holo_illum_kernel(const double* pr, const double* pi, const double* rr, const double* ri, long n,
                                  int copies, double* ore, double* oim) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    const double re = __dsub_rn(__dmul_rn(pr[k], rr[k]), __dmul_rn(pi[k], ri[k]));
    const double im = __dadd_rn(__dmul_rn(pr[k], ri[k]), __dmul_rn(pi[k], rr[k]));
    for (int c = 0; c < copies; ++c) {
      ore[c * n + k] = re;
      oim[c * n + k] = im;
    }
  }
}

// sum = object + reference, recorded = |sum|^2, running maximum (non-negative:
// integer max on the FP64 bit pattern is exact)
__global__ void holo_record_kernel(const double* orr, const double* oi, const double* rr, const double* ri, long n,
                                   double* sre, double* sim, double* rec, unsigned long long* mx) {
  double m = 0.0;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    const double a = __dadd_rn(orr[k], rr[k]), b = __dadd_rn(oi[k], ri[k]);
    sre[k] = a;
    sim[k] = b;
    const double v = __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b));
    rec[k] = v;
    m = fmax(m, v);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, (unsigned long long)__double_as_longlong(m));
}

__device__ __forceinline__ double js_round_d(double x) {
  const double f = floor(x);
  return (__dsub_rn(x, f) >= 0.5) ? f + 1.0 : f;
}

// normalise and encode (0 raw, 1 binary, 2 phase; levels > 1 quantises the phase)
__global__ void holo_encode_kernel(const double* sre, const double* sim, double* rec, long n,
                                   const unsigned long long* mx, int encode, int levels, double* pre, double* pim) {
  const double norm = __longlong_as_double((long long)*mx);
  const double pi = 3.141592653589793, two_pi = 6.283185307179586;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    double v = rec[k];
    if (norm > 0) v = v / norm;
    rec[k] = v;
    double re = 0.0, im = 0.0;
    if (encode == 0) {
      re = v;
    } else if (encode == 1) {
      re = v > 0.5 ? 1.0 : 0.0;
    } else {
      double ph = atan2(sim[k], sre[k]);
      ph = fmod(ph, two_pi);  // wrapPhase (src/propagate.js:410-420)
      if (ph > pi) ph -= two_pi;
      else if (ph <= -pi) ph += two_pi;
      re = cos(ph);
      im = sin(ph);
      if (levels > 1) {
        const double step = two_pi / levels;
        const double q = __dmul_rn(js_round_d(atan2(im, re) / step), step);
        re = cos(q);
        im = sin(q);
      }
    }
    pre[k] = re;
    pim[k] = im;
  }
}

// intensity[k] = sum_m w_m |U_m[k]|^2 / sum_m w_m, modes in order
__global__ void modal_sum_kernel(const double* re, const double* im, int M, long n, const double* w, double wsum,
                                 double* out) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int m = 0; m < M; ++m) {
      const double a = re[(long)m * n + k], b = im[(long)m * n + k];
      acc = __dadd_rn(acc, __dmul_rn(w ? w[m] : 1.0, __dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b))));
    }
    out[k] = wsum > 0 ? acc / wsum : acc;
  }
}

// smoothInPlace (src/interference.js:104-125), rows: one thread per (mode, row),
// the reference's running sum in its order (circular indices).
__global__ void box_rows_kernel(const double* in, double* out, int nx, int ny, int rows, int r, double norm) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows) return;
  const double* a = in + (long)t * nx;
  double* o = out + (long)t * nx;
  double acc = 0.0;
  for (int i = -r; i <= r; ++i) acc = __dadd_rn(acc, a[((i % nx) + nx) % nx]);
  for (int i = 0; i < nx; ++i) {
    o[i] = __dmul_rn(acc, norm);
    acc = __dsub_rn(acc, a[(((i - r) % nx) + nx) % nx]);
    acc = __dadd_rn(acc, a[(((i + r + 1) % nx) + nx) % nx]);
  }
}

// columns: one thread per (mode, column), then the Gaussian envelope times
// exp(i * smoothed phase) (src/interference.js:87-96)
__global__ void box_cols_envelope_kernel(const double* tmp, int nx, int ny, int modes, int r, double norm, double dx,
                                        double dy, double waist2, double* re, double* im) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= modes * nx) return;
  const int m = t / nx, i = t % nx;
  const long n = (long)nx * ny;
  const double* a = tmp + (long)m * n + i;
  double acc = 0.0;
  for (int j = -r; j <= r; ++j) acc = __dadd_rn(acc, a[(long)(((j % ny) + ny) % ny) * nx]);
  const double x = __dmul_rn(i - nx / 2.0, dx);
  for (int j = 0; j < ny; ++j) {
    const double ph = __dmul_rn(acc, norm);
    acc = __dsub_rn(acc, a[(long)((((j - r) % ny) + ny) % ny) * nx]);
    acc = __dadd_rn(acc, a[(long)((((j + r + 1) % ny) + ny) % ny) * nx]);
    const double y = __dmul_rn(j - ny / 2.0, dy);
    const double amp = exp(-__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)) / waist2);
    double s, c;
    sincos(ph, &s, &c);
    const long k = (long)m * n + (long)j * nx + i;
    re[k] = __dmul_rn(amp, c);
    im[k] = __dmul_rn(amp, s);
  }
}

// In-place angular-spectrum propagation of P FP64 plane pairs (plane p to z[p]).
int asm_f64_planes(doe_ctx* c, double* dre, double* dim, int P, int nx, int ny, double dx, double dy, double lambda,
                   const double* z, int band_limit, int evanescent, double soft_edge) {
  const long n = (long)nx * ny;
  void* dw;
  DOE_TRY(ensure_slot(c, kSlotW0, (size_t)std::min(P, kMaxGroup) * n * sizeof(float2), &dw));
  float2* w = (float2*)dw;
  for (int p0 = 0; p0 < P; p0 += kMaxGroup) {
    const int pn = std::min(kMaxGroup, P - p0);
    AsmGroupArgs a = group_args(nx, ny, dx, dy, band_limit, evanescent, soft_edge);
    a.nplanes = pn;
    for (int i = 0; i < pn; ++i) {
      a.lam[i] = lambda;
      a.z[i] = z[p0 + i];
    }
    AsmTables tab;
    DOE_TRY(asm_build_tables(c, a, &tab));
    double* re = dre + (long)p0 * n;
    double* im = dim + (long)p0 * n;
    DOE_TRY(with_row0(nx, [&](auto S) {
      return launch_row<decltype(S)>(c, RowF64In<false>{{}, re, im, w, nx, ny, 0, 0}, pn, ny);
    }));
    DOE_TRY(with_col0(ny, [&](auto S) {
      return launch_col<decltype(S)>(c, ColAsm{{}, w, w, tab, nx, ny}, pn, nx);
    }));
    DOE_TRY(with_row0(nx, [&](auto S) {
      return launch_row<decltype(S)>(c, RowInvToF64{{}, w, re, im, nx, ny, n, 1.f / (float)n}, pn, ny);
    }));
  }
  return DOE_OK;
}

}  // namespace
}  // namespace doe

using namespace doe;

// recordHologram: encode 0 'raw', 1 'binary', 2 'phase'; all arrays host FP64 of n.
extern "C" int doe_hologram_record(doe_ctx* c, const double* obj_re, const double* obj_im, const double* ref_re,
                                   const double* ref_im, long long n, int encode, int levels, double* plate_re,
                                   double* plate_im, double* recorded, double* sum_re, double* sum_im) {
  if (!c) return DOE_ERR_BAD_ARG;
  if (!obj_re || !obj_im || !ref_re || !ref_im || !plate_re || !plate_im || !recorded || n < 1)
    return set_err(c, DOE_ERR_BAD_ARG, "recordHologram: bad argument");
  if (encode < 0 || encode > 2) return set_err(c, DOE_ERR_BAD_ARG, "recordHologram: unknown encoding");
  void* p;
  DOE_TRY(ensure_slot(c, kSlotIn, (size_t)9 * n * sizeof(double) + 64, &p));
  double* d = (double*)p;
  double *orr = d, *oi = d + n, *rr = d + 2 * n, *ri = d + 3 * n, *sre = d + 4 * n, *sim = d + 5 * n,
         *rec = d + 6 * n, *pre = d + 7 * n, *pim = d + 8 * n;
  unsigned long long* mx = (unsigned long long*)(d + 9 * n);
  DOE_TRY(host_upload(c, orr, obj_re, n * sizeof(double)));
  DOE_TRY(host_upload(c, oi, obj_im, n * sizeof(double)));
  DOE_TRY(host_upload(c, rr, ref_re, n * sizeof(double)));
  DOE_TRY(host_upload(c, ri, ref_im, n * sizeof(double)));
  DOE_CUDA(c, cudaMemsetAsync(mx, 0, sizeof(unsigned long long), c->stream));
  {
    LaunchScope ls(c, "hologram_record");
    holo_record_kernel<<<grid_n(n), 256, 0, c->stream>>>(orr, oi, rr, ri, n, sre, sim, rec, mx);
    DOE_CUDA(c, cudaGetLastError());
  }
  {
    LaunchScope ls(c, "hologram_encode");
    holo_encode_kernel<<<grid_n(n), 256, 0, c->stream>>>(sre, sim, rec, n, mx, encode, levels, pre, pim);
    DOE_CUDA(c, cudaGetLastError());
  }
  DOE_TRY(host_download(c, plate_re, pre, n * sizeof(double)));
  DOE_TRY(host_download(c, plate_im, pim, n * sizeof(double)));
  DOE_TRY(host_download(c, recorded, rec, n * sizeof(double)));
  if (sum_re) DOE_TRY(host_download(c, sum_re, sre, n * sizeof(double)));
  if (sum_im) DOE_TRY(host_download(c, sum_im, sim, n * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

// reconstructHologram: illumination = plate * reference, propagated to +z (real
// image) and -z (virtual image) in one batch of two planes.
extern "C" int doe_hologram_reconstruct(doe_ctx* c, const double* plate_re, const double* plate_im,
                                        const double* ref_re, const double* ref_im, int nx, int ny, double dx,
                                        double dy, double lambda, double z, int band_limit, int evanescent,
                                        double soft_edge, double* real_re, double* real_im, double* virt_re,
                                        double* virt_im, double* illum_re, double* illum_im) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "reconstructHologram"));
  if (!plate_re || !plate_im || !ref_re || !ref_im || !real_re || !real_im || !virt_re || !virt_im)
    return set_err(c, DOE_ERR_BAD_ARG, "reconstructHologram: null plane");
  const long n = (long)nx * ny;
  void* p;
  DOE_TRY(ensure_slot(c, kSlotOut, (size_t)8 * n * sizeof(double), &p));
  double* d = (double*)p;
  double *pr = d, *pi = d + n, *rr = d + 2 * n, *ri = d + 3 * n, *ore = d + 4 * n, *oim = d + 6 * n;
  DOE_TRY(host_upload(c, pr, plate_re, n * sizeof(double)));
  DOE_TRY(host_upload(c, pi, plate_im, n * sizeof(double)));
  DOE_TRY(host_upload(c, rr, ref_re, n * sizeof(double)));
  DOE_TRY(host_upload(c, ri, ref_im, n * sizeof(double)));
  {
    LaunchScope ls(c, "hologram_illum");
    holo_illum_kernel<<<grid_n(n), 256, 0, c->stream>>>(pr, pi, rr, ri, n, 2, ore, oim);
    DOE_CUDA(c, cudaGetLastError());
  }
  if (illum_re) DOE_TRY(host_download(c, illum_re, ore, n * sizeof(double)));
  if (illum_im) DOE_TRY(host_download(c, illum_im, oim, n * sizeof(double)));
  if (z != 0.0) {  // src/propagate.js:113: z = 0 leaves the field unchanged
    const double zz[2] = {z, -z};
    DOE_TRY(asm_f64_planes(c, ore, oim, 2, nx, ny, dx, dy, lambda, zz, band_limit, evanescent, soft_edge));
  }
  DOE_TRY(host_download(c, real_re, ore, n * sizeof(double)));
  DOE_TRY(host_download(c, real_im, oim, n * sizeof(double)));
  DOE_TRY(host_download(c, virt_re, ore + n, n * sizeof(double)));
  DOE_TRY(host_download(c, virt_im, oim + n, n * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

// modalIntensity of M modes [M][n] (weights may be NULL = all 1); with z != 0 each
// mode is first propagated by the angular spectrum to z (one batch).
extern "C" int doe_modal_intensity(doe_ctx* c, int M, const double* re, const double* im, int nx, int ny,
                                   const double* weights, double dx, double dy, double lambda, double z,
                                   int band_limit, int evanescent, double soft_edge, double* out) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "modalIntensity"));
  if (M < 1 || !re || !im || !out) return set_err(c, DOE_ERR_BAD_ARG, "modalIntensity: bad argument");
  const long n = (long)nx * ny;
  void* p;
  DOE_TRY(ensure_slot(c, kSlotIn, ((size_t)2 * M + 1) * n * sizeof(double) + (size_t)M * sizeof(double) + 64, &p));
  double* dre = (double*)p;
  double* dim = dre + (long)M * n;
  double* dout = dim + (long)M * n;
  double* dw = dout + n;
  DOE_TRY(host_upload(c, dre, re, (size_t)M * n * sizeof(double)));
  DOE_TRY(host_upload(c, dim, im, (size_t)M * n * sizeof(double)));
  double wsum = 0.0;
  if (weights) {
    for (int m = 0; m < M; ++m) wsum += weights[m];
    DOE_TRY(host_upload(c, dw, weights, (size_t)M * sizeof(double)));
  } else {
    wsum = M;
  }
  if (z != 0.0) {
    std::vector<double> zz(M, z);
    DOE_TRY(asm_f64_planes(c, dre, dim, M, nx, ny, dx, dy, lambda, zz.data(), band_limit, evanescent, soft_edge));
  }
  {
    LaunchScope ls(c, "modal_intensity");
    modal_sum_kernel<<<grid_n(n), 256, 0, c->stream>>>(dre, dim, M, n, weights ? dw : nullptr, wsum, dout);
    DOE_CUDA(c, cudaGetLastError());
  }
  DOE_TRY(host_download(c, out, dout, n * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

// partiallyCoherentModes (src/interference.js:79-101): the uniform phase screens
// come from one xorshift32 stream on the host (src/doe.js:65-75, sequential by
// definition); smoothing and the envelope run on the device.
extern "C" int doe_partially_coherent_modes(doe_ctx* c, int nx, int ny, double dx, double dy, int modes,
                                            double sigma, double waist, double seed, double* re, double* im) {
  if (!c) return DOE_ERR_BAD_ARG;
  if (nx < 1 || ny < 1 || modes < 1 || !re || !im || !(dx > 0) || !(waist != 0))
    return set_err(c, DOE_ERR_BAD_ARG, "partiallyCoherentModes: bad argument");
  const long n = (long)nx * ny;
  const long total = (long)modes * n;
  std::vector<double> ph(total);
  {
    const double t = std::trunc(seed);
    double m = std::fmod(t, 4294967296.0);
    if (m < 0) m += 4294967296.0;
    uint32_t s = (uint32_t)m;
    if (!s) s = 1;
    for (long k = 0; k < total; ++k) {
      s ^= s << 13;
      s ^= s >> 17;
      s ^= s << 5;
      ph[k] = ((double)s / 4294967296.0 * 2 - 1) * M_PI;
    }
  }
  const double sigma_pix = std::max(1.0, sigma / dx);
  const double fl = std::floor(sigma_pix);
  const int r = (int)std::max(1.0, (sigma_pix - fl >= 0.5) ? fl + 1.0 : fl);  // Math.round
  const double norm = 1.0 / (2 * r + 1);
  void* p;
  DOE_TRY(ensure_slot(c, kSlotIn, (size_t)4 * total * sizeof(double), &p));
  double* d_ph = (double*)p;
  double* d_tmp = d_ph + total;
  double* d_re = d_tmp + total;
  double* d_im = d_re + total;
  DOE_TRY(host_upload(c, d_ph, ph.data(), total * sizeof(double)));
  {
    LaunchScope ls(c, "coherence_box_rows");
    const int rows = modes * ny;
    box_rows_kernel<<<(rows + 127) / 128, 128, 0, c->stream>>>(d_ph, d_tmp, nx, ny, rows, r, norm);
    DOE_CUDA(c, cudaGetLastError());
  }
  {
    LaunchScope ls(c, "coherence_box_cols_envelope");
    const int cols = modes * nx;
    box_cols_envelope_kernel<<<(cols + 127) / 128, 128, 0, c->stream>>>(d_tmp, nx, ny, modes, r, norm, dx, dy,
                                                                        waist * waist, d_re, d_im);
    DOE_CUDA(c, cudaGetLastError());
  }
  DOE_TRY(host_download(c, re, d_re, total * sizeof(double)));
  DOE_TRY(host_download(c, im, d_im, total * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}
