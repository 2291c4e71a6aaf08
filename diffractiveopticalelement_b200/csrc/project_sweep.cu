// project_sweep.cu -- ProjectorSystem.simulate at many screen distances from one
// element (reference: src/projector.js:475-498 simulate, called per distance by
// defocusCurve :622-642 and focusStack :645-653).
//
// Every distance sees the same element field, so its forward transform is
// computed once. Angular-spectrum mode: one forward 2-D FFT of the padded
// element, then per distance only the transfer-function product with the inverse
// column FFT and the inverse row FFT (the focus-sweep passes), then the centre
// crop. Lens mode: one forward FFT, then per throw only the fftshift, chirp and
// amplitude factor of focalPlaneSpectrum (src/propagate.js:342-374), evaluated
// with the same FP32 operations as the single-distance lens pass.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ops_propagate.cuh"

namespace doe {
__global__ void element_field_kernel(const double* __restrict__ A, const double* __restrict__ ph, int nx, int ny,
                                     int pad, int rot, float2* __restrict__ out);

namespace {

unsigned grid_for_n(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

// Centre crop of nz (nx*pad)-by-(ny*pad) complex64 planes into FP64 planes [nz][nx*ny].
__global__ void crop_planes_kernel(const float2* __restrict__ in, int nx, int ny, int pad, int nz,
                                   double* __restrict__ re, double* __restrict__ im) {
  const int NX = nx * pad, NY = ny * pad;
  const int ox = (NX - nx) / 2, oy = (NY - ny) / 2;
  const long n = (long)nx * ny, N = (long)NX * NY;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nz * n; i += (long)gridDim.x * blockDim.x) {
    const long p = i / n, k = i % n;
    const int x = (int)(k % nx), y = (int)(k / nx);
    const float2 v = in[p * N + (x + ox) + (long)(y + oy) * NX];
    re[i] = v.x;
    im[i] = v.y;
  }
}

// Lens focal planes of nz throws from one forward spectrum (unshifted): output
// sample (i, j) of throw p is bin ((i + nx/2) mod nx, (j + ny/2) mod ny) times
// amp0_p exp(i 2 pi (cx_p[i] + cy_p[j] - 1/4)), the per-axis cycles reduced mod 1
// in FP64 on the host (the single-throw lens pass evaluates the same expression).
__global__ void focal_planes_kernel(const float2* __restrict__ spec, int nx, int ny, int nz,
                                    const float* __restrict__ cxy, const float* __restrict__ amp0,
                                    double* __restrict__ re, double* __restrict__ im) {
  const long n = (long)nx * ny;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nz * n; t += (long)gridDim.x * blockDim.x) {
    const int p = (int)(t / n);
    const long k = t % n;
    const int i = (int)(k % nx), j = (int)(k / nx);
    const int x = (i + (nx >> 1)) & (nx - 1), y = (j + (ny >> 1)) & (ny - 1);
    const float2 v = spec[x + (long)y * nx];
    const float* cx = cxy + (long)p * (nx + ny);
    float c = cx[i] + cx[nx + j] - 0.25f;
    c -= rintf(c);
    float sn, cs;
    sincospif(2.f * c, &sn, &cs);
    const float a = amp0[p];
    const float2 z = cmul(v, make_float2(a * cs, a * sn));
    re[t] = (double)z.x;
    im[t] = (double)z.y;
  }
}

}  // namespace
}  // namespace doe

using namespace doe;

// simulate at nz distances (z[] in metres): out_re / out_im [nz][nx*ny] FP64,
// out_d [nz][2] the screen pitch of each plane.
extern "C" int doe_simulate_sweep(doe_ctx* c, const double* illumination, const double* phase, int nx, int ny,
                                  double dx, double dy, double lambda, const double* z, int nz, int band_limit,
                                  int far_field, int pad, double* out_re, double* out_im, double* out_d) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "ProjectorSystem.simulate"));
  if (!illumination || !phase || !z || !out_re || !out_im || nz < 0)
    return set_err(c, DOE_ERR_BAD_ARG, "simulate: bad argument");
  if (nz == 0) return DOE_OK;
  if (pad < 1 || (pad & (pad - 1))) return set_err(c, DOE_ERR_BAD_ARG, "simulate: pad must be a power of two");
  if (far_field) {
    for (int p = 0; p < nz; ++p)
      if (!(z[p] > 0))
        return set_err(c, DOE_ERR_BAD_ARG, "ProjectorSystem.simulate: far-field mode needs a positive throw");
    pad = 1;  // src/projector.js:481-490 (no padding in the lens geometry)
  }
  DOE_TRY(check_grid(c, nx * pad, ny * pad, "ProjectorSystem.simulate"));
  const long n = (long)nx * ny, NX = (long)nx * pad, NY = (long)ny * pad, N = NX * NY;
  void *pin, *pw, *pout;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &pin));
  DOE_TRY(ensure_slot(c, kSlotW0, 2 * N * sizeof(float2), &pw));
  DOE_TRY(ensure_slot(c, kSlotOut, 2 * (size_t)nz * n * sizeof(double), &pout));
  double* dA = (double*)pin;
  double* dP = dA + n;
  float2* elem = (float2*)pw;  // padded element field
  float2* spec = elem + N;     // its forward spectrum
  double* ore = (double*)pout;
  double* oim = ore + (long)nz * n;
  DOE_TRY(host_upload(c, dA, illumination, n * sizeof(double)));
  DOE_TRY(host_upload(c, dP, phase, n * sizeof(double)));
  {
    LaunchScope ls(c, "element_field");
    element_field_kernel<<<grid_for_n(N), 256, 0, c->stream>>>(dA, dP, nx, ny, pad, far_field ? 1 : 0, elem);
    DOE_CUDA(c, cudaGetLastError());
  }
  DOE_TRY(with_row0((int)NX, [&](auto S) {
    return launch_row<decltype(S)>(c, RowC64<false>{{}, elem, spec, (int)NX, (int)NY, N, N, 1.f}, 1, (int)NY);
  }));
  DOE_TRY(with_col0((int)NY, [&](auto S) {
    return launch_col<decltype(S)>(c, ColC64<false>{{}, spec, spec, (int)NX, (int)NY, N, N, 1.f}, 1, (int)NX);
  }));
  if (far_field) {
    std::vector<float> h((size_t)nz * (nx + ny) + nz);
    float* amp = h.data() + (size_t)nz * (nx + ny);
    for (int p = 0; p < nz; ++p) {
      const double dux = (lambda * z[p]) / (nx * dx), duy = (lambda * z[p]) / (ny * dy);
      float* cx = h.data() + (size_t)p * (nx + ny);
      for (int i = 0; i < nx; ++i) {
        const double u = (i - nx / 2.0) * dux, cyc = (u * u) / (2.0 * lambda * z[p]);
        cx[i] = (float)(cyc - std::nearbyint(cyc));
      }
      for (int j = 0; j < ny; ++j) {
        const double v = (j - ny / 2.0) * duy, cyc = (v * v) / (2.0 * lambda * z[p]);
        cx[nx + j] = (float)(cyc - std::nearbyint(cyc));
      }
      amp[p] = (float)((dx * dy) / (lambda * z[p]));
      if (out_d) {
        out_d[2 * p] = dux;
        out_d[2 * p + 1] = duy;
      }
    }
    void* pt;
    DOE_TRY(ensure_slot(c, kSlotTab, h.size() * sizeof(float), &pt));
    float* dt = (float*)pt;
    DOE_TRY(host_upload(c, dt, h.data(), h.size() * sizeof(float)));
    LaunchScope ls(c, "focal_planes");
    focal_planes_kernel<<<grid_for_n((long)nz * n), 256, 0, c->stream>>>(spec, nx, ny, nz, dt,
                                                                         dt + (size_t)nz * (nx + ny), ore, oim);
    DOE_CUDA(c, cudaGetLastError());
  } else {
    // plane groups bounded by 1 GiB of complex64 work planes
    const int G = (int)std::max<long>(1, std::min<long>({(long)nz, (long)kMaxGroup, (1L << 30) / (N * 8)}));
    void* pw1;
    DOE_TRY(ensure_slot(c, kSlotW1, (size_t)G * N * sizeof(float2), &pw1));
    float2* work = (float2*)pw1;
    for (int p0 = 0; p0 < nz; p0 += G) {
      const int gn = std::min(G, nz - p0);
      AsmGroupArgs a = group_args((int)NX, (int)NY, dx, dy, band_limit, 1, 0.02);
      a.nplanes = gn;
      for (int i = 0; i < gn; ++i) {
        a.lam[i] = lambda;
        a.z[i] = z[p0 + i];
      }
      AsmTables tab;
      DOE_TRY(asm_build_tables(c, a, &tab));
      DOE_TRY(with_col0((int)NY, [&](auto S) {
        return launch_col<decltype(S)>(c, ColSweep{ColSweepBase{{}, spec, work, tab, (int)NX, (int)NY, 0}}, gn,
                                       (int)NX);
      }));
      DOE_TRY(with_row0((int)NX, [&](auto S) {
        return launch_row<decltype(S)>(c, RowC64<true>{{}, work, work, (int)NX, (int)NY, N, N, 1.f / (float)N}, gn,
                                       (int)NY);
      }));
      for (int i = 0; i < gn; ++i)  // src/propagate.js:113: z = 0 leaves the field unchanged
        if (a.z[i] == 0.0)
          DOE_CUDA(c, cudaMemcpyAsync(work + (long)i * N, elem, N * sizeof(float2), cudaMemcpyDeviceToDevice,
                                      c->stream));
      LaunchScope ls(c, "crop");
      crop_planes_kernel<<<grid_for_n((long)gn * n), 256, 0, c->stream>>>(work, nx, ny, pad, gn, ore + (long)p0 * n,
                                                                          oim + (long)p0 * n);
      DOE_CUDA(c, cudaGetLastError());
    }
    if (out_d)
      for (int p = 0; p < nz; ++p) {
        out_d[2 * p] = dx;
        out_d[2 * p + 1] = dy;
      }
  }
  DOE_TRY(host_download(c, out_re, ore, (size_t)nz * n * sizeof(double)));
  DOE_TRY(host_download(c, out_im, oim, (size_t)nz * n * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}
