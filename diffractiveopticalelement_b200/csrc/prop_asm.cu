// prop_asm.cu -- angular-spectrum propagation, transfer function and the lens
// focal-plane transform (reference: src/propagate.js:57-133, :342-374).
#include "ops_propagate.cuh"

namespace doe {

// Centred transfer function as FP64 planes (angularSpectrumTransferFunction) and
// the propagating count (w > 0.5, or any non-evanescent bin when evanescent=0).
static __global__ void asm_transfer_kernel(AsmTables t, int nx, int ny, double* hre, double* him,
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

}  // namespace doe

using namespace doe;

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
  DOE_TRY(with_row0(nx, [&](auto S) {
    return launch_row<decltype(S)>(c, RowF64In<false>{{}, dre, dim, w, nx, ny, 0, 0}, 1, ny);
  }));
  DOE_TRY(with_col0(ny, [&](auto S) {
    return launch_col<decltype(S)>(c, ColAsm{{}, w, w, tab, nx, ny}, 1, nx);
  }));
  DOE_TRY(with_row0(nx, [&](auto S) {
    return launch_row<decltype(S)>(c, RowInvToF64{{}, w, dre, dim, nx, ny, (long)n, 1.f / (float)n}, 1, ny);
  }));
  DOE_TRY(download_f64(c, re, dre, n));
  DOE_TRY(download_f64(c, im, dim, n));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
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
  DOE_TRY(with_row0(nx, [&](auto S) {
    return launch_row<decltype(S)>(c, RowF64In<false>{{}, dre, dim, w, nx, ny, nx >> 1, ny >> 1}, 1, ny);
  }));
  DOE_TRY(with_col0(ny, [&](auto S) {
    return launch_col<decltype(S)>(c, ColFocal{{}, w, dre, dim, cxy, cxy + nx, nx, ny, (float)amp0}, 1, nx);
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

