// prop_fft.cu -- 2-D FFT entry points (reference: src/fft.js:148-154) and the
// shared helpers of the propagation translation units.
#include "ops_propagate.cuh"

namespace doe {

// ------------------------------------------------------------------ helpers
int upload_f64(doe_ctx* c, double* d, const double* h, size_t n) { return host_upload(c, d, h, n * sizeof(double)); }
int download_f64(doe_ctx* c, double* h, const double* d, size_t n) { return host_download(c, h, d, n * sizeof(double)); }

AsmGroupArgs group_args(int nx, int ny, double dx, double dy, int band_limit, int evanescent,
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
  DOE_TRY(with_row(c, nx, kTuneFft, [&](auto S) {
    if (inverse) {
      RowC64<true> op{{}, d, d, nx, ny, pe, pe, 1.f};
      return launch_row<decltype(S)>(c, op, nplanes, ny);
    }
    RowC64<false> op{{}, d, d, nx, ny, pe, pe, 1.f};
    return launch_row<decltype(S)>(c, op, nplanes, ny);
  }));
  return with_col(c, ny, kTuneFft, [&](auto S) {
    if (inverse) {
      ColC64<true> op{{}, d, d, nx, ny, pe, pe, scale};
      return launch_col<decltype(S)>(c, op, nplanes, nx);
    }
    ColC64<false> op{{}, d, d, nx, ny, pe, pe, scale};
    return launch_col<decltype(S)>(c, op, nplanes, nx);
  });
}

// Propagate nplanes complex64 planes in place (used by the design loops too).
int asm_c64_inplace(doe_ctx* c, float2* d, int nplanes, const AsmTables& tab, int nx, int ny, float2* work) {
  const long pe = (long)nx * ny;
  DOE_TRY(with_row0(nx, [&](auto S) {
    RowC64<false> op{{}, d, work, nx, ny, pe, pe, 1.f};
    return launch_row<decltype(S)>(c, op, nplanes, ny);
  }));
  DOE_TRY(with_col0(ny, [&](auto S) {
    ColAsm op{{}, work, work, tab, nx, ny};
    return launch_col<decltype(S)>(c, op, nplanes, nx);
  }));
  return with_row0(nx, [&](auto S) {
    RowC64<true> op{{}, work, d, nx, ny, pe, pe, 1.f / (float)pe};
    return launch_row<decltype(S)>(c, op, nplanes, ny);
  });
}

}  // namespace doe

using namespace doe;

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
  DOE_TRY(with_row0(nx, [&](auto S) {
    if (inverse) return launch_row<decltype(S)>(c, RowF64In<true>{{}, dre, dim, w, nx, ny, 0, 0}, 1, ny);
    return launch_row<decltype(S)>(c, RowF64In<false>{{}, dre, dim, w, nx, ny, 0, 0}, 1, ny);
  }));
  DOE_TRY(with_col0(ny, [&](auto S) {
    if (inverse) return launch_col<decltype(S)>(c, ColToF64<true>{{}, w, dre, dim, nx, ny, scale}, 1, nx);
    return launch_col<decltype(S)>(c, ColToF64<false>{{}, w, dre, dim, nx, ny, scale}, 1, nx);
  }));
  DOE_TRY(download_f64(c, re, dre, n));
  DOE_TRY(download_f64(c, im, dim, n));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

extern "C" int doe_fft2d_dev(doe_ctx* c, void* d_planes, int nx, int ny, int nplanes, int inverse) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "fft2d"));
  if (!d_planes || nplanes < 0) return set_err(c, DOE_ERR_BAD_ARG, "fft2d: bad argument");
  return fft2d_c64(c, (float2*)d_planes, nx, ny, nplanes, inverse != 0);
}

