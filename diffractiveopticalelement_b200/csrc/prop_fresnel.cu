// prop_fresnel.cu -- single-FFT Fresnel propagation to the magnified grid and its
// exact inverse (reference: src/propagate.js:155-230 propagateFresnelFFT,
// :237-308 propagateFresnelFFTInverse).
//
// Both are one row pass and one column pass over the plane: the input quadratic
// factor (with its checkerboard) is applied on load of the row FFT, the constant
// prefactor and the output quadratic factor (with its checkerboard) on store of
// the column FFT. No shifts are involved: the reference transforms the centred
// grids with the checkerboards instead.
#include <cmath>
#include <vector>

#include "ops_propagate.cuh"

using namespace doe;

namespace {

double frac_cycles(double c) { return c - std::nearbyint(c); }

// cycles of sgn * pi * (i - n/2)^2 d^2 / (lambda az) (/ 2 pi) plus half a cycle on
// odd indices, reduced to [-1/2, 1/2]
void chirp_axis(int n, double d, double lambda, double az, double sgn, float* out) {
  for (int i = 0; i < n; ++i) {
    const double x = (i - n / 2.0) * d;
    const double cyc = sgn * (x * x) / (2.0 * lambda * az) + ((i & 1) ? 0.5 : 0.0);
    out[i] = (float)frac_cycles(cyc);
  }
}

int fresnel_run(doe_ctx* c, const double* re, const double* im, int nx, int ny, bool inverse,
                const std::vector<float>& tabs, float2 pre, double* out_re, double* out_im) {
  const size_t n = (size_t)nx * ny;
  void *din, *dw, *dtab;
  DOE_TRY(ensure_slot(c, kSlotIn, 2 * n * sizeof(double), &din));
  DOE_TRY(ensure_slot(c, kSlotW0, n * sizeof(float2), &dw));
  DOE_TRY(ensure_slot(c, kSlotTab, tabs.size() * sizeof(float), &dtab));
  double* dre = (double*)din;
  double* dim = dre + n;
  float2* w = (float2*)dw;
  float* t = (float*)dtab;
  const float* cx = t;
  const float* cy = t + nx;
  const float* cu = t + nx + ny;
  const float* cv = t + 2 * nx + ny;
  DOE_CUDA(c, cudaMemcpyAsync(t, tabs.data(), tabs.size() * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  DOE_TRY(upload_f64(c, dre, re, n));
  DOE_TRY(upload_f64(c, dim, im, n));
  if (inverse) {
    DOE_TRY(with_row0(nx, [&](auto S) {
      return launch_row<decltype(S)>(c, RowChirpIn<true>{{}, dre, dim, w, cx, cy, nx, ny}, 1, ny);
    }));
    DOE_TRY(with_col0(ny, [&](auto S) {
      return launch_col<decltype(S)>(c, ColChirpOut<true>{{}, w, dre, dim, cu, cv, nx, ny, pre}, 1, nx);
    }));
  } else {
    DOE_TRY(with_row0(nx, [&](auto S) {
      return launch_row<decltype(S)>(c, RowChirpIn<false>{{}, dre, dim, w, cx, cy, nx, ny}, 1, ny);
    }));
    DOE_TRY(with_col0(ny, [&](auto S) {
      return launch_col<decltype(S)>(c, ColChirpOut<false>{{}, w, dre, dim, cu, cv, nx, ny, pre}, 1, nx);
    }));
  }
  DOE_TRY(download_f64(c, out_re, dre, n));
  DOE_TRY(download_f64(c, out_im, dim, n));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  return DOE_OK;
}

}  // namespace

// propagateFresnelFFT: out_d receives the output pitch {lambda|z|/(nx dx), lambda|z|/(ny dy)}.
extern "C" int doe_fresnel(doe_ctx* c, const double* re, const double* im, int nx, int ny, double dx, double dy,
                           double lambda, double z, double* out_re, double* out_im, double* out_d) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "propagateFresnelFFT"));
  if (!re || !im || !out_re || !out_im) return set_err(c, DOE_ERR_BAD_ARG, "propagateFresnelFFT: null plane");
  if (!(z != 0.0) || !(lambda > 0.0)) return set_err(c, DOE_ERR_BAD_ARG, "propagateFresnelFFT: z must be non-zero");
  const double az = std::fabs(z);
  const double dux = (lambda * az) / (nx * dx), duy = (lambda * az) / (ny * dy);
  std::vector<float> tabs(2 * (size_t)(nx + ny));
  chirp_axis(nx, dx, lambda, az, 1.0, tabs.data());
  chirp_axis(ny, dy, lambda, az, 1.0, tabs.data() + nx);
  chirp_axis(nx, dux, lambda, az, 1.0, tabs.data() + nx + ny);
  chirp_axis(ny, duy, lambda, az, 1.0, tabs.data() + 2 * nx + ny);
  // e^{i kz} / (i lambda |z|) with kz = k z - pi (nx + ny) / 2 (src/propagate.js:196-202),
  // kz reduced in cycles in FP64: z / lambda - (nx + ny) / 4
  const double amp = (dx * dy) / (lambda * az);
  const double kz = 2.0 * M_PI * frac_cycles(z / lambda - (nx + ny) / 4.0);
  const float2 pre = make_float2((float)(amp * std::sin(kz)), (float)(-amp * std::cos(kz)));
  DOE_TRY(fresnel_run(c, re, im, nx, ny, false, tabs, pre, out_re, out_im));
  if (out_d) {
    out_d[0] = dux;
    out_d[1] = duy;
  }
  return DOE_OK;
}

// propagateFresnelFFTInverse: the input lives on the magnified grid (pitch dux,
// duy); dx, dy are the DOE-plane pitch of the output.
extern "C" int doe_fresnel_inverse(doe_ctx* c, const double* re, const double* im, int nx, int ny, double dux,
                                   double duy, double lambda, double z, double dx, double dy, double* out_re,
                                   double* out_im) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_grid(c, nx, ny, "propagateFresnelFFTInverse"));
  if (!re || !im || !out_re || !out_im) return set_err(c, DOE_ERR_BAD_ARG, "propagateFresnelFFTInverse: null plane");
  if (!(dx > 0.0) || !(dy > 0.0))
    return set_err(c, DOE_ERR_BAD_ARG, "propagateFresnelFFTInverse: pass the DOE-plane pitch as {dx, dy}");
  if (!(z != 0.0) || !(lambda > 0.0))
    return set_err(c, DOE_ERR_BAD_ARG, "propagateFresnelFFTInverse: z must be non-zero");
  const double az = std::fabs(z);
  std::vector<float> tabs(2 * (size_t)(nx + ny));
  // step 1: conjugate output factor on the magnified grid; step 4: conjugate input factor
  chirp_axis(nx, dux, lambda, az, -1.0, tabs.data());
  chirp_axis(ny, duy, lambda, az, -1.0, tabs.data() + nx);
  chirp_axis(nx, dx, lambda, az, -1.0, tabs.data() + nx + ny);
  chirp_axis(ny, dy, lambda, az, -1.0, tabs.data() + 2 * nx + ny);
  // 1/A = lambda |z| e^{-i kg} / (dx dy), kg = k z - pi (nx + ny)/2 - pi/2
  // (src/propagate.js:279-287), times the 1/(nx ny) of the inverse DFT
  const double amp = (lambda * az) / (dx * dy) / ((double)nx * ny);
  const double kg = 2.0 * M_PI * frac_cycles(z / lambda - (nx + ny) / 4.0 - 0.25);
  const float2 pre = make_float2((float)(amp * std::cos(kg)), (float)(-amp * std::sin(kg)));
  return fresnel_run(c, re, im, nx, ny, true, tabs, pre, out_re, out_im);
}
