// design_loss.cu -- intensity loss of B DOE phases and its gradient with respect
// to the phase, through the image-plane propagation of the design loops (the
// training signal of the warm-start surrogate; no reference counterpart).
// Five passes: A e^{i phi} + row FFT | column (x H) | row: U, loss sums, G, row FFT |
// column (x conj H) | row: inverse, gradient.
#include <cstring>
#include <vector>

#include "design_ops.cuh"

using namespace doe;

namespace doe {
int design_prepare(doe_ctx* c, DesignBufs& b, int B, int nx, int ny, double dx, double dy, const double* lam,
                   const double* z, int ntab, bool wgs, bool needU);
}

extern "C" int doe_phase_loss_grad(doe_ctx* c, const doe_phase_loss_desc* a) {
  if (!c || !a) return DOE_ERR_BAD_ARG;
  if (!a->illumination || !a->target_amp || !a->phase || !a->grad)
    return set_err(c, DOE_ERR_BAD_ARG, "phase loss: null plane");
  const int B = a->batch, nx = a->nx, ny = a->ny;
  if (B <= 0 || B > 65535) return set_err(c, DOE_ERR_BAD_ARG, "phase loss: batch must be in [1, 65535]");
  DesignBufs b;
  DOE_TRY(design_prepare(c, b, B, nx, ny, a->dx, a->dy, &a->lambda, &a->z, 1, false, false));
  b.illum = a->illumination;
  b.tgt = a->target_amp;
  b.roi = a->roi;
  b.phase = const_cast<float*>(a->phase);
  const float scale = 1.f / (float)((long)nx * ny);
  const ColAsmTab<false> fwd{{}, b.W, b.htab, 0, nx, ny};
  const ColAsmTab<true> back{{}, b.W, b.htab, 0, nx, ny};
  DOE_TRY(design_row(c, RowDoeFwd<false>{{}, b}, B, nx, ny));
  DOE_TRY(design_col(c, fwd, B, nx, ny));
  DOE_TRY(design_row(c, RowLossField{b, scale}, B, nx, ny));
  DOE_TRY(design_col(c, back, B, nx, ny));
  return design_row(c, RowPhaseGrad{{}, b, scale, a->grad, a->loss}, B, nx, ny);
}
