// design_fourier.cu -- pass sequence of fourierCgh, plain or under the weighted
// wrapper (src/doe.js:639-730, :898-905).
#include "design_ops.cuh"

namespace doe {

int design_run_fourier(doe_ctx* c, const DesignBufs& b, int B, int I, bool wgs) {
  const int nx = b.nx, ny = b.ny;
  const float norm = (float)(1.0 / std::sqrt((double)nx * ny));
  DOE_TRY(design_row(c, RowDoeFwd<true>{{}, b}, B, nx, ny));
  for (int it = 0; it < I; ++it) {
    const bool last = it + 1 == I;
    if (wgs) {
      DOE_TRY(design_col(c, ColFourier<true>{b, it, norm}, B, nx, ny));
      if (!last) DOE_TRY(design_row(c, RowDoeUpdate<true, true, true>{{}, b, it}, B, nx, ny));
      else DOE_TRY(design_row(c, RowDoeUpdate<false, true, true>{{}, b, it}, B, nx, ny));
    } else {
      DOE_TRY(design_col(c, ColFourier<false>{b, it, norm}, B, nx, ny));
      if (!last) DOE_TRY(design_row(c, RowDoeUpdate<true, true, false>{{}, b, it}, B, nx, ny));
      else DOE_TRY(design_row(c, RowDoeUpdate<false, true, false>{{}, b, it}, B, nx, ny));
    }
  }
  return DOE_OK;
}

}  // namespace doe
