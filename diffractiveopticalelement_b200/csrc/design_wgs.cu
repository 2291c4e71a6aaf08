// design_wgs.cu -- pass sequence of weightedGerchbergSaxton over the
// angular-spectrum loop (src/doe.js:455-546 driving :327-437).
#include "design_ops.cuh"

namespace doe {

int design_run_wgs(doe_ctx* c, const DesignBufs& b, int B, int I) {
  // 64^2, 128^2, 256^2 (when selected): the whole loop in one cluster per design
  if (b.nx == b.ny && ((c->tune_design_cluster >> ilog2i(b.nx)) & 1u)) {
    const int rc = design_run_wgs_cluster(c, b, B, I);
    if (rc != DOE_ERR_UNSUPPORTED) return rc;
  }
  const int nx = b.nx, ny = b.ny;
  const float scale = 1.f / (float)((long)nx * ny);
  const ColAsmTab<false> fwd{{}, b.W, b.htab, b.htab_stride, nx, ny, b.st};
  const ColAsmTab<true> back{{}, b.W, b.htab, b.htab_stride, nx, ny, b.st};
  DOE_TRY(design_row(c, RowDoeFwd<false>{{}, b}, B, nx, ny));
  DOE_TRY(design_col(c, fwd, B, nx, ny));
  if (b.rmse_goal > 0) {
    DOE_TRY(design_row(c, RowWgsTarget<true, true>{b, 0, scale}, B, nx, ny));
  } else {
    DOE_TRY(design_row(c, RowWgsTarget<true>{b, 0, scale}, B, nx, ny));
  }
  for (int it = 0; it < I; ++it) {
    DOE_TRY(design_row(c, RowWgsConstrain{{}, b, it - 1}, B, nx, ny));
    DOE_TRY(design_col(c, back, B, nx, ny));
    DOE_TRY(design_row(c, RowDoeUpdate<true, false, false>{{}, b, 0}, B, nx, ny));
    DOE_TRY(design_col(c, fwd, B, nx, ny));
    if (b.rmse_goal > 0) {
      DOE_TRY(design_row(c, RowWgsTarget<false, true>{b, it, scale}, B, nx, ny));
    } else {
      DOE_TRY(design_row(c, RowWgsTarget<false>{b, it, scale}, B, nx, ny));
    }
  }
  return DOE_OK;
}

}  // namespace doe
