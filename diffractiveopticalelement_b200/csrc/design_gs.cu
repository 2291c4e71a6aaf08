// design_gs.cu -- pass sequences of gerchbergSaxton / HIO (src/doe.js:327-437)
// and gerchbergSaxtonMultiPlane (src/doe.js:557-626).
#include "design_ops.cuh"

namespace doe {

int design_run_gs(doe_ctx* c, const DesignBufs& b, int B, int I) {
  const int nx = b.nx, ny = b.ny;
  const float scale = 1.f / (float)((long)nx * ny);
  const ColAsmTab<false> fwd{{}, b.W, b.htab, b.htab_stride, nx, ny};
  const ColAsmTab<true> back{{}, b.W, b.htab, b.htab_stride, nx, ny};
  DOE_TRY(design_row(c, RowDoeFwd<false>{{}, b}, B, nx, ny));
  DOE_TRY(design_col(c, fwd, B, nx, ny));
  for (int it = 0; it < I; ++it) {
    DOE_TRY(design_row(c, RowGsTarget<false, false>{b, it, scale}, B, nx, ny));
    DOE_TRY(design_col(c, back, B, nx, ny));
    DOE_TRY(design_row(c, RowDoeUpdate<true, false, false>{{}, b, 0}, B, nx, ny));
    DOE_TRY(design_col(c, fwd, B, nx, ny));
  }
  return design_row(c, RowGsTarget<true, false>{b, I, scale}, B, nx, ny);
}

int design_run_multiplane(doe_ctx* c, DesignBufs b, int B, int I, int P, const float2* htab, const float* tgt0,
                          const float* roi0) {
  const int nx = b.nx, ny = b.ny;
  const long n = (long)nx * ny;
  const float scale = 1.f / (float)n;
  if (I > 0) DOE_TRY(design_row(c, RowDoeFwd<false>{{}, b}, B, nx, ny));
  for (int it = 0; it < I; ++it) {
    for (int p = 0; p < P; ++p) {
      // plane p of design d: tgt0 + d * P n + p n (tgt_stride = P n)
      const float2* hp = htab + (long)p * n;
      b.tgt = tgt0 + (long)p * n;
      b.roi = roi0 ? roi0 + (long)p * n : nullptr;
      b.mp_plane = p;
      DOE_TRY(design_col(c, ColAsmTab<false>{{}, b.W, hp, 0, nx, ny}, B, nx, ny));
      DOE_TRY(design_row(c, RowGsTarget<false, true>{b, it, scale}, B, nx, ny));
      DOE_TRY(design_col(c, ColAsmTab<true>{{}, b.W, hp, 0, nx, ny}, B, nx, ny));
      if (it + 1 == I && p + 1 == P) DOE_TRY(design_row(c, RowDoeUpdate<false, false, false>{{}, b, 0}, B, nx, ny));
      else DOE_TRY(design_row(c, RowDoeUpdate<true, false, false>{{}, b, 0}, B, nx, ny));
    }
  }
  return DOE_OK;
}

}  // namespace doe
