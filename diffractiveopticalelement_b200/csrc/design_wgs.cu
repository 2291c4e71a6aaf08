// design_wgs.cu -- pass sequence of weightedGerchbergSaxton over the
// angular-spectrum loop (src/doe.js:455-546 driving :327-437).
#include "design_ops.cuh"

namespace doe {
namespace {

unsigned grid_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

// Cluster-resident loop: it snapshots every improved iterate but the last itself;
// the last iteration's, when it improved, is taken here from the final phase and field.
__global__ void cluster_last_snapshot_kernel(DesignBufs b, int B, int it) {
  const long n = b.pe();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)B * n; i += (long)gridDim.x * blockDim.x) {
    const long d = i / n;
    if (!b.improved[d * b.iters + it]) continue;
    const float2 u = b.U[i];
    b.best_phase[i] = b.phase[i];
    b.best_amp[i] = sqrtf(u.x * u.x + u.y * u.y);
  }
}

// Passes: a design's best iterate k that no constraint pass copied (k is one of
// the last two iterations, or the design stopped at k) is still in the
// alternating buffers -- its phase in buffer (k + 1) mod 2, its field in k mod 2.
__global__ void best_iterate_kernel(DesignBufs b, int B, int I) {
  const long n = b.pe();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)B * n; i += (long)gridDim.x * blockDim.x) {
    const DesignState& S = b.st[i / n];
    const int k = S.best_it;
    if (k < 0 || (S.stop < 0 && k <= I - 3)) continue;  // none yet, or copied by the constraint pass
    const float* ph = ((k + 1) & 1) ? b.phase2 : b.phase;
    const float2 u = ((k & 1) ? b.U2 : b.U)[i];
    b.best_phase[i] = ph[i];
    b.best_amp[i] = sqrtf(u.x * u.x + u.y * u.y);
  }
}

}  // namespace

// Runs the loop and leaves every design's best iterate in b.best_phase / b.best_amp.
int design_run_wgs(doe_ctx* c, const DesignBufs& b, int B, int I) {
  const long Bn = (long)B * b.nx * b.ny;
  // 64^2, 128^2, 256^2 (when selected): the whole loop in one cluster per design
  if (b.nx == b.ny && ((c->tune_design_cluster >> ilog2i(b.nx)) & 1u)) {
    const int rc = design_run_wgs_cluster(c, b, B, I);
    if (rc != DOE_ERR_UNSUPPORTED) {
      DOE_TRY(rc);
      LaunchScope ls(c, "design_snapshot");
      cluster_last_snapshot_kernel<<<grid_for(Bn), 256, 0, c->stream>>>(b, B, I - 1);
      DOE_CUDA(c, cudaGetLastError());
      return DOE_OK;
    }
  }
  const int nx = b.nx, ny = b.ny;
  const float scale = 1.f / (float)((long)nx * ny);
  // phase produced by iteration k (k = -1: the initial phase) and field of iteration k
  auto phase_of = [&](int k) { return ((k + 1) & 1) ? b.phase2 : b.phase; };
  auto field_of = [&](int k) { return (k & 1) ? b.U2 : b.U; };
  const ColAsmTab<false> fwd{{}, b.W, b.htab, b.htab_stride, nx, ny, b.st};
  const ColAsmTab<true> back{{}, b.W, b.htab, b.htab_stride, nx, ny, b.st};
  DesignBufs bk = b;
  bk.U = field_of(-1);
  DOE_TRY(design_row(c, RowDoeFwd<false>{{}, b}, B, nx, ny));
  DOE_TRY(design_col(c, fwd, B, nx, ny));
  if (b.rmse_goal > 0) {
    DOE_TRY(design_row(c, RowWgsTarget<true, true>{bk, 0, scale}, B, nx, ny));
  } else {
    DOE_TRY(design_row(c, RowWgsTarget<true>{bk, 0, scale}, B, nx, ny));
  }
  for (int it = 0; it < I; ++it) {
    bk = b;
    bk.U = field_of(it - 1);
    DOE_TRY(design_row(c, RowWgsConstrain{{}, bk, it, phase_of(it - 2), field_of(it - 2)}, B, nx, ny));
    DOE_TRY(design_col(c, back, B, nx, ny));
    bk = b;
    bk.phase = phase_of(it);
    DOE_TRY(design_row(c, RowDoeUpdate<true, false, false>{{}, bk, 0}, B, nx, ny));
    DOE_TRY(design_col(c, fwd, B, nx, ny));
    bk = b;
    bk.U = field_of(it);
    if (b.rmse_goal > 0) {
      DOE_TRY(design_row(c, RowWgsTarget<false, true>{bk, it, scale}, B, nx, ny));
    } else {
      DOE_TRY(design_row(c, RowWgsTarget<false>{bk, it, scale}, B, nx, ny));
    }
  }
  LaunchScope ls(c, "design_best");
  best_iterate_kernel<<<grid_for(Bn), 256, 0, c->stream>>>(b, B, I);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

}  // namespace doe
