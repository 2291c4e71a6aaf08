// design_tune.cu -- autotuner of the design loops (no reference counterpart):
// times the design-pass shape variants (and, for image-plane WGS on square
// 64^2-256^2 grids, the cluster-resident loop) on the caller's own batch and keeps
// the fastest for that grid in the context.
#include <vector>

#include "design_ops.cuh"

using namespace doe;

namespace {

// Time one configuration: the faster of two runs after one warm-up run, each
// from the caller's initial phase.
int time_design(doe_ctx* c, const doe_design_dev_desc& d, const float* phase0, size_t phase_bytes, float* ms_out) {
  float best = 1e30f;
  cudaEvent_t a, b;
  DOE_CUDA(c, cudaEventCreate(&a));
  if (cudaEventCreate(&b) != cudaSuccess) {
    cudaEventDestroy(a);
    return set_err(c, DOE_ERR_CUDA, "autotune design: event creation failed");
  }
  int rc = DOE_OK;
  for (int r = 0; r < 3 && rc == DOE_OK; ++r) {
    if (cudaMemcpyAsync(d.phase, phase0, phase_bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) {
      rc = set_err(c, DOE_ERR_CUDA, "autotune design: phase restore failed");
      break;
    }
    cudaEventRecord(a, c->stream);
    rc = doe_design_dev(c, &d);
    cudaEventRecord(b, c->stream);
    if (rc == DOE_OK && cudaEventSynchronize(b) != cudaSuccess) rc = set_err(c, DOE_ERR_CUDA, "autotune design: run failed");
    float ms = 0.f;
    if (rc == DOE_OK && r > 0 && cudaEventElapsedTime(&ms, a, b) == cudaSuccess) best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc == DOE_OK) rc = design_error_check(c);
  *ms_out = best;
  return rc;
}

}  // namespace

extern "C" int doe_autotune_design(doe_ctx* c, const doe_design_dev_desc* desc, int iterations, int* chosen) {
  if (!c || !desc || !desc->phase || desc->batch < 1) return DOE_ERR_BAD_ARG;
  DOE_CUDA(c, cudaSetDevice(c->device));
  const int nx = desc->nx, ny = desc->ny;
  if (!is_pow2(nx) || !is_pow2(ny) || nx > kDesignMaxN || ny > kDesignMaxN)
    return set_err(c, DOE_ERR_BAD_ARG, "autotune design: grid must have power-of-two axes up to %d", kDesignMaxN);
  doe_design_dev_desc d = *desc;
  d.iterations = iterations > 0 ? std::min(iterations, desc->iterations) : std::min(4, desc->iterations);
  d.rmse_goal = 0.0;  // every design runs every timed iteration
  d.iterations_used = nullptr;
  const size_t pbytes = sizeof(float) * (size_t)d.batch * nx * ny;
  float* phase0 = nullptr;
  DOE_CUDA(c, cudaMalloc(&phase0, pbytes));
  const bool saved = cudaMemcpyAsync(phase0, desc->phase, pbytes, cudaMemcpyDeviceToDevice, c->stream) == cudaSuccess;
  int rc = saved ? DOE_OK : set_err(c, DOE_ERR_CUDA, "autotune design: phase copy failed");

  const int lx = ilog2i(nx), ly = ilog2i(ny);
  const int nr = design_row_variants(nx), nc = design_col_variants(ny);
  const unsigned char r0 = c->tune_row[kTuneDesign][lx], c0 = c->tune_col[kTuneDesign][ly];
  const unsigned cl0 = c->tune_design_cluster, bit = 1u << lx;
  int best_r = r0, best_c = c0, best_cl = (cl0 & bit) ? 1 : 0;
  float best_pass = 1e30f, best_cluster = 1e30f;
  // the cluster-resident loop applies to image-plane WGS on square 64^2..256^2 grids
  const bool cl_ok = desc->algorithm == DOE_ALG_WGS && nx == ny && nx >= 64 && nx <= 256;
  c->tune_design_cluster = cl0 & ~bit;
  for (int r = 0; r < nr && rc == DOE_OK; ++r) {
    for (int k = 0; k < nc && rc == DOE_OK; ++k) {
      c->tune_row[kTuneDesign][lx] = (unsigned char)r;
      c->tune_col[kTuneDesign][ly] = (unsigned char)k;
      float ms = 0.f;
      rc = time_design(c, d, phase0, pbytes, &ms);
      if (rc == DOE_OK && ms < best_pass) {
        best_pass = ms;
        best_r = r;
        best_c = k;
      }
    }
  }
  if (cl_ok && rc == DOE_OK) {
    c->tune_design_cluster = cl0 | bit;
    rc = time_design(c, d, phase0, pbytes, &best_cluster);
  }
  best_cl = best_cluster < best_pass ? 1 : 0;
  // restore the caller's initial phase, also after a failed trial; keep the
  // fastest configuration (or the previous one when a trial failed)
  if (saved && cudaMemcpyAsync(desc->phase, phase0, pbytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess &&
      rc == DOE_OK)
    rc = set_err(c, DOE_ERR_CUDA, "autotune design: phase restore failed");
  cudaStreamSynchronize(c->stream);
  cudaFree(phase0);
  if (rc != DOE_OK) {
    c->tune_row[kTuneDesign][lx] = r0;
    c->tune_col[kTuneDesign][ly] = c0;
    c->tune_design_cluster = cl0;
    return rc;
  }
  c->tune_row[kTuneDesign][lx] = (unsigned char)best_r;
  c->tune_col[kTuneDesign][ly] = (unsigned char)best_c;
  c->tune_design_cluster = best_cl ? (cl0 | bit) : (cl0 & ~bit);
  if (chosen) {
    chosen[0] = best_r;
    chosen[1] = best_c;
    chosen[2] = best_cl;
  }
  return DOE_OK;
}
