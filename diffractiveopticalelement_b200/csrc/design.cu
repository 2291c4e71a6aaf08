// design.cu -- batched Gerchberg-Saxton family on the device
// (reference: src/doe.js:327-437, :455-546, :557-626, :639-730).
//
// One call runs B designs of one grid size together: every pass below is one
// kernel launch over all B designs. Per iteration:
//   GS / HIO (image plane)  4 passes: col(+z) | row: inverse, measure, constrain,
//                           forward | col(-z) | row: inverse, phase, A e^{i phi}, forward
//   WGS (image plane)       5 passes: the constraint needs the weight
//                           normalisation of the same field, so measuring and
//                           constraining sit on either side of a pass boundary
//   Fourier CGH (GS / WGS)  2 passes: the column pass measures and constrains
//                           between its forward and inverse column FFTs
//   multi-plane             4 passes per plane step, like GS
// Inside each weighted iteration the reference recomputes the forward field that
// the previous iteration's final pass already produced (src/doe.js:350-352 and
// :417-419 take identical inputs); here it is computed once and reused.
#include <cstring>
#include <memory>
#include <vector>

#include "design_ops.cuh"

namespace doe {

__global__ void f64_to_f32_kernel(const double* __restrict__ in, float* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void f32_to_f64_kernel(const float* __restrict__ in, double* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// Weights 1 inside the ROI, 0 elsewhere (src/doe.js:461-468); norm 1, best +inf.
__global__ void design_init_kernel(DesignBufs b, int B, bool wgs) {
  const long n = b.pe();
  if (wgs) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)B * n; i += (long)gridDim.x * blockDim.x) {
      const long d = i / n, k = i % n;
      const float m = b.roi ? b.roi[d * b.tgt_stride + k] : 1.f;
      b.wraw[i] = m > 0.f ? 1.f : 0.f;
    }
  }
  if (blockIdx.x == 0) {
    for (int d = threadIdx.x; d < B; d += blockDim.x) {
      b.st[d].norm = 1.0;
      b.st[d].best = __longlong_as_double(0x7ff0000000000000LL);  // +inf
      b.st[d].eff_cur = 0.0;
      b.st[d].stop = -1;
      b.st[d].best_it = -2;
      b.st[d].sT = 0.0;
      b.st[d].sTT = 0.0;
    }
  }
}

// Designs stopped by the screen goal: iterations run, and the histories past the
// stop repeat its last entry. One thread per design.
__global__ void design_goal_out_kernel(DesignBufs b, int B, int iters, int* used) {
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < B; d += gridDim.x * blockDim.x) {
    const int stop = b.st[d].stop;
    if (used) used[d] = stop >= 0 ? stop + 1 : iters;
    if (stop < 0) continue;
    for (int i = stop + 1; i < iters; ++i) {
      b.err_hist[(long)d * b.iters + i] = b.err_hist[(long)d * b.iters + stop];
      b.eff_hist[(long)d * b.iters + i] = b.eff_hist[(long)d * b.iters + stop];
    }
  }
}

// Final weights = w_raw * norm (src/doe.js:523-524).
__global__ void design_weights_out_kernel(DesignBufs b, int B, float* out) {
  const long n = b.pe();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)B * n; i += (long)gridDim.x * blockDim.x)
    out[i] = b.wraw[i] * (float)b.st[i / n].norm;
}

// Transfer function of the design loops (bandLimit false, evanescent zeroed:
// src/doe.js:352) tabulated in FFT bin order, one plane per geometry.
__global__ void design_htab_kernel(AsmTables t, int nx, int ny, int ntab, float2* htab) {
  const long n = (long)nx * ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (long)ntab * n; i += (long)gridDim.x * blockDim.x) {
    const int p = (int)(i / n);
    const long k = i % n;
    htab[i] = asm_h(t, nx, ny, p, (int)(k % nx), (int)(k / nx));
  }
}

static unsigned grid_for(long n) { return (unsigned)std::max<long>(1, std::min<long>((n + 255) / 256, 148L * 16)); }

static int check_design_grid(doe_ctx* c, int nx, int ny, const char* who) {
  DOE_TRY(check_grid(c, nx, ny, who));
  if (nx < kDesignMinN || ny < kDesignMinN || nx > kDesignMaxN || ny > kDesignMaxN)
    return set_err(c, DOE_ERR_UNSUPPORTED, "%s: design grids must have power-of-two axes in [%d, %d], got %dx%d", who,
                   kDesignMinN, kDesignMaxN, nx, ny);
  return DOE_OK;
}

static char* take(char*& q, size_t bytes) {
  char* r = q;
  q += (bytes + 255) / 256 * 256;
  return r;
}

// Build `ntab` transfer-function planes (wavelength / distance per plane).
static int build_htab(doe_ctx* c, int nx, int ny, double dx, double dy, int ntab, const double* lam,
                      const double* z, float2* htab) {
  const long n = (long)nx * ny;
  for (int t0 = 0; t0 < ntab; t0 += kMaxGroup) {
    const int tn = std::min(kMaxGroup, ntab - t0);
    AsmGroupArgs g = group_args(nx, ny, dx, dy, 0, 1, 0.02);
    g.nplanes = tn;
    for (int i = 0; i < tn; ++i) {
      g.lam[i] = lam[t0 + i];
      g.z[i] = z[t0 + i];
    }
    AsmTables tab;
    DOE_TRY(asm_build_tables(c, g, &tab));
    LaunchScope ls(c, "design_htab");
    design_htab_kernel<<<grid_for((long)tn * n), 256, 0, c->stream>>>(tab, nx, ny, tn, htab + (long)t0 * n);
    DOE_CUDA(c, cudaGetLastError());
  }
  return DOE_OK;
}

// Carve the design state of B designs (histories `Ih` long) from kSlotDesign2.
static int carve_state(doe_ctx* c, DesignBufs& b, int B, int Ih, int bpp, int pp_planes) {
  const size_t bytes = 256 * 8 + sizeof(DesignState) * B + sizeof(double) * (size_t)B * Ih * (2 + pp_planes) +
                       (size_t)B * Ih + sizeof(double) * (size_t)B * bpp * kRedKGoal + sizeof(unsigned) * B +
                       sizeof(double) * B * kRedKGoal;
  void* p2;
  DOE_TRY(ensure_slot(c, kSlotDesign2, bytes, &p2));
  char* q = (char*)p2;
  b.st = (DesignState*)take(q, sizeof(DesignState) * B);
  if (!b.err_hist) b.err_hist = (double*)take(q, sizeof(double) * (size_t)B * Ih);
  if (!b.eff_hist) b.eff_hist = (double*)take(q, sizeof(double) * (size_t)B * Ih);
  b.pp_err = pp_planes ? (double*)take(q, sizeof(double) * (size_t)B * Ih * pp_planes) : nullptr;
  b.improved = (unsigned char*)take(q, (size_t)B * Ih);
  b.partials = (double*)take(q, sizeof(double) * (size_t)B * bpp * kRedKGoal);
  b.counters = (unsigned*)take(q, sizeof(unsigned) * B);
  b.totals = (double*)take(q, sizeof(double) * B * kRedKGoal);
  DOE_CUDA(c, cudaMemsetAsync(b.counters, 0, sizeof(unsigned) * B, c->stream));
  DOE_CUDA(c, cudaMemsetAsync(b.improved, 0, (size_t)B * Ih, c->stream));
  return DOE_OK;
}

// Work plane, one transfer table and reduction state for B designs of one
// geometry (the phase-gradient passes); planes are attached by the caller.
int design_prepare(doe_ctx* c, DesignBufs& b, int B, int nx, int ny, double dx, double dy, const double* lam,
                   const double* z, int ntab, bool wgs, bool needU) {
  (void)wgs;
  (void)needU;
  DOE_TRY(check_design_grid(c, nx, ny, "phase loss"));
  const long n = (long)nx * ny;
  void* p0;
  DOE_TRY(ensure_slot(c, kSlotDesign0, (size_t)B * n * sizeof(float2) + (size_t)ntab * n * sizeof(float2) + 1024, &p0));
  char* q0 = (char*)p0;
  memset(&b, 0, sizeof(b));
  b.nx = nx;
  b.ny = ny;
  b.iters = 1;
  b.dx = dx;
  b.dy = dy;
  b.tgt_stride = n;
  b.W = (float2*)take(q0, (size_t)B * n * sizeof(float2));
  float2* htab = (float2*)take(q0, (size_t)ntab * n * sizeof(float2));
  b.htab = htab;
  b.htab_stride = ntab > 1 ? n : 0;
  DOE_TRY(carve_state(c, b, B, 1, design_bpp(nx, ny), 0));
  return build_htab(c, nx, ny, dx, dy, ntab, lam, z, htab);
}

}  // namespace doe

using namespace doe;

extern "C" int doe_design_dev(doe_ctx* c, const doe_design_dev_desc* a) {
  if (!c || !a) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_design_grid(c, a->nx, a->ny, "designDOE"));
  const int B = a->batch, nx = a->nx, ny = a->ny, I = a->iterations;
  if (B <= 0 || I < 0 || !a->illumination || !a->target_amp || !a->phase)
    return set_err(c, DOE_ERR_BAD_ARG, "designDOE: bad argument");
  const int alg = a->algorithm;
  if (alg < 0 || alg > 3) return set_err(c, DOE_ERR_BAD_ARG, "designDOE: unknown algorithm %d", alg);
  const bool fourier = alg == DOE_ALG_FOURIER || alg == DOE_ALG_WGS_FOURIER;
  const bool wgs = alg == DOE_ALG_WGS || alg == DOE_ALG_WGS_FOURIER;
  if (wgs && I < 1) return set_err(c, DOE_ERR_BAD_ARG, "weightedGerchbergSaxton: needs at least one iteration");
  if (a->rmse_goal < 0 || a->rmse_goal != a->rmse_goal)
    return set_err(c, DOE_ERR_BAD_ARG, "designDOE: rmse_goal must be >= 0");
  if (a->rmse_goal > 0 && alg != DOE_ALG_WGS)
    return set_err(c, DOE_ERR_UNSUPPORTED, "designDOE: a screen RMSE goal needs image-plane WGS");
  if (B > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "designDOE: at most 65535 designs per call");
  const long n = (long)nx * ny;
  const long Bn = (long)B * n;
  const int Ih = std::max(I, 1);

  const bool tab_shared = (a->lambdas == nullptr && a->zs == nullptr);
  const int ntab = fourier ? 0 : (tab_shared ? 1 : B);
  const bool needU = wgs && !fourier;
  void *p0, *p1;
  DOE_TRY(ensure_slot(c, kSlotDesign0, (size_t)(needU ? 3 : 1) * Bn * sizeof(float2) + (size_t)ntab * n * sizeof(float2) + 1024, &p0));
  DOE_TRY(ensure_slot(c, kSlotDesign1, (size_t)(needU ? 5 : 4) * Bn * sizeof(float) + 1024, &p1));
  char* q0 = (char*)p0;
  char* q1 = (char*)p1;
  DesignBufs b;
  memset(&b, 0, sizeof(b));
  b.nx = nx;
  b.ny = ny;
  b.iters = Ih;
  b.dx = a->dx;
  b.dy = a->dy;
  b.feedback = (float)a->feedback;
  b.escape = a->escape;
  b.beta = (float)a->beta;
  b.illum = a->illumination;
  b.tgt = a->target_amp;
  b.roi = a->roi;
  b.tgt_stride = n;
  b.phase = a->phase;
  b.W = (float2*)take(q0, Bn * sizeof(float2));
  b.U = needU ? (float2*)take(q0, Bn * sizeof(float2)) : nullptr;
  b.U2 = needU ? (float2*)take(q0, Bn * sizeof(float2)) : nullptr;
  float2* htab = ntab ? (float2*)take(q0, (size_t)ntab * n * sizeof(float2)) : nullptr;
  b.htab = htab;
  b.htab_stride = ntab > 1 ? n : 0;
  b.amp = a->amplitude ? a->amplitude : (float*)take(q1, Bn * sizeof(float));
  b.wraw = wgs ? (float*)take(q1, Bn * sizeof(float)) : nullptr;
  b.best_phase = wgs ? (float*)take(q1, Bn * sizeof(float)) : nullptr;
  b.best_amp = wgs ? (float*)take(q1, Bn * sizeof(float)) : nullptr;
  b.phase2 = needU ? (float*)take(q1, Bn * sizeof(float)) : nullptr;
  b.err_hist = a->error;
  b.eff_hist = a->efficiency;
  b.rmse_goal = a->rmse_goal;
  b.screen_irr = a->screen_irr;
  DOE_TRY(carve_state(c, b, B, Ih, design_bpp(nx, ny), 0));
  {
    LaunchScope ls(c, "design_init");
    design_init_kernel<<<grid_for(Bn), 256, 0, c->stream>>>(b, B, wgs);
    DOE_CUDA(c, cudaGetLastError());
  }
  if (ntab) {
    std::vector<double> lam(ntab), zz(ntab);
    for (int i = 0; i < ntab; ++i) {
      lam[i] = a->lambdas ? a->lambdas[i] : a->lambda;
      zz[i] = a->zs ? a->zs[i] : a->z;
    }
    DOE_TRY(build_htab(c, nx, ny, a->dx, a->dy, ntab, lam.data(), zz.data(), htab));
  }

  if (!fourier && !wgs) {
    DOE_TRY(design_run_gs(c, b, B, I));
  } else if (!fourier) {
    DOE_TRY(design_run_wgs(c, b, B, I));  // leaves the best iterates in best_phase / best_amp
    if (b.rmse_goal > 0 || a->iterations_used) {
      LaunchScope ls(c, "design_goal_out");
      design_goal_out_kernel<<<(B + 255) / 256, 256, 0, c->stream>>>(b, B, I, a->iterations_used);
      DOE_CUDA(c, cudaGetLastError());
    }
  } else {
    DOE_TRY(design_run_fourier(c, b, B, I, wgs));
  }

  if (wgs) {
    DOE_CUDA(c, cudaMemcpyAsync(a->phase, b.best_phase, Bn * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
    if (a->amplitude)
      DOE_CUDA(c, cudaMemcpyAsync(a->amplitude, b.best_amp, Bn * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
    if (a->weights) {
      LaunchScope ls(c, "design_weights");
      design_weights_out_kernel<<<grid_for(Bn), 256, 0, c->stream>>>(b, B, a->weights);
      DOE_CUDA(c, cudaGetLastError());
    }
    if (a->rmse)
      DOE_CUDA(c, cudaMemcpy2DAsync(a->rmse, sizeof(double), &b.st[0].best, sizeof(DesignState), sizeof(double), B,
                                    cudaMemcpyDeviceToDevice, c->stream));
  }
  return DOE_OK;
}

// ------------------------------------------------------------------ host-buffer API
static void random_phase_host(int nx, int ny, double seed, double* out) {
  // makeRng (src/doe.js:65-75) + randomPhase (:81-86)
  const double t = std::trunc(seed);
  double m = std::fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  uint32_t s = (uint32_t)m;
  if (!s) s = 1;
  const long n = (long)nx * ny;
  for (long k = 0; k < n; ++k) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    out[k] = ((double)s / 4294967296.0 * 2 - 1) * M_PI;
  }
}

extern "C" int doe_random_phase(int nx, int ny, double seed, double* out) {
  if (nx <= 0 || ny <= 0 || !out) return DOE_ERR_BAD_ARG;
  random_phase_host(nx, ny, seed, out);
  return DOE_OK;
}

static int convert_launch(doe_ctx* c, const double* in, float* out, long n) {
  LaunchScope ls(c, "f64_to_f32");
  f64_to_f32_kernel<<<grid_for(n), 256, 0, c->stream>>>(in, out, n);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}
static int convert_back_launch(doe_ctx* c, const float* in, double* out, long n) {
  LaunchScope ls(c, "f32_to_f64");
  f32_to_f64_kernel<<<grid_for(n), 256, 0, c->stream>>>(in, out, n);
  DOE_CUDA(c, cudaGetLastError());
  return DOE_OK;
}

extern "C" int doe_design_batch(doe_ctx* c, int nb, const doe_design_desc* d, doe_design_result* r) {
  if (!c || !d || !r || nb <= 0) return DOE_ERR_BAD_ARG;
  const doe_design_desc& d0 = d[0];
  DOE_TRY(check_design_grid(c, d0.nx, d0.ny, "designDOE"));
  for (int i = 1; i < nb; ++i) {
    if (d[i].nx != d0.nx || d[i].ny != d0.ny || d[i].algorithm != d0.algorithm || d[i].iterations != d0.iterations ||
        d[i].dx != d0.dx || d[i].dy != d0.dy)
      return set_err(c, DOE_ERR_BAD_ARG, "designDOE batch: designs must share grid, pitch, algorithm and iterations");
  }
  const bool has_roi = d0.roi != nullptr;
  for (int i = 0; i < nb; ++i) {
    if (!d[i].illumination || !d[i].target_amp || !r[i].phase)
      return set_err(c, DOE_ERR_BAD_ARG, "designDOE: missing illumination, target or output phase");
    if ((d[i].roi != nullptr) != has_roi)
      return set_err(c, DOE_ERR_BAD_ARG, "designDOE batch: roi given for some designs only");
  }
  const int nx = d0.nx, ny = d0.ny, I = d0.iterations;
  const long n = (long)nx * ny, Bn = (long)nb * n;
  const int Ih = std::max(I, 1);
  const bool fourier = d0.algorithm == DOE_ALG_FOURIER || d0.algorithm == DOE_ALG_WGS_FOURIER;
  const bool wgs = d0.algorithm == DOE_ALG_WGS || d0.algorithm == DOE_ALG_WGS_FOURIER;
  const int nf = has_roi ? 4 : 3;
  std::vector<double> lam(nb), zz(nb);
  bool same = true;
  int ngen = 0;  // designs whose initial phase is the seeded random phase
  for (int i = 0; i < nb; ++i) {
    if (!d[i].init_phase && fourier) ++ngen;
    lam[i] = d[i].lambda;
    zz[i] = d[i].z;
    same = same && lam[i] == lam[0] && zz[i] == zz[0];
  }
  void *pin, *pout, *pw;
  DOE_TRY(ensure_slot(c, kSlotIn, (size_t)Bn * nf * sizeof(double), &pin));
  const size_t fbytes = ((size_t)Bn * 5 * sizeof(float) + 255) / 256 * 256;
  DOE_TRY(ensure_slot(c, kSlotOut, fbytes + sizeof(double) * ((size_t)nb * Ih * 2 + nb) + 256, &pout));
  DOE_TRY(ensure_slot(c, kSlotParams, (size_t)Bn * sizeof(float) + 256, &pw));
  double* din = (double*)pin;
  // the FP64 inputs (converted to FP32 on the device) go straight from the caller's
  // arrays; only seeded initial phases are made on the host first
  std::unique_ptr<double[]> gen(ngen ? new double[(size_t)ngen * n] : nullptr);
  {
    double* dph = din + 2 * Bn;
    auto up = [&](double* dst, const double* src) { return host_upload(c, dst, src, n * sizeof(double)); };
    for (int i = 0, g = 0; i < nb; ++i) {
      DOE_TRY(up(din + i * n, d[i].illumination));
      DOE_TRY(up(din + Bn + i * n, d[i].target_amp));
      if (has_roi) DOE_TRY(up(din + 3 * Bn + i * n, d[i].roi));
      if (d[i].init_phase) {
        DOE_TRY(up(dph + i * n, d[i].init_phase));
      } else if (fourier) {
        double* gp = gen.get() + (size_t)g++ * n;
        random_phase_host(nx, ny, d[i].seed, gp);  // src/doe.js:651
        DOE_TRY(up(dph + i * n, gp));
      } else {
        DOE_CUDA(c, cudaMemsetAsync(dph + i * n, 0, n * sizeof(double), c->stream));  // flatPhase, src/doe.js:339
      }
    }
  }
  float* f = (float*)pout;
  float* fill = f;
  float* ftgt = f + Bn;
  float* fph = f + 2 * Bn;
  float* froi = has_roi ? f + 3 * Bn : nullptr;
  float* famp = f + 4 * Bn;
  double* hist = (double*)((char*)pout + fbytes);
  double* err = hist;
  double* eff = hist + (size_t)nb * Ih;
  double* rms = eff + (size_t)nb * Ih;
  float* fw = wgs ? (float*)pw : nullptr;
  DOE_TRY(convert_launch(c, din, f, Bn * nf));
  doe_design_dev_desc a;
  memset(&a, 0, sizeof(a));
  a.batch = nb;
  a.nx = nx;
  a.ny = ny;
  a.dx = d0.dx;
  a.dy = d0.dy;
  a.lambda = d0.lambda;
  a.z = d0.z;
  a.lambdas = same ? nullptr : lam.data();
  a.zs = same ? nullptr : zz.data();
  a.algorithm = d0.algorithm;
  a.iterations = I;
  a.feedback = d0.feedback;
  a.escape = d0.escape;
  a.beta = d0.beta;
  a.illumination = fill;
  a.target_amp = ftgt;
  a.roi = froi;
  a.phase = fph;
  a.amplitude = famp;
  a.weights = fw;
  a.error = err;
  a.efficiency = eff;
  a.rmse = wgs ? rms : nullptr;
  DOE_TRY(doe_design_dev(c, &a));
  // results back to FP64 in the input staging area
  double* o = din;
  DOE_TRY(convert_back_launch(c, fph, o, Bn));
  DOE_TRY(convert_back_launch(c, famp, o + Bn, Bn));
  if (wgs) DOE_TRY(convert_back_launch(c, fw, o + 2 * Bn, Bn));
  std::vector<double> hh((size_t)nb * Ih * 2 + nb);
  DOE_TRY(host_download(c, hh.data(), hist, hh.size() * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  DOE_TRY(design_error_check(c));
  // every result plane straight into the caller's array
  std::unique_ptr<double[]> tmp;
  auto down = [&](double* dst, const double* src) { return host_download(c, dst, src, n * sizeof(double)); };
  for (int i = 0; i < nb; ++i) {
    DOE_TRY(down(r[i].phase, o + i * n));
    if (r[i].amplitude || r[i].intensity) {
      double* am = r[i].amplitude;
      if (!am) {
        if (!tmp) tmp.reset(new double[n]);
        am = tmp.get();
      }
      DOE_TRY(down(am, o + Bn + i * n));
      if (r[i].intensity) {
        DOE_CUDA(c, cudaStreamSynchronize(c->stream));
        for (long k = 0; k < n; ++k) r[i].intensity[k] = am[k] * am[k];
      }
    }
    if (wgs && r[i].weights) DOE_TRY(down(r[i].weights, o + 2 * Bn + i * n));
    if (r[i].error) memcpy(r[i].error, hh.data() + (size_t)i * Ih, I * sizeof(double));
    if (r[i].efficiency) memcpy(r[i].efficiency, hh.data() + (size_t)nb * Ih + (size_t)i * Ih, I * sizeof(double));
    r[i].rmse = wgs ? hh[(size_t)nb * Ih * 2 + i] : 0.0;
  }
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));  // pinned result arrays complete asynchronously
  return DOE_OK;
}

extern "C" int doe_design(doe_ctx* c, const doe_design_desc* d, doe_design_result* r) {
  return doe_design_batch(c, 1, d, r);
}

// ------------------------------------------------------------------ multi-plane
extern "C" int doe_multiplane(doe_ctx* c, int nx, int ny, double dx, double dy, double lambda,
                              const double* illumination, int P, const double* zs, const double* target_amp,
                              const double* roi, const double* weight, int I, const double* init_phase,
                              double* phase, double* error, double* efficiency, double* per_plane_error) {
  if (!c) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_design_grid(c, nx, ny, "gerchbergSaxtonMultiPlane"));
  if (P <= 0) return set_err(c, DOE_ERR_BAD_ARG, "gerchbergSaxtonMultiPlane: no planes");  // src/doe.js:564
  if (!illumination || !zs || !target_amp || !phase || I < 0)
    return set_err(c, DOE_ERR_BAD_ARG, "gerchbergSaxtonMultiPlane: bad argument");
  const long n = (long)nx * ny;
  const int Ih = std::max(I, 1);
  const int nf = 2 + P * (roi ? 2 : 1);
  void *pin, *pf, *p0;
  DOE_TRY(ensure_slot(c, kSlotIn, (size_t)n * nf * sizeof(double), &pin));
  DOE_TRY(ensure_slot(c, kSlotOut, (size_t)n * (nf + 1) * sizeof(float) + 256, &pf));
  DOE_TRY(ensure_slot(c, kSlotDesign0, (size_t)n * sizeof(float2) + (size_t)P * n * sizeof(float2) + 1024, &p0));
  double* din = (double*)pin;
  float* f = (float*)pf;
  // the caller's planes straight to the device (no host-side gather)
  DOE_TRY(host_upload(c, din, illumination, n * sizeof(double)));
  if (init_phase) {
    DOE_TRY(host_upload(c, din + n, init_phase, n * sizeof(double)));
  } else {
    DOE_CUDA(c, cudaMemsetAsync(din + n, 0, n * sizeof(double), c->stream));  // flatPhase (src/doe.js:568)
  }
  DOE_TRY(host_upload(c, din + 2 * n, target_amp, (size_t)P * n * sizeof(double)));
  if (roi)
    DOE_TRY(host_upload(c, din + (2 + P) * n, roi, (size_t)P * n * sizeof(double)));
  DOE_TRY(convert_launch(c, din, f, n * nf));
  char* q0 = (char*)p0;
  DesignBufs b;
  memset(&b, 0, sizeof(b));
  b.nx = nx;
  b.ny = ny;
  b.iters = Ih;
  b.dx = dx;
  b.dy = dy;
  b.illum = f;
  b.phase = f + n;
  b.amp = f + (long)nf * n;
  b.tgt_stride = (long)P * n;
  b.W = (float2*)take(q0, n * sizeof(float2));
  float2* htab = (float2*)take(q0, (size_t)P * n * sizeof(float2));
  b.htab_stride = 0;
  b.mp_nplanes = P;
  DOE_TRY(carve_state(c, b, 1, Ih, design_bpp(nx, ny), P));
  {
    LaunchScope ls(c, "design_init");
    design_init_kernel<<<1, 256, 0, c->stream>>>(b, 1, false);
    DOE_CUDA(c, cudaGetLastError());
  }
  std::vector<double> lam(P, lambda);
  DOE_TRY(build_htab(c, nx, ny, dx, dy, P, lam.data(), zs, htab));
  DOE_TRY(design_run_multiplane(c, b, 1, I, P, htab, f + 2 * n, roi ? f + (long)(2 + P) * n : nullptr));
  DOE_TRY(convert_back_launch(c, b.phase, din, n));
  std::vector<double> ppe((size_t)P * Ih);
  DOE_TRY(host_download(c, phase, din, n * sizeof(double)));
  DOE_TRY(host_download(c, ppe.data(), b.pp_err, ppe.size() * sizeof(double)));
  DOE_CUDA(c, cudaStreamSynchronize(c->stream));
  // per-iteration error: mean of the weighted per-plane errors (src/doe.js:601, :618-619)
  for (int it = 0; it < I; ++it) {
    double iterErr = 0;
    for (int p = 0; p < P; ++p) iterErr += ppe[(size_t)p * Ih + it] * (weight ? weight[p] : 1.0);
    if (error) error[it] = iterErr / P;
    if (efficiency) efficiency[it] = 1 - iterErr / P;
  }
  if (per_plane_error)
    for (int p = 0; p < P; ++p)
      for (int it = 0; it < I; ++it) per_plane_error[(size_t)p * I + it] = ppe[(size_t)p * Ih + it];
  return DOE_OK;
}

// Per-iteration multi-plane error / efficiency of B designs from the per-plane
// errors (src/doe.js:601, :618-619). One thread per (design, iteration).
__global__ void multiplane_hist_kernel(const double* ppe, int B, int P, int Ih, int I, const double* w, double* err,
                                       double* eff, double* ppe_out) {
  const long total = (long)B * I;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int d = (int)(i / I), it = (int)(i % I);
    double e = 0;
    for (int p = 0; p < P; ++p) {
      const double v = ppe[((long)d * P + p) * Ih + it];
      e += v * w[p];
      if (ppe_out) ppe_out[((long)d * P + p) * I + it] = v;
    }
    if (err) err[i] = e / P;
    if (eff) eff[i] = 1 - e / P;
  }
}

extern "C" int doe_multiplane_dev(doe_ctx* c, const doe_multiplane_dev_desc* a) {
  if (!c || !a) return DOE_ERR_BAD_ARG;
  DOE_TRY(check_design_grid(c, a->nx, a->ny, "gerchbergSaxtonMultiPlane"));
  const int B = a->batch, nx = a->nx, ny = a->ny, P = a->nplanes, I = a->iterations;
  if (P <= 0) return set_err(c, DOE_ERR_BAD_ARG, "gerchbergSaxtonMultiPlane: no planes");
  if (B <= 0 || I < 0 || !a->z || !a->illumination || !a->target_amp || !a->phase)
    return set_err(c, DOE_ERR_BAD_ARG, "gerchbergSaxtonMultiPlane: bad argument");
  if (B > 65535) return set_err(c, DOE_ERR_UNSUPPORTED, "gerchbergSaxtonMultiPlane: at most 65535 designs per call");
  const long n = (long)nx * ny;
  const int Ih = std::max(I, 1);
  void* p0;
  DOE_TRY(ensure_slot(c, kSlotDesign0, (size_t)B * n * sizeof(float2) + (size_t)P * n * sizeof(float2) +
                                           (size_t)B * n * sizeof(float) + sizeof(double) * (P + 2) + 2048, &p0));
  char* q0 = (char*)p0;
  DesignBufs b;
  memset(&b, 0, sizeof(b));
  b.nx = nx;
  b.ny = ny;
  b.iters = Ih;
  b.dx = a->dx;
  b.dy = a->dy;
  b.illum = a->illumination;
  b.phase = a->phase;
  b.tgt_stride = (long)P * n;
  b.W = (float2*)take(q0, (size_t)B * n * sizeof(float2));
  float2* htab = (float2*)take(q0, (size_t)P * n * sizeof(float2));
  b.amp = (float*)take(q0, (size_t)B * n * sizeof(float));
  double* dw = (double*)take(q0, sizeof(double) * P);
  b.htab_stride = 0;
  b.mp_nplanes = P;
  DOE_TRY(carve_state(c, b, B, Ih, design_bpp(nx, ny), P));
  {
    LaunchScope ls(c, "design_init");
    design_init_kernel<<<1, 256, 0, c->stream>>>(b, B, false);
    DOE_CUDA(c, cudaGetLastError());
  }
  std::vector<double> lam(P, a->lambda), w(P, 1.0);
  if (a->weight)
    for (int p = 0; p < P; ++p) w[p] = a->weight[p];
  DOE_TRY(host_upload(c, dw, w.data(), sizeof(double) * P));
  DOE_TRY(build_htab(c, nx, ny, a->dx, a->dy, P, lam.data(), a->z, htab));
  DOE_TRY(design_run_multiplane(c, b, B, I, P, htab, a->target_amp, a->roi));
  if (I > 0 && (a->error || a->efficiency || a->per_plane_error)) {
    LaunchScope ls(c, "multiplane_hist");
    multiplane_hist_kernel<<<grid_for((long)B * I), 256, 0, c->stream>>>(b.pp_err, B, P, Ih, I, dw, a->error,
                                                                         a->efficiency, a->per_plane_error);
    DOE_CUDA(c, cudaGetLastError());
  }
  return DOE_OK;
}
