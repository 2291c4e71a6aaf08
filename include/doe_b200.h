/*
 * doe_b200.h -- C ABI of the B200 engine for the propagate-and-retrieve path of
 * Ziggyware/DiffractiveOpticalElement (a plain-JavaScript optics toolkit).
 *
 * The reference exposes ES-module functions over ComplexField objects whose data
 * are split Float64Array planes (re, im), row-major, idx = x + y*nx, optical axis
 * at the array centre (src/field.js:8-16). Each entry point below replaces one of
 * those functions (cited as file:line inside the reference project) and takes the
 * same planes as plain `double*` buffers owned by the caller. A Node N-API addon,
 * Python ctypes, or any C caller binds these symbols directly; no C++ or torch
 * types appear in any signature.
 *
 * Conventions
 *   - Every function returns a doe_status; DOE_OK is 0. On failure the message of
 *     the failing call is available from doe_last_error(ctx) and uses the
 *     reference's wording where the reference throws for the same condition.
 *   - Host-buffer entry points ("doe_*" without the _dev suffix) are synchronous:
 *     they copy the planes to HBM, run the CUDA kernels, copy results back and
 *     return when the results are in the caller's buffers. Page-locked buffers
 *     (doe_host_alloc) make those copies run at full PCIe rate.
 *   - Device entry points (suffix _dev) take device pointers to complex64
 *     (interleaved float2) planes already resident in HBM and are asynchronous on
 *     the context's stream (doe_ctx_stream / doe_ctx_synchronize).
 *   - A context owns one CUDA stream and its scratch memory; it is not
 *     thread-safe. Use one context per host thread.
 *   - Arithmetic: FP32 transforms and pointwise maths; FP64 for the angular-
 *     spectrum phase argument (reduced mod 2*pi before FP32 sincos) and for every
 *     power / efficiency / error / weight-normalisation reduction.
 *   - Grids: power-of-two nx, ny in [1, 8192] (the reference accepts any power of
 *     two; larger axes return DOE_ERR_UNSUPPORTED).
 */
#ifndef DOE_B200_H
#define DOE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define DOE_B200_ABI_VERSION 1

typedef struct doe_ctx doe_ctx;

typedef enum doe_status {
  DOE_OK = 0,
  DOE_ERR_NOT_POW2 = 1,      /* src/field.js:30-32, src/fft.js:88 */
  DOE_ERR_SIZE_MISMATCH = 2, /* src/fft.js:149-151, src/field.js:78-80 */
  DOE_ERR_BAD_ARG = 3,       /* e.g. src/propagate.js:248-250, src/doe.js:564 */
  DOE_ERR_CUDA = 4,          /* a CUDA runtime call failed */
  DOE_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up */
  DOE_ERR_UNSUPPORTED = 6,   /* outside the engine's supported range */
  DOE_ERR_NO_DEVICE = 7      /* no CUDA device / library not usable */
} doe_status;

/* ------------------------------------------------------------ context */
int doe_abi_version(void);
int doe_ctx_create(int device, doe_ctx** out);
void doe_ctx_destroy(doe_ctx* ctx);
const char* doe_last_error(const doe_ctx* ctx);
void* doe_ctx_stream(doe_ctx* ctx); /* the context's cudaStream_t */
int doe_ctx_synchronize(doe_ctx* ctx);
/* Page-locked host allocation for fast host<->device copies. */
int doe_host_alloc(doe_ctx* ctx, void** ptr, unsigned long long bytes);
int doe_host_free(doe_ctx* ctx, void* ptr);

/* Instrumentation (engine-only; no reference counterpart). */
unsigned long long doe_ctx_launch_count(doe_ctx* ctx); /* kernels launched so far */
int doe_ctx_set_profiling(doe_ctx* ctx, int on); /* bracket each launch with events */
/* Per-kernel totals since the last read: returns the number of labels written
 * (names: max_entries rows of name_len chars). Synchronises the stream. */
int doe_ctx_profile_read(doe_ctx* ctx, int max_entries, char* names, int name_len,
                         double* total_ms, unsigned long long* count);

/* Tuning knobs (engine-only): "sweep_group" = planes per focus-sweep launch pair
 * (0 = sized from the L2 cache); "sweep_fused" = 1 to read and multiply per
 * element in the sweep column pass (0: all reads first); "sweep_graph" = 0 to
 * disable CUDA-graph replay of repeated device sweeps; "sweep_hsym" = 1 to have
 * the sweep column pass evaluate the transfer function once per pair of mirrored
 * rows (H depends on fy^2) into shared memory, 2 to also have its spectrum tile
 * staged into shared memory by TMA; "sweep_res" = K in 2..64 to have one CTA of
 * the sweep column pass keep its spectrum tile in shared memory (one TMA copy)
 * across K planes (1, the default: one plane per CTA); "sweep_tc" = 0 to run
 * 1024 x 1024 focus sweeps on the FP32 CUDA-core passes instead of the tcgen05
 * tensor-core passes (default 1); "design_cluster" = 1 to run image-plane
 * weightedGerchbergSaxton on square 64^2, 128^2 and 256^2 grids as one
 * on-chip loop per design (a thread-block cluster holding the plane in
 * distributed shared memory) instead of five passes per iteration, 0 for the
 * passes on all three (default), or (log2(n) << 8) | on for one grid size;
 * its current value reads back as a mask with bit log2(n) set per size on;
 * "surrogate_tc" selects the surrogate's convolution kernel where the layer
 * allows tcgen05 (a multiple of 64 input channels): 0 mma.sync, 1 tcgen05 with
 * cp.async operand staging, 2 tcgen05 with TMA operand staging and a 4-stage ring
 * (default), 3 the same with 3 stages; "host_copy_threads" = host threads that
 * stage pageable caller planes of 1 MB or more through pinned chunks of the
 * context (default a quarter of the host's threads, at most 4; 0 = hand them
 * to the driver as they are);
 * "fft_row", "fft_col",
 * "sweep_row", "sweep_col", "design_row", "design_col" = (log2(n) << 8) | shape
 * variant for that pass. */
int doe_ctx_set_tuning(doe_ctx* ctx, const char* key, long long value);
/* Current value of "sweep_group", "sweep_fused", "sweep_graph", "sweep_hsym",
 * "sweep_res", "sweep_tc", "design_cluster", "surrogate_tc" or "host_copy_threads". */
int doe_ctx_get_tuning(doe_ctx* ctx, const char* key, long long* value);
/* Autotuner (engine-only): times the compiled FFT-pass shape variants for an
 * nx-by-ny grid at the given geometry on this device and keeps the fastest for
 * the plain FFT and focus-sweep passes (and the sweep column pass's load
 * formulations: "sweep_fused", "sweep_hsym", "sweep_res" 2/4/8), then times the pipelined sweep for
 * several group sizes ("sweep_group") on the CUDA-core passes and, for 1024^2
 * grids with "sweep_tc" on, on the tensor-core passes, keeping the fastest pair
 * ("sweep_tc", "sweep_group"). chosen (5 ints, may be NULL) receives the picked
 * {fft row, fft column, sweep row, sweep column} variants and group size. */
int doe_autotune(doe_ctx* ctx, int nx, int ny, double dx, double dy, double lambda, double z,
                 int* chosen);

/* ------------------------------------------------------------ transforms */
/* fft2d(re, im, nx, ny, inverse) -- src/fft.js:148-154. In place; forward
 * unscaled, inverse scaled by 1/(nx*ny). */
int doe_fft2d(doe_ctx* ctx, double* re, double* im, int nx, int ny, int inverse);

/* angularSpectrumTransferFunction -- src/propagate.js:57-102. Writes the centred
 * transfer function and the propagating fraction (entries with w > 0.5). */
int doe_asm_transfer(doe_ctx* ctx, int nx, int ny, double dx, double dy, double lambda,
                     double z, int band_limit, int evanescent, double soft_edge,
                     double* h_re, double* h_im, double* propagating_fraction);

/* propagateAngularSpectrumInPlace -- src/propagate.js:112-133 (z may be negative;
 * z == 0 leaves the field untouched). propagateAngularSpectrum (:105-109) is the
 * same call on a copy. */
int doe_asm(doe_ctx* ctx, double* re, double* im, int nx, int ny, double dx, double dy,
            double lambda, double z, int band_limit, int evanescent, double soft_edge);

/* focusSweep -- src/propagate.js:427-434: one input field propagated to nz
 * distances; out_re/out_im hold nz consecutive planes. */
int doe_asm_sweep(doe_ctx* ctx, const double* re, const double* im, int nx, int ny,
                  double dx, double dy, double lambda, const double* z, int nz,
                  int band_limit, int evanescent, double soft_edge, double* out_re,
                  double* out_im);

/* focalPlaneSpectrum -- src/propagate.js:342-374. Output pitch in out_d[0..1]. */
int doe_focal_plane(doe_ctx* ctx, const double* re, const double* im, int nx, int ny,
                    double dx, double dy, double lambda, double f, double* out_re,
                    double* out_im, double* out_d);

/* propagateFresnelFFT -- src/propagate.js:155-230: single-FFT Fresnel transform
 * of the nx*ny FP64 planes to the magnified grid; out_d receives its pitch
 * {lambda|z|/(nx dx), lambda|z|/(ny dy)}. z must be non-zero. Inputs and outputs
 * may alias. The undersampling check (throwOnUndersampled) is host-side. */
int doe_fresnel(doe_ctx* ctx, const double* re, const double* im, int nx, int ny, double dx,
                double dy, double lambda, double z, double* out_re, double* out_im, double* out_d);

/* propagateFresnelFFTInverse -- src/propagate.js:237-308: the exact inverse,
 * from the magnified grid (pitch dux, duy) back to the DOE grid (pitch dx, dy). */
int doe_fresnel_inverse(doe_ctx* ctx, const double* re, const double* im, int nx, int ny,
                        double dux, double duy, double lambda, double z, double dx, double dy,
                        double* out_re, double* out_im);

/* ------------------------------------------------------------ device-resident */
/* Batched 2-D FFT of nplanes complex64 planes in place (device pointer). */
int doe_fft2d_dev(doe_ctx* ctx, void* d_planes, int nx, int ny, int nplanes, int inverse);

/* Batched focus sweep on device-resident complex64 fields: field f (of nfields)
 * with wavelength lambda[f] is propagated to z[f*nz + k] for k < nz and written
 * to plane f*nz + k of d_out. lambda and z are host arrays. */
int doe_asm_sweep_dev(doe_ctx* ctx, const void* d_fields, int nfields, int nx, int ny,
                      double dx, double dy, const double* lambda, const double* z, int nz,
                      int band_limit, int evanescent, double soft_edge, void* d_out);

/* ------------------------------------------------------------ design loops */
typedef enum doe_algorithm {
  DOE_ALG_GS = 0,          /* gerchbergSaxton (HIO when feedback > 0) -- src/doe.js:327-437 */
  DOE_ALG_WGS = 1,         /* weightedGerchbergSaxton over gerchbergSaxton -- src/doe.js:455-546 */
  DOE_ALG_FOURIER = 2,     /* fourierCgh -- src/doe.js:639-730 */
  DOE_ALG_WGS_FOURIER = 3  /* weightedGerchbergSaxton over fourierCgh -- src/doe.js:898-905 */
} doe_algorithm;

/* One design; planes are nx*ny FP64 arrays in the reference's layout. Option
 * meanings follow src/doe.js:49-59 and :327-335. roi, init_phase may be NULL
 * (NULL init_phase: flat for GS/WGS, randomPhase(seed) for the Fourier loop). */
typedef struct doe_design_desc {
  int nx, ny;
  double dx, dy, lambda, z;
  int algorithm;
  int iterations;
  double feedback; /* HIO feedback, 0 = plain GS */
  int escape;      /* iterations before the feedback applies */
  double beta;     /* WGS exponent */
  double seed;
  const double* illumination;
  const double* target_amp; /* target amplitude (already power-matched, src/doe.js:817-829) */
  const double* roi;
  const double* init_phase;
} doe_design_desc;

/* Caller-owned outputs: phase/amplitude/intensity/weights nx*ny, error/efficiency
 * `iterations` entries; any may be NULL except phase. */
typedef struct doe_design_result {
  double* phase;
  double* amplitude;
  double* intensity;
  double* error;
  double* efficiency;
  double* weights; /* WGS only */
  double rmse;     /* WGS only: best unweighted ROI RMSE */
} doe_design_result;

/* randomPhase(nx, ny, seed) -- src/doe.js:81-86 (xorshift32 makeRng, :65-75):
 * the seeded initial phase in (-pi, pi]. Host-side, needs no context. */
int doe_random_phase(int nx, int ny, double seed, double* out);

/* errorDiffusionQuantize -- src/doe.js:185-226: serpentine (snake) Floyd-Steinberg
 * quantisation of `batch` phase planes of n samples each to `levels` levels, the
 * error taken on the unit circle; wrap_first wraps the input into (-pi, pi] first.
 * The grid is inferred as the reference does (nx = round(sqrt(n))); when nx does
 * not divide n the call fails with "expected a square grid" (the reference then
 * indexes past its array). Host FP64 arrays [batch][n]; one element per GPU
 * thread, bitwise the FP64 scan. */
int doe_error_diffusion(doe_ctx* ctx, int batch, long long n, int levels, int snake, int wrap_first,
                        const double* phase, double* out);

/* recordHologram -- src/interference.js:347-388: sum = object + reference,
 * recorded = |sum|^2 / max, plate encoded as encode 0 'raw' (recorded), 1 'binary'
 * (recorded > 0.5) or 2 'phase' (exp(i wrapPhase(arg sum)), quantised to `levels`
 * when levels > 1). Host FP64 planes of n samples; sum_re / sum_im may be NULL. */
int doe_hologram_record(doe_ctx* ctx, const double* obj_re, const double* obj_im, const double* ref_re,
                        const double* ref_im, long long n, int encode, int levels, double* plate_re,
                        double* plate_im, double* recorded, double* sum_re, double* sum_im);

/* reconstructHologram -- src/interference.js:397-411: illumination = plate *
 * reference, angular-spectrum propagated to +z (real image) and -z (virtual image)
 * as one two-plane batch. The reference's default is band_limit = 0. illum_re /
 * illum_im may be NULL. */
int doe_hologram_reconstruct(doe_ctx* ctx, const double* plate_re, const double* plate_im,
                             const double* ref_re, const double* ref_im, int nx, int ny, double dx, double dy,
                             double lambda, double z, int band_limit, int evanescent, double soft_edge,
                             double* real_re, double* real_im, double* virt_re, double* virt_im,
                             double* illum_re, double* illum_im);

/* modalIntensity -- src/interference.js:57-69: sum_m w_m |U_m|^2 / sum_m w_m over
 * M modes [M][nx*ny] (weights NULL = all 1). With z != 0 every mode is first
 * angular-spectrum propagated to z in one batch (the reference's tests propagate
 * each mode with propagateAngularSpectrumInPlace, then call modalIntensity). */
int doe_modal_intensity(doe_ctx* ctx, int modes, const double* re, const double* im, int nx, int ny,
                        const double* weights, double dx, double dy, double lambda, double z, int band_limit,
                        int evanescent, double soft_edge, double* out);

/* partiallyCoherentModes -- src/interference.js:79-125: `modes` fields [modes][nx*ny]
 * = Gaussian envelope exp(-(x^2+y^2)/waist^2) times exp(i phi), phi a uniform
 * (-pi, pi] screen from one xorshift32 stream (src/doe.js:65-75) smoothed by a
 * circular box blur of radius max(1, round(max(1, sigma/dx))) pixels. */
int doe_partially_coherent_modes(doe_ctx* ctx, int nx, int ny, double dx, double dy, int modes, double sigma,
                                 double waist, double seed, double* re, double* im);

/* gerchbergSaxton / weightedGerchbergSaxton / fourierCgh on one design. */
int doe_design(doe_ctx* ctx, const doe_design_desc* desc, doe_design_result* result);
/* n designs sharing grid, pitch, algorithm and iterations, run as one batch. */
int doe_design_batch(doe_ctx* ctx, int n, const doe_design_desc* desc, doe_design_result* result);

/* Device-resident batch: FP32 planes [batch][nx*ny] in HBM, asynchronous on the
 * context's stream. lambdas/zs (host, batch entries) may be NULL: lambda/z apply
 * to all. phase holds the initial phase on entry and the result on return. */
typedef struct doe_design_dev_desc {
  int batch, nx, ny;
  double dx, dy, lambda, z;
  const double* lambdas;
  const double* zs;
  int algorithm, iterations;
  double feedback;
  int escape;
  double beta;
  const float* illumination;
  const float* target_amp;
  const float* roi;  /* may be NULL */
  float* phase;
  float* amplitude;  /* may be NULL */
  float* weights;    /* may be NULL */
  double* error;     /* [batch][iterations], may be NULL */
  double* efficiency;
  double* rmse;      /* [batch], WGS, may be NULL */
  /* Per-design stopping goal (image-plane WGS only; no counterpart in the
   * reference, whose loop always runs `iterations`). When rmse_goal > 0 the
   * screen RMSE of src/projector.js:554-595 (target scaled to the in-ROI power,
   * intensity RMSE over the ROI) is measured on every iteration's forward field,
   * fused into the iteration's last pass; a design whose screen RMSE reaches the
   * goal returns that iterate and drops out of all later passes. screen_irr is
   * the target irradiance [batch][nx*ny] (NULL: target_amp^2, equivalent for the
   * scale-invariant RMSE). iterations_used [batch] (may be NULL) receives the
   * iterations each design ran; error/efficiency entries past that repeat the
   * last value. */
  double rmse_goal;
  const float* screen_irr;
  int* iterations_used;
} doe_design_dev_desc;
int doe_design_dev(doe_ctx* ctx, const doe_design_dev_desc* desc);

/* Autotuner of the design loops (engine-only; no reference counterpart): runs
 * the design described by desc for `iterations` iterations (<= 0: 4; the
 * screen-RMSE goal is ignored) with every shape variant of its row and column
 * passes -- the same FFT plan in every variant, so the arithmetic of a pass does
 * not change, only how its lines are grouped into CTAs and its register cap --
 * and, for image-plane WGS on a square 64^2, 128^2 or 256^2 grid, with the
 * cluster-resident loop; keeps the fastest in the context ("design_row" /
 * "design_col" variants for those lengths, the grid's "design_cluster" entry).
 * desc's output arrays are scratch during the trials; desc->phase is restored to
 * the initial phase. Allocates one phase-sized buffer for the duration of the
 * call and synchronises the stream. chosen (3 ints, may be NULL) receives {row
 * variant, column variant, cluster loop 0/1}. */
int doe_autotune_design(doe_ctx* ctx, const doe_design_dev_desc* desc, int iterations, int* chosen);

/* Designs of uneven sizes in one submission (no reference counterpart): each
 * descriptor is one size class (B designs of one grid) and runs on its own
 * sub-context and stream, forked from and joined into the context's stream.
 * mode 0 runs directly; mode 1 captures the whole submission (every pass of
 * every iteration of every class) into a CUDA graph and launches it -- call mode
 * 0 with the same shapes first so that no scratch is allocated in the capture;
 * mode 2 relaunches the last captured graph (same descriptors and arrays). */
typedef struct doe_design_multi doe_design_multi;
int doe_design_multi_create(doe_ctx* ctx, doe_design_multi** out);
void doe_design_multi_destroy(doe_design_multi* m);
int doe_design_multi_run(doe_design_multi* m, int nclasses, const doe_design_dev_desc* descs,
                         int mode);

/* gerchbergSaxtonMultiPlane -- src/doe.js:557-626. nplanes target planes at
 * distances z[p] with target_amp / roi planes p*nx*ny (roi may be NULL) and
 * weights weight[p] (NULL = 1). per_plane_error is nplanes*iterations (row p =
 * plane p); error and efficiency follow the reference (mean weighted error,
 * 1 - error). */
int doe_multiplane(doe_ctx* ctx, int nx, int ny, double dx, double dy, double lambda,
                   const double* illumination, int nplanes, const double* z,
                   const double* target_amp, const double* roi, const double* weight,
                   int iterations, const double* init_phase, double* phase, double* error,
                   double* efficiency, double* per_plane_error);

/* Batched, device-resident gerchbergSaxtonMultiPlane: B designs of one grid and
 * one set of planes (z, weight: host arrays of nplanes; weight may be NULL).
 * Device FP32 planes: illumination [batch][n], target_amp and roi
 * [batch][nplanes][n] (roi may be NULL), phase [batch][n] (initial phase in,
 * result out). Device FP64 outputs (may be NULL): error and efficiency
 * [batch][iterations], per_plane_error [batch][nplanes][iterations].
 * Asynchronous on the context's stream. */
typedef struct doe_multiplane_dev_desc {
  int batch, nx, ny;
  double dx, dy, lambda;
  int nplanes;
  const double* z;
  const double* weight;
  int iterations;
  const float* illumination;
  const float* target_amp;
  const float* roi;
  float* phase;
  double* error;
  double* efficiency;
  double* per_plane_error;
} doe_multiplane_dev_desc;
int doe_multiplane_dev(doe_ctx* ctx, const doe_multiplane_dev_desc* desc);

/* ------------------------------------------------------------ projector */
/* ProjectorSystem.simulate -- src/projector.js:475-498: the element A exp(i phi)
 * (illumination, phase: nx*ny FP64) is formed on the device, zero-padded to
 * pad*nx x pad*ny (image plane, src/field.js:443-461), propagated by the angular
 * spectrum to z (band_limit as given), centre-cropped; far_field instead applies
 * focalPlaneSpectrum with f = z. out_d receives the screen pitch. */
int doe_simulate(doe_ctx* ctx, const double* illumination, const double* phase, int nx, int ny,
                 double dx, double dy, double lambda, double z, int band_limit, int far_field,
                 int pad, double* out_re, double* out_im, double* out_d);

/* ProjectorSystem.simulate at nz distances z[] (defocusCurve / focusStack,
 * src/projector.js:622-653, call simulate once per distance): the element's
 * forward transform is computed once and shared by every distance. out_re /
 * out_im are [nz][nx*ny]; out_d (may be NULL) receives nz (dx, dy) pairs, the
 * screen pitch of each plane (lens throws give lambda*z/(n*dx)). Same planes as
 * nz calls of doe_simulate. */
int doe_simulate_sweep(doe_ctx* ctx, const double* illumination, const double* phase, int nx, int ny,
                       double dx, double dy, double lambda, const double* z, int nz, int band_limit,
                       int far_field, int pad, double* out_re, double* out_im, double* out_d);

/* ProjectorSystem.screenMetrics, radiometric subset -- src/projector.js:554-595
 * with src/metrics.js:10-18, :73-84: out = {rmse, efficiency, fluxFraction,
 * powerInSignal, powerAtScreen, powerIncident}. roi may be NULL. */
int doe_screen_metrics(doe_ctx* ctx, const double* re, const double* im, int nx, int ny,
                       double sdx, double sdy, const double* target_irr, const double* roi,
                       const double* illumination, double dx, double dy, double* out);

/* ProjectorSystem.screenMetrics, every field -- src/projector.js:554-614 with
 * src/metrics.js:37-321: out[18] = {efficiency, fluxFraction, uniformity,
 * spotUniformity (NaN unless grid_cols, grid_rows > 0), flatness, contrast, rmse,
 * fidelity, correlation, ssim (8x8 windows, target-weighted), snr, zeroOrder (of
 * the element field illumination * exp(i phase)), rmsRadius, meanIntensity,
 * peakIntensity, powerInSignal, powerAtScreen, powerIncident}. roi may be NULL. */
int doe_screen_metrics_full(doe_ctx* ctx, const double* re, const double* im, int nx, int ny,
                            double sdx, double sdy, const double* target_irr, const double* roi,
                            const double* illumination, const double* phase, double dx, double dy,
                            int grid_cols, int grid_rows, double* out);

/* Batched screen metrics of B device-resident screens given by their amplitudes
 * (FP32 [B][nx*ny]); target/roi/illumination use the given design strides (0 =
 * shared). out is a device array [B][6] in the order of doe_screen_metrics.
 * Asynchronous on the context's stream. */
int doe_screen_metrics_dev(doe_ctx* ctx, int batch, int nx, int ny, const float* amplitude,
                           const float* target_irr, long long target_stride, const float* roi,
                           const float* illumination, long long illumination_stride, double sdx,
                           double sdy, double dx, double dy, double* out);

/* ------------------------------------------------------------ warm-start surrogate */
/* No counterpart in the reference. Intensity loss of B DOE phases through the
 * image-plane propagation of the design loops (bandLimit false) and its gradient:
 *   L = sum m (|U|^2 - t^2)^2 / sum m t^4,  U = P(A e^{i phase}),
 * grad = dL/dphase. Device FP32 planes [batch][nx*ny] (roi may be NULL); loss is a
 * device FP64 array [batch] (may be NULL). Asynchronous on the context's stream. */
typedef struct doe_phase_loss_desc {
  int batch, nx, ny;
  double dx, dy, lambda, z;
  const float* illumination;
  const float* target_amp;
  const float* roi;
  const float* phase;
  float* grad;
  double* loss;
} doe_phase_loss_desc;
int doe_phase_loss_grad(doe_ctx* ctx, const doe_phase_loss_desc* desc);

/* A U-Net (levels of base << l channels, 3x3 convolutions + ReLU, 2x2 average
 * pooling, nearest up-sampling, skip concatenation, 1x1 head to (c, s), phase =
 * atan2(s, c)) with BF16 weights and activations, FP32 accumulation and FP32
 * master weights under Adam. Input: target irradiance (scaled by its maximum) and
 * ROI planes of n x n (plus a constant plane). All device arrays; calls are asynchronous on the context's
 * stream except the parameter copies. */
typedef struct doe_surrogate doe_surrogate;
int doe_surrogate_create(doe_ctx* ctx, int n, int base, int levels, int max_batch,
                         unsigned long long seed, doe_surrogate** out);
void doe_surrogate_destroy(doe_surrogate* s);
long long doe_surrogate_param_count(const doe_surrogate* s);
/* which = 0: FP32 weights, 1: accumulated gradients (host array of param_count) */
int doe_surrogate_params(doe_surrogate* s, float* host_out, int which);
int doe_surrogate_set_params(doe_surrogate* s, const float* host_in);
int doe_surrogate_forward(doe_surrogate* s, int batch, const float* d_irr, const float* d_roi,
                          float* d_phase);
/* back-propagates d_dphase = dL/dphase [batch][n*n] of the last forward pass and
 * accumulates the parameter gradients */
int doe_surrogate_backward(doe_surrogate* s, const float* d_dphase);
int doe_surrogate_zero_grad(doe_surrogate* s);
/* device copies of the FP32 gradient buffer (param_count floats), for the
 * all-reduce of data-parallel training between backward and Adam */
int doe_surrogate_grads_dev(doe_surrogate* s, float* d_out);
int doe_surrogate_set_grads_dev(doe_surrogate* s, const float* d_in);
/* Adam with decoupled weight decay on grad * grad_scale; zeroes the gradients */
int doe_surrogate_adam(doe_surrogate* s, float lr, float beta1, float beta2, float eps,
                       float weight_decay, float grad_scale);
/* supervised phase loss L = mean(1 - cos(phase - target)) over B*n pixels:
 * grad = sin(phase - target) / (B n); loss (device FP64 [1], may be NULL) */
int doe_phase_supervised_grad(doe_ctx* ctx, long long count, const float* d_phase,
                              const float* d_target, float* d_grad, double* d_loss);

/* ------------------------------------------------------------ allocation-free */
/* No counterpart in the reference. Angular-spectrum propagation of one complex64
 * plane for callers that must not allocate device memory (a host runtime that owns
 * every device allocation, or a latency-critical loop that cannot afford the
 * allocator's implicit synchronisation). The caller passes device input and
 * output planes (they may alias) and a CUDA stream (NULL = default stream); the
 * routine needs no context and allocates nothing: its scratch is a fixed
 * 2.6 MiB array that every GPU loading this library holds until exit. Limit:
 * nx*ny <= 262144 samples (e.g. 512x512), each axis <= 8192; larger grids return
 * DOE_ERR_UNSUPPORTED. The first call on a device sets the scratch up and
 * synchronises the stream once; make it before any stream capture. Calls whose
 * work overlaps on the GPU share the scratch and race: serialise them. The error
 * message, if any, is written to err (err_len bytes, may be NULL). */
int doe_asm_c64_noalloc(const void* d_in, void* d_out, int nx, int ny, double dx, double dy,
                        double lambda, double z, int band_limit, int evanescent,
                        double soft_edge, void* stream, char* err, int err_len);

#ifdef __cplusplus
}
#endif
#endif /* DOE_B200_H */
