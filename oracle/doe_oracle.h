/*
 * doe_oracle.h -- FP64 CPU restatement of the reference's propagate-and-retrieve
 * path (Ziggyware/DiffractiveOpticalElement, plain JavaScript).
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker for the CUDA
 * engine and the timed CPU baseline of bench.py. Nothing in the product package
 * links or calls it.
 *
 * Every routine keeps the reference's operation order (same loops, same
 * accumulation order, same twiddle tables) so that its results differ from the
 * JavaScript only by the last-ulp differences between V8's and glibc's
 * cos/sin/atan2/pow/hypot. Each function names the reference file:line it follows.
 *
 * Layout: complex fields are split re/im double planes, row-major, idx = i + j*nx,
 * optical axis at the array centre (src/field.js:8-16).
 */
#ifndef DOE_ORACLE_H
#define DOE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/fft.js:86-139 -- in-place radix-2 DIT over a strided slice. */
int orc_fft1d(double* re, double* im, int n, long stride, long offset, int inverse);
/* src/fft.js:148-154 -- rows then columns; inverse carries 1/(nx*ny). */
int orc_fft2d(double* re, double* im, int nx, int ny, int inverse);
/* src/fft.js:188-202 -- quadrant swap (shift=1 fftshift, 0 ifftshift). */
void orc_fftshift2d(double* re, double* im, int nx, int ny, int shift);
/* src/fft.js:208-237 -- O(N^4) oracle DFT. */
void orc_dft2d_naive(const double* re, const double* im, int nx, int ny, int inverse,
                     double* out_re, double* out_im);

/* src/propagate.js:48-51 */
double orc_local_frequency_limit(int n, double d, double lambda, double z);
/* src/propagate.js:57-102; returns propagatingFraction. */
double orc_asm_transfer(int nx, int ny, double dx, double dy, double lambda, double z,
                        int band_limit, int evanescent, double soft_edge,
                        double* h_re, double* h_im);
/* src/propagate.js:112-133 */
void orc_asm_inplace(double* re, double* im, int nx, int ny, double dx, double dy,
                     double lambda, double z, int band_limit, int evanescent, double soft_edge);
/* src/propagate.js:342-374 (output pitch written to out_d[0..1]). */
void orc_focal_plane(const double* re, const double* im, int nx, int ny, double dx, double dy,
                     double lambda, double f, double* out_re, double* out_im, double* out_d);
/* src/propagate.js:155-239 (out_d = {dux, duy}). */
void orc_fresnel_fft(const double* re, const double* im, int nx, int ny, double dx, double dy,
                     double lambda, double z, double* out_re, double* out_im, double* out_d);
/* src/propagate.js:246-316 (field pitch dux/duy in, DOE pitch dx/dy out). */
void orc_fresnel_fft_inverse(const double* re, const double* im, int nx, int ny, double dux,
                             double duy, double lambda, double z, double dx, double dy,
                             double* out_re, double* out_im);

/* src/field.js:516-536 */
void orc_disc_mask(int nx, int ny, double dx, double dy, double radius, double soft,
                   double cx, double cy, double* out);
/* src/field.js:539-558 */
void orc_rect_mask(int nx, int ny, double dx, double dy, double width, double height,
                   double soft, double* out);

/* src/doe.js:65-75 -- xorshift32; state carried by the caller. */
double orc_rng_next(uint32_t* state);
uint32_t orc_rng_seed(double seed);
/* src/doe.js:81-86 */
void orc_random_phase(int nx, int ny, double seed, double* out);

/*
 * Design options shared by the GS-family loops (src/doe.js:49-59, :327-335).
 * Null pointers mean "absent" exactly as `undefined` does in the reference.
 */
typedef struct {
  int nx, ny;
  double dx, dy, lambda, z;
  int iterations;
  double feedback; /* HIO feedback */
  int escape;      /* iterations before feedback kicks in */
  double beta;     /* WGS exponent */
  double seed;     /* fourierCgh default init phase seed */
  const double* roi;        /* may be NULL */
  const double* weights;    /* may be NULL */
  const double* init_phase; /* may be NULL */
} orc_design_opts;

/*
 * Results. Arrays are caller-allocated: phase, amplitude, intensity have nx*ny
 * entries, error/efficiency have `iterations` entries; weights (WGS only) nx*ny.
 */
typedef struct {
  double* phase;
  double* amplitude;
  double* intensity;
  double* error;
  double* efficiency;
  double* weights; /* WGS: final weights */
  double rmse;     /* WGS: best unweighted ROI RMSE */
} orc_design_result;

/* src/doe.js:327-437 */
int orc_gerchberg_saxton(const double* illumination, const double* target_amp,
                         const orc_design_opts* o, orc_design_result* r);
/* src/doe.js:639-730 */
int orc_fourier_cgh(const double* illumination, const double* target_amp,
                    const orc_design_opts* o, orc_design_result* r);
/* src/doe.js:455-546; base = 0 gerchbergSaxton, 1 fourierCgh */
int orc_weighted_gs(const double* illumination, const double* target_amp,
                    const orc_design_opts* o, int base, orc_design_result* r);
/* Image-plane WGS stopped at a screen-RMSE goal (engine extension, see the .c). */
int orc_weighted_gs_goal(const double* illumination, const double* target_amp,
                         const orc_design_opts* o, const double* screen_irr, double goal,
                         int* used, orc_design_result* r);
/* src/doe.js:557-626. Plane p uses z[p], target_amp + p*n, roi + p*n (roi may be NULL),
 * weight[p]. per_plane_error is nplanes*iterations (row p = plane p). */
int orc_gs_multiplane(const double* illumination, int nplanes, const double* z,
                      const double* target_amp, const double* roi, const double* weight,
                      const orc_design_opts* o, double* phase, double* error,
                      double* efficiency, double* per_plane_error);

/* src/projector.js:262-315 */
void orc_auto_roi(const double* irr, int nx, int ny, double dilate, double soft,
                  double threshold, double* out);
/*
 * src/projector.js:554-595 rmse / efficiency / fluxFraction subset of screenMetrics.
 * out = {rmse, efficiency, fluxFraction, powerInSignal, powerAtScreen, powerIncident}.
 */
/* src/doe.js:164-173, :185-226 */
void orc_quantize_phase(const double* phi, long n, int levels, double* out);
int orc_error_diffusion(const double* phi, long n, int levels, int snake, int wrap_first, double* out);
void orc_screen_metrics(const double* field_re, const double* field_im, int nx, int ny,
                        double sdx, double sdy, const double* target_irr, const double* roi,
                        const double* illumination, double dx, double dy, double* out);
/* src/projector.js:554-614 with src/metrics.js (all fields), out[18] */
void orc_screen_metrics_full(const double* field_re, const double* field_im, int nx, int ny,
                             double sdx, double sdy, const double* target_irr, const double* roi,
                             const double* illumination, const double* phase, double dx, double dy,
                             int grid_cols, int grid_rows, double* out);

/* src/doe.js:817-829 target amplitude and power match. */
void orc_prepare_target(const double* irr, const double* illumination, long n, double* out);

/* src/interference.js:57-69 modalIntensity of M modes [M][n] (w NULL = all 1). */
void orc_modal_intensity(int M, const double* re, const double* im, long n, const double* w, double* out);
/* src/interference.js:347-388 recordHologram (encode 0 raw, 1 binary, 2 phase). */
void orc_record_hologram(const double* obj_re, const double* obj_im, const double* ref_re, const double* ref_im,
                         long n, int encode, int levels, double* plate_re, double* plate_im, double* recorded,
                         double* sum_re, double* sum_im);
/* src/interference.js:397-411 reconstructHologram (real image at +z, virtual at -z). */
void orc_reconstruct_hologram(const double* plate_re, const double* plate_im, const double* ref_re,
                              const double* ref_im, int nx, int ny, double dx, double dy, double lambda, double z,
                              int band_limit, int evanescent, double soft_edge, double* real_re, double* real_im,
                              double* virt_re, double* virt_im, double* illum_re, double* illum_im);
/* src/interference.js:79-125 partiallyCoherentModes, modes [M][n]. */
void orc_partially_coherent_modes(int nx, int ny, double dx, double dy, int modes, double sigma, double waist,
                                  double seed, double* re, double* im);

#ifdef __cplusplus
}
#endif
#endif
