/*
 * doe_oracle.c -- FP64 CPU restatement of the reference's propagate-and-retrieve
 * path. TEST INFRASTRUCTURE ONLY: the parity checker and timed CPU baseline.
 * The product (diffractiveopticalelement_b200) never links or calls it.
 *
 * Build without -ffast-math (see oracle/Makefile): operation order matters.
 * Each function cites the reference file:line (paths inside the reference
 * project) whose loop it restates.
 */
#include "doe_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ */
/* Twiddles: src/fft.js:29-48. One table per power-of-two length, built once
 * for every length up to 2^MAX_LOG2 (the reference caches them lazily; the
 * values are identical). */
#define MAX_LOG2 16
static double* g_tw_cos[MAX_LOG2 + 1];
static double* g_tw_sin[MAX_LOG2 + 1];
static pthread_once_t g_tw_once = PTHREAD_ONCE_INIT;

static void build_twiddles(void) {
  for (int lg = 1; lg <= MAX_LOG2; lg++) {
    int n = 1 << lg;
    int half = n >> 1;
    g_tw_cos[lg] = (double*)malloc(sizeof(double) * half);
    g_tw_sin[lg] = (double*)malloc(sizeof(double) * half);
    for (int k = 0; k < half; k++) {
      double a = (-2.0 * M_PI * (double)k) / (double)n;
      g_tw_cos[lg][k] = cos(a);
      g_tw_sin[lg][k] = sin(a);
    }
  }
}

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

/* src/fft.js:86-139 */
int orc_fft1d(double* re, double* im, int n, long stride, long offset, int inverse) {
  if (n <= 1) return 0;
  if (!is_pow2(n) || n > (1 << MAX_LOG2)) return -1;
  pthread_once(&g_tw_once, build_twiddles);
  /* bit-reversal permutation (src/fft.js:91-105) */
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      long ia = offset + (long)i * stride;
      long ja = offset + (long)j * stride;
      double tr = re[ia];
      re[ia] = re[ja];
      re[ja] = tr;
      double ti = im[ia];
      im[ia] = im[ja];
      im[ja] = ti;
    }
  }
  /* butterflies (src/fft.js:108-129) */
  for (int len = 2, lg = 1; len <= n; len <<= 1, lg++) {
    int half = len >> 1;
    const double* cs = g_tw_cos[lg];
    const double* sn = g_tw_sin[lg];
    for (int base = 0; base < n; base += len) {
      long b0 = offset + (long)base * stride;
      for (int k = 0; k < half; k++) {
        double wr = cs[k];
        double wi = inverse ? -sn[k] : sn[k];
        long p = b0 + (long)k * stride;
        long q = p + (long)half * stride;
        double xr = re[q];
        double xi = im[q];
        double tr = xr * wr - xi * wi;
        double ti = xr * wi + xi * wr;
        re[q] = re[p] - tr;
        im[q] = im[p] - ti;
        re[p] += tr;
        im[p] += ti;
      }
    }
  }
  /* per-pass 1/n (src/fft.js:131-138) */
  if (inverse) {
    double s = 1.0 / (double)n;
    for (int i = 0; i < n; i++) {
      long p = offset + (long)i * stride;
      re[p] *= s;
      im[p] *= s;
    }
  }
  return 0;
}

/* src/fft.js:148-154 */
int orc_fft2d(double* re, double* im, int nx, int ny, int inverse) {
  if (!is_pow2(nx) || !is_pow2(ny)) return -1;
  for (int y = 0; y < ny; y++)
    if (orc_fft1d(re, im, nx, 1, (long)y * nx, inverse)) return -1;
  for (int x = 0; x < nx; x++)
    if (orc_fft1d(re, im, ny, nx, x, inverse)) return -1;
  return 0;
}

/* src/fft.js:170-181 */
static void fftshift1d(double* arr, int n, int shift, long stride, long offset) {
  int m = n >> 1;
  int d = shift ? m : n - m;
  for (int i = 0; i < m; i++) {
    long a = offset + (long)i * stride;
    long b = offset + (long)((i + d) % n) * stride;
    double t = arr[a];
    arr[a] = arr[b];
    arr[b] = t;
  }
}

/* src/fft.js:188-202 */
void orc_fftshift2d(double* re, double* im, int nx, int ny, int shift) {
  for (int y = 0; y < ny; y++) {
    long row = (long)y * nx;
    fftshift1d(re, nx, shift, 1, row);
    if (im) fftshift1d(im, nx, shift, 1, row);
  }
  for (int x = 0; x < nx; x++) {
    fftshift1d(re, ny, shift, nx, x);
    if (im) fftshift1d(im, ny, shift, nx, x);
  }
}

/* src/fft.js:208-237 */
void orc_dft2d_naive(const double* re, const double* im, int nx, int ny, int inverse,
                     double* out_re, double* out_im) {
  double sign = inverse ? 1.0 : -1.0;
  double scale = inverse ? 1.0 / (double)(nx * ny) : 1.0;
  for (int ky = 0; ky < ny; ky++) {
    for (int kx = 0; kx < nx; kx++) {
      double sr = 0, si = 0;
      for (int y = 0; y < ny; y++) {
        double ay = (sign * 2.0 * M_PI * ky * y) / ny;
        double cy = cos(ay), sy = sin(ay);
        for (int x = 0; x < nx; x++) {
          double ax = (sign * 2.0 * M_PI * kx * x) / nx;
          double c = cos(ax) * cy - sin(ax) * sy;
          double s = sin(ax) * cy + cos(ax) * sy;
          double vr = re[x + y * nx];
          double vi = im[x + y * nx];
          sr += vr * c - vi * s;
          si += vr * s + vi * c;
        }
      }
      long o = kx + (long)ky * nx;
      out_re[o] = sr * scale;
      out_im[o] = si * scale;
    }
  }
}

/* ------------------------------------------------------------------ */
/* src/propagate.js:38-42 */
static double soft_window(double v, double lim, double inner) {
  if (v <= inner) return 1;
  if (v >= lim) return 0;
  return 0.5 * (1 + cos((M_PI * (v - inner)) / (lim - inner)));
}

/* src/propagate.js:48-51 */
double orc_local_frequency_limit(int n, double d, double lambda, double z) {
  double df = 1.0 / (n * d);
  return 1.0 / (lambda * sqrt(pow(2 * df * z, 2) + 1));
}

/* src/propagate.js:57-102 */
double orc_asm_transfer(int nx, int ny, double dx, double dy, double lambda, double z,
                        int band_limit, int evanescent, double soft_edge, double* re,
                        double* im) {
  double dfx = 1.0 / (nx * dx);
  double dfy = 1.0 / (ny * dy);
  double invL2 = 1.0 / (lambda * lambda);
  double fxLim = band_limit ? orc_local_frequency_limit(nx, dx, lambda, z) : INFINITY;
  double fyLim = band_limit ? orc_local_frequency_limit(ny, dy, lambda, z) : INFINITY;
  double fxn = 1.0 / (2 * dx);
  double fyn = 1.0 / (2 * dy);
  long propagating = 0;
  for (int j = 0; j < ny; j++) {
    double fy = (j - ny / 2.0) * dfy;
    double limY = fmin(fyLim, fyn);
    double wy = isinf(fyLim) ? 1 : soft_window(fabs(fy), limY, limY * (1 - soft_edge));
    for (int i = 0; i < nx; i++) {
      double fx = (i - nx / 2.0) * dfx;
      double limX = fmin(fxLim, fxn);
      double wx = isinf(fxLim) ? 1 : soft_window(fabs(fx), limX, limX * (1 - soft_edge));
      double arg = invL2 - fx * fx - fy * fy;
      long k = i + (long)j * nx;
      if (arg >= 0) {
        double phase = 2 * M_PI * z * sqrt(arg);
        double w = wx * wy;
        re[k] = w * cos(phase);
        im[k] = w * sin(phase);
        if (w > 0.5) propagating++;
      } else if (evanescent) {
        re[k] = 0;
        im[k] = 0;
      } else {
        double w = wx * wy;
        double phase = 2 * M_PI * z * sqrt(-arg);
        re[k] = w * cos(phase);
        im[k] = w * sin(phase);
        propagating++;
      }
    }
  }
  return (double)propagating / (double)((long)nx * ny);
}

/* src/propagate.js:112-133 */
void orc_asm_inplace(double* re, double* im, int nx, int ny, double dx, double dy,
                     double lambda, double z, int band_limit, int evanescent,
                     double soft_edge) {
  if (z == 0) return;
  long n = (long)nx * ny;
  orc_fftshift2d(re, im, nx, ny, 0);
  orc_fft2d(re, im, nx, ny, 0);
  orc_fftshift2d(re, im, nx, ny, 1);
  double* hr = (double*)malloc(sizeof(double) * n);
  double* hi = (double*)malloc(sizeof(double) * n);
  orc_asm_transfer(nx, ny, dx, dy, lambda, z, band_limit, evanescent, soft_edge, hr, hi);
  for (long k = 0; k < n; k++) {
    double ur = re[k], ui = im[k];
    re[k] = ur * hr[k] - ui * hi[k];
    im[k] = ur * hi[k] + ui * hr[k];
  }
  free(hr);
  free(hi);
  orc_fftshift2d(re, im, nx, ny, 0);
  orc_fft2d(re, im, nx, ny, 1);
  orc_fftshift2d(re, im, nx, ny, 1);
}

/* src/propagate.js:342-374 */
void orc_focal_plane(const double* in_re, const double* in_im, int nx, int ny, double dx,
                     double dy, double lambda, double f, double* re, double* im,
                     double* out_d) {
  long n = (long)nx * ny;
  memcpy(re, in_re, sizeof(double) * n);
  memcpy(im, in_im, sizeof(double) * n);
  orc_fftshift2d(re, im, nx, ny, 0);
  orc_fft2d(re, im, nx, ny, 0);
  orc_fftshift2d(re, im, nx, ny, 1);
  double dux = (lambda * f) / (nx * dx);
  double duy = (lambda * f) / (ny * dy);
  double amp0 = (dx * dy) / (lambda * f);
  for (int j = 0; j < ny; j++) {
    double v = (j - ny / 2.0) * duy;
    for (int i = 0; i < nx; i++) {
      double u = (i - nx / 2.0) * dux;
      long idx = i + (long)j * nx;
      double q = (M_PI * (u * u + v * v)) / (lambda * f) - M_PI / 2;
      double c = amp0 * cos(q);
      double s = amp0 * sin(q);
      double ur = re[idx], ui = im[idx];
      re[idx] = ur * c - ui * s;
      im[idx] = ur * s + ui * c;
    }
  }
  if (out_d) {
    out_d[0] = dux;
    out_d[1] = duy;
  }
}

/* src/propagate.js:155-239 */
void orc_fresnel_fft(const double* in_re, const double* in_im, int nx, int ny, double dx,
                     double dy, double lambda, double z, double* re, double* im,
                     double* out_d) {
  double az = fabs(z);
  double k = (2 * M_PI) / lambda;
  double dux = (lambda * az) / (nx * dx);
  double duy = (lambda * az) / (ny * dy);
  for (int j = 0; j < ny; j++) {
    double y = (j - ny / 2.0) * dy;
    for (int i = 0; i < nx; i++) {
      double x = (i - nx / 2.0) * dx;
      double q = (M_PI * (x * x + y * y)) / (lambda * az);
      double c = ((i + j) % 2) ? -cos(q) : cos(q);
      double s = ((i + j) % 2) ? -sin(q) : sin(q);
      long idx = i + (long)j * nx;
      double ur = in_re[idx], ui = in_im[idx];
      re[idx] = ur * c - ui * s;
      im[idx] = ur * s + ui * c;
    }
  }
  orc_fft2d(re, im, nx, ny, 0);
  double amp = (dx * dy) / (lambda * az);
  double kz = k * z - (M_PI * (nx + ny)) / 2;
  double ckz = cos(kz), skz = sin(kz);
  double pr = amp * skz;
  double pj = -amp * ckz;
  for (int j = 0; j < ny; j++) {
    double v = ((j - ny / 2.0) * dy) * 0 + (j - ny / 2.0) * duy;
    for (int i = 0; i < nx; i++) {
      double u = (i - nx / 2.0) * dux;
      double q = (M_PI * (u * u + v * v)) / (lambda * az);
      double c = ((i + j) % 2) ? -cos(q) : cos(q);
      double s = ((i + j) % 2) ? -sin(q) : sin(q);
      long idx = i + (long)j * nx;
      double ur = re[idx], ui = im[idx];
      double tr = ur * pr - ui * pj;
      double ti = ur * pj + ui * pr;
      re[idx] = tr * c - ti * s;
      im[idx] = tr * s + ti * c;
    }
  }
  if (out_d) {
    out_d[0] = dux;
    out_d[1] = duy;
  }
}

/* src/propagate.js:246-316 */
void orc_fresnel_fft_inverse(const double* in_re, const double* in_im, int nx, int ny,
                             double dux, double duy, double lambda, double z, double dx,
                             double dy, double* re, double* im) {
  double az = fabs(z);
  double k = (2 * M_PI) / lambda;
  for (int j = 0; j < ny; j++) {
    double v = (j - ny / 2.0) * duy;
    for (int i = 0; i < nx; i++) {
      double u = (i - nx / 2.0) * dux;
      double q = (M_PI * (u * u + v * v)) / (lambda * az);
      double sg = ((i + j) % 2) ? -1 : 1;
      double c = sg * cos(q);
      double s = -sg * sin(q);
      long idx = i + (long)j * nx;
      double ur = in_re[idx], ui = in_im[idx];
      re[idx] = ur * c - ui * s;
      im[idx] = ur * s + ui * c;
    }
  }
  orc_fft2d(re, im, nx, ny, 1);
  double amp = (lambda * az) / (dx * dy);
  double kg = k * z - (M_PI * (nx + ny)) / 2 - M_PI / 2;
  double cg = cos(kg), sg2 = sin(kg);
  double pr = amp * cg;
  double pj = -amp * sg2;
  for (int j = 0; j < ny; j++) {
    double y = (j - ny / 2.0) * dy;
    for (int i = 0; i < nx; i++) {
      double x = (i - nx / 2.0) * dx;
      double q = (M_PI * (x * x + y * y)) / (lambda * az);
      double sg = ((i + j) % 2) ? -1 : 1;
      double c = sg * cos(q);
      double s = -sg * sin(q);
      long idx = i + (long)j * nx;
      double ur = re[idx], ui = im[idx];
      double tr = ur * pr - ui * pj;
      double ti = ur * pj + ui * pr;
      re[idx] = tr * c - ti * s;
      im[idx] = tr * s + ti * c;
    }
  }
}

/* ------------------------------------------------------------------ */
/* src/field.js:516-536 */
void orc_disc_mask(int nx, int ny, double dx, double dy, double radius, double soft,
                   double cx, double cy, double* m) {
  for (int j = 0; j < ny; j++) {
    double y = (j - ny / 2.0) * dy - cy;
    for (int i = 0; i < nx; i++) {
      double x = (i - nx / 2.0) * dx - cx;
      double r = hypot(x, y);
      double v;
      if (soft > 0) {
        v = r <= radius - soft ? 1
            : r >= radius      ? 0
                               : 0.5 * (1 + cos((M_PI * (r - radius + soft)) / soft));
      } else {
        v = r <= radius ? 1 : 0;
      }
      m[i + (long)j * nx] = v;
    }
  }
}

/* src/field.js:554-558 */
static double edge_fn(double x, double half, double soft) {
  if (x <= half - soft) return 1;
  if (x >= half) return 0;
  return 0.5 * (1 + cos((M_PI * (x - half + soft)) / soft));
}

/* src/field.js:539-552 */
void orc_rect_mask(int nx, int ny, double dx, double dy, double width, double height,
                   double soft, double* m) {
  for (int j = 0; j < ny; j++) {
    double y = fabs((j - ny / 2.0) * dy);
    for (int i = 0; i < nx; i++) {
      double x = fabs((i - nx / 2.0) * dx);
      double fx = soft > 0 ? edge_fn(x, width / 2, soft) : (x <= width / 2 ? 1 : 0);
      double fy = soft > 0 ? edge_fn(y, height / 2, soft) : (y <= height / 2 ? 1 : 0);
      m[i + (long)j * nx] = fx * fy;
    }
  }
}

/* ------------------------------------------------------------------ */
/* src/doe.js:65-75: `seed >>> 0 || 1` then xorshift32 (13, 17, 5). */
uint32_t orc_rng_seed(double seed) {
  /* ToUint32: truncate toward zero, modulo 2^32. */
  double t = trunc(seed);
  double m = fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  uint32_t s = (uint32_t)m;
  return s ? s : 1u;
}

double orc_rng_next(uint32_t* state) {
  uint32_t s = *state;
  s ^= s << 13;
  s ^= s >> 17;
  s ^= s << 5;
  *state = s;
  return (double)s / 4294967296.0;
}

/* src/doe.js:81-86 */
void orc_random_phase(int nx, int ny, double seed, double* p) {
  uint32_t st = orc_rng_seed(seed);
  long n = (long)nx * ny;
  for (long k = 0; k < n; k++) p[k] = (orc_rng_next(&st) * 2 - 1) * M_PI;
}

/* ------------------------------------------------------------------ */
/* src/doe.js:327-437 */
int orc_gerchberg_saxton(const double* illumination, const double* targetAmp,
                         const orc_design_opts* o, orc_design_result* r) {
  int nx = o->nx, ny = o->ny;
  long n = (long)nx * ny;
  double dx = o->dx, dy = o->dy;
  const double* roi = o->roi;
  const double* weights = o->weights;
  double* re = (double*)malloc(sizeof(double) * n);
  double* im = (double*)malloc(sizeof(double) * n);
  double* amp = (double*)malloc(sizeof(double) * n);
  if (!re || !im || !amp) return -2;
  double* phase = r->phase;
  if (o->init_phase) {
    if (phase != o->init_phase) memcpy(phase, o->init_phase, sizeof(double) * n);
  } else {
    memset(phase, 0, sizeof(double) * n);
  }
  for (int it = 0; it < o->iterations; it++) {
    /* forward: setAmplitudePhase + copyFrom + ASM(+z) (src/doe.js:350-352) */
    for (long k = 0; k < n; k++) {
      re[k] = illumination[k] * cos(phase[k]);
      im[k] = illumination[k] * sin(phase[k]);
    }
    orc_asm_inplace(re, im, nx, ny, dx, dy, o->lambda, o->z, 0, 1, 0.02);
    /* measurement (src/doe.js:355-377) */
    double errNum = 0, errDen = 0, inRoi = 0, total = 0;
    for (long k = 0; k < n; k++) {
      double a = hypot(re[k], im[k]);
      double i2 = a * a;
      amp[k] = a;
      total += i2;
      double m = roi ? roi[k] : 1;
      double t = targetAmp[k] * (weights ? weights[k] : 1);
      if (m > 0) {
        inRoi += i2 * m;
        if (t > 0 || i2 > 0) {
          double d = a * m - t * m;
          errNum += d * d;
          errDen += t * t;
        }
      }
    }
    if (r->error) r->error[it] = errDen > 0 ? sqrt(errNum / errDen) : 0;
    if (r->efficiency) r->efficiency[it] = total > 0 ? (inRoi * dx * dy) / (total * dx * dy) : 0;
    /* constraint (src/doe.js:380-397) */
    double fb = it >= o->escape ? o->feedback : 0;
    for (long k = 0; k < n; k++) {
      double m = roi ? roi[k] : 1;
      double t = targetAmp[k] * (weights ? weights[k] : 1);
      double a = amp[k];
      double newAmp;
      if (m > 0) {
        newAmp = t;
        if (fb > 0 && a > 0) newAmp = t + fb * (a - t);
      } else {
        newAmp = a * (1 - fb) + fb * a;
      }
      if (a > 0) {
        double s = newAmp / a;
        re[k] *= s;
        im[k] *= s;
      }
    }
    /* back-propagate, keep the phase (src/doe.js:400-410) */
    orc_asm_inplace(re, im, nx, ny, dx, dy, o->lambda, -o->z, 0, 1, 0.02);
    for (long k = 0; k < n; k++) phase[k] = atan2(im[k], re[k]);
  }
  /* final honest forward pass (src/doe.js:418-426) */
  for (long k = 0; k < n; k++) {
    re[k] = illumination[k] * cos(phase[k]);
    im[k] = illumination[k] * sin(phase[k]);
  }
  orc_asm_inplace(re, im, nx, ny, dx, dy, o->lambda, o->z, 0, 1, 0.02);
  for (long k = 0; k < n; k++) {
    double a = hypot(re[k], im[k]);
    if (r->amplitude) r->amplitude[k] = a;
    if (r->intensity) r->intensity[k] = a * a;
  }
  free(re);
  free(im);
  free(amp);
  return 0;
}

/* src/doe.js:639-730 */
int orc_fourier_cgh(const double* illumination, const double* targetAmp,
                    const orc_design_opts* o, orc_design_result* r) {
  int nx = o->nx, ny = o->ny;
  long n = (long)nx * ny;
  const double* roi = o->roi;
  const double* weights = o->weights;
  double* re = (double*)malloc(sizeof(double) * n);
  double* im = (double*)malloc(sizeof(double) * n);
  if (!re || !im) return -2;
  double* phase = r->phase;
  if (o->init_phase) {
    if (phase != o->init_phase) memcpy(phase, o->init_phase, sizeof(double) * n);
  } else {
    orc_random_phase(nx, ny, o->seed, phase);
  }
  double norm = 1.0 / sqrt((double)nx * ny);
  for (int it = 0; it < o->iterations; it++) {
    for (long k = 0; k < n; k++) {
      double a = illumination[k];
      re[k] = a * cos(phase[k]);
      im[k] = a * sin(phase[k]);
    }
    orc_fftshift2d(re, im, nx, ny, 0);
    orc_fft2d(re, im, nx, ny, 0);
    orc_fftshift2d(re, im, nx, ny, 1);
    for (long k = 0; k < n; k++) {
      re[k] *= norm;
      im[k] *= norm;
    }
    double errNum = 0, errDen = 0, inRoi = 0, total = 0;
    for (long k = 0; k < n; k++) {
      double a = hypot(re[k], im[k]);
      if (r->amplitude) r->amplitude[k] = a;
      if (r->intensity) r->intensity[k] = a * a;
      total += a * a;
      double m = roi ? roi[k] : 1;
      double t = targetAmp[k] * (weights ? weights[k] : 1);
      if (m > 0) {
        inRoi += a * a * m;
        double d = (a - t) * m;
        errNum += d * d;
        errDen += t * t;
      }
    }
    if (r->error) r->error[it] = errDen > 0 ? sqrt(errNum / errDen) : 0;
    if (r->efficiency) r->efficiency[it] = total > 0 ? inRoi / total : 0;
    for (long k = 0; k < n; k++) {
      double m = roi ? roi[k] : 1;
      double a = hypot(re[k], im[k]);
      double t = m > 0 ? targetAmp[k] * (weights ? weights[k] : 1) : a;
      if (a > 0) {
        double s = t / a;
        re[k] *= s;
        im[k] *= s;
      } else {
        re[k] = t;
        im[k] = 0;
      }
    }
    orc_fftshift2d(re, im, nx, ny, 0);
    orc_fft2d(re, im, nx, ny, 1);
    orc_fftshift2d(re, im, nx, ny, 1);
    for (long k = 0; k < n; k++) {
      re[k] *= sqrt((double)nx * ny);
      im[k] *= sqrt((double)nx * ny);
      phase[k] = atan2(im[k], re[k]);
    }
  }
  free(re);
  free(im);
  return 0;
}

/* src/doe.js:455-546 */
/* Screen RMSE of src/projector.js:554-595 on an intensity plane (the pitch
 * cancels): target scaled to the in-ROI power, RMSE over the ROI. */
static double screen_rmse(const double* inten, const double* T, const double* roi, long n) {
  double im = 0, tt = 0, ii = 0, it = 0, t2 = 0;
  for (long k = 0; k < n; k++) {
    double m = roi ? roi[k] : 1;
    im += inten[k] * m;
    tt += T[k];
    if (m > 0) {
      ii += inten[k] * inten[k];
      it += inten[k] * T[k];
      t2 += T[k] * T[k];
    }
  }
  double s = tt > 0 ? im / tt : 0;
  double den = s * s * t2;
  double num = fmax(0.0, ii - 2 * s * it + s * s * t2);
  return den > 0 ? sqrt(num / den) : 0;
}

static int weighted_gs_impl(const double* illumination, const double* targetAmp,
                            const orc_design_opts* o, int base, const double* screen_irr,
                            double goal, int* used, orc_design_result* r);

int orc_weighted_gs(const double* illumination, const double* targetAmp,
                    const orc_design_opts* o, int base, orc_design_result* r) {
  return weighted_gs_impl(illumination, targetAmp, o, base, NULL, 0.0, NULL, r);
}

/* Image-plane WGS with the engine's per-design stopping goal (no counterpart in
 * the reference): after every iteration the screen RMSE of its forward field is
 * measured; at or below `goal` that iterate is returned and the loop ends.
 * screen_irr NULL uses targetAmp^2. *used receives the iterations run. */
int orc_weighted_gs_goal(const double* illumination, const double* targetAmp,
                         const orc_design_opts* o, const double* screen_irr, double goal,
                         int* used, orc_design_result* r) {
  return weighted_gs_impl(illumination, targetAmp, o, 0, screen_irr, goal, used, r);
}

static int weighted_gs_impl(const double* illumination, const double* targetAmp,
                            const orc_design_opts* o, int base, const double* screen_irr,
                            double goal, int* used, orc_design_result* r) {
  int nx = o->nx, ny = o->ny;
  long n = (long)nx * ny;
  const double* roi = o->roi;
  if (o->iterations < 1) return -1; /* the reference dereferences a null result */
  double* weights = r->weights ? r->weights : (double*)malloc(sizeof(double) * n);
  double* cur_phase = (double*)malloc(sizeof(double) * n);
  double* amp = (double*)malloc(sizeof(double) * n);
  double* inten = (double*)malloc(sizeof(double) * n);
  double* eff = (double*)malloc(sizeof(double));
  double* best_phase = (double*)malloc(sizeof(double) * n);
  double* best_amp = (double*)malloc(sizeof(double) * n);
  double* best_int = (double*)malloc(sizeof(double) * n);
  if (!weights || !cur_phase || !amp || !inten || !eff || !best_phase || !best_amp || !best_int)
    return -2;
  for (long k = 0; k < n; k++) weights[k] = ((roi ? roi[k] : 1) > 0) ? 1 : 0;
  double bestRmse = INFINITY;
  int have_best = 0;
  double beta = o->beta;
  double* T2 = NULL;
  if (goal > 0 && !screen_irr) {
    T2 = (double*)malloc(sizeof(double) * n);
    if (!T2) return -2;
    for (long k = 0; k < n; k++) T2[k] = targetAmp[k] * targetAmp[k];
    screen_irr = T2;
  }
  int ran = o->iterations;
  for (int it = 0; it < o->iterations; it++) {
    orc_design_opts so = *o;
    so.weights = weights;
    so.iterations = 1;
    so.init_phase = it > 0 ? cur_phase : o->init_phase;
    orc_design_result sr;
    memset(&sr, 0, sizeof(sr));
    sr.phase = cur_phase;
    sr.amplitude = amp;
    sr.intensity = inten;
    sr.efficiency = eff;
    int rc = base == 1 ? orc_fourier_cgh(illumination, targetAmp, &so, &sr)
                       : orc_gerchberg_saxton(illumination, targetAmp, &so, &sr);
    if (rc) return rc;
    /* unweighted ROI RMSE and best-iterate snapshot (src/doe.js:489-504) */
    double num = 0, den = 0;
    for (long k = 0; k < n; k++) {
      if ((roi ? roi[k] : 1) <= 0) continue;
      double d = amp[k] - targetAmp[k];
      num += d * d;
      den += targetAmp[k] * targetAmp[k];
    }
    double rmse = den > 0 ? sqrt(num / den) : 0;
    int stop = goal > 0 && screen_rmse(inten, screen_irr, roi, n) <= goal;
    if (rmse < bestRmse || stop) {
      bestRmse = rmse;
      memcpy(best_phase, cur_phase, sizeof(double) * n);
      memcpy(best_amp, amp, sizeof(double) * n);
      memcpy(best_int, inten, sizeof(double) * n);
      have_best = 1;
    }
    /* multiplicative weight update + renormalisation (src/doe.js:510-524) */
    double wsum = 0, tsum = 0;
    for (long k = 0; k < n; k++) {
      if ((roi ? roi[k] : 1) <= 0) continue;
      double measured = amp[k];
      double desired = targetAmp[k];
      double ratio = measured > 1e-30 ? desired / measured : 2;
      weights[k] *= pow(fmin(fmax(ratio, 0.25), 4), beta);
      weights[k] = fmin(fmax(weights[k], 1e-4), 1e4);
      wsum += weights[k] * weights[k] * desired * desired;
      tsum += desired * desired;
    }
    double nrm = wsum > 0 ? sqrt(tsum / wsum) : 1;
    for (long k = 0; k < n; k++) weights[k] *= nrm;
    if (r->error) r->error[it] = bestRmse;
    if (r->efficiency) r->efficiency[it] = eff[0];
    if (stop) {
      ran = it + 1;
      for (int j = it + 1; j < o->iterations; j++) {
        if (r->error) r->error[j] = bestRmse;
        if (r->efficiency) r->efficiency[j] = eff[0];
      }
      break;
    }
  }
  if (used) *used = ran;
  free(T2);
  if (have_best) {
    memcpy(r->phase, best_phase, sizeof(double) * n);
    if (r->amplitude) memcpy(r->amplitude, best_amp, sizeof(double) * n);
    if (r->intensity) memcpy(r->intensity, best_int, sizeof(double) * n);
  } else {
    memcpy(r->phase, cur_phase, sizeof(double) * n);
    if (r->amplitude) memcpy(r->amplitude, amp, sizeof(double) * n);
    if (r->intensity) memcpy(r->intensity, inten, sizeof(double) * n);
  }
  r->rmse = bestRmse;
  if (!r->weights) free(weights);
  free(cur_phase);
  free(amp);
  free(inten);
  free(eff);
  free(best_phase);
  free(best_amp);
  free(best_int);
  return 0;
}

/* src/doe.js:557-626 */
int orc_gs_multiplane(const double* illumination, int nplanes, const double* zs,
                      const double* target_amp, const double* roi_all,
                      const double* weight, const orc_design_opts* o, double* phase,
                      double* error, double* efficiency, double* per_plane_error) {
  int nx = o->nx, ny = o->ny;
  long n = (long)nx * ny;
  if (nplanes == 0) return -1;
  double* re = (double*)malloc(sizeof(double) * n);
  double* im = (double*)malloc(sizeof(double) * n);
  double* amps = (double*)malloc(sizeof(double) * n);
  if (!re || !im || !amps) return -2;
  if (o->init_phase) {
    if (phase != o->init_phase) memcpy(phase, o->init_phase, sizeof(double) * n);
  } else {
    memset(phase, 0, sizeof(double) * n);
  }
  for (int it = 0; it < o->iterations; it++) {
    double iterErr = 0;
    for (int p = 0; p < nplanes; p++) {
      double z = zs[p];
      const double* targetAmp = target_amp + (long)p * n;
      const double* roi = roi_all ? roi_all + (long)p * n : NULL;
      double w = weight ? weight[p] : 1;
      for (long k = 0; k < n; k++) {
        re[k] = illumination[k] * cos(phase[k]);
        im[k] = illumination[k] * sin(phase[k]);
      }
      orc_asm_inplace(re, im, nx, ny, o->dx, o->dy, o->lambda, z, 0, 1, 0.02);
      double errNum = 0, errDen = 0, inRoi = 0, total = 0;
      for (long k = 0; k < n; k++) {
        double a = hypot(re[k], im[k]);
        amps[k] = a;
        double i2 = a * a;
        total += i2;
        double m = roi ? roi[k] : 1;
        if (m > 0) {
          inRoi += i2 * m;
          double d = (a - targetAmp[k]) * m;
          errNum += d * d;
          errDen += targetAmp[k] * targetAmp[k];
        }
      }
      (void)inRoi;
      (void)total;
      double e = errDen > 0 ? sqrt(errNum / errDen) : 0;
      if (per_plane_error) per_plane_error[(long)p * o->iterations + it] = e;
      iterErr += e * w;
      for (long k = 0; k < n; k++) {
        double m = roi ? roi[k] : 1;
        double t = m > 0 ? targetAmp[k] : amps[k];
        if (amps[k] > 0) {
          double s = t / amps[k];
          re[k] *= s;
          im[k] *= s;
        }
      }
      orc_asm_inplace(re, im, nx, ny, o->dx, o->dy, o->lambda, -z, 0, 1, 0.02);
      for (long k = 0; k < n; k++) phase[k] = atan2(im[k], re[k]);
    }
    if (error) error[it] = iterErr / nplanes;
    if (efficiency) efficiency[it] = 1 - iterErr / nplanes;
  }
  free(re);
  free(im);
  free(amps);
  return 0;
}

/* ------------------------------------------------------------------ */
/* JavaScript Math.round: the nearest integer, ties toward +infinity (x - floor(x)
 * is exact, so values just below a half do not round up as floor(x + 0.5) can). */
static double js_round(double x) {
  double f = floor(x);
  return (x - f >= 0.5) ? f + 1.0 : f;
}

/* src/projector.js:262-315 */
void orc_auto_roi(const double* irr, int nx, int ny, double dilate, double soft,
                  double threshold, double* out) {
  long n = (long)nx * ny;
  double mx = 0;
  for (long k = 0; k < n; k++)
    if (irr[k] > mx) mx = irr[k];
  double* bin = (double*)malloc(sizeof(double) * n);
  double* tmp = (double*)malloc(sizeof(double) * n);
  double* dil = (double*)malloc(sizeof(double) * n);
  for (long k = 0; k < n; k++) bin[k] = irr[k] > threshold * mx ? 1 : 0;
  int r = (int)fmax(1, js_round(dilate));
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      double v = 0;
      for (int d = -r; d <= r && v == 0; d++) {
        int ii = i + d;
        if (ii < 0 || ii >= nx) continue;
        if (bin[ii + (long)j * nx] > 0) v = 1;
      }
      tmp[i + (long)j * nx] = v;
    }
  }
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      double v = 0;
      for (int d = -r; d <= r && v == 0; d++) {
        int jj = j + d;
        if (jj < 0 || jj >= ny) continue;
        if (tmp[i + (long)jj * nx] > 0) v = 1;
      }
      dil[i + (long)j * nx] = v;
    }
  }
  if (soft <= 0) {
    memcpy(out, dil, sizeof(double) * n);
  } else {
    int s = (int)fmax(1, js_round(soft));
    for (int j = 0; j < ny; j++) {
      for (int i = 0; i < nx; i++) {
        double acc = 0;
        int cnt = 0;
        for (int dj = -s; dj <= s; dj++) {
          int jj = j + dj;
          if (jj < 0 || jj >= ny) continue;
          for (int di = -s; di <= s; di++) {
            int ii = i + di;
            if (ii < 0 || ii >= nx) continue;
            acc += dil[ii + (long)jj * nx];
            cnt++;
          }
        }
        out[i + (long)j * nx] = cnt > 0 ? acc / cnt : 0;
      }
    }
  }
  free(bin);
  free(tmp);
  free(dil);
}

/* src/projector.js:554-595 (rmse / efficiency / flux subset), src/metrics.js:10-18,73-84 */
void orc_screen_metrics(const double* fre, const double* fim, int nx, int ny, double sdx,
                        double sdy, const double* target_irr, const double* roi,
                        const double* illumination, double dx, double dy, double* out) {
  long n = (long)nx * ny;
  double* irr = (double*)malloc(sizeof(double) * n);
  double* tgt = (double*)malloc(sizeof(double) * n);
  for (long k = 0; k < n; k++) irr[k] = fre[k] * fre[k] + fim[k] * fim[k];
  double cell = sdx * sdy;
  memcpy(tgt, target_irr, sizeof(double) * n);
  double spt = 0, stt = 0;
  for (long k = 0; k < n; k++) spt += roi ? irr[k] * roi[k] : irr[k];
  for (long k = 0; k < n; k++) stt += tgt[k];
  double pt = spt * cell, tt = stt * cell;
  double s = tt > 0 ? pt / tt : 0;
  for (long k = 0; k < n; k++) tgt[k] *= s;
  double sinc = 0;
  for (long k = 0; k < n; k++) sinc += illumination[k];
  double incident = sinc * dx * dy;
  double stot = 0;
  for (long k = 0; k < n; k++) stot += irr[k];
  double total = stot * cell;
  double inSignal = spt * cell;
  double num = 0, den = 0;
  for (long k = 0; k < n; k++) {
    double m = roi ? roi[k] : 1;
    if (m <= 0) continue;
    double d = irr[k] - tgt[k];
    num += d * d;
    den += tgt[k] * tgt[k];
  }
  out[0] = den > 0 ? sqrt(num / den) : 0;
  out[1] = incident > 0 ? inSignal / incident : 0;
  out[2] = total > 0 ? inSignal / total : 0;
  out[3] = inSignal;
  out[4] = total;
  out[5] = incident;
  free(irr);
  free(tgt);
}

/* ---------------------------------------------------------------- quantisation */
static double wrap1(double p) { /* src/propagate.js:410-420 */
  double two_pi = 2 * M_PI;
  p = fmod(p, two_pi);
  if (p > M_PI) p -= two_pi;
  else if (p <= -M_PI) p += two_pi;
  return p;
}

/* src/doe.js:164-173 quantizePhase */
void orc_quantize_phase(const double* phi, long n, int levels, double* out) {
  double step = (2 * M_PI) / levels;
  for (long k = 0; k < n; k++) out[k] = wrap1(js_round(phi[k] / step) * step);
}

/* src/doe.js:185-226 errorDiffusionQuantize; returns -1 for a non-square length */
int orc_error_diffusion(const double* phi, long n, int levels, int snake, int wrap_first, double* out) {
  long nx = lround(sqrt((double)n));
  long ny = nx > 0 ? n / nx : 0;
  if (nx * ny != n) return -1;
  double* buf = (double*)malloc(sizeof(double) * n);
  for (long k = 0; k < n; k++) buf[k] = wrap_first ? wrap1(phi[k]) : phi[k];
  double step = (2 * M_PI) / levels, two_pi = 2 * M_PI;
  for (long j = 0; j < ny; j++) {
    int ltr = snake ? (j % 2 == 0) : 1;
    long iStart = ltr ? 0 : nx - 1, iEnd = ltr ? nx : -1, iStep = ltr ? 1 : -1;
    for (long i = iStart; i != iEnd; i += iStep) {
      long k = i + j * nx;
      double v = buf[k];
      double q = js_round(v / step) * step;
      out[k] = q;
      double e = v - q;
      if (e > M_PI) e -= two_pi;
      else if (e <= -M_PI) e += two_pi;
      const long di[4] = {1, -1, 0, 1}, dj[4] = {0, 1, 1, 1};
      const double w[4] = {7.0 / 16, 3.0 / 16, 5.0 / 16, 1.0 / 16};
      for (int t = 0; t < 4; t++) {
        long ii = i + iStep * di[t], jj = j + dj[t];
        if (ii < 0 || ii >= nx || jj < 0 || jj >= ny) continue;
        buf[ii + jj * nx] += e * w[t];
      }
    }
  }
  for (long k = 0; k < n; k++) out[k] = wrap1(out[k]);
  free(buf);
  return 0;
}

/* ---------------------------------------------------------------- full screenMetrics */
/* src/metrics.js:37-67 regionStats -> {n, mean, min, max, std, uniformity, flatness, cv} */
static void region_stats(const double* plane, const double* mask, long n, double threshold, double* o) {
  long cnt = 0;
  double sum = 0, sumSq = 0, mn = INFINITY, mx = -INFINITY;
  for (long k = 0; k < n; k++) {
    if (mask && mask[k] <= 0) continue;
    double v = plane[k];
    if (v <= threshold) continue;
    cnt++;
    sum += v;
    sumSq += v * v;
    if (v < mn) mn = v;
    if (v > mx) mx = v;
  }
  if (cnt == 0) {
    for (int i = 0; i < 8; i++) o[i] = 0;
    return;
  }
  double mean = sum / cnt;
  double var = fmax(0, sumSq / cnt - mean * mean);
  double sd = sqrt(var);
  o[0] = (double)cnt;
  o[1] = mean;
  o[2] = mn;
  o[3] = mx;
  o[4] = sd;
  o[5] = mx + mn > 0 ? 1 - (mx - mn) / (mx + mn) : 1;
  o[6] = mean > 0 ? 1 - sd / mean : 1;
  o[7] = mean > 0 ? sd / mean : 0;
}

/* src/metrics.js:87-118 correlation (two passes) */
static double correlation(const double* p, const double* t, const double* mask, long n) {
  double sp = 0, st = 0;
  long cnt = 0;
  for (long k = 0; k < n; k++) {
    if (mask && mask[k] <= 0) continue;
    sp += p[k];
    st += t[k];
    cnt++;
  }
  if (cnt == 0) return 0;
  double mp = sp / cnt, mt = st / cnt, cov = 0, vp = 0, vt = 0;
  for (long k = 0; k < n; k++) {
    if (mask && mask[k] <= 0) continue;
    double dp = p[k] - mp, dt = t[k] - mt;
    cov += dp * dt;
    vp += dp * dp;
    vt += dt * dt;
  }
  return vp > 0 && vt > 0 ? cov / sqrt(vp * vt) : 0;
}

/* src/metrics.js:198-259 ssim, window 8, dataRange from the peaks, weight 'target' */
static double ssim_target(const double* p, const double* t, int nx, int ny, int window) {
  long n = (long)nx * ny;
  double mx = 0;
  for (long k = 0; k < n; k++) {
    if (p[k] > mx) mx = p[k];
    if (t[k] > mx) mx = t[k];
  }
  double L = mx > 0 ? mx : 1;
  double C1 = 0.01 * L * (0.01 * L), C2 = 0.03 * L * (0.03 * L);
  double total = 0, wsum = 0;
  for (int wy = 0; wy + window <= ny; wy += window) {
    for (int wx = 0; wx + window <= nx; wx += window) {
      double sp = 0, st = 0, spp = 0, stt = 0, spt = 0;
      double w2 = (double)window * window;
      for (int j = 0; j < window; j++) {
        for (int i = 0; i < window; i++) {
          long k = wx + i + (long)(wy + j) * nx;
          sp += p[k];
          st += t[k];
          spp += p[k] * p[k];
          stt += t[k] * t[k];
          spt += p[k] * t[k];
        }
      }
      double mp = sp / w2, mt = st / w2;
      double vp = fabs(spp / w2 - mp * mp), vt = fabs(stt / w2 - mt * mt);
      double cpt = spt / w2 - mp * mt;
      double num = (2 * mp * mt + C1) * (2 * cpt + C2);
      double den = (mp * mp + mt * mt + C1) * (vp + vt + C2);
      double wt = st / w2;
      total += (den != 0 ? num / den : 0) * wt;
      wsum += wt;
    }
  }
  return wsum > 0 ? total / wsum : 0;
}

/* src/metrics.js:284-321 spotUniformity (minPeak 0.05) -> uniformity */
static double spot_uniformity(const double* plane, int nx, int ny, int cols, int rows) {
  long n = (long)nx * ny;
  double* cells = (double*)calloc((size_t)cols * rows, sizeof(double));
  double peak = 0;
  for (long k = 0; k < n; k++)
    if (plane[k] > peak) peak = plane[k];
  double cut = 0.05 * peak;
  for (int j = 0; j < ny; j++) {
    int cj = (int)fmin(rows - 1, floor(((double)j / ny) * rows));
    for (int i = 0; i < nx; i++) {
      int ci = (int)fmin(cols - 1, floor(((double)i / nx) * cols));
      double v = plane[i + (long)j * nx];
      if (v >= cut) cells[ci + cj * cols] += v;
    }
  }
  double mn = INFINITY, mx = 0;
  int cnt = 0;
  for (int c = 0; c < cols * rows; c++) {
    if (cells[c] <= 0) continue;
    mn = fmin(mn, cells[c]);
    mx = fmax(mx, cells[c]);
    cnt++;
  }
  free(cells);
  if (cnt == 0) return 0;
  return mx + mn > 0 ? (2 * mn) / (mx + mn) : 1;
}

/* src/projector.js:554-614 screenMetrics (all fields; spot uniformity when
 * grid_cols > 0) with src/metrics.js:145-157 zeroOrderFraction of the element
 * field illumination * exp(i phase) and :164-185 rmsRadius. out[18] in the
 * order of the engine's doe_screen_metrics_full. */
void orc_screen_metrics_full(const double* fre, const double* fim, int nx, int ny, double sdx,
                             double sdy, const double* target_irr, const double* roi,
                             const double* illumination, const double* phase, double dx, double dy,
                             int grid_cols, int grid_rows, double* out) {
  long n = (long)nx * ny;
  double* irr = (double*)malloc(sizeof(double) * n);
  double* tgt = (double*)malloc(sizeof(double) * n);
  for (long k = 0; k < n; k++) irr[k] = fre[k] * fre[k] + fim[k] * fim[k];
  double cell = sdx * sdy;
  memcpy(tgt, target_irr, sizeof(double) * n);
  double spt = 0, stt = 0;
  for (long k = 0; k < n; k++) spt += roi ? irr[k] * roi[k] : irr[k];
  for (long k = 0; k < n; k++) stt += tgt[k];
  double pt = spt * cell, tt = stt * cell;
  double s = tt > 0 ? pt / tt : 0;
  for (long k = 0; k < n; k++) tgt[k] *= s;
  double prov[8], st8[8];
  region_stats(irr, roi, n, 0.0, prov);
  region_stats(irr, roi, n, 0.1 * prov[3], st8);
  double spots = grid_cols > 0 ? spot_uniformity(irr, nx, ny, grid_cols, grid_rows) : NAN;
  double sinc = 0;
  for (long k = 0; k < n; k++) sinc += illumination[k];
  double incident = sinc * dx * dy;
  double stot = 0;
  for (long k = 0; k < n; k++) stot += irr[k];
  double total = stot * cell, inSignal = spt * cell;
  double num = 0, den = 0;
  for (long k = 0; k < n; k++) {
    double m = roi ? roi[k] : 1;
    if (m <= 0) continue;
    double d = irr[k] - tgt[k];
    num += d * d;
    den += tgt[k] * tgt[k];
  }
  double rms = den > 0 ? sqrt(num / den) : 0;
  double corr = correlation(irr, tgt, roi, n);
  double ss = ssim_target(irr, tgt, nx, ny, 8);
  /* rmsRadius(irr, nx, sdx, 0, 0, sdy) */
  double p = 0, sx = 0, sy = 0;
  for (int j = 0; j < ny; j++) {
    double y = (j - ny / 2.0) * sdy;
    for (int i = 0; i < nx; i++) {
      double x = (i - nx / 2.0) * sdx;
      double v = irr[i + (long)j * nx];
      p += v;
      sx += v * x * x;
      sy += v * y * y;
    }
  }
  double rr = p == 0 ? 0 : hypot(sqrt(sx / p), sqrt(sy / p));
  /* zeroOrderFraction of A exp(i phase) (src/field.js:168-179 setAmplitudePhase) */
  double zr = 0, zi = 0, zp = 0;
  for (long k = 0; k < n; k++) {
    double re = illumination[k] * cos(phase[k]), im = illumination[k] * sin(phase[k]);
    zr += re;
    zi += im;
    zp += re * re + im * im;
  }
  double zero = zp == 0 ? 0 : (zr * zr + zi * zi) / (n * zp);
  out[0] = incident > 0 ? inSignal / incident : 0;            /* efficiency */
  out[1] = total > 0 ? inSignal / total : 0;                  /* fluxFraction */
  out[2] = grid_cols > 0 ? spots : st8[5];                    /* uniformity */
  out[3] = spots;                                             /* spotUniformity (NaN: none) */
  out[4] = st8[6];                                            /* flatness */
  out[5] = st8[7];                                            /* contrast (cv) */
  out[6] = rms;                                               /* rmse */
  out[7] = (corr + 1) / 2;                                    /* fidelity */
  out[8] = corr;                                              /* correlation */
  out[9] = ss;                                                /* ssim */
  out[10] = rms > 0 ? 20 * log10(1 / rms) : INFINITY;         /* snr */
  out[11] = zero;                                             /* zeroOrder */
  out[12] = rr;                                               /* rmsRadius */
  out[13] = st8[1];                                           /* meanIntensity */
  out[14] = st8[3];                                           /* peakIntensity */
  out[15] = inSignal;                                         /* powerInSignal */
  out[16] = total;                                            /* powerAtScreen */
  out[17] = incident;                                         /* powerIncident */
  free(irr);
  free(tgt);
}

/* src/doe.js:817-829: targetAmp = sqrt(max(0, irr)), then scaled so that
 * sum(targetAmp^2) equals sum(illumination^2), both summed sequentially. */
void orc_prepare_target(const double* irr, const double* illumination, long n, double* out) {
  for (long k = 0; k < n; k++) out[k] = sqrt(fmax(0, irr[k]));
  double inPower = 0;
  for (long k = 0; k < n; k++) inPower += illumination[k] * illumination[k];
  double tPower = 0;
  for (long k = 0; k < n; k++) tPower += out[k] * out[k];
  if (tPower > 0) {
    double s = sqrt(inPower / tPower);
    for (long k = 0; k < n; k++) out[k] *= s;
  }
}

/* ------------------------------------------------------------------ */
/* src/interference.js:57-69 modalIntensity over M modes [M][n]; w NULL = all 1. */
void orc_modal_intensity(int M, const double* re, const double* im, long n, const double* w, double* out) {
  double wsum = 0;
  for (long k = 0; k < n; k++) out[k] = 0;
  for (int m = 0; m < M; m++) {
    double wm = w ? w[m] : 1;
    wsum += wm;
    const double* r = re + (long)m * n;
    const double* q = im + (long)m * n;
    for (long k = 0; k < n; k++) out[k] += wm * (r[k] * r[k] + q[k] * q[k]);
  }
  if (wsum > 0)
    for (long k = 0; k < n; k++) out[k] /= wsum;
}

/* src/interference.js:347-388 recordHologram; encode 0 'raw', 1 'binary', 2 'phase'. */
void orc_record_hologram(const double* obj_re, const double* obj_im, const double* ref_re, const double* ref_im,
                         long n, int encode, int levels, double* plate_re, double* plate_im, double* recorded,
                         double* sum_re, double* sum_im) {
  for (long k = 0; k < n; k++) {
    sum_re[k] = obj_re[k] + ref_re[k];
    sum_im[k] = obj_im[k] + ref_im[k];
  }
  for (long k = 0; k < n; k++) recorded[k] = sum_re[k] * sum_re[k] + sum_im[k] * sum_im[k];
  double norm = 0;
  for (long k = 0; k < n; k++)
    if (recorded[k] > norm) norm = recorded[k];
  if (norm > 0)
    for (long k = 0; k < n; k++) recorded[k] /= norm;
  for (long k = 0; k < n; k++) {
    plate_re[k] = 0;
    plate_im[k] = 0;
  }
  if (encode == 0) {
    for (long k = 0; k < n; k++) plate_re[k] = recorded[k];
  } else if (encode == 1) {
    for (long k = 0; k < n; k++) plate_re[k] = recorded[k] > 0.5 ? 1 : 0;
  } else {
    for (long k = 0; k < n; k++) {
      double ph = wrap1(atan2(sum_im[k], sum_re[k]));
      plate_re[k] = cos(ph);
      plate_im[k] = sin(ph);
    }
    if (levels > 1) {
      double step = (2 * M_PI) / levels;
      for (long k = 0; k < n; k++) {
        double ph = js_round(atan2(plate_im[k], plate_re[k]) / step) * step;
        plate_re[k] = cos(ph);
        plate_im[k] = sin(ph);
      }
    }
  }
}

/* src/interference.js:397-411 reconstructHologram: illumination = plate * reference,
 * then angular-spectrum propagation of two copies to +z (real) and -z (virtual). */
void orc_reconstruct_hologram(const double* plate_re, const double* plate_im, const double* ref_re,
                              const double* ref_im, int nx, int ny, double dx, double dy, double lambda, double z,
                              int band_limit, int evanescent, double soft_edge, double* real_re, double* real_im,
                              double* virt_re, double* virt_im, double* illum_re, double* illum_im) {
  long n = (long)nx * ny;
  for (long k = 0; k < n; k++) {
    illum_re[k] = plate_re[k] * ref_re[k] - plate_im[k] * ref_im[k];
    illum_im[k] = plate_re[k] * ref_im[k] + plate_im[k] * ref_re[k];
  }
  memcpy(real_re, illum_re, sizeof(double) * n);
  memcpy(real_im, illum_im, sizeof(double) * n);
  memcpy(virt_re, illum_re, sizeof(double) * n);
  memcpy(virt_im, illum_im, sizeof(double) * n);
  orc_asm_inplace(real_re, real_im, nx, ny, dx, dy, lambda, z, band_limit, evanescent, soft_edge);
  orc_asm_inplace(virt_re, virt_im, nx, ny, dx, dy, lambda, -z, band_limit, evanescent, soft_edge);
}

/* src/interference.js:104-125 smoothInPlace: separable circular box blur of
 * radius r by running sums (rows into tmp, then columns back into arr). */
static void box_blur_circular(double* arr, int nx, int ny, int r) {
  long n = (long)nx * ny;
  double* tmp = (double*)malloc(sizeof(double) * n);
  double norm = 1.0 / (2 * r + 1);
  for (int j = 0; j < ny; j++) {
    double acc = 0;
    for (int i = -r; i <= r; i++) acc += arr[((i % nx) + nx) % nx + (long)j * nx];
    for (int i = 0; i < nx; i++) {
      tmp[i + (long)j * nx] = acc * norm;
      acc -= arr[(((i - r) % nx) + nx) % nx + (long)j * nx];
      acc += arr[(((i + r + 1) % nx) + nx) % nx + (long)j * nx];
    }
  }
  for (int i = 0; i < nx; i++) {
    double acc = 0;
    for (int j = -r; j <= r; j++) acc += tmp[i + (long)(((j % ny) + ny) % ny) * nx];
    for (int j = 0; j < ny; j++) {
      arr[i + (long)j * nx] = acc * norm;
      acc -= tmp[i + (long)((((j - r) % ny) + ny) % ny) * nx];
      acc += tmp[i + (long)((((j + r + 1) % ny) + ny) % ny) * nx];
    }
  }
  free(tmp);
}

/* src/interference.js:79-101 partiallyCoherentModes: M modes [M][n] from one
 * xorshift32 stream (src/doe.js:65-75), each a Gaussian envelope of waist
 * `waist` times a box-smoothed uniform phase screen. */
void orc_partially_coherent_modes(int nx, int ny, double dx, double dy, int modes, double sigma, double waist,
                                  double seed, double* re, double* im) {
  long n = (long)nx * ny;
  uint32_t st = orc_rng_seed(seed);
  double sigma_pix = fmax(1, sigma / dx);
  int r = (int)fmax(1, js_round(sigma_pix));
  double* ph = (double*)malloc(sizeof(double) * n);
  for (int m = 0; m < modes; m++) {
    for (long k = 0; k < n; k++) ph[k] = (orc_rng_next(&st) * 2 - 1) * M_PI;
    box_blur_circular(ph, nx, ny, r);
    for (int j = 0; j < ny; j++) {
      double y = (j - ny / 2.0) * dy;
      for (int i = 0; i < nx; i++) {
        double x = (i - nx / 2.0) * dx;
        long k = i + (long)j * nx;
        double a = exp(-(x * x + y * y) / (waist * waist));
        re[(long)m * n + k] = a * cos(ph[k]);
        im[(long)m * n + k] = a * sin(ph[k]);
      }
    }
  }
  free(ph);
}
