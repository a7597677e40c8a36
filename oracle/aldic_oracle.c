/*
 * aldic_oracle.c -- CPU FP64 restatement of the AL-DIC hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Nothing in the product library
 * links this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline / reference arm load liboracle.so.
 *
 * Parity: orc_ba_interp2_* is pinned bit-exactly against the reference's own
 * ba_interp2.cpp (compiled from the reference sources into oracle/_ref by
 * oracle/Makefile).  Everything else restates the reference MATLAB (file:line
 * cited per function); MATLAB/Octave is absent, so those parts are
 * "parity unpinned" against the reference itself and are pinned by
 * known-answer tests built from the algorithms' definitions.
 *
 * Compile with -ffp-contract=off: several kernels of the CUDA path reproduce
 * these operation orders with explicit round-to-nearest intrinsics so that the
 * FP64 results (and the integer-exact NCC maps) are bit-identical.
 */
#include "aldic_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;
void orc_set_threads(int n) {
  g_threads = n;
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ======================================================================
 * a3: bicubic sampling.  Follows ba_interp2.cpp:60-182: Keys cubic
 * convolution (a = -1/2) on a column-major M x N image, X indexing columns
 * (N) and Y rows (M), 1-based, clamp-to-edge.  The arithmetic order of the
 * weights and of the 4x4 sum is kept so that results are bit-identical.
 * ==================================================================== */
static inline int64_t clamp64(int64_t v, int64_t lo, int64_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

/* floor(c)-1 as an index, with the coordinate clamped first so the
 * conversion is defined for any finite input (values outside the image
 * clamp to the same border samples as the reference's access()). */
static inline int64_t corner_index(double c_floor, int64_t extent) {
  double lo = -4.0, hi = (double)extent + 4.0;
  double c = c_floor < lo ? lo : (c_floor > hi ? hi : c_floor);
  return (int64_t)(c - 1.0);
}

void orc_ba_interp2_f64(const double *F, int64_t M, int64_t N, int64_t P,
                        const double *X, const double *Y, int64_t n, double *out) {
  const int64_t LO = M * N;
#pragma omp parallel for schedule(static) if (n > 65536)
  for (int64_t i = 0; i < n; ++i) {
    const double x = X[i], y = Y[i];
    if (!isfinite(x) || !isfinite(y)) {
      for (int64_t j = 0; j < P; ++j) out[i + j * n] = NAN;
      continue;
    }
    const double xf = floor(x), yf = floor(y);
    const double dx = x - xf, dy = y - yf;
    const double dxx = dx * dx, dxxx = dxx * dx;
    const double dyy = dy * dy, dyyy = dyy * dy;
    const double wx0 = 0.5 * ((-dx + 2.0 * dxx) - dxxx);
    const double wx1 = 0.5 * ((2.0 - 5.0 * dxx) + 3.0 * dxxx);
    const double wx2 = 0.5 * ((dx + 4.0 * dxx) - 3.0 * dxxx);
    const double wx3 = 0.5 * (-dxx + dxxx);
    const double wy0 = 0.5 * ((-dy + 2.0 * dyy) - dyyy);
    const double wy1 = 0.5 * ((2.0 - 5.0 * dyy) + 3.0 * dyyy);
    const double wy2 = 0.5 * ((dy + 4.0 * dyy) - 3.0 * dyyy);
    const double wy3 = 0.5 * (-dyy + dyyy);
    const int64_t xc = corner_index(xf, N), yc = corner_index(yf, M);
    int64_t c[4], r[4];
    for (int k = 0; k < 4; ++k) {
      c[k] = clamp64(xc - 1 + k, 0, N - 1) * M;
      r[k] = clamp64(yc - 1 + k, 0, M - 1);
    }
    for (int64_t j = 0; j < P; ++j) {
      const double *Fj = F + j * LO;
      double s0 = wx0 * Fj[c[0] + r[0]] + wx1 * Fj[c[1] + r[0]] + wx2 * Fj[c[2] + r[0]] + wx3 * Fj[c[3] + r[0]];
      double s1 = wx0 * Fj[c[0] + r[1]] + wx1 * Fj[c[1] + r[1]] + wx2 * Fj[c[2] + r[1]] + wx3 * Fj[c[3] + r[1]];
      double s2 = wx0 * Fj[c[0] + r[2]] + wx1 * Fj[c[1] + r[2]] + wx2 * Fj[c[2] + r[2]] + wx3 * Fj[c[3] + r[2]];
      double s3 = wx0 * Fj[c[0] + r[3]] + wx1 * Fj[c[1] + r[3]] + wx2 * Fj[c[2] + r[3]] + wx3 * Fj[c[3] + r[3]];
      out[i + j * n] = wy0 * s0 + wy1 * s1 + wy2 * s2 + wy3 * s3;
    }
  }
}

/* Single precision: as in the reference's REAL=float instantiation the
 * weight polynomials are evaluated in double (the literals are double) and
 * rounded to float; wx3's inner sum stays in float; the 4x4 sum is float. */
void orc_ba_interp2_f32(const float *F, int64_t M, int64_t N, int64_t P,
                        const float *X, const float *Y, int64_t n, float *out) {
  const int64_t LO = M * N;
#pragma omp parallel for schedule(static) if (n > 65536)
  for (int64_t i = 0; i < n; ++i) {
    const float x = X[i], y = Y[i];
    if (!isfinite(x) || !isfinite(y)) {
      for (int64_t j = 0; j < P; ++j) out[i + j * n] = NAN;
      continue;
    }
    const float xf = floorf(x), yf = floorf(y);
    const float dx = x - xf, dy = y - yf;
    const float dxx = dx * dx, dxxx = dxx * dx;
    const float dyy = dy * dy, dyyy = dyy * dy;
    const float wx0 = (float)(0.5 * (((double)(-dx) + 2.0 * (double)dxx) - (double)dxxx));
    const float wx1 = (float)(0.5 * ((2.0 - 5.0 * (double)dxx) + 3.0 * (double)dxxx));
    const float wx2 = (float)(0.5 * (((double)dx + 4.0 * (double)dxx) - 3.0 * (double)dxxx));
    const float wx3 = (float)(0.5 * (double)(-dxx + dxxx));
    const float wy0 = (float)(0.5 * (((double)(-dy) + 2.0 * (double)dyy) - (double)dyyy));
    const float wy1 = (float)(0.5 * ((2.0 - 5.0 * (double)dyy) + 3.0 * (double)dyyy));
    const float wy2 = (float)(0.5 * (((double)dy + 4.0 * (double)dyy) - 3.0 * (double)dyyy));
    const float wy3 = (float)(0.5 * (double)(-dyy + dyyy));
    const int64_t xc = corner_index((double)xf, N), yc = corner_index((double)yf, M);
    int64_t c[4], r[4];
    for (int k = 0; k < 4; ++k) {
      c[k] = clamp64(xc - 1 + k, 0, N - 1) * M;
      r[k] = clamp64(yc - 1 + k, 0, M - 1);
    }
    for (int64_t j = 0; j < P; ++j) {
      const float *Fj = F + j * LO;
      float s0 = wx0 * Fj[c[0] + r[0]] + wx1 * Fj[c[1] + r[0]] + wx2 * Fj[c[2] + r[0]] + wx3 * Fj[c[3] + r[0]];
      float s1 = wx0 * Fj[c[0] + r[1]] + wx1 * Fj[c[1] + r[1]] + wx2 * Fj[c[2] + r[1]] + wx3 * Fj[c[3] + r[1]];
      float s2 = wx0 * Fj[c[0] + r[2]] + wx1 * Fj[c[1] + r[2]] + wx2 * Fj[c[2] + r[2]] + wx3 * Fj[c[3] + r[2]];
      float s3 = wx0 * Fj[c[0] + r[3]] + wx1 * Fj[c[1] + r[3]] + wx2 * Fj[c[2] + r[3]] + wx3 * Fj[c[3] + r[3]];
      out[i + j * n] = wy0 * s0 + wy1 * s1 + wy2 * s2 + wy3 * s3;
    }
  }
}

/* ======================================================================
 * a1: funNormalizeImg.m:22-39.  Integer images: ROI sums are exact
 * integers, mean = S1/n, std = sqrt((S2 - mean*S1)/(n-1)).
 * ==================================================================== */
static inline double px_value(const void *img, int dtype, int64_t i) {
  switch (dtype) {
    case 0: return (double)((const uint8_t *)img)[i];
    case 1: return (double)((const uint16_t *)img)[i];
    case 2: return (double)((const float *)img)[i];
    default: return ((const double *)img)[i];
  }
}

static void clamp_roi(int W, int H, const int roi_in[4], int roi[4]) {
  roi[0] = roi_in[0] < 1 ? 1 : roi_in[0];
  roi[1] = roi_in[1] > W ? W : roi_in[1];
  roi[2] = roi_in[2] < 1 ? 1 : roi_in[2];
  roi[3] = roi_in[3] > H ? H : roi_in[3];
}

static void roi_stats(const void *img, int dtype, int W, const int roi[4],
                      double *mean, double *stdev) {
  const int64_t n = (int64_t)(roi[1] - roi[0] + 1) * (roi[3] - roi[2] + 1);
  if (dtype <= 1) {
    uint64_t s1 = 0, s2 = 0;
    for (int y = roi[2]; y <= roi[3]; ++y)
      for (int x = roi[0]; x <= roi[1]; ++x) {
        uint64_t v = (uint64_t)px_value(img, dtype, (int64_t)(y - 1) * W + (x - 1));
        s1 += v;
        s2 += v * v;
      }
    double m = (double)s1 / (double)n;
    double ssd = (double)s2 - m * (double)s1;
    *mean = m;
    *stdev = sqrt(ssd / (double)(n - 1));
  } else {
    double s = 0.0;
    for (int y = roi[2]; y <= roi[3]; ++y)
      for (int x = roi[0]; x <= roi[1]; ++x) s += px_value(img, dtype, (int64_t)(y - 1) * W + (x - 1));
    double m = s / (double)n, ss = 0.0;
    for (int y = roi[2]; y <= roi[3]; ++y)
      for (int x = roi[0]; x <= roi[1]; ++x) {
        double d = px_value(img, dtype, (int64_t)(y - 1) * W + (x - 1)) - m;
        ss += d * d;
      }
    *mean = m;
    *stdev = sqrt(ss / (double)(n - 1));
  }
}

int orc_normalize(const void *img, int dtype, int W, int H, const int roi_in[4],
                  double *out, double *mean, double *stdev) {
  int roi[4];
  clamp_roi(W, H, roi_in, roi);
  if (roi[1] < roi[0] || roi[3] < roi[2]) return -1;
  double m, s;
  roi_stats(img, dtype, W, roi, &m, &s);
  const int64_t total = (int64_t)W * H;
  for (int64_t i = 0; i < total; ++i) out[i] = (px_value(img, dtype, i) - m) / s;
  if (mean) *mean = m;
  if (stdev) *stdev = s;
  return 0;
}

/* ======================================================================
 * a2: funImgGradient.m:53-78.  Correlation with
 * [-1/60 3/20 -3/4 0 3/4 -3/20 1/60] along x (DfDx) and y (DfDy), kept on
 * x,y in [4, size-3] (1-based), times the mask.  The symmetric taps are
 * paired so that a flat neighbourhood gives an exact 0 (the masked-subset
 * test of funICGN.m:54 counts exact zeros).
 * ==================================================================== */
#define GC1 0.75
#define GC2 (3.0 / 20.0)
#define GC3 (1.0 / 60.0)

void orc_gradient(const double *f, const double *mask, int W, int H,
                  double *dfdx, double *dfdy) {
  const int64_t total = (int64_t)W * H;
  memset(dfdx, 0, sizeof(double) * total);
  memset(dfdy, 0, sizeof(double) * total);
#pragma omp parallel for schedule(static)
  for (int y = 3; y < H - 3; ++y) {
    for (int x = 3; x < W - 3; ++x) {
      const int64_t i = (int64_t)y * W + x;
      double tx = (GC1 * (f[i + 1] - f[i - 1]) - GC2 * (f[i + 2] - f[i - 2])) + GC3 * (f[i + 3] - f[i - 3]);
      double ty = (GC1 * (f[i + W] - f[i - W]) - GC2 * (f[i + 2 * W] - f[i - 2 * W])) +
                  GC3 * (f[i + 3 * W] - f[i - 3 * W]);
      double m = mask ? mask[i] : 1.0;
      dfdx[i] = tx * m;
      dfdy[i] = ty * m;
    }
  }
}

/* ======================================================================
 * a4/a5: integer search.
 * ==================================================================== */
int orc_search_dims(int W, int H, const int gridx[2], const int gridy[2],
                    int winsize, int step, const int search[2],
                    int *nx, int *ny, int *x_first, int *y_first) {
  /* funIntegerSearch.m:14-25 */
  int gx1 = gridx[0], gx2 = gridx[1], gy1 = gridy[0], gy2 = gridy[1];
  const double hw = 0.5 * winsize, w15 = 1.5 * winsize;
  if (step <= 0 || winsize <= 0) return -1;
  while (gx1 - search[0] - hw < 1) gx1++;
  while (gy1 - search[1] - hw < 1) gy1++;
  while (gx2 + w15 + search[0] > W) gx2--;
  while (gy2 + w15 + search[1] > H) gy2--;
  /* funIntegerSearch.m:90-91: XList = gx1 : step : gx2-step */
  int cx = (gx2 - step >= gx1) ? (gx2 - step - gx1) / step + 1 : 0;
  int cy = (gy2 - step >= gy1) ? (gy2 - step - gy1) / step + 1 : 0;
  *nx = cx;
  *ny = cy;
  if (x_first) *x_first = gx1;
  if (y_first) *y_first = gy1;
  return 0;
}

/* Exact-integer partial sums of one template placement.  Template T is
 * (w+1)^2 with x fastest, region D is (w+1+2sx) x (w+1+2sy).  The template's
 * top-left sits at D offset (ox, oy) (0-based, may be negative or overhang). */
typedef struct {
  int64_t st, st2;              /* template sums (integer images) */
  double stf, st2f;             /* template sums (floating-point images) */
  const int64_t *T, *D;         /* integer-valued copies */
  const double *Tf, *Df;        /* float-valued copies (dtype >= 2) */
  int tw, th, dw, dh;           /* template and region extents */
  int integer;
} ncc_ctx;

/* NCC at one offset: the published normalised cross-correlation (Lewis,
 * "Fast Normalized Cross-Correlation", 1995) over the whole template, with
 * D zero-padded in normalised units, i.e. padded with mu_g in raw units.
 * Combination formula (FP64, fixed order) shared with the CUDA kernel. */
static double ncc_at(const ncc_ctx *c, int ox, int oy, double mu) {
  const int64_t mn = (int64_t)c->tw * c->th;
  int x0 = ox < 0 ? -ox : 0, y0 = oy < 0 ? -oy : 0;
  int x1 = c->tw, y1 = c->th;
  if (ox + x1 > c->dw) x1 = c->dw - ox;
  if (oy + y1 > c->dh) y1 = c->dh - oy;
  if (x1 <= x0 || y1 <= y0) {
    /* no overlap at all: all padding -> flat window */
    return 0.0;
  }
  const int64_t n_in = (int64_t)(x1 - x0) * (y1 - y0);
  const int64_t n_pad = mn - n_in;
  double A, B = 0.0, C0, Cc = 0.0, denT;
  if (c->integer) {
    denT = (double)(mn * c->st2 - c->st * c->st);
    int64_t sd = 0, sd2 = 0, std_ = 0, st_in = 0;
    for (int ty = y0; ty < y1; ++ty) {
      const int64_t *Tr = c->T + (int64_t)ty * c->tw;
      const int64_t *Dr = c->D + (int64_t)(ty + oy) * c->dw + ox;
      for (int tx = x0; tx < x1; ++tx) {
        int64_t d = Dr[tx], t = Tr[tx];
        sd += d;
        sd2 += d * d;
        std_ += t * d;
        st_in += t;
      }
    }
    A = (double)(mn * std_ - c->st * sd);
    C0 = (double)(mn * sd2 - sd * sd);
    if (n_pad > 0) {
      const int64_t st_pad = c->st - st_in;
      B = mu * (double)(mn * st_pad - c->st * n_pad);
      Cc = mu * ((double)(n_pad * (mn - n_pad)) * mu - 2.0 * (double)(sd * n_pad));
    }
  } else {
    double sd = 0, sd2 = 0, std_ = 0, st_in = 0;
    for (int ty = y0; ty < y1; ++ty) {
      const double *Tr = c->Tf + (int64_t)ty * c->tw;
      const double *Dr = c->Df + (int64_t)(ty + oy) * c->dw + ox;
      for (int tx = x0; tx < x1; ++tx) {
        double d = Dr[tx], t = Tr[tx];
        sd += d;
        sd2 += d * d;
        std_ += t * d;
        st_in += t;
      }
    }
    denT = (double)mn * c->st2f - c->stf * c->stf;
    A = (double)mn * std_ - c->stf * sd;
    C0 = (double)mn * sd2 - sd * sd;
    if (n_pad > 0) {
      const double st_pad = c->stf - st_in;
      B = mu * ((double)mn * st_pad - c->stf * (double)n_pad);
      Cc = mu * ((double)(n_pad * (mn - n_pad)) * mu - 2.0 * (sd * (double)n_pad));
    }
  }
  const double num = A + B;
  const double den = C0 + Cc;
  if (!(den > 0.0)) return 0.0;
  double r = num / sqrt(denT * den);
  if (fabs(r) - 1.0 > sqrt(DBL_EPSILON)) r = 0.0;
  return r;
}

/* findpeak.m:27-66 with the 3x3 least-squares quadratic written in closed
 * form (the 9x6 design matrix of findpeak.m:43 has a fixed pseudo-inverse).
 * map is nr x nc column-major (rows = x shifts).  Outputs 1-based
 * (row, col) peak positions and the fitted maximum. */
static void findpeak_restated(const double *map, int nr, int nc, double *row_pk,
                              double *col_pk, double *max_f) {
  int im = 0;
  double mv = map[0];
  for (int i = 1; i < nr * nc; ++i)
    if (map[i] > mv) {
      mv = map[i];
      im = i;
    }
  int r = im % nr, c = im / nr; /* 0-based */
  *row_pk = r + 1;
  *col_pk = c + 1;
  *max_f = mv;
  if (r == 0 || r == nr - 1 || c == 0 || c == nc - 1) return;
  /* u over the 3x3 block; xo = column offset, yo = row offset */
  double s0 = 0, sxu = 0, syu = 0, sxyu = 0, sxxu = 0, syyu = 0;
  for (int dc = -1; dc <= 1; ++dc)
    for (int dr = -1; dr <= 1; ++dr) {
      double u = map[(c + dc) * nr + (r + dr)];
      s0 += u;
      sxu += dc * u;
      syu += dr * u;
      sxyu += (dc * dr) * u;
      sxxu += (dc * dc) * u;
      syyu += (dr * dr) * u;
    }
  const double A2 = sxu / 6.0, A3 = syu / 6.0, A4 = sxyu / 4.0;
  const double p = 0.5 * (sxxu + syyu) - (2.0 / 3.0) * s0;
  const double q = 0.5 * (sxxu - syyu);
  const double A5 = 0.5 * (p + q), A6 = 0.5 * (p - q);
  const double A1 = (s0 - 6.0 * p) / 9.0;
  const double den = A4 * A4 - 4.0 * A5 * A6;
  double xo = (-A3 * A4 + 2.0 * A6 * A2) / den;
  double yo = -1.0 / den * (A4 * A2 - 2.0 * A5 * A3);
  if (fabs(xo) > 1.0 || fabs(yo) > 1.0) return;
  xo = round(1000.0 * xo) / 1000.0;
  yo = round(1000.0 * yo) / 1000.0;
  *col_pk = (c + 1) + xo;
  *row_pk = (r + 1) + yo;
  *max_f = A1 + A2 * xo + A3 * yo + A4 * (xo * yo) + A5 * (xo * xo) + A6 * (yo * yo);
}

/* compute_qFactor (funIntegerSearch.m:211-264) on the full NCC map:
 * PCE = peak^2 / mean(cc_min.^2) and 1/entropy of a 30-bin histogram of
 * cc_min (uniform bins over [0, peak]; MATLAB's histcounts bin picker is not
 * restated -- parity unpinned). */
static void qfactor(const double *cc, int n, double *pce, double *ppe) {
  double mn = cc[0];
  for (int i = 1; i < n; ++i)
    if (cc[i] < mn) mn = cc[i];
  double peak = 0.0, ss = 0.0;
  for (int i = 0; i < n; ++i) {
    double v = cc[i] - mn;
    if (v > peak) peak = v;
    ss += v * v;
  }
  *pce = (peak * peak) / (ss / n);
  int hist[30] = {0};
  for (int i = 0; i < n; ++i) {
    double v = cc[i] - mn;
    int b = peak > 0 ? (int)floor(v / peak * 30.0) : 0;
    if (b > 29) b = 29;
    if (b < 0) b = 0;
    hist[b]++;
  }
  double ent = 0.0;
  for (int b = 0; b < 30; ++b) {
    double pb = (double)hist[b] / n;
    if (pb > 0) ent += pb * log(1.0 / pb);
  }
  *ppe = 1.0 / ent;
}

int orc_int_search(const void *f_raw, const void *g_raw, int dtype, int W, int H,
                   double mu_g, const int gridx[2], const int gridy[2],
                   int winsize, int step, const int search[2],
                   double *xo, double *yo, double *uo, double *vo, double *ccmax,
                   double *qfac) {
  int nx, ny, gx1, gy1;
  if (orc_search_dims(W, H, gridx, gridy, winsize, step, search, &nx, &ny, &gx1, &gy1)) return -1;
  const int w = winsize, sx = search[0], sy = search[1];
  const int tw = w + 1, th = w + 1, dw = w + 1 + 2 * sx, dh = w + 1 + 2 * sy;
  const int cr = 2 * sx + 3, cc = 2 * sy + 3;          /* cropped map */
  const int fr = 2 * w + 2 * sx + 1, fc = 2 * w + 2 * sy + 1; /* full map */
  const int64_t npts = (int64_t)nx * ny;
  double *pce = qfac ? (double *)malloc(sizeof(double) * npts) : NULL;
  double *ppe = qfac ? (double *)malloc(sizeof(double) * npts) : NULL;
  const int integer = dtype <= 1;
#pragma omp parallel
  {
    int64_t *T = (int64_t *)malloc(sizeof(int64_t) * tw * th);
    int64_t *D = (int64_t *)malloc(sizeof(int64_t) * dw * dh);
    double *Tf = (double *)malloc(sizeof(double) * tw * th);
    double *Df = (double *)malloc(sizeof(double) * dw * dh);
    double *map = (double *)malloc(sizeof(double) * cr * cc);
    double *full = qfac ? (double *)malloc(sizeof(double) * fr * fc) : NULL;
#pragma omp for schedule(dynamic, 4)
    for (int64_t k = 0; k < npts; ++k) {
      /* tempi runs over ndgrid(XList,YList)(:) -> x fastest */
      const int ix = (int)(k % nx), iy = (int)(k / nx);
      const int ii = gx1 + ix * step, jj = gy1 + iy * step; /* 1-based */
      ncc_ctx c;
      memset(&c, 0, sizeof(c));
      c.tw = tw; c.th = th; c.dw = dw; c.dh = dh; c.integer = integer;
      int64_t st = 0, st2 = 0;
      double stf = 0, st2f = 0;
      for (int ty = 0; ty < th; ++ty)
        for (int tx = 0; tx < tw; ++tx) {
          double v = px_value(f_raw, dtype, (int64_t)(jj - 1 + ty) * W + (ii - 1 + tx));
          Tf[ty * tw + tx] = v;
          T[ty * tw + tx] = (int64_t)v;
          st += (int64_t)v;
          st2 += (int64_t)v * (int64_t)v;
          stf += v;
          st2f += v * v;
        }
      for (int dy = 0; dy < dh; ++dy)
        for (int dx = 0; dx < dw; ++dx) {
          double v = px_value(g_raw, dtype, (int64_t)(jj - 1 - sy + dy) * W + (ii - 1 - sx + dx));
          Df[dy * dw + dx] = v;
          D[dy * dw + dx] = (int64_t)v;
        }
      c.T = T; c.D = D; c.Tf = Tf; c.Df = Df;
      c.st = st; c.st2 = st2; c.stf = stf; c.st2f = st2f;
      const int64_t out_idx = (int64_t)iy + (int64_t)ix * ny; /* ny x nx column-major */
      xo[out_idx] = (ii + ii + w) / 2.0;
      yo[out_idx] = (jj + jj + w) / 2.0;
      int flat = integer ? ((int64_t)tw * th * st2 - st * st) == 0 : 0;
      if (!integer) {
        double m = stf / (tw * th), s = 0;
        for (int i = 0; i < tw * th; ++i) s += (Tf[i] - m) * (Tf[i] - m);
        flat = !(s > 0);
      }
      if (flat) {
        /* normxcorr2 rejects a constant template: the catch branch of
         * funIntegerSearch.m:153-157 */
        uo[out_idx] = NAN; vo[out_idx] = NAN; ccmax[out_idx] = NAN;
        if (qfac) { pce[k] = INFINITY; ppe[k] = INFINITY; }
        continue;
      }
      /* cropped map entry (a,b), 0-based: D offset (a-1, b-1) */
      for (int b = 0; b < cc; ++b)
        for (int a = 0; a < cr; ++a) map[b * cr + a] = ncc_at(&c, a - 1, b - 1, mu_g);
      double rpk, cpk, mf;
      findpeak_restated(map, cr, cc, &rpk, &cpk, &mf);
      /* funIntegerSearch.m:134-151: [v1,u1] = findpeak -> u from rows */
      uo[out_idx] = rpk - (sx + 2);
      vo[out_idx] = cpk - (sy + 2);
      ccmax[out_idx] = mf;
      if (qfac) {
        for (int b = 0; b < fc; ++b)
          for (int a = 0; a < fr; ++a) full[b * fr + a] = ncc_at(&c, a - w, b - w, mu_g);
        qfactor(full, fr * fc, &pce[k], &ppe[k]);
      }
    }
    free(T); free(D); free(Tf); free(Df); free(map); free(full);
  }
  if (qfac) {
    /* funIntegerSearch.m:174-177, over tempi order (x fastest) */
    double *q[2] = {pce, ppe};
    for (int kk = 0; kk < 2; ++kk) {
      double mn = INFINITY;
      for (int64_t k = 0; k < npts; ++k)
        if (q[kk][k] < mn) mn = q[kk][k];
      double mx = -INFINITY;
      for (int64_t k = 0; k < npts; ++k) {
        double v = q[kk][k] - mn;
        if (v > mx) mx = v;
      }
      for (int64_t k = 0; k < npts; ++k) qfac[k + kk * npts] = (q[kk][k] - mn) / mx;
    }
    free(pce);
    free(ppe);
  }
  return 0;
}

/* ======================================================================
 * Multigrid search primitives (func/funIntegerSearchMg.m): normxcorr2 of an
 * arbitrary template rectangle of f against a region rectangle of g, at a
 * rectangle of offsets; findpeak and compute_qFactor on a given map.
 * ==================================================================== */
int orc_ncc_map(const void *f_raw, const void *g_raw, int dtype, int W, int H, double mu_g,
                const int trect[4], const int drect[4], int ox0, int ox1, int oy0, int oy1,
                double *out) {
  const int tw = trect[1] - trect[0] + 1, th = trect[3] - trect[2] + 1;
  const int dw = drect[1] - drect[0] + 1, dh = drect[3] - drect[2] + 1;
  if (tw < 1 || th < 1 || dw < 1 || dh < 1) return -1;
  if (trect[0] < 1 || trect[1] > W || trect[2] < 1 || trect[3] > H) return -1;
  if (drect[0] < 1 || drect[1] > W || drect[2] < 1 || drect[3] > H) return -1;
  const int integer = dtype <= 1;
  int64_t *T = (int64_t *)malloc(sizeof(int64_t) * tw * th);
  int64_t *D = (int64_t *)malloc(sizeof(int64_t) * dw * dh);
  double *Tf = (double *)malloc(sizeof(double) * tw * th);
  double *Df = (double *)malloc(sizeof(double) * dw * dh);
  int64_t st = 0, st2 = 0;
  double stf = 0, st2f = 0;
  for (int ty = 0; ty < th; ++ty)
    for (int tx = 0; tx < tw; ++tx) {
      const double v = px_value(f_raw, dtype, (int64_t)(trect[2] - 1 + ty) * W + (trect[0] - 1 + tx));
      Tf[ty * tw + tx] = v;
      T[ty * tw + tx] = (int64_t)v;
      st += (int64_t)v;
      st2 += (int64_t)v * (int64_t)v;
      stf += v;
      st2f += v * v;
    }
  for (int dy = 0; dy < dh; ++dy)
    for (int dx = 0; dx < dw; ++dx) {
      const double v = px_value(g_raw, dtype, (int64_t)(drect[2] - 1 + dy) * W + (drect[0] - 1 + dx));
      Df[dy * dw + dx] = v;
      D[dy * dw + dx] = (int64_t)v;
    }
  int flat;
  if (integer) {
    flat = ((int64_t)tw * th * st2 - st * st) == 0;
  } else {
    double m = stf / ((double)tw * th), q = 0;
    for (int i = 0; i < tw * th; ++i) q += (Tf[i] - m) * (Tf[i] - m);
    flat = !(q > 0);
  }
  if (!flat) {
    ncc_ctx c;
    memset(&c, 0, sizeof(c));
    c.tw = tw; c.th = th; c.dw = dw; c.dh = dh; c.integer = integer;
    c.T = T; c.D = D; c.Tf = Tf; c.Df = Df;
    c.st = st; c.st2 = st2; c.stf = stf; c.st2f = st2f;
    const int nr = ox1 - ox0 + 1, nc = oy1 - oy0 + 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nc; ++b)
      for (int a = 0; a < nr; ++a) out[(int64_t)b * nr + a] = ncc_at(&c, ox0 + a, oy0 + b, mu_g);
  }
  free(T); free(D); free(Tf); free(Df);
  return flat ? 1 : 0;
}

void orc_findpeak(const double *map, int nr, int nc, double out[3]) {
  findpeak_restated(map, nr, nc, &out[0], &out[1], &out[2]);
}

void orc_qfactor(const double *cc, int n, double out[2]) { qfactor(cc, n, &out[0], &out[1]); }

/* ======================================================================
 * a6: MeshSetUp.m:23-39.
 * ==================================================================== */
void orc_mesh(int M, int N, const double *xlist, const double *ylist, double *coords,
              int32_t *elems) {
  const int64_t n = (int64_t)M * N, ne = (int64_t)(M - 1) * (N - 1);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      coords[(int64_t)j * M + i] = xlist[i];
      coords[n + (int64_t)j * M + i] = ylist[j];
    }
  for (int j = 1; j <= N - 1; ++j)
    for (int i = 1; i <= M - 1; ++i) {
      int64_t e = (int64_t)(j - 1) * (M - 1) + (i - 1);
      elems[e] = (j - 1) * M + i;
      elems[ne + e] = (j - 1) * M + i + 1;
      elems[2 * ne + e] = j * M + i + 1;
      elems[3 * ne + e] = j * M + i;
    }
}

/* ======================================================================
 * small dense solves
 * ==================================================================== */
/* H\b for symmetric H: Cholesky, falling back to Gaussian elimination with
 * partial pivoting (MATLAB's backslash tries chol first for symmetric
 * matrices with a positive diagonal).  Returns 0 ok, -1 singular. */
static int solve_sym(int n, const double *Hin, const double *b, double *x) {
  double L[36], y[6];
  int ok = 1;
  for (int j = 0; j < n && ok; ++j) {
    double s = Hin[j * n + j];
    for (int k = 0; k < j; ++k) s -= L[j * n + k] * L[j * n + k];
    if (!(s > 0.0)) { ok = 0; break; }
    L[j * n + j] = sqrt(s);
    for (int i = j + 1; i < n; ++i) {
      double t = Hin[i * n + j];
      for (int k = 0; k < j; ++k) t -= L[i * n + k] * L[j * n + k];
      L[i * n + j] = t / L[j * n + j];
    }
  }
  if (ok) {
    for (int i = 0; i < n; ++i) {
      double t = b[i];
      for (int k = 0; k < i; ++k) t -= L[i * n + k] * y[k];
      y[i] = t / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double t = y[i];
      for (int k = i + 1; k < n; ++k) t -= L[k * n + i] * x[k];
      x[i] = t / L[i * n + i];
    }
    return 0;
  }
  double A[36], r[6];
  memcpy(A, Hin, sizeof(double) * n * n);
  memcpy(r, b, sizeof(double) * n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (fabs(A[i * n + k]) > fabs(A[p * n + k])) p = i;
    if (A[p * n + k] == 0.0) {
      for (int i = 0; i < n; ++i) x[i] = NAN;
      return -1;
    }
    if (p != k) {
      for (int j = 0; j < n; ++j) { double t = A[k * n + j]; A[k * n + j] = A[p * n + j]; A[p * n + j] = t; }
      double t = r[k]; r[k] = r[p]; r[p] = t;
    }
    for (int i = k + 1; i < n; ++i) {
      double f = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; ++j) A[i * n + j] -= f * A[k * n + j];
      r[i] -= f * r[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double t = r[i];
    for (int j = i + 1; j < n; ++j) t -= A[i * n + j] * x[j];
    x[i] = t / A[i * n + i];
  }
  return 0;
}

/* inverse-compositional update, funICGN.m:268-286 */
static int ic_compose(double P[6], const double d[6]) {
  const double det = (1 + d[0]) * (1 + d[3]) - d[1] * d[2];
  if (!(det != 0.0)) return -1;
  const double t1 = (-d[0] - d[0] * d[3] + d[1] * d[2]) / det;
  const double t2 = -d[1] / det;
  const double t3 = -d[2] / det;
  const double t4 = (-d[3] - d[0] * d[3] + d[1] * d[2]) / det;
  const double t5 = (-d[4] - d[3] * d[4] + d[2] * d[5]) / det;
  const double t6 = (-d[5] - d[0] * d[5] + d[1] * d[4]) / det;
  const double a11 = 1 + P[0], a12 = P[2], a13 = P[4];
  const double a21 = P[1], a22 = 1 + P[3], a23 = P[5];
  const double m11 = a11 * (1 + t1) + a12 * t2;
  const double m12 = a11 * t3 + a12 * (1 + t4);
  const double m13 = a11 * t5 + a12 * t6 + a13;
  const double m21 = a21 * (1 + t1) + a22 * t2;
  const double m22 = a21 * t3 + a22 * (1 + t4);
  const double m23 = a21 * t5 + a22 * t6 + a23;
  P[0] = m11 - 1;
  P[1] = m21;
  P[2] = m12;
  P[3] = m22 - 1;
  P[4] = m13;
  P[5] = m23;
  return 0;
}

/* ======================================================================
 * a7: funICGN.m per subset.
 * ==================================================================== */
typedef struct {
  const double *f, *g, *dfdx, *dfdy;
  int W, H;
} img_set;

/* subset bounds of funICGN.m:34-50 (1-based, inclusive).  Returns 0 when
 * MATLAB's indexing would succeed (integral, Df and ImgRef in range). */
static int subset_bounds(const img_set *im, double x0, double y0, int w, int *xl,
                         int *xr, int *yl, int *yr) {
  const double a = x0 - 0.5 * w, b = y0 - 0.5 * w;
  if (a != floor(a) || b != floor(b)) return -1;
  *xl = (int)a; *xr = (int)a + w;
  *yl = (int)b; *yr = (int)b + w;
  /* Df is the (W-6)x(H-6) crop starting at x=4: index x-3 in [1, W-6] */
  if (*xl < 4 || *yl < 4 || *xr > im->W - 3 || *yr > im->H - 3) return -1;
  return 0;
}

static inline int64_t pidx(const img_set *im, int x, int y) { /* 1-based */
  return (int64_t)(y - 1) * im->W + (x - 1);
}

/* funICGN.m:54-65 / funICGN_Subpb1.m:59-70: count DfDx == 0 and grow. */
static int masked_window(const img_set *im, double x0, double y0, int *w, int *xl,
                         int *xr, int *yl, int *yr) {
  int64_t cnt = 0;
  for (int y = *yl; y <= *yr; ++y)
    for (int x = *xl; x <= *xr; ++x)
      if (im->dfdx[pidx(im, x, y)] == 0.0) cnt++;
  const double n = (double)(*w + 1) * (*w + 1);
  if (!((double)cnt < 0.5 * n)) return 102;
  if ((double)cnt > 0.1 * n) {
    *w = (int)round(sqrt(2.0) * (*w));
    if (subset_bounds(im, x0, y0, *w, xl, xr, yl, yr)) return -1;
  }
  return 0;
}

static int icgn_one(const img_set *im, double x0, double y0, const double U0[2], int w,
                    double tol, double Uo[2], double Fo[4], double H21[21]) {
  int xl, xr, yl, yr;
  if (subset_bounds(im, x0, y0, w, &xl, &xr, &yl, &yr)) goto fail;
  double P[6] = {0, 0, 0, 0, U0[0], U0[1]};
  int st = masked_window(im, x0, y0, &w, &xl, &xr, &yl, &yr);
  if (st == -1) goto fail;
  if (st == 102) {
    Uo[0] = P[4]; Uo[1] = P[5];
    for (int k = 0; k < 4; ++k) Fo[k] = P[k];
    for (int k = 0; k < 21; ++k) H21[k] = 0.0;
    return 102;
  }
  const int nw = w + 1;
  const int64_t npx = (int64_t)nw * nw;
  /* H (funICGN.m:67-79) */
  double h11 = 0, h12 = 0, h13 = 0, h14 = 0, h15 = 0, h16 = 0, h22 = 0, h24 = 0, h26 = 0;
  double h33 = 0, h34 = 0, h35 = 0, h36 = 0, h44 = 0, h46 = 0, h55 = 0, h56 = 0, h66 = 0;
  double sf = 0;
  for (int y = yl; y <= yr; ++y)
    for (int x = xl; x <= xr; ++x) {
      const int64_t i = pidx(im, x, y);
      const double fx = im->dfdx[i], fy = im->dfdy[i];
      const double X = x - x0, Y = y - y0;
      const double fxx = fx * fx, fyy = fy * fy, fxy = fx * fy;
      const double XX = X * X, YY = Y * Y, XY = X * Y;
      h11 += XX * fxx; h12 += XX * fxy; h13 += XY * fxx; h14 += XY * fxy;
      h15 += X * fxx; h16 += X * fxy; h22 += XX * fyy; h24 += XY * fyy;
      h26 += X * fyy; h33 += YY * fxx; h34 += YY * fxy; h35 += Y * fxx;
      h36 += Y * fxy; h44 += YY * fyy; h46 += Y * fyy; h55 += fxx;
      h56 += fxy; h66 += fyy;
      sf += im->f[i];
    }
  double H[36] = {h11, h12, h13, h14, h15, h16, h12, h22, h14, h24, h16, h26,
                  h13, h14, h33, h34, h35, h36, h14, h24, h34, h44, h36, h46,
                  h15, h16, h35, h36, h55, h56, h16, h26, h36, h46, h56, h66};
  const double meanf = sf / (double)npx;
  double ssf = 0;
  for (int y = yl; y <= yr; ++y)
    for (int x = xl; x <= xr; ++x) {
      double d = im->f[pidx(im, x, y)] - meanf;
      ssf += d * d;
    }
  const double bottomf = sqrt((double)(npx - 1) * (ssf / (double)(npx - 1)));
  double *tg = (double *)malloc(sizeof(double) * npx * 3);
  double *uu = tg + npx, *vv = uu + npx;
  double normNew = 1, normAbs = 1, normInit = 1;
  int step = 0;
  while (step <= 100 && normNew > tol && normAbs > tol) {
    step++;
    int out = 0;
    int64_t k = 0;
    for (int y = yl; y <= yr; ++y)
      for (int x = xl; x <= xr; ++x, ++k) {
        const double X = x - x0, Y = y - y0;
        const double u22 = (1 + P[0]) * X + P[2] * Y + (x0 + P[4]);
        const double v22 = P[1] * X + (1 + P[3]) * Y + (y0 + P[5]);
        if (u22 < 3 || u22 > im->W - 2 || v22 < 3 || v22 > im->H - 2) out = 1;
        uu[k] = u22;
        vv[k] = v22;
      }
    if (out) {
      normNew = 1e6;
      break;
    }
    /* ba_interp2(ImgDef, v22, u22): F is W x H column-major (M=W) */
    orc_ba_interp2_f64(im->g, im->W, im->H, 1, vv, uu, npx, tg);
    double sg = 0;
    for (k = 0; k < npx; ++k) sg += tg[k];
    const double meang = sg / (double)npx;
    double ssg = 0;
    for (k = 0; k < npx; ++k) {
      double d = tg[k] - meang;
      ssg += d * d;
    }
    const double bottomg = sqrt((double)(npx - 1) * (ssg / (double)(npx - 1)));
    double b2[6] = {0, 0, 0, 0, 0, 0};
    k = 0;
    for (int y = yl; y <= yr; ++y)
      for (int x = xl; x <= xr; ++x, ++k) {
        const int64_t i = pidx(im, x, y);
        const double r = (im->f[i] - meanf) / bottomf - (tg[k] - meang) / bottomg;
        const double X = x - x0, Y = y - y0;
        const double fx = im->dfdx[i], fy = im->dfdy[i];
        b2[0] += X * fx * r;
        b2[1] += X * fy * r;
        b2[2] += Y * fx * r;
        b2[3] += Y * fy * r;
        b2[4] += fx * r;
        b2[5] += fy * r;
      }
    double b[6], nb = 0;
    for (int q = 0; q < 6; ++q) {
      b[q] = bottomf * b2[q];
      nb += b[q] * b[q];
    }
    normNew = sqrt(nb);
    normAbs = normNew;
    if (step == 1) normInit = normNew;
    if (normInit > tol) normNew = normNew / normInit;
    else normNew = 0;
    if (normNew < tol || normAbs < tol) break;
    double dP[6];
    solve_sym(6, H, b, dP);
    for (int q = 0; q < 6; ++q) dP[q] = -dP[q];
    if (ic_compose(P, dP)) break;
  }
  free(tg);
  if (!(normNew < tol || normAbs < tol)) step = 101;
  if (isnan(normNew)) step = 101;
  Uo[0] = P[4]; Uo[1] = P[5];
  for (int q = 0; q < 4; ++q) Fo[q] = P[q];
  {
    /* funICGN.m:320 packing */
    int idx = 0;
    for (int c = 0; c < 6; ++c)
      for (int r = c; r < 6; ++r) H21[idx++] = H[r * 6 + c];
  }
  return step;
fail:
  /* LocalICGN.m:75-80: catch -> -1 and NaN; HtempPar row stays zero */
  Uo[0] = Uo[1] = NAN;
  for (int q = 0; q < 4; ++q) Fo[q] = NAN;
  for (int q = 0; q < 21; ++q) H21[q] = 0.0;
  return -1;
}

void orc_icgn_batch(const double *f, const double *g, const double *dfdx,
                    const double *dfdy, int W, int H, const double *coords,
                    int64_t n, const double *U0, const int32_t *winsize_arr,
                    int winsize, double tol, double *U, double *F,
                    int32_t *iters, double *H21) {
  img_set im = {f, g, dfdx, dfdy, W, H};
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t j = 0; j < n; ++j) {
    double Uo[2], Fo[4], h[21];
    const int w = winsize_arr ? winsize_arr[j] : winsize;
    int it = icgn_one(&im, coords[j], coords[n + j], U0 + 2 * j, w, tol, Uo, Fo, h);
    iters[j] = it;
    U[2 * j] = Uo[0]; U[2 * j + 1] = Uo[1];
    for (int q = 0; q < 4; ++q) F[4 * j + q] = Fo[q];
    for (int q = 0; q < 21; ++q) H21[(int64_t)q * n + j] = h[q];
  }
}

/* ======================================================================
 * a9: funICGN_Subpb1.m per subset.
 * ==================================================================== */
static int subpb1_one(const img_set *im, double x0, double y0, const double UOld[2],
                      const double FOld[4], const double vdual[2], double h55,
                      double h65, double h66, int w, double mu, double tol,
                      double Uo[2]) {
  int xl, xr, yl, yr;
  double P[6] = {FOld[0], FOld[1], FOld[2], FOld[3], UOld[0], UOld[1]};
  if (subset_bounds(im, x0, y0, w, &xl, &xr, &yl, &yr)) goto fail;
  int st = masked_window(im, x0, y0, &w, &xl, &xr, &yl, &yr);
  if (st == -1) goto fail;
  if (st == 102) {
    Uo[0] = P[4]; Uo[1] = P[5];
    return 102;
  }
  const int nw = w + 1;
  const int64_t npx = (int64_t)nw * nw;
  double sf = 0;
  for (int y = yl; y <= yr; ++y)
    for (int x = xl; x <= xr; ++x) sf += im->f[pidx(im, x, y)];
  const double meanf = sf / (double)npx;
  double ssf = 0;
  for (int y = yl; y <= yr; ++y)
    for (int x = xl; x <= xr; ++x) {
      double d = im->f[pidx(im, x, y)] - meanf;
      ssf += d * d;
    }
  const double bottomf = sqrt((double)(npx - 1) * (ssf / (double)(npx - 1)));
  const double s2 = 2.0 / (bottomf * bottomf);
  /* funICGN_Subpb1.m:73,281-283 */
  const double H2a = h55 * s2 + mu, H2b = h65 * s2, H2d = h66 * s2 + mu;
  const double dmax = H2a > H2d ? H2a : H2d;
  const double Ha = H2a + 1e-3 * dmax, Hb = H2b, Hd = H2d + 1e-3 * dmax;
  const double Hs[4] = {Ha, Hb, Hb, Hd};
  double *tg = (double *)malloc(sizeof(double) * npx * 3);
  double *uu = tg + npx, *vv = uu + npx;
  double normNew = 1, normAbs = 1, normInit = 1;
  int step = 0;
  while (step <= 100 && normNew > tol && normAbs > tol) {
    step++;
    int out = 0;
    int64_t k = 0;
    for (int y = yl; y <= yr; ++y)
      for (int x = xl; x <= xr; ++x, ++k) {
        const double X = x - x0, Y = y - y0;
        const double u22 = (1 + P[0]) * X + P[2] * Y + (x0 + P[4]);
        const double v22 = P[1] * X + (1 + P[3]) * Y + (y0 + P[5]);
        if (u22 < 3 || u22 > im->W - 2 || v22 < 3 || v22 > im->H - 2) out = 1;
        uu[k] = u22;
        vv[k] = v22;
      }
    if (out) {
      normNew = 1e6;
      break;
    }
    orc_ba_interp2_f64(im->g, im->W, im->H, 1, vv, uu, npx, tg);
    double sg = 0;
    for (k = 0; k < npx; ++k) sg += tg[k];
    const double meang = sg / (double)npx;
    double ssg = 0;
    for (k = 0; k < npx; ++k) {
      double d = tg[k] - meang;
      ssg += d * d;
    }
    const double bottomg = sqrt((double)(npx - 1) * (ssg / (double)(npx - 1)));
    double b5 = 0, b6 = 0;
    k = 0;
    for (int y = yl; y <= yr; ++y)
      for (int x = xl; x <= xr; ++x, ++k) {
        const int64_t i = pidx(im, x, y);
        const double r = (im->f[i] - meanf) / bottomf - (tg[k] - meang) / bottomg;
        b5 += im->dfdx[i] * r;
        b6 += im->dfdy[i] * r;
      }
    /* funICGN_Subpb1.m:267-269 */
    double tb[2];
    tb[0] = bottomf * b5 * s2 + mu * (P[4] - UOld[0] - vdual[0]);
    tb[1] = bottomf * b6 * s2 + mu * (P[5] - UOld[1] - vdual[1]);
    double dP[6] = {0, 0, 0, 0, 0, 0}, sol[2];
    solve_sym(2, Hs, tb, sol);
    dP[4] = -sol[0];
    dP[5] = -sol[1];
    normNew = sqrt(tb[0] * tb[0] + tb[1] * tb[1]);
    normAbs = normNew;
    if (step == 1) normInit = normNew;
    if (normInit > tol) normNew = normNew / normInit;
    else normNew = 0;
    if (normNew < tol || normAbs < tol) break;
    if (ic_compose(P, dP)) break;
  }
  free(tg);
  if (!(normNew < tol || normAbs < tol)) step = 101;
  if (isnan(normNew)) step = 101;
  Uo[0] = P[4]; Uo[1] = P[5];
  return step;
fail:
  Uo[0] = Uo[1] = NAN;
  return -1;
}

void orc_subpb1_batch(const double *f, const double *g, const double *dfdx,
                      const double *dfdy, int W, int H, const double *coords,
                      int64_t n, const double *UOld, const double *FOld,
                      const double *vdual, const double *H21,
                      const int32_t *winsize_arr, int winsize, double mu,
                      double tol, double *U, int32_t *iters) {
  img_set im = {f, g, dfdx, dfdy, W, H};
#pragma omp parallel for schedule(dynamic, 8)
  for (int64_t j = 0; j < n; ++j) {
    double Uo[2];
    const int w = winsize_arr ? winsize_arr[j] : winsize;
    iters[j] = subpb1_one(&im, coords[j], coords[n + j], UOld + 2 * j, FOld + 4 * j,
                          vdual + 2 * j, H21[18 * n + j], H21[19 * n + j], H21[20 * n + j],
                          w, mu, tol, Uo);
    U[2 * j] = Uo[0];
    U[2 * j + 1] = Uo[1];
  }
}

/* ======================================================================
 * Grid solvers: gridfit 'springs' and inpaint_nans method 4 by FP64 CG.
 * ==================================================================== */
typedef void (*matvec_fn)(const void *ctx, const double *x, double *y);

static int cg_solve(int64_t n, matvec_fn A, const void *ctx, const double *b, double *x,
                    double rtol, int maxit) {
  double *r = (double *)malloc(sizeof(double) * n * 3);
  double *p = r + n, *Ap = p + n;
  A(ctx, x, Ap);
  double bb = 0, rr = 0;
  for (int64_t i = 0; i < n; ++i) {
    r[i] = b[i] - Ap[i];
    p[i] = r[i];
    bb += b[i] * b[i];
    rr += r[i] * r[i];
  }
  int it = 0;
  const double stop = rtol * rtol * (bb > 0 ? bb : 1.0);
  while (rr > stop && it < maxit) {
    A(ctx, p, Ap);
    double pAp = 0;
    for (int64_t i = 0; i < n; ++i) pAp += p[i] * Ap[i];
    const double alpha = rr / pAp;
    double rr2 = 0;
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
      rr2 += r[i] * r[i];
    }
    const double beta = rr2 / rr;
    for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
    rr = rr2;
    it++;
  }
  free(r);
  return it;
}

typedef struct {
  int M, N;
  const double *wdata; /* 1 where data present */
  double lam2;
} gf_ctx;

/* (A'A + lam^2 Areg'Areg) x with the springs of gridfit.m:523-550 on a
 * uniform grid: axial springs of stiffness 1, the two diagonals 1/sqrt(2). */
static void gf_matvec(const void *vctx, const double *x, double *y) {
  const gf_ctx *c = (const gf_ctx *)vctx;
  const int M = c->M, N = c->N;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      const int64_t k = (int64_t)j * M + i;
      const double xk = x[k];
      double s = 0;
      if (i > 0) s += xk - x[k - 1];
      if (i < M - 1) s += xk - x[k + 1];
      if (j > 0) s += xk - x[k - M];
      if (j < N - 1) s += xk - x[k + M];
      double sd = 0;
      if (i > 0 && j > 0) sd += xk - x[k - M - 1];
      if (i < M - 1 && j > 0) sd += xk - x[k - M + 1];
      if (i > 0 && j < N - 1) sd += xk - x[k + M - 1];
      if (i < M - 1 && j < N - 1) sd += xk - x[k + M + 1];
      y[k] = c->wdata[k] * xk + c->lam2 * (s + 0.5 * sd);
    }
}

/* norm(Areg,1) of gridfit.m:592: max column sum of |Areg| */
static double springs_norm1(int M, int N) {
  double best = 0;
  const double d = 1.0 / sqrt(2.0);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      double s = 0;
      s += (i > 0) + (i < M - 1) + (j > 0) + (j < N - 1);
      s += d * ((i > 0 && j > 0) + (i < M - 1 && j > 0) + (i > 0 && j < N - 1) + (i < M - 1 && j < N - 1));
      if (s > best) best = s;
    }
  return best;
}

int orc_gridfit_springs(int M, int N, int nf, const double *in, double *out) {
  const int64_t n = (int64_t)M * N;
  double *w = (double *)malloc(sizeof(double) * n);
  double *b = (double *)malloc(sizeof(double) * n);
  double *x = (double *)malloc(sizeof(double) * n);
  const double NR = springs_norm1(M, N);
  int maxit_used = 0;
  for (int fi = 0; fi < nf; ++fi) {
    const double *d = in + fi * n;
    int64_t nd = 0;
    for (int64_t k = 0; k < n; ++k) {
      const int ok = !isnan(d[k]);
      w[k] = ok ? 1.0 : 0.0;
      b[k] = ok ? d[k] : 0.0;
      x[k] = ok ? d[k] : 0.0;
      nd += ok;
    }
    if (nd < 3) {
      free(w); free(b); free(x);
      return -1;
    }
    gf_ctx c = {M, N, w, 1.0 / (NR * NR)}; /* smoothness 1, norm(A,1) = 1 */
    int it = cg_solve(n, gf_matvec, &c, b, x, 1e-13, 20000);
    if (it > maxit_used) maxit_used = it;
    memcpy(out + fi * n, x, sizeof(double) * n);
  }
  free(w); free(b); free(x);
  return maxit_used;
}

typedef struct {
  int M, N;
  const unsigned char *unk;
} ip_ctx;

/* inpaint_nans.m method 4: springs between each NaN node and its 4
 * neighbours; normal equations restricted to the unknown nodes. */
static void ip_matvec(const void *vctx, const double *x, double *y) {
  const ip_ctx *c = (const ip_ctx *)vctx;
  const int M = c->M, N = c->N;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      const int64_t k = (int64_t)j * M + i;
      if (!c->unk[k]) { y[k] = 0; continue; }
      double s = 0;
      const int64_t nb[4] = {i > 0 ? k - 1 : -1, i < M - 1 ? k + 1 : -1, j > 0 ? k - M : -1,
                             j < N - 1 ? k + M : -1};
      for (int q = 0; q < 4; ++q) {
        if (nb[q] < 0) continue;
        s += x[k];
        if (c->unk[nb[q]]) s -= x[nb[q]];
      }
      y[k] = s;
    }
}

int orc_inpaint_springs(int M, int N, double *z) {
  const int64_t n = (int64_t)M * N;
  unsigned char *unk = (unsigned char *)malloc(n);
  int64_t nn = 0;
  for (int64_t k = 0; k < n; ++k) {
    unk[k] = isnan(z[k]) ? 1 : 0;
    nn += unk[k];
  }
  if (nn == 0) { free(unk); return 0; }
  if (nn == n) { free(unk); return -1; }
  double *b = (double *)calloc(n, sizeof(double));
  double *x = (double *)calloc(n, sizeof(double));
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      const int64_t k = (int64_t)j * M + i;
      if (!unk[k]) continue;
      const int64_t nb[4] = {i > 0 ? k - 1 : -1, i < M - 1 ? k + 1 : -1, j > 0 ? k - M : -1,
                             j < N - 1 ? k + M : -1};
      for (int q = 0; q < 4; ++q)
        if (nb[q] >= 0 && !unk[nb[q]]) b[k] += z[nb[q]];
    }
  ip_ctx c = {M, N, unk};
  int it = cg_solve(n, ip_matvec, &c, b, x, 1e-13, 50000);
  for (int64_t k = 0; k < n; ++k)
    if (unk[k]) z[k] = x[k];
  free(unk); free(b); free(x);
  return it;
}

/* ======================================================================
 * LocalICGN.m:114-161 and Subpb1.m:162-199 post-processing
 * ==================================================================== */
int orc_localicgn_post(int M, int N, const int32_t *iters, double *U, double *F) {
  const int64_t n = (int64_t)M * N;
  unsigned char *bad = (unsigned char *)calloc(n, 1);
  int64_t nbad = 0, n102 = 0, ngood = 0;
  double sum = 0;
  for (int64_t k = 0; k < n; ++k) {
    bad[k] = (iters[k] < 0 || iters[k] > 99);
    nbad += bad[k];
    n102 += (iters[k] == 102);
    if (!bad[k]) { ngood++; sum += iters[k]; }
  }
  double mean = ngood ? sum / ngood : NAN, ss = 0;
  for (int64_t k = 0; k < n; ++k)
    if (!bad[k]) ss += (iters[k] - mean) * (iters[k] - mean);
  const double sd = ngood > 1 ? sqrt(ss / (ngood - 1)) : (ngood == 1 ? 0.0 : NAN);
  const double thr = mean + 0.15 * sd;
  for (int64_t k = 0; k < n; ++k)
    if ((double)iters[k] > thr) bad[k] = 1;
  double *fld = (double *)malloc(sizeof(double) * n);
  for (int c = 0; c < 6; ++c) {
    double *base = c < 2 ? U : F;
    const int stride = c < 2 ? 2 : 4, off = c < 2 ? c : c - 2;
    for (int64_t k = 0; k < n; ++k) fld[k] = bad[k] ? NAN : base[k * stride + off];
    orc_inpaint_springs(M, N, fld);
    for (int64_t k = 0; k < n; ++k) base[k * stride + off] = fld[k];
  }
  free(fld);
  free(bad);
  return (int)(nbad - n102);
}

int orc_subpb1_post(int M, int N, const int32_t *iters, double *U) {
  const int64_t n = (int64_t)M * N;
  double *fld = (double *)malloc(sizeof(double) * 2 * n);
  int nbad = 0;
  for (int64_t k = 0; k < n; ++k) {
    const int b = iters[k] < 0 || iters[k] > 99;
    nbad += b;
    fld[k] = b ? NAN : U[2 * k];
    fld[n + k] = b ? NAN : U[2 * k + 1];
  }
  int rc = orc_gridfit_springs(M, N, 2, fld, fld);
  for (int64_t k = 0; k < n; ++k) {
    U[2 * k] = fld[k];
    U[2 * k + 1] = fld[n + k];
  }
  free(fld);
  return rc < 0 ? rc : nbad;
}

/* ======================================================================
 * a10: Subpb2.m:72-195 on the uniform Q4 mesh
 * ==================================================================== */
typedef struct {
  int M, N;
  double *blk; /* per node: 9 neighbours x 2x2 block (row-major) */
} fe_ctx;

static void fe_matvec(const void *vctx, const double *x, double *y) {
  const fe_ctx *c = (const fe_ctx *)vctx;
  const int M = c->M, N = c->N;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      const int64_t k = (int64_t)j * M + i;
      double s0 = 0, s1 = 0;
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          const int ii = i + di, jj = j + dj;
          if (ii < 0 || ii >= M || jj < 0 || jj >= N) continue;
          const double *B = c->blk + (k * 9 + (dj + 1) * 3 + (di + 1)) * 4;
          const int64_t q = (int64_t)jj * M + ii;
          s0 += B[0] * x[2 * q] + B[1] * x[2 * q + 1];
          s1 += B[2] * x[2 * q] + B[3] * x[2 * q + 1];
        }
      y[2 * k] = s0;
      y[2 * k + 1] = s1;
    }
}

/* Shape-function derivatives of Subpb2.m:201-224 */
static void dN_dksi_deta(double ksi, double eta, double dks[4], double det_[4]) {
  dks[0] = -(1 - eta) / 4; det_[0] = -(1 - ksi) / 4;
  dks[1] = (1 - eta) / 4;  det_[1] = -(1 + ksi) / 4;
  dks[2] = (1 + eta) / 4;  det_[2] = (1 + ksi) / 4;
  dks[3] = -(1 + eta) / 4; det_[3] = (1 - ksi) / 4;
}

int orc_subpb2(int M, int N, double step, double beta, double mu,
               const double *U, const double *F, const double *udual,
               const double *vdual, double *Uhat) {
  const int64_t n = (int64_t)M * N;
  fe_ctx c = {M, N, (double *)calloc((size_t)n * 36, sizeof(double))};
  double *b = (double *)calloc((size_t)2 * n, sizeof(double));
  const double gp[3] = {-sqrt(3.0 / 5.0), 0.0, sqrt(3.0 / 5.0)};
  const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  for (int ej = 0; ej < N - 1; ++ej)
    for (int ei = 0; ei < M - 1; ++ei) {
      /* elementsFEM row: [(j-1)M+i, (j-1)M+i+1, jM+i+1, jM+i] (1-based) */
      int64_t nd[4] = {(int64_t)ej * M + ei, (int64_t)ej * M + ei + 1,
                       (int64_t)(ej + 1) * M + ei + 1, (int64_t)(ej + 1) * M + ei};
      double px[4], py[4];
      for (int a = 0; a < 4; ++a) {
        px[a] = (nd[a] % M) * step;
        py[a] = (nd[a] / M) * step;
      }
      /* DOF k = 2a (u), 2a+1 (v).  FMinusW rows: [F11 F12 F21 F22] with
       * the index order [4a-3, 4a-1, 4a-2, 4a] of Subpb2.m:88-94 */
      double FW[8][4], UV[8];
      for (int k = 0; k < 8; ++k) {
        const int64_t a = nd[k / 2];
        const int64_t fi[4] = {4 * a + 0, 4 * a + 2, 4 * a + 1, 4 * a + 3};
        for (int q = 0; q < 4; ++q) FW[k][q] = F[fi[q]] - udual[fi[q]];
        const int64_t ui = 2 * a + (k & 1);
        UV[k] = U[ui] - vdual[ui];
      }
      double A8[8][8], b8[8];
      memset(A8, 0, sizeof(A8));
      memset(b8, 0, sizeof(b8));
      for (int ti = 0; ti < 3; ++ti)
        for (int tj = 0; tj < 3; ++tj) {
          const double ksi = gp[ti], eta = gp[tj];
          const double wgt = gw[ti] * gw[tj];
          const double N4[4] = {(1 - ksi) * (1 - eta) * 0.25, (1 + ksi) * (1 - eta) * 0.25,
                                (1 + ksi) * (1 + eta) * 0.25, (1 - ksi) * (1 + eta) * 0.25};
          double dks[4], det_[4];
          dN_dksi_deta(ksi, eta, dks, det_);
          double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
          for (int a = 0; a < 4; ++a) {
            J11 += dks[a] * px[a]; J12 += dks[a] * py[a];
            J21 += det_[a] * px[a]; J22 += det_[a] * py[a];
          }
          const double Jac = J11 * J22 - J12 * J21;
          const double i11 = J22 / Jac, i12 = -J12 / Jac, i21 = -J21 / Jac, i22 = J11 / Jac;
          /* DN (4x8): rows du/dx du/dy dv/dx dv/dy */
          double DN[4][8];
          memset(DN, 0, sizeof(DN));
          for (int a = 0; a < 4; ++a) {
            const double gx = i11 * dks[a] + i12 * det_[a];
            const double gy = i21 * dks[a] + i22 * det_[a];
            DN[0][2 * a] = gx; DN[1][2 * a] = gy;
            DN[2][2 * a + 1] = gx; DN[3][2 * a + 1] = gy;
          }
          double Nm[2][8];
          memset(Nm, 0, sizeof(Nm));
          for (int a = 0; a < 4; ++a) { Nm[0][2 * a] = N4[a]; Nm[1][2 * a + 1] = N4[a]; }
          const double s = Jac * wgt;
          for (int r = 0; r < 8; ++r) {
            for (int q = 0; q < 8; ++q) {
              double kk = 0, mm = 0;
              for (int t = 0; t < 4; ++t) kk += DN[t][r] * DN[t][q];
              for (int t = 0; t < 2; ++t) mm += Nm[t][r] * Nm[t][q];
              A8[r][q] += s * (beta * kk + mu * mm);
            }
            /* diag(DN' * FMinusW') and N'N (U - V) */
            double dd = 0, nn = 0;
            for (int t = 0; t < 4; ++t) dd += DN[t][r] * FW[r][t];
            for (int q = 0; q < 8; ++q) {
              double mm = 0;
              for (int t = 0; t < 2; ++t) mm += Nm[t][r] * Nm[t][q];
              nn += mm * UV[q];
            }
            b8[r] += s * (beta * dd + mu * nn);
          }
        }
      for (int r = 0; r < 8; ++r) {
        const int64_t nr = nd[r / 2];
        b[2 * nr + (r & 1)] += b8[r];
        for (int q = 0; q < 8; ++q) {
          const int64_t nq = nd[q / 2];
          const int di = (int)(nq % M) - (int)(nr % M), dj = (int)(nq / M) - (int)(nr / M);
          double *B = c.blk + (nr * 9 + (dj + 1) * 3 + (di + 1)) * 4;
          B[(r & 1) * 2 + (q & 1)] += A8[r][q];
        }
      }
    }
  for (int64_t k = 0; k < 2 * n; ++k) Uhat[k] = 0.0;
  int it = cg_solve(2 * n, fe_matvec, &c, b, Uhat, 1e-13, 100000);
  free(c.blk);
  free(b);
  return it;
}

/* ======================================================================
 * a11: funGlobal_NodalStrainAvg.m:32-144 on the uniform mesh.  The output
 * slots per node are [du/dx du/dy dv/dx dv/dy] exactly as :97,123-137 write
 * them (DN*U), which differs from funICGN's [F11 F21 F12 F22] order in the
 * two middle slots; the reference's ADMM loop consumes them as written.
 * ==================================================================== */
void orc_nodal_strain(int M, int N, double step, const double *U, double *Fout) {
  const int64_t n = (int64_t)M * N;
  double *acc = (double *)calloc((size_t)4 * n, sizeof(double));
  double *cnt = (double *)calloc((size_t)4 * n, sizeof(double));
  const double r3 = 1.0 / sqrt(3.0);
  const double gks[4] = {-r3, r3, r3, -r3}, get_[4] = {-r3, -r3, r3, r3};
  const double s3 = sqrt(3.0);
  const double E[4][4] = {{1 + 0.5 * s3, -0.5, 1 - 0.5 * s3, -0.5},
                          {-0.5, 1 + 0.5 * s3, -0.5, 1 - 0.5 * s3},
                          {1 - 0.5 * s3, -0.5, 1 + 0.5 * s3, -0.5},
                          {-0.5, 1 - 0.5 * s3, -0.5, 1 + 0.5 * s3}};
  for (int ej = 0; ej < N - 1; ++ej)
    for (int ei = 0; ei < M - 1; ++ei) {
      int64_t nd[4] = {(int64_t)ej * M + ei, (int64_t)ej * M + ei + 1,
                       (int64_t)(ej + 1) * M + ei + 1, (int64_t)(ej + 1) * M + ei};
      double px[4], py[4], ue[8];
      for (int a = 0; a < 4; ++a) {
        px[a] = (nd[a] % M) * step;
        py[a] = (nd[a] / M) * step;
        ue[2 * a] = U[2 * nd[a]];
        ue[2 * a + 1] = U[2 * nd[a] + 1];
      }
      double G[4][4]; /* gauss point x component */
      for (int g = 0; g < 4; ++g) {
        double dks[4], det_[4];
        dN_dksi_deta(gks[g], get_[g], dks, det_);
        double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
        for (int a = 0; a < 4; ++a) {
          J11 += dks[a] * px[a]; J12 += dks[a] * py[a];
          J21 += det_[a] * px[a]; J22 += det_[a] * py[a];
        }
        const double Jac = J11 * J22 - J12 * J21;
        const double i11 = J22 / Jac, i12 = -J12 / Jac, i21 = -J21 / Jac, i22 = J11 / Jac;
        double v[4] = {0, 0, 0, 0};
        for (int a = 0; a < 4; ++a) {
          const double gx = i11 * dks[a] + i12 * det_[a];
          const double gy = i21 * dks[a] + i22 * det_[a];
          v[0] += gx * ue[2 * a];
          v[1] += gy * ue[2 * a];
          v[2] += gx * ue[2 * a + 1];
          v[3] += gy * ue[2 * a + 1];
        }
        for (int q = 0; q < 4; ++q) G[g][q] = v[q];
      }
      for (int a = 0; a < 4; ++a)
        for (int q = 0; q < 4; ++q) {
          double s = 0;
          for (int g = 0; g < 4; ++g) s += E[a][g] * G[g][q];
          acc[4 * nd[a] + q] += s;
          cnt[4 * nd[a] + q] += 1.0;
        }
    }
  for (int64_t k = 0; k < 4 * n; ++k) Fout[k] = acc[k] / cnt[k];
  free(acc);
  free(cnt);
}

/* ======================================================================
 * a14: funSmoothDisp.m:64-101 / funSmoothStrain.m:63-109 core.
 * ==================================================================== */
int orc_smooth_fields(int M, int N, int nf, double *vals) {
  const int64_t n = (int64_t)M * N;
  double *fld = (double *)malloc(sizeof(double) * n * nf);
  double *tmp = (double *)malloc(sizeof(double) * n);
  /* fspecial('gaussian',3,0.5) */
  double k[3][3], ks = 0;
  for (int a = -1; a <= 1; ++a)
    for (int b = -1; b <= 1; ++b) {
      k[a + 1][b + 1] = exp(-(a * a + b * b) / (2 * 0.25));
      ks += k[a + 1][b + 1];
    }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) k[a][b] /= ks;
  for (int pass = 0; pass < 2; ++pass) {
    for (int fi = 0; fi < nf; ++fi)
      for (int64_t q = 0; q < n; ++q) fld[fi * n + q] = vals[q * nf + fi];
    if (orc_gridfit_springs(M, N, nf, fld, fld) < 0) {
      free(fld); free(tmp);
      return -1;
    }
    for (int fi = 0; fi < nf; ++fi) {
      double *z = fld + fi * n;
      /* nanconv(z, k, 'edge', 'nanout') with no NaN left after gridfit */
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < M; ++i) {
          double s = 0, w = 0;
          for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di) {
              const int ii = i + di, jj = j + dj;
              if (ii < 0 || ii >= M || jj < 0 || jj >= N) continue;
              s += k[di + 1][dj + 1] * z[(int64_t)jj * M + ii];
              w += k[di + 1][dj + 1];
            }
          tmp[(int64_t)j * M + i] = s / w;
        }
      memcpy(z, tmp, sizeof(double) * n);
    }
    for (int fi = 0; fi < nf; ++fi)
      for (int64_t q = 0; q < n; ++q) vals[q * nf + fi] = fld[fi * n + q];
  }
  free(fld);
  free(tmp);
  return 0;
}

/* ======================================================================
 * a12: ADMM core, main_ALDIC.m:166-451 (one frame, accumulative mode).
 * ==================================================================== */
static double vec_norm_diff(const double *a, const double *b, int64_t n) {
  double s = 0;
  for (int64_t i = 0; i < n; ++i) s += (a[i] - b[i]) * (a[i] - b[i]);
  return sqrt(s);
}

int orc_frame(const void *f_raw, const void *g_raw, int dtype, int W, int H,
              const orc_frame_params *p, orc_frame_result *r) {
  memset(r, 0, sizeof(*r));
  const double t0 = now_s();
  const int64_t npx = (int64_t)W * H;
  const int roi[4] = {p->gridx[0], p->gridx[1], p->gridy[0], p->gridy[1]};
  double *f = (double *)malloc(sizeof(double) * npx);
  double *g = (double *)malloc(sizeof(double) * npx);
  double *dfdx = (double *)malloc(sizeof(double) * npx);
  double *dfdy = (double *)malloc(sizeof(double) * npx);
  double mf, sf, mg, sg;
  orc_normalize(f_raw, dtype, W, H, roi, f, &mf, &sf);
  orc_normalize(g_raw, dtype, W, H, roi, g, &mg, &sg);
  orc_gradient(f, NULL, W, H, dfdx, dfdy);
  /* Section 3: search, MeshSetUp, Init */
  double ts = now_s();
  int nx, ny;
  orc_search_dims(W, H, p->gridx, p->gridy, p->winsize, p->step, p->search, &nx, &ny, NULL, NULL);
  const int M = nx, N = ny;
  const int64_t n = (int64_t)M * N;
  double *sx = (double *)malloc(sizeof(double) * n * 5);
  double *sy = sx + n, *su = sy + n, *sv = su + n, *scc = sv + n;
  if (!p->init_U) {
    orc_int_search(f_raw, g_raw, dtype, W, H, mg, p->gridx, p->gridy, p->winsize, p->step,
                   p->search, sx, sy, su, sv, scc, NULL);
  } else {
    /* the node grid of the search (funIntegerSearch.m:158-159), no search */
    int gx1, gy1;
    orc_search_dims(W, H, p->gridx, p->gridy, p->winsize, p->step, p->search, &nx, &ny, &gx1, &gy1);
    for (int i = 0; i < ny; ++i)
      for (int j = 0; j < nx; ++j) {
        const int64_t o = (int64_t)i + (int64_t)j * ny; /* ny x nx column-major */
        const double ii = gx1 + (double)j * p->step, jj = gy1 + (double)i * p->step;
        sx[o] = (ii + ii + p->winsize) / 2.0;
        sy[o] = (jj + jj + p->winsize) / 2.0;
        su[o] = sv[o] = scc[o] = 0.0;
      }
  }
  r->t_search = now_s() - ts;
  /* x (ny x nx) -> coordinatesFEM x-fastest; Init inpaints u,v (Init.m:13) */
  r->M = M; r->N = N;
  r->x0 = (double *)malloc(sizeof(double) * n);
  r->y0 = (double *)malloc(sizeof(double) * n);
  double *coords = (double *)malloc(sizeof(double) * 2 * n);
  double *ug = (double *)malloc(sizeof(double) * n), *vg = (double *)malloc(sizeof(double) * n);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) {
      const int64_t k = (int64_t)j * M + i, src = (int64_t)j + (int64_t)i * N;
      coords[k] = sx[src];
      coords[n + k] = sy[src];
      r->x0[k] = sx[src];
      r->y0[k] = sy[src];
      ug[k] = su[src];
      vg[k] = sv[src];
    }
  double *U0 = (double *)malloc(sizeof(double) * 2 * n);
  if (!p->init_U) {
    orc_inpaint_springs(M, N, ug);
    orc_inpaint_springs(M, N, vg);
    for (int64_t k = 0; k < n; ++k) { U0[2 * k] = ug[k]; U0[2 * k + 1] = vg[k]; }
  } else {
    memcpy(U0, p->init_U, sizeof(double) * 2 * n);
  }
  /* Section 4: LocalICGN */
  double ti = now_s();
  double *U1 = (double *)malloc(sizeof(double) * 2 * n);
  double *F1 = (double *)malloc(sizeof(double) * 4 * n);
  double *H21 = (double *)malloc(sizeof(double) * 21 * n);
  int32_t *it1 = (int32_t *)malloc(sizeof(int32_t) * n);
  orc_icgn_batch(f, g, dfdx, dfdy, W, H, coords, n, U0, NULL, p->winsize, p->tol, U1, F1, it1, H21);
  orc_localicgn_post(M, N, it1, U1, F1);
  r->t_icgn = now_s() - ti;
  r->iters_icgn = it1;
  r->U_icgn = (double *)malloc(sizeof(double) * 2 * n);
  r->F_icgn = (double *)malloc(sizeof(double) * 4 * n);
  memcpy(r->U_icgn, U1, sizeof(double) * 2 * n);
  memcpy(r->F_icgn, F1, sizeof(double) * 4 * n);
  /* Section 5 */
  double tsub2 = now_s();
  if (p->smooth) orc_smooth_fields(M, N, 4, F1);
  const double mu = p->mu, step = (double)p->step;
  double *udual = (double *)calloc(4 * n, sizeof(double));
  double *vdual = (double *)calloc(2 * n, sizeof(double));
  double *U2 = (double *)malloc(sizeof(double) * 2 * n);
  double *F2 = (double *)malloc(sizeof(double) * 4 * n);
  double beta = p->beta;
  if (!(beta > 0)) {
    /* main_ALDIC.m:237,285-301 */
    const double bl[6] = {1e-3, sqrt(1e-5), 1e-2, sqrt(1e-3), 1e-1, sqrt(1e-1)};
    double e1[6], e2[6], bs[6];
    for (int k = 0; k < 6; ++k) {
      bs[k] = bl[k] * step * step * mu;
      orc_subpb2(M, N, step, bs[k], mu, U1, F1, udual, vdual, U2);
      orc_nodal_strain(M, N, step, U2, F2);
      e1[k] = vec_norm_diff(U1, U2, 2 * n);
      e2[k] = vec_norm_diff(F1, F2, 4 * n);
    }
    double m1 = 0, m2 = 0;
    for (int k = 0; k < 6; ++k) { m1 += e1[k]; m2 += e2[k]; }
    m1 /= 6; m2 /= 6;
    double v1 = 0, v2 = 0;
    for (int k = 0; k < 6; ++k) { v1 += (e1[k] - m1) * (e1[k] - m1); v2 += (e2[k] - m2) * (e2[k] - m2); }
    v1 = sqrt(v1 / 5); v2 = sqrt(v2 / 5);
    double es[6];
    int ib = 0;
    for (int k = 0; k < 6; ++k) {
      es[k] = (e1[k] - m1) / v1 + (e2[k] - m2) / v2;
      if (es[k] < es[ib]) ib = k;
    }
    if (ib >= 1 && ib <= 4) {
      /* poly2 through three points in log10(beta); vertex -p2/(2 p1) */
      const double x0 = log10(bs[ib - 1]), x1 = log10(bs[ib]), x2 = log10(bs[ib + 1]);
      const double y0 = es[ib - 1], y1 = es[ib], y2 = es[ib + 1];
      const double d01 = (y1 - y0) / (x1 - x0), d12 = (y2 - y1) / (x2 - x1);
      const double p1 = (d12 - d01) / (x2 - x0);
      const double p2 = d01 - p1 * (x0 + x1);
      beta = pow(10.0, -p2 / 2.0 / p1);
    } else {
      beta = bs[ib];
    }
  }
  r->beta = beta;
  orc_subpb2(M, N, step, beta, mu, U1, F1, udual, vdual, U2);
  orc_nodal_strain(M, N, step, U2, F2);
  if (p->smooth) orc_smooth_fields(M, N, 4, F2);
  for (int64_t k = 0; k < 4 * n; ++k) udual[k] = F2[k] - F1[k];
  for (int64_t k = 0; k < 2 * n; ++k) vdual[k] = U2[k] - U1[k];
  r->t_subpb2 += now_s() - tsub2;
  /* Section 6 */
  double *U2old = (double *)malloc(sizeof(double) * 2 * n);
  double *U1old = (double *)malloc(sizeof(double) * 2 * n);
  int32_t *itb = (int32_t *)malloc(sizeof(int32_t) * n);
  memcpy(U1old, U1, sizeof(double) * 2 * n);
  int steps = 0;
  for (int a = 0; a < p->n_admm; ++a) {
    double t1 = now_s();
    memcpy(U2old, U2, sizeof(double) * 2 * n);
    orc_subpb1_batch(f, g, dfdx, dfdy, W, H, coords, n, U2, F2, vdual, H21, NULL, p->winsize,
                     mu, p->tol, U1, itb);
    orc_subpb1_post(M, N, itb, U1);
    memcpy(F1, F2, sizeof(double) * 4 * n);
    r->t_subpb1 += now_s() - t1;
    const double uy2 = vec_norm_diff(U1old, U1, 2 * n) / sqrt((double)(2 * n));
    memcpy(U1old, U1, sizeof(double) * 2 * n);
    if (p->smooth) orc_smooth_fields(M, N, 2, U1);
    double t2 = now_s();
    orc_subpb2(M, N, step, beta, mu, U1, F1, udual, vdual, U2);
    if (p->smooth) orc_smooth_fields(M, N, 2, U2);
    orc_nodal_strain(M, N, step, U2, F2);
    if (p->smooth) orc_smooth_fields(M, N, 4, F2);
    r->t_subpb2 += now_s() - t2;
    const double uy = vec_norm_diff(U2old, U2, 2 * n) / sqrt((double)(2 * n));
    if (a < 16) { r->update_y[a] = uy; r->update_y2[a] = uy2; }
    for (int64_t k = 0; k < 4 * n; ++k) udual[k] = F2[k] - F1[k];
    for (int64_t k = 0; k < 2 * n; ++k) vdual[k] = U2[k] - U1[k];
    steps++;
    if (p->tol2 > 0 && (uy < p->tol2 || uy2 < p->tol2)) break;
  }
  r->admm_steps = steps;
  r->U = U2;
  r->F = F2;
  r->t_total = now_s() - t0;
  free(f); free(g); free(dfdx); free(dfdy); free(sx); free(coords); free(ug); free(vg);
  free(U0); free(U1); free(F1); free(H21); free(udual); free(vdual); free(U2old);
  free(U1old); free(itb);
  return 0;
}

void orc_frame_free(orc_frame_result *r) {
  free(r->x0); free(r->y0); free(r->U); free(r->F); free(r->U_icgn); free(r->F_icgn);
  free(r->iters_icgn);
  memset(r, 0, sizeof(*r));
}
