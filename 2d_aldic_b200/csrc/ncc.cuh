// ncc.cuh -- normalised cross-correlation from exact partial sums and the
// findpeak.m sub-pixel fit, shared by the whole-field search (k_search.cu)
// and the multigrid search (k_searchmg.cu).  The FP64 operation order is the
// CPU restatement's, so argmax and the 1e-3-rounded peaks are bit-identical
// to it wherever the partial sums are.
#pragma once
#include <cuda_runtime.h>

namespace aldic {

constexpr double kSqrtEps = 1.4901161193847656e-08;  // sqrt(DBL_EPSILON) = 2^-26

// Numerator and window part of the denominator of one cropped-map entry:
// the template is correlated with the window whose n_pad pixels beyond the
// search region read as mu (the mean the padding stands for).
__device__ __forceinline__ void ncc_parts(long long mn, long long st, long long stdv,
                                          long long sd, long long sd2, long long st_pad,
                                          long long n_pad, double mu, double *num, double *den) {
  const double A = (double)(mn * stdv - st * sd);
  const double C0 = (double)(mn * sd2 - sd * sd);
  double B = 0.0, Cc = 0.0;
  if (n_pad > 0) {
    B = __dmul_rn(mu, (double)(mn * st_pad - st * n_pad));
    Cc = __dmul_rn(mu, __dsub_rn(__dmul_rn((double)(n_pad * (mn - n_pad)), mu),
                                 __dmul_rn(2.0, (double)(sd * n_pad))));
  }
  *num = __dadd_rn(A, B);
  *den = __dadd_rn(C0, Cc);
}

// NCC at one cropped-map entry from the exact partial sums (same arithmetic
// as the CPU restatement's ncc_at).
__device__ __forceinline__ double ncc_combine(long long mn, long long st, long long st2,
                                              long long stdv, long long sd, long long sd2,
                                              long long st_pad, long long n_pad, double mu) {
  const double denT = (double)(mn * st2 - st * st);
  double num, den;
  ncc_parts(mn, st, stdv, sd, sd2, st_pad, n_pad, mu, &num, &den);
  if (!(den > 0.0)) return 0.0;
  double r = __ddiv_rn(num, __dsqrt_rn(__dmul_rn(denT, den)));
  if (__dsub_rn(fabs(r), 1.0) > kSqrtEps) r = 0.0;
  return r;
}

__device__ __forceinline__ double ncc_combine_f(double mn, double st, double st2, double stdv,
                                                double sd, double sd2, double st_pad,
                                                double n_pad, double mu) {
  const double denT = mn * st2 - st * st;
  const double A = mn * stdv - st * sd;
  const double C0 = mn * sd2 - sd * sd;
  double B = 0.0, Cc = 0.0;
  if (n_pad > 0) {
    B = mu * (mn * st_pad - st * n_pad);
    Cc = mu * ((n_pad * (mn - n_pad)) * mu - 2.0 * (sd * n_pad));
  }
  const double num = A + B, den = C0 + Cc;
  if (!(den > 0.0)) return 0.0;
  double r = num / sqrt(denT * den);
  if (fabs(r) - 1.0 > kSqrtEps) r = 0.0;
  return r;
}

// The same combination with 128-bit integer products, for templates large
// enough that mn * sum(d^2) leaves the 64-bit range (the multigrid levels);
// identical to ncc_combine wherever that one does not overflow.
__device__ __forceinline__ double ncc_combine_wide(long long mn, long long st, long long st2,
                                                   long long stdv, long long sd, long long sd2,
                                                   long long st_pad, long long n_pad, double mu) {
  typedef __int128 W;
  const double denT = (double)((W)mn * st2 - (W)st * st);
  const double A = (double)((W)mn * stdv - (W)st * sd);
  const double C0 = (double)((W)mn * sd2 - (W)sd * sd);
  double B = 0.0, Cc = 0.0;
  if (n_pad > 0) {
    B = __dmul_rn(mu, (double)((W)mn * st_pad - (W)st * n_pad));
    Cc = __dmul_rn(mu, __dsub_rn(__dmul_rn((double)((W)n_pad * (mn - n_pad)), mu),
                                 __dmul_rn(2.0, (double)((W)sd * n_pad))));
  }
  const double num = __dadd_rn(A, B);
  const double den = __dadd_rn(C0, Cc);
  if (!(den > 0.0)) return 0.0;
  double r = __ddiv_rn(num, __dsqrt_rn(__dmul_rn(denT, den)));
  if (__dsub_rn(fabs(r), 1.0) > kSqrtEps) r = 0.0;
  return r;
}

// findpeak.m:27-66 with the closed-form 3x3 quadratic fit (same operation
// order as the CPU restatement).  u holds the 3x3 neighbourhood of the
// maximum (r, c) (0-based, not on the map edge) as u[(dc + 1) * 3 + dr + 1];
// on return the 1-based peak row/column and the fitted value (unchanged when
// the fitted offset leaves the cell).
__device__ __forceinline__ void findpeak_fit9(const double u9[9], int r, int c, double *row_pk,
                                              double *col_pk, double *max_f) {
  double s0 = 0, sxu = 0, syu = 0, sxyu = 0, sxxu = 0, syyu = 0;
  for (int dc = -1; dc <= 1; ++dc)
    for (int dr = -1; dr <= 1; ++dr) {
      const double u = u9[(dc + 1) * 3 + dr + 1];
      s0 = __dadd_rn(s0, u);
      sxu = __dadd_rn(sxu, __dmul_rn((double)dc, u));
      syu = __dadd_rn(syu, __dmul_rn((double)dr, u));
      sxyu = __dadd_rn(sxyu, __dmul_rn((double)(dc * dr), u));
      sxxu = __dadd_rn(sxxu, __dmul_rn((double)(dc * dc), u));
      syyu = __dadd_rn(syyu, __dmul_rn((double)(dr * dr), u));
    }
  const double A2 = __ddiv_rn(sxu, 6.0), A3 = __ddiv_rn(syu, 6.0), A4 = __ddiv_rn(sxyu, 4.0);
  const double p = __dsub_rn(__dmul_rn(0.5, __dadd_rn(sxxu, syyu)), __dmul_rn(2.0 / 3.0, s0));
  const double q = __dmul_rn(0.5, __dsub_rn(sxxu, syyu));
  const double A5 = __dmul_rn(0.5, __dadd_rn(p, q)), A6 = __dmul_rn(0.5, __dsub_rn(p, q));
  const double A1 = __ddiv_rn(__dsub_rn(s0, __dmul_rn(6.0, p)), 9.0);
  const double den = __dsub_rn(__dmul_rn(A4, A4), __dmul_rn(__dmul_rn(4.0, A5), A6));
  double xo = __ddiv_rn(__dadd_rn(__dmul_rn(-A3, A4), __dmul_rn(__dmul_rn(2.0, A6), A2)), den);
  double yo = __dmul_rn(__ddiv_rn(-1.0, den),
                        __dsub_rn(__dmul_rn(A4, A2), __dmul_rn(__dmul_rn(2.0, A5), A3)));
  if (fabs(xo) > 1.0 || fabs(yo) > 1.0) return;
  xo = __ddiv_rn(round(__dmul_rn(1000.0, xo)), 1000.0);
  yo = __ddiv_rn(round(__dmul_rn(1000.0, yo)), 1000.0);
  *col_pk = __dadd_rn((double)(c + 1), xo);
  *row_pk = __dadd_rn((double)(r + 1), yo);
  double m = __dadd_rn(A1, __dmul_rn(A2, xo));
  m = __dadd_rn(m, __dmul_rn(A3, yo));
  m = __dadd_rn(m, __dmul_rn(A4, __dmul_rn(xo, yo)));
  m = __dadd_rn(m, __dmul_rn(A5, __dmul_rn(xo, xo)));
  m = __dadd_rn(m, __dmul_rn(A6, __dmul_rn(yo, yo)));
  *max_f = m;
}

// findpeak on an nr x nc column-major map whose maximum is at index im.
__device__ __forceinline__ void findpeak_fit(const double *map, int nr, int nc, int im,
                                             double *row_pk, double *col_pk, double *max_f) {
  const int r = im % nr, c = im / nr;
  *row_pk = r + 1;
  *col_pk = c + 1;
  *max_f = map[im];
  if (r == 0 || r == nr - 1 || c == 0 || c == nc - 1) return;
  double u9[9];
  for (int dc = -1; dc <= 1; ++dc)
    for (int dr = -1; dr <= 1; ++dr) u9[(dc + 1) * 3 + dr + 1] = map[(c + dc) * nr + (r + dr)];
  findpeak_fit9(u9, r, c, row_pk, col_pk, max_f);
}

}  // namespace aldic
