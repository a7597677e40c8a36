// k_searchmg.cu -- multigrid integer search (func/funIntegerSearchMg.m), the
// search IntegerSearch.m:117-120 runs when InitFFTSearchMethod is neither 1
// nor 2: one global shift from the whole ROI, then regions split level by
// level down to the subset size, each refined within +-5 px of its parent's
// shift, and the last level's displacements fitted onto the node grid.
//
// Device side:
//   * summed-area tables of f, f^2, g, g^2 (exact 64-bit for integer images)
//     give every window sum of the normalised cross-correlation in O(1);
//   * level 1: normxcorr2 of the whole f ROI against the g ROI for every
//     shift by an FP64 FFT cross-correlation (own radix-2 kernels: rows in
//     shared memory, tiled transposes; the two real transforms packed into
//     one complex one), then an argmax reduction and findpeak's 3x3 fit;
//   * intermediate levels: the 13 x 14 cropped map of every region from
//     exact integer products -- CTAs over (region, 8-row band, 256-column
//     tile), each thread a register window over 13 horizontal shifts;
//   * last level: the full (2a+9) x (2b+9) map of every region in shared
//     memory (for compute_qFactor), with register-blocked strips of 8 shifts.
// Host side: the region bookkeeping of funIntegerSearchMg.m (splits, border
// clamps, even widths, NaN propagation) and the gridfit 'springs' normal
// equations of the scattered last-level data, solved by the CSR PCG.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <type_traits>
#include <vector>

#include "aldic_internal.cuh"
#include "kernels.cuh"
#include "ncc.cuh"

namespace aldic {

namespace {

constexpr int kCropR = 13, kCropC = 14, kCrop = kCropR * kCropC;  // 13 x 14 crop
constexpr int kBand = 8, kSegs = 16;                               // intermediate levels
constexpr int kStrip = 8;                                          // last level
constexpr int kMaxFinal = 80;  // largest last-level region side (about winsize + 1)
constexpr int kMaxFFT = 8192;  // largest FFT length (ROI up to 4096 px per side)

template <typename P> struct MgT;
template <> struct MgT<uint8_t> {
  using S = long long;       // window sums
  using V = unsigned int;    // shared-memory pixel
  using A = unsigned int;    // per-thread product sums (<= 16 * 8 * 255^2)
  using G = unsigned long long;
  static constexpr bool integer = true;
};
template <> struct MgT<uint16_t> {
  using S = long long;
  using V = unsigned int;
  using A = unsigned long long;
  using G = unsigned long long;
  static constexpr bool integer = true;
};
template <> struct MgT<float> {
  using S = double;
  using V = double;
  using A = double;
  using G = double;
  static constexpr bool integer = false;
};
template <> struct MgT<double> : MgT<float> {};

struct MgReg {
  int tx, ty, a, b;  // template f(tx : tx+a-1, ty : ty+b-1), 1-based
  int dx, dy;        // region g(dx : dx+a+9, dy : dy+b+9), 1-based
  int valid;
  int pad;
};

// rectangle sum of a (W+1) x (H+1) summed-area table over 0-based pixels
// [x0, x1) x [y0, y1)
template <typename S>
__device__ __forceinline__ S rect_sum(const S *__restrict__ sat, int W1, int x0, int x1, int y0,
                                      int y1) {
  return sat[(long long)y1 * W1 + x1] - sat[(long long)y0 * W1 + x1] -
         sat[(long long)y1 * W1 + x0] + sat[(long long)y0 * W1 + x0];
}

template <typename S>
__device__ __forceinline__ double combine(long long mn, S st, S st2, S stdv, S sd, S sd2, S st_pad,
                                          long long n_pad, double mu) {
  if constexpr (std::is_integral<S>::value) {
    return ncc_combine_wide(mn, (long long)st, (long long)st2, (long long)stdv, (long long)sd,
                            (long long)sd2, (long long)st_pad, n_pad, mu);
  } else {
    return ncc_combine_f((double)mn, (double)st, (double)st2, (double)stdv, (double)sd,
                         (double)sd2, (double)st_pad, (double)n_pad, mu);
  }
}

// ------------------------------------------------------------ summed-area tables
// sat[0..3] = f, f^2, g, g^2, each (W+1) x (H+1), row 0 and column 0 zero.
// Pass 1: one block per image row, block-wide scan along x.
template <typename P>
__global__ void k_sat_rows(const P *__restrict__ f, const P *__restrict__ g, int W, int H,
                           typename MgT<P>::S *__restrict__ sat) {
  using S = typename MgT<P>::S;
  const int y = blockIdx.x;  // image row -> table row y + 1
  const int q = blockIdx.y;  // 0 f, 1 f^2, 2 g, 3 g^2
  const P *img = q < 2 ? f : g;
  const bool sq = q & 1;
  const long long W1 = W + 1, plane = W1 * (H + 1);
  S *row = sat + q * plane + (long long)(y + 1) * W1;
  __shared__ S wsum[32];
  __shared__ S carry;
  if (threadIdx.x == 0) {
    carry = 0;
    row[0] = 0;
    if (y == 0) sat[q * plane] = 0;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int x0 = 0; x0 < W; x0 += blockDim.x) {
    const int x = x0 + threadIdx.x;
    S v = 0;
    if (x < W) {
      const S p = (S)img[(long long)y * W + x];
      v = sq ? p * p : p;
    }
    for (int o = 1; o < 32; o <<= 1) {
      const S t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) wsum[wid] = v;
    __syncthreads();
    if (wid == 0) {
      S t = lane < nw ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const S u = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += u;
      }
      if (lane < nw) wsum[lane] = t;
    }
    __syncthreads();
    const S base = carry + (wid ? wsum[wid - 1] : 0);
    if (x < W) row[x + 1] = base + v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = base + v;
    __syncthreads();
  }
  // first table row (zeros) for columns > 0
  if (y == 0)
    for (int x = threadIdx.x; x < W; x += blockDim.x) sat[q * plane + x + 1] = 0;
}

// Pass 2: columns, in chunks of rows: scan each chunk, then add the totals
// of the chunks above.
constexpr int kSatChunk = 64;
template <typename S>
__global__ void k_sat_cols_chunk(S *__restrict__ sat, int W, int H, S *__restrict__ tot) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.z, ch = blockIdx.y;
  const long long W1 = W + 1, plane = W1 * (H + 1);
  if (x > W) return;
  S *p = sat + q * plane;
  const int y0 = 1 + ch * kSatChunk, y1 = min(H + 1, y0 + kSatChunk);
  S acc = 0;
  for (int y = y0; y < y1; ++y) {
    acc += p[(long long)y * W1 + x];
    p[(long long)y * W1 + x] = acc;
  }
  tot[((long long)q * gridDim.y + ch) * W1 + x] = acc;
}
template <typename S>
__global__ void k_sat_cols_fix(S *__restrict__ sat, int W, int H, const S *__restrict__ tot) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.z, ch = blockIdx.y;
  const long long W1 = W + 1, plane = W1 * (H + 1);
  if (x > W || ch == 0) return;
  S off = 0;
  for (int c = 0; c < ch; ++c) off += tot[((long long)q * gridDim.y + c) * W1 + x];
  S *p = sat + q * plane;
  const int y0 = 1 + ch * kSatChunk, y1 = min(H + 1, y0 + kSatChunk);
  for (int y = y0; y < y1; ++y) p[(long long)y * W1 + x] += off;
}

// ------------------------------------------------------------ FFT (FP64)
// Stockham autosort transform of one row in shared memory: passes of radix
// 8 (a radix-2 or radix-4 pass first when log2 L is not a multiple of 3),
// each thread loading R values L/R apart, twiddling, an R-point DFT in
// registers and writing them Ns apart -- natural order in and out, no
// bit reversal.  Twiddles come from a table of exp(-2 pi i t / L).
__global__ void k_fft_twiddle(double2 *tw, int L) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L) return;
  double s, c;
  sincospi(2.0 * (double)k / (double)L, &s, &c);
  tw[k] = make_double2(c, -s);  // exp(-2 pi i k / L)
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// times -i (forward) or +i (inverse)
__device__ __forceinline__ double2 cmi(double2 a, bool inv) {
  return inv ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <int R>
__device__ __forceinline__ void dft_reg(double2 *a, bool inv) {
  if constexpr (R == 2) {
    const double2 t = a[0];
    a[0] = cadd(t, a[1]);
    a[1] = csub(t, a[1]);
  } else if constexpr (R == 4) {
    const double2 c0 = cadd(a[0], a[2]), c2 = csub(a[0], a[2]);
    const double2 c1 = cadd(a[1], a[3]), c3 = cmi(csub(a[1], a[3]), inv);
    a[0] = cadd(c0, c1);
    a[2] = csub(c0, c1);
    a[1] = cadd(c2, c3);
    a[3] = csub(c2, c3);
  } else {
    constexpr double h = 0.70710678118654752440;
    // decimation in frequency: sums feed the even outputs, twiddled
    // differences the odd ones
    const double2 b0 = cadd(a[0], a[4]), b1 = cadd(a[1], a[5]), b2 = cadd(a[2], a[6]),
                  b3 = cadd(a[3], a[7]);
    const double2 d1 = csub(a[1], a[5]), d3 = csub(a[3], a[7]);
    const double2 b4 = csub(a[0], a[4]);
    const double2 b6 = cmi(csub(a[2], a[6]), inv);
    // W8 = (1 - i)/sqrt2, W8^3 = (-1 - i)/sqrt2 (conjugates for the inverse)
    const double2 b5 = inv ? make_double2(h * (d1.x - d1.y), h * (d1.x + d1.y))
                           : make_double2(h * (d1.x + d1.y), h * (d1.y - d1.x));
    const double2 b7 = inv ? make_double2(-h * (d3.x + d3.y), h * (d3.x - d3.y))
                           : make_double2(h * (d3.y - d3.x), -h * (d3.x + d3.y));
    const double2 c0 = cadd(b0, b2), c2 = csub(b0, b2), c1 = cadd(b1, b3), c3 = cmi(csub(b1, b3), inv);
    const double2 c4 = cadd(b4, b6), c6 = csub(b4, b6), c5 = cadd(b5, b7), c7 = cmi(csub(b5, b7), inv);
    a[0] = cadd(c0, c1);
    a[4] = csub(c0, c1);
    a[2] = cadd(c2, c3);
    a[6] = csub(c2, c3);
    a[1] = cadd(c4, c5);
    a[5] = csub(c4, c5);
    a[3] = cadd(c6, c7);
    a[7] = csub(c6, c7);
  }
}

// index groups per thread in a radix-R pass: every value of an 8192-point
// row is held in registers by the 512 threads between read and write
template <int R> struct FftJ { static constexpr int J = kMaxFFT / (R * 512); };

template <int R>
__device__ void stockham_pass(double2 *s, int L, int Ns, const double2 *__restrict__ tw, bool inv) {
  constexpr int kFftJ = FftJ<R>::J;
  const int nj = L / R, tstep = L / (Ns * R);
  double2 v[kFftJ][R];
#pragma unroll
  for (int t = 0; t < kFftJ; ++t) {
    const int j = threadIdx.x + t * blockDim.x;
    if (j < nj) {
#pragma unroll
      for (int q = 0; q < R; ++q) v[t][q] = s[j + q * nj];
    }
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < kFftJ; ++t) {
    const int j = threadIdx.x + t * blockDim.x;
    if (j < nj) {
      const int k = j % Ns;
#pragma unroll
      for (int q = 1; q < R; ++q) {
        double2 w = __ldg(&tw[k * q * tstep]);
        if (inv) w.y = -w.y;
        v[t][q] = cmul(v[t][q], w);
      }
      dft_reg<R>(v[t], inv);
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int q = 0; q < R; ++q) s[base + q * Ns] = v[t][q];
    }
  }
  __syncthreads();
}

// the whole row: s[0..L) in natural order, L = 2^logL <= 8192
__device__ void fft_smem(double2 *s, int L, int logL, const double2 *__restrict__ tw, bool inv) {
  int Ns = 1;
  const int rem = logL % 3;
  if (rem == 1) { stockham_pass<2>(s, L, Ns, tw, inv); Ns *= 2; }
  else if (rem == 2) { stockham_pass<4>(s, L, Ns, tw, inv); Ns *= 4; }
  while (Ns < L) { stockham_pass<8>(s, L, Ns, tw, inv); Ns *= 8; }
}

// Level-1 forward row transforms with the packing fused: row y < b holds
// z(x) = (f - mean f) + i (g - mu) over the ROI, zero beyond; rows >= b are
// zero (their transform too).
template <typename P>
__global__ void __launch_bounds__(512) k_fft_pack_rows(const P *__restrict__ f, const P *__restrict__ g, int W, int H,
                                int x1, int y1, int a, int b, const typename MgT<P>::S *__restrict__ sat,
                                const double *__restrict__ mu_g, double2 *__restrict__ Z, int L,
                                int logL, const double2 *__restrict__ tw) {
  extern __shared__ double2 s[];
  const int y = blockIdx.x;
  double2 *row = Z + (long long)y * L;
  if (y >= b) {
    for (int x = threadIdx.x; x < L; x += blockDim.x) row[x] = make_double2(0.0, 0.0);
    return;
  }
  const long long W1 = W + 1;
  const double st = (double)rect_sum(sat, (int)W1, x1 - 1, x1 - 1 + a, y1 - 1, y1 - 1 + b);
  const double mean_t = st / ((double)a * (double)b);
  const double mu = *mu_g;
  for (int x = threadIdx.x; x < L; x += blockDim.x) {
    double2 z = make_double2(0.0, 0.0);
    if (x < a) {
      const long long o = (long long)(y1 - 1 + y) * W + (x1 - 1 + x);
      z = make_double2((double)f[o] - mean_t, (double)g[o] - mu);
    }
    s[x] = z;
  }
  __syncthreads();
  fft_smem(s, L, logL, tw, false);
  for (int x = threadIdx.x; x < L; x += blockDim.x) row[x] = s[x];
}

template <bool INV>
__global__ void __launch_bounds__(512) k_fft_rows(double2 *__restrict__ Z, int L, int logL,
                                                  const double2 *__restrict__ tw, int row0, int row1) {
  extern __shared__ double2 s[];
  const int y = blockIdx.x;
  if (y >= row0 && y < row1) return;  // rows nobody reads
  double2 *row = Z + (long long)y * L;
  for (int x = threadIdx.x; x < L; x += blockDim.x) s[x] = row[x];
  __syncthreads();
  fft_smem(s, L, logL, tw, INV);
  for (int x = threadIdx.x; x < L; x += blockDim.x) row[x] = s[x];
}

// out (C x R) = in (R x C)^T
__global__ void k_transpose_c(const double2 *__restrict__ in, double2 *__restrict__ out, int R,
                              int Cn) {
  __shared__ double2 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < R && c < Cn) t[k][threadIdx.x] = in[(long long)r * Cn + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < R && c < Cn) out[(long long)c * R + r] = t[threadIdx.x][k];
  }
}

// Spectrum of the correlation: with Z = F + i G (F, G transforms of the two
// real inputs), F(k) = (Z(k) + conj Z(-k)) / 2, G(k) = (Z(k) - conj Z(-k)) / 2i,
// and sum_p t(p) d(p + s) has the transform conj(F) G.  Z is [kx][ky].
__global__ void k_mg_spectrum(const double2 *__restrict__ Z, double2 *__restrict__ Cs, int P1,
                              int P2) {
  const long long n = (long long)P1 * P2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(e / P2), ky = (int)(e - (long long)kx * P2);
    const long long m = (long long)((P1 - kx) & (P1 - 1)) * P2 + ((P2 - ky) & (P2 - 1));
    const double2 z = Z[e], w = Z[m];
    const double2 F = make_double2(0.5 * (z.x + w.x), 0.5 * (z.y - w.y));
    const double2 Gm = make_double2(z.x - w.x, z.y + w.y);  // Z(k) - conj Z(-k)
    const double2 G = make_double2(0.5 * Gm.y, -0.5 * Gm.x);
    Cs[e] = make_double2(F.x * G.x + F.y * G.y, F.x * G.y - F.y * G.x);
  }
}

// Level-1 normalised cross-correlation at map entry e of the (2a-1) x (2b-1)
// map (column-major, rows = x shifts): D offset (ox, oy) of the template.
template <bool INT, typename S>
struct L1Args {
  const S *sat;          // g, g^2 planes used
  int W1, gx0, gy0;      // table row length, 0-based ROI origin
  int a, b;
  long long mn;
  S st, st2;             // template sums
  const double2 *c;      // [oy][ox] cyclic correlation, unscaled
  int P1, P2;
  double inv;            // 1 / (P1 P2)
  double mu;
};

template <bool INT, typename S>
__device__ double l1_ncc(const L1Args<INT, S> &A, const S *satg, const S *satg2, long long e) {
  const int nr = 2 * A.a - 1;
  const int i = (int)(e % nr), j = (int)(e / nr);
  const int ox = i - (A.a - 1), oy = j - (A.b - 1);
  const int x0 = max(0, ox), x1 = min(A.a, A.a + ox), y0 = max(0, oy), y1 = min(A.b, A.b + oy);
  if (x1 <= x0 || y1 <= y0) return 0.0;
  const long long n_in = (long long)(x1 - x0) * (y1 - y0), n_pad = A.mn - n_in;
  const S sd = rect_sum(satg, A.W1, A.gx0 + x0, A.gx0 + x1, A.gy0 + y0, A.gy0 + y1);
  const S sd2 = rect_sum(satg2, A.W1, A.gx0 + x0, A.gx0 + x1, A.gy0 + y0, A.gy0 + y1);
  const double cv = A.c[(long long)(oy & (A.P2 - 1)) * A.P1 + (ox & (A.P1 - 1))].x * A.inv;
  const double num = (double)A.mn * cv;
  double denT, C0, Cc = 0.0;
  if constexpr (INT) {
    typedef __int128 Wd;
    denT = (double)((Wd)A.mn * (long long)A.st2 - (Wd)(long long)A.st * (long long)A.st);
    C0 = (double)((Wd)A.mn * (long long)sd2 - (Wd)(long long)sd * (long long)sd);
    if (n_pad > 0)
      Cc = A.mu * ((double)((Wd)n_pad * (A.mn - n_pad)) * A.mu - 2.0 * (double)((Wd)(long long)sd * n_pad));
  } else {
    denT = (double)A.mn * (double)A.st2 - (double)A.st * (double)A.st;
    C0 = (double)A.mn * (double)sd2 - (double)sd * (double)sd;
    if (n_pad > 0)
      Cc = A.mu * ((double)n_pad * (double)(A.mn - n_pad) * A.mu - 2.0 * ((double)sd * (double)n_pad));
  }
  const double den = C0 + Cc;
  if (!(den > 0.0)) return 0.0;
  double r = num / sqrt(denT * den);
  if (fabs(r) - 1.0 > kSqrtEps) r = 0.0;
  return r;
}

__device__ __forceinline__ void argmax_merge(double &bv, long long &bi, double v, long long i) {
  if (v > bv || (v == bv && i < bi)) {
    bv = v;
    bi = i;
  }
}

template <bool INT, typename S>
__global__ void k_mg_l1_argmax(L1Args<INT, S> A, const S *__restrict__ satg,
                               const S *__restrict__ satg2, double *__restrict__ pv,
                               long long *__restrict__ pi) {
  const long long nm = (long long)(2 * A.a - 1) * (2 * A.b - 1);
  double bv = -1e300;
  long long bi = 0x7fffffffffffffffll;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nm;
       e += (long long)gridDim.x * blockDim.x)
    argmax_merge(bv, bi, l1_ncc(A, satg, satg2, e), e);
  for (int o = 16; o > 0; o >>= 1)
    argmax_merge(bv, bi, __shfl_xor_sync(0xffffffffu, bv, o), __shfl_xor_sync(0xffffffffu, bi, o));
  __shared__ double sv[32];
  __shared__ long long si[32];
  if ((threadIdx.x & 31) == 0) {
    sv[threadIdx.x >> 5] = bv;
    si[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) argmax_merge(bv, bi, sv[k], si[k]);
    pv[blockIdx.x] = bv;
    pi[blockIdx.x] = bi;
  }
}

// out = {row, col, max_f} of findpeak over the level-1 map
template <bool INT, typename S>
__global__ void k_mg_l1_peak(L1Args<INT, S> A, const S *__restrict__ satg,
                             const S *__restrict__ satg2, const double *__restrict__ pv,
                             const long long *__restrict__ pi, int np, double *__restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double bv = -1e300;
  long long bi = 0x7fffffffffffffffll;
  for (int k = 0; k < np; ++k) argmax_merge(bv, bi, pv[k], pi[k]);
  const int nr = 2 * A.a - 1, nc = 2 * A.b - 1;
  const int r = (int)(bi % nr), c = (int)(bi / nr);
  double rp = r + 1, cp = c + 1, mf = bv;
  if (!(r == 0 || r == nr - 1 || c == 0 || c == nc - 1)) {
    double u9[9];
    for (int dc = -1; dc <= 1; ++dc)
      for (int dr = -1; dr <= 1; ++dr)
        u9[(dc + 1) * 3 + dr + 1] = l1_ncc(A, satg, satg2, (long long)(c + dc) * nr + (r + dr));
    findpeak_fit9(u9, r, c, &rp, &cp, &mf);
  }
  out[0] = rp;
  out[1] = cp;
  out[2] = mf;
}

// ------------------------------------------------------------ intermediate levels
// Exact sum of t * d over one (region, 8-row band, 256-column tile) for the
// 13 x 14 shifts of the crop, added into acc[region][182] (column-major,
// rows = ox + 1, ox in [-1, 11]; columns oy + 1, oy in [-1, 12]).  D pixels
// outside the region read 0 (their padding is the mu term of the NCC).
// Column segment per thread: 16 columns (8 for FP64 pixels, to keep the
// static shared memory of the tile under 48 KB); 16 segments per tile.
template <typename P> struct CropCfg {
  static constexpr int SW = sizeof(typename MgT<P>::V) == 8 ? 8 : 16;
  static constexpr int TILE = kSegs * SW;
};

template <typename P>
__global__ void __launch_bounds__(224) k_mg_crop(const P *__restrict__ f, const P *__restrict__ g,
                                                 int W, const MgReg *__restrict__ regs,
                                                 typename MgT<P>::G *__restrict__ acc) {
  using V = typename MgT<P>::V;
  using A = typename MgT<P>::A;
  using G = typename MgT<P>::G;
  constexpr int kTile = CropCfg<P>::TILE, kSeg = CropCfg<P>::SW;
  constexpr int TS = kTile + 4;             // template row stride
  constexpr int DS = kTile + 16 + 4;        // region row stride (tile + 12 halo, padded)
  constexpr int DR = kBand + kCropC - 1;    // region rows: band + 13
  __shared__ V Ts[kBand][TS];
  __shared__ V Ds[DR][DS];
  const MgReg R = regs[blockIdx.x];
  if (!R.valid) return;
  const int q0 = blockIdx.y * kBand, x0 = blockIdx.z * kTile;
  if (q0 >= R.b || x0 >= R.a) return;
  const int nq = min(kBand, R.b - q0), nx = min(kTile, R.a - x0);
  const int dwid = R.a + 10, dhgt = R.b + 10;
  for (int e = threadIdx.x; e < kBand * kTile; e += blockDim.x) {
    const int qq = e / kTile, xx = e - qq * kTile;
    V t = 0;
    if (qq < nq && xx < nx)
      t = (V)f[(long long)(R.ty - 1 + q0 + qq) * W + (R.tx - 1 + x0 + xx)];
    Ts[qq][xx] = t;
  }
  for (int e = threadIdx.x; e < DR * (kTile + 16); e += blockDim.x) {
    const int r = e / (kTile + 16), cidx = e - r * (kTile + 16);
    const int yl = q0 - 1 + r, xl = x0 - 1 + cidx;  // region-local
    V d = 0;
    if (yl >= 0 && yl < dhgt && xl >= 0 && xl < dwid && cidx < nx + 12)
      d = (V)g[(long long)(R.dy - 1 + yl) * W + (R.dx - 1 + xl)];
    Ds[r][cidx] = d;
  }
  __syncthreads();
  const int oyi = threadIdx.x / kSegs, seg = threadIdx.x - oyi * kSegs;  // oy = oyi - 1
  const int xs = seg * kSeg;
  A s[kCropR];
#pragma unroll
  for (int k = 0; k < kCropR; ++k) s[k] = 0;
  if (xs < nx) {
    for (int qq = 0; qq < nq; ++qq) {
      const V *dr = &Ds[qq + oyi][xs];  // region row q0 + qq + oy
      const V *tr = &Ts[qq][xs];
      V win[kSeg + kCropR - 1];
#pragma unroll
      for (int k = 0; k < kSeg + kCropR - 1; ++k) win[k] = dr[k];
#pragma unroll
      for (int xx = 0; xx < kSeg; ++xx) {
        const A t = (A)tr[xx];
#pragma unroll
        for (int k = 0; k < kCropR; ++k) s[k] += t * (A)win[xx + k];
      }
    }
  }
  // reduce over the 16 column segments of the same oy (consecutive lanes)
#pragma unroll
  for (int k = 0; k < kCropR; ++k) {
    G v = (G)s[k];
#pragma unroll
    for (int o = kSegs / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, kSegs);
    if (seg == 0 && v != G(0)) atomicAdd(&acc[(long long)blockIdx.x * kCrop + oyi * kCropR + k], v);
  }
}

// NCC of the 182 crop entries from the products and the window sums, then
// findpeak: res[region] = {u offset, v offset, Phi, ok}.
template <typename P>
__global__ void k_mg_crop_peak(const MgReg *__restrict__ regs, int W, int H,
                               const typename MgT<P>::S *__restrict__ sat,
                               const typename MgT<P>::G *__restrict__ acc,
                               const double *__restrict__ mu_g, double *__restrict__ res) {
  using S = typename MgT<P>::S;
  __shared__ double map[kCrop];
  __shared__ int s_flat;
  const MgReg R = regs[blockIdx.x];
  double *o = res + (long long)blockIdx.x * 8;
  if (!R.valid) {
    if (threadIdx.x == 0) o[3] = 0.0;
    return;
  }
  const int W1 = W + 1;
  const long long plane = (long long)W1 * (H + 1);
  const S *sf = sat, *sf2 = sat + plane, *sg = sat + 2 * plane, *sg2 = sat + 3 * plane;
  const long long mn = (long long)R.a * R.b;
  const int tx0i = R.tx - 1, ty0i = R.ty - 1, dx0i = R.dx - 1, dy0i = R.dy - 1;
  const S st = rect_sum(sf, W1, tx0i, tx0i + R.a, ty0i, ty0i + R.b);
  const S st2 = rect_sum(sf2, W1, tx0i, tx0i + R.a, ty0i, ty0i + R.b);
  if (threadIdx.x == 0) {
    bool flat;
    if constexpr (MgT<P>::integer)
      flat = ((__int128)mn * (long long)st2 - (__int128)(long long)st * (long long)st) == 0;
    else
      flat = !((double)mn * (double)st2 - (double)st * (double)st > 0.0);
    s_flat = flat;
  }
  const double mu = *mu_g;
  for (int e = threadIdx.x; e < kCrop; e += blockDim.x) {
    const int ox = e % kCropR - 1, oy = e / kCropR - 1;
    const int tx0 = max(0, -ox), tx1 = min(R.a, R.a + 10 - ox);
    const int ty0 = max(0, -oy), ty1 = min(R.b, R.b + 10 - oy);
    double r = 0.0;
    if (tx1 > tx0 && ty1 > ty0) {
      const long long n_in = (long long)(tx1 - tx0) * (ty1 - ty0);
      const S st_in = rect_sum(sf, W1, tx0i + tx0, tx0i + tx1, ty0i + ty0, ty0i + ty1);
      const S sd = rect_sum(sg, W1, dx0i + tx0 + ox, dx0i + tx1 + ox, dy0i + ty0 + oy, dy0i + ty1 + oy);
      const S sd2 = rect_sum(sg2, W1, dx0i + tx0 + ox, dx0i + tx1 + ox, dy0i + ty0 + oy, dy0i + ty1 + oy);
      const S stdv = (S)acc[(long long)blockIdx.x * kCrop + e];
      r = combine<S>(mn, st, st2, stdv, sd, sd2, st - st_in, mn - n_in, mu);
    }
    map[e] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (s_flat) {
      o[3] = 0.0;
      return;
    }
    int im = 0;
    double mv = map[0];
    for (int e = 1; e < kCrop; ++e)
      if (map[e] > mv) {
        mv = map[e];
        im = e;
      }
    double rp, cp, mf;
    findpeak_fit(map, kCropR, kCropC, im, &rp, &cp, &mf);
    o[0] = __dsub_rn(rp, 7.0);
    o[1] = __dsub_rn(cp, 7.0);
    o[2] = mf;
    o[3] = 1.0;
  }
}

// ------------------------------------------------------------ last level
// One CTA per region: the full normxcorr2 map (2a+9) x (2b+9) in shared
// memory, compute_qFactor over it, findpeak on its 13 x 14 crop.
// res[region] = {u offset, v offset, Phi, ok, PCE, 1/entropy}.
template <typename P>
__global__ void __launch_bounds__(256) k_mg_full(const P *__restrict__ f, const P *__restrict__ g,
                                                 int W, int H, const MgReg *__restrict__ regs,
                                                 const typename MgT<P>::S *__restrict__ sat,
                                                 const double *__restrict__ mu_g,
                                                 double *__restrict__ res) {
  using S = typename MgT<P>::S;
  using V = typename MgT<P>::V;
  using A = typename MgT<P>::A;  // u8: <= 80 * 80 * 255^2 < 2^32
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[64];
  __shared__ int hist[30];
  __shared__ double crop[kCrop];
  const MgReg R = regs[blockIdx.x];
  double *o = res + (long long)blockIdx.x * 8;
  if (!R.valid) {
    if (threadIdx.x == 0) o[3] = 0.0;
    return;
  }
  const int a = R.a, b = R.b, dw = a + 10, dh = b + 10;
  const int fr = a + dw - 1, fc = b + dh - 1, nm = fr * fc;
  // template rows padded with 8 zero columns, region rows with kStrip zero
  // columns on the left and kStrip + 8 on the right
  const int TP = a + 8, DP = dw + 2 * kStrip + 8;
  double *map = (double *)smem;
  V *Ts = (V *)(map + nm);
  V *Ds = Ts + TP * b;
  for (int e = threadIdx.x; e < TP * b; e += blockDim.x) {
    const int ty = e / TP, tx = e - ty * TP;
    Ts[e] = tx < a ? (V)f[(long long)(R.ty - 1 + ty) * W + (R.tx - 1 + tx)] : (V)0;
  }
  for (int e = threadIdx.x; e < dh * DP; e += blockDim.x) {
    const int yy = e / DP, xx = e - yy * DP - kStrip;
    Ds[e] = (xx >= 0 && xx < dw) ? (V)g[(long long)(R.dy - 1 + yy) * W + (R.dx - 1 + xx)] : (V)0;
  }
  if (threadIdx.x < 30) hist[threadIdx.x] = 0;
  const int W1 = W + 1;
  const long long plane = (long long)W1 * (H + 1);
  const S *sf = sat, *sf2 = sat + plane, *sg = sat + 2 * plane, *sg2 = sat + 3 * plane;
  const long long mn = (long long)a * b;
  const int tx0i = R.tx - 1, ty0i = R.ty - 1, dx0i = R.dx - 1, dy0i = R.dy - 1;
  const S st = rect_sum(sf, W1, tx0i, tx0i + a, ty0i, ty0i + b);
  const S st2 = rect_sum(sf2, W1, tx0i, tx0i + a, ty0i, ty0i + b);
  bool flat;
  if constexpr (MgT<P>::integer)
    flat = ((__int128)mn * (long long)st2 - (__int128)(long long)st * (long long)st) == 0;
  else
    flat = !((double)mn * (double)st2 - (double)st * (double)st > 0.0);
  if (flat) {
    if (threadIdx.x == 0) o[3] = 0.0;
    return;
  }
  const double mu = *mu_g;
  __syncthreads();
  // strips of kStrip consecutive x shifts (map rows) at one y shift; the
  // template columns run in chunks of 8 over zero-padded rows, so the 8 x 8
  // products of a chunk are fully unrolled in registers
  const int nsr = (fr + kStrip - 1) / kStrip, nstrips = nsr * fc;
  for (int sI = threadIdx.x; sI < nstrips; sI += blockDim.x) {
    const int j = sI / nsr, i0 = (sI - j * nsr) * kStrip;
    const int oy = j - (b - 1), ox0 = i0 - (a - 1);
    const int ty0 = max(0, -oy), ty1 = min(b, dh - oy);
    const int txa = max(0, -(ox0 + kStrip - 1)), txb = min(a, dw - ox0);
    A s[kStrip];
#pragma unroll
    for (int k = 0; k < kStrip; ++k) s[k] = 0;
    for (int ty = ty0; ty < ty1; ++ty) {
      const V *tr = Ts + ty * TP;
      const V *dr = Ds + (ty + oy) * DP + kStrip + ox0;  // dr[tx + k]: region x = tx + ox0 + k
      for (int tx = txa; tx < txb; tx += 8) {
        V tv[8], dv[15];
#pragma unroll
        for (int q = 0; q < 8; ++q) tv[q] = tr[tx + q];
#pragma unroll
        for (int q = 0; q < 15; ++q) dv[q] = dr[tx + q];
#pragma unroll
        for (int q = 0; q < 8; ++q)
#pragma unroll
          for (int k = 0; k < kStrip; ++k) s[k] += (A)tv[q] * (A)dv[q + k];
      }
    }
#pragma unroll
    for (int k = 0; k < kStrip; ++k) {
      const int i = i0 + k;
      if (i >= fr) break;
      const int ox = ox0 + k;
      const int tx0 = max(0, -ox), tx1 = min(a, dw - ox);
      double r = 0.0;
      if (tx1 > tx0 && ty1 > ty0) {
        const long long n_in = (long long)(tx1 - tx0) * (ty1 - ty0);
        const S st_in = rect_sum(sf, W1, tx0i + tx0, tx0i + tx1, ty0i + ty0, ty0i + ty1);
        const S sd = rect_sum(sg, W1, dx0i + tx0 + ox, dx0i + tx1 + ox, dy0i + ty0 + oy, dy0i + ty1 + oy);
        const S sd2 = rect_sum(sg2, W1, dx0i + tx0 + ox, dx0i + tx1 + ox, dy0i + ty0 + oy, dy0i + ty1 + oy);
        r = combine<S>(mn, st, st2, (S)s[k], sd, sd2, st - st_in, mn - n_in, mu);
      }
      map[(long long)j * fr + i] = r;
    }
  }
  __syncthreads();
  // compute_qFactor: min, then peak and sum of squares of cc - min, histogram
  const int tid = threadIdx.x, nth = blockDim.x;
  double mnv = 1e300;
  for (int e = tid; e < nm; e += nth) mnv = fmin(mnv, map[e]);
  for (int k = 16; k > 0; k >>= 1) mnv = fmin(mnv, __shfl_xor_sync(0xffffffffu, mnv, k));
  if ((tid & 31) == 0) red[tid >> 5] = mnv;
  __syncthreads();
  if (tid == 0) {
    for (int k = 1; k < nth / 32; ++k) mnv = fmin(mnv, red[k]);
    red[32] = mnv;
  }
  __syncthreads();
  mnv = red[32];
  __syncthreads();
  double pk = 0, ss = 0;
  for (int e = tid; e < nm; e += nth) {
    const double v = map[e] - mnv;
    pk = fmax(pk, v);
    ss += v * v;
  }
  for (int k = 16; k > 0; k >>= 1) {
    pk = fmax(pk, __shfl_xor_sync(0xffffffffu, pk, k));
    ss += __shfl_xor_sync(0xffffffffu, ss, k);
  }
  if ((tid & 31) == 0) {
    red[tid >> 5] = pk;
    red[32 + (tid >> 5)] = ss;
  }
  __syncthreads();
  if (tid == 0) {
    double Pk = 0, Sq = 0;
    for (int k = 0; k < nth / 32; ++k) {
      Pk = fmax(Pk, red[k]);
      Sq += red[32 + k];
    }
    red[0] = Pk;
    red[1] = Sq;
  }
  __syncthreads();
  const double peak = red[0], sumsq = red[1];
  for (int e = tid; e < nm; e += nth) {
    const double v = map[e] - mnv;
    int bb = peak > 0 ? (int)floor(v / peak * 30.0) : 0;
    bb = bb > 29 ? 29 : (bb < 0 ? 0 : bb);
    atomicAdd(&hist[bb], 1);
  }
  // crop rows a-2 .. a+10, columns b-2 .. b+11 (0-based) of the full map
  for (int e = tid; e < kCrop; e += nth) {
    const int r = e % kCropR, c = e / kCropR;
    crop[e] = map[(long long)(b - 2 + c) * fr + (a - 2 + r)];
  }
  __syncthreads();
  if (tid == 0) {
    const double n = (double)nm;
    o[4] = (peak * peak) / (sumsq / n);
    double ent = 0;
    for (int k = 0; k < 30; ++k) {
      const double p = hist[k] / n;
      if (p > 0) ent += p * log(1.0 / p);
    }
    o[5] = 1.0 / ent;
    int im = 0;
    double mv = crop[0];
    for (int e = 1; e < kCrop; ++e)
      if (crop[e] > mv) {
        mv = crop[e];
        im = e;
      }
    double rp, cp, mf;
    findpeak_fit(crop, kCropR, kCropC, im, &rp, &cp, &mf);
    o[0] = __dsub_rn(rp, 7.0);
    o[1] = __dsub_rn(cp, 7.0);
    o[2] = mf;
    o[3] = 1.0;
  }
}

// ------------------------------------------------------------ gridfit gather
// A'A (9 coefficients per node, (di, dj) in row-major 3 x 3 order) and A'z of
// gridfit's triangle interpolation (gridfit.m:484-493) from the points of the
// four cells around each node.  Points are sorted by cell (cell = iy (nx-1) +
// ix, start[] its offsets); px, py their coordinates, pz their nr values
// (point-major).  rhs is field-major (nr x nx*ny).
__global__ void k_mg_ata(int nx, int ny, double x0, double y0, double h,
                         const int *__restrict__ start, const double *__restrict__ px,
                         const double *__restrict__ py, const double *__restrict__ pz, int nr,
                         double *__restrict__ ata, double *__restrict__ rhs) {
  const long long n = (long long)nx * ny;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % nx), j = (int)(k / nx);
    double c9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double r[5] = {0, 0, 0, 0, 0};
    for (int cj = j - 1; cj <= j; ++cj)
      for (int ci = i - 1; ci <= i; ++ci) {
        if (ci < 0 || ci >= nx - 1 || cj < 0 || cj >= ny - 1) continue;
        const int c = cj * (nx - 1) + ci;
        for (int p = start[c]; p < start[c + 1]; ++p) {
          const double tx = fmin(1.0, fmax(0.0, (px[p] - (x0 + ci * h)) / h));
          const double ty = fmin(1.0, fmax(0.0, (py[p] - (y0 + cj * h)) / h));
          const double t1 = fmin(tx, ty), t2 = fmax(tx, ty);
          // the triangle's nodes and weights
          const int ni[3] = {ci, ci + 1, tx > ty ? ci + 1 : ci};
          const int nj[3] = {cj, cj + 1, tx > ty ? cj : cj + 1};
          const double wt[3] = {1 - t2, t1, t2 - t1};
          int me = -1;
          for (int q = 0; q < 3; ++q)
            if (ni[q] == i && nj[q] == j) me = q;
          if (me < 0) continue;
          const double wk = wt[me];
          for (int q = 0; q < 3; ++q) c9[(nj[q] - j + 1) * 3 + (ni[q] - i + 1)] += wk * wt[q];
          for (int m = 0; m < nr; ++m) r[m] += wk * pz[(long long)p * nr + m];
        }
      }
    for (int q = 0; q < 9; ++q) ata[9 * k + q] = c9[q];
    for (int m = 0; m < nr; ++m) rhs[m * n + k] = r[m];
  }
}

// ------------------------------------------------------------ host bookkeeping
struct Region {
  double xf[2], yf[2], xg[2], yg[2];
};

inline double mceil(double v) { return std::isfinite(v) ? std::ceil(v) : NAN; }
inline long long mround(double v) { return v >= 0 ? (long long)std::floor(v + 0.5) : -(long long)std::floor(-v + 0.5); }

// funIntegerSearchMg.m:37-46 / :180-199 (comparisons with NaN are false)
void clamp_region(Region &q, double bg, int W, int H) {
  if (q.xg[0] < bg) { const double t = q.xg[0]; q.xg[0] = bg; q.xf[0] = q.xf[0] + bg - t; }
  if (q.yg[0] < bg) { const double t = q.yg[0]; q.yg[0] = bg; q.yf[0] = q.yf[0] + bg - t; }
  if (q.xg[1] > W - bg) { const double t = q.xg[1]; q.xg[1] = W - bg; q.xf[1] = q.xf[1] + (W - bg) - t; }
  if (q.yg[1] > H - bg) { const double t = q.yg[1]; q.yg[1] = H - bg; q.yf[1] = q.yf[1] + (H - bg) - t; }
}
// :47-48 / :200-208: mod(width, 2) == 1 -> shrink both by one
void make_even(Region &q) {
  const double dx = q.xf[1] - q.xf[0], dy = q.yf[1] - q.yf[0];
  if (std::isfinite(dx) && std::fmod(dx, 2.0) == 1.0) { q.xf[1] -= 1; q.xg[1] -= 1; }
  if (std::isfinite(dy) && std::fmod(dy, 2.0) == 1.0) { q.yf[1] -= 1; q.yg[1] -= 1; }
}

bool int_range(double lo, double hi, int lim) {
  return std::isfinite(lo) && std::isfinite(hi) && lo == std::floor(lo) && hi == std::floor(hi) &&
         lo >= 1 && lo <= hi && hi <= lim;
}

// Device descriptor of one region (valid = the correlation does not raise).
MgReg describe(const Region &q, int W, int H) {
  MgReg r{};
  const bool ok = int_range(q.xf[0], q.xf[1], W) && int_range(q.yf[0], q.yf[1], H) &&
                  int_range(q.xg[0] - 5, q.xg[1] + 5, W) && int_range(q.yg[0] - 5, q.yg[1] + 5, H);
  if (!ok) return r;
  r.tx = (int)q.xf[0];
  r.ty = (int)q.yf[0];
  r.a = (int)(q.xf[1] - q.xf[0]) + 1;
  r.b = (int)(q.yf[1] - q.yf[0]) + 1;
  r.dx = (int)q.xg[0] - 5;
  r.dy = (int)q.yg[0] - 5;
  // g is sliced with the f width (xg = xf + shift), so the region is a + 10 wide
  r.valid = (int)(q.xg[1] - q.xg[0]) == r.a - 1 && (int)(q.yg[1] - q.yg[0]) == r.b - 1 &&
            (long long)r.a * r.b >= 2;
  return r;
}

template <typename P>
int run_levels(MgWork &w, const P *f, const P *g, int W, int H, const double *mu_g,
               const int gridx_in[2], const int gridy_in[2], int winsize, bool qfactors,
               MgData &out, cudaStream_t st) {
  using S = typename MgT<P>::S;
  using G = typename MgT<P>::G;
  const long long W1 = W + 1, plane = W1 * (H + 1);
  int rc;
  auto t_last = std::chrono::steady_clock::now();
  auto lap = [&](int slot) {
    const auto now = std::chrono::steady_clock::now();
    out.t_ms[slot] += std::chrono::duration<double, std::milli>(now - t_last).count();
    t_last = now;
  };
  // summed-area tables
  const int nch = (H + kSatChunk - 1) / kSatChunk;
  if ((rc = w.sat.ensure(sizeof(S) * 4 * plane))) return rc;
  if ((rc = w.tot.ensure(sizeof(S) * 4 * (size_t)nch * W1))) return rc;
  S *sat = w.sat.as<S>();
  k_sat_rows<P><<<dim3(H, 4), 256, 0, st>>>(f, g, W, H, sat);
  k_sat_cols_chunk<S><<<dim3((unsigned)((W1 + 127) / 128), nch, 4), 128, 0, st>>>(sat, W, H, w.tot.as<S>());
  k_sat_cols_fix<S><<<dim3((unsigned)((W1 + 127) / 128), nch, 4), 128, 0, st>>>(sat, W, H, w.tot.as<S>());
  ALDIC_CUDA(cudaGetLastError());

  // ---- level 1: whole ROI (funIntegerSearchMg.m:9-35)
  const double bg = (double)(1 + mround(0.75 * winsize));
  int gx[2] = {gridx_in[0], gridx_in[1]}, gy[2] = {gridy_in[0], gridy_in[1]};
  if (gx[0] < bg) gx[0] = (int)bg;
  if (gy[0] < bg) gy[0] = (int)bg;
  if (gx[1] > W - bg) gx[1] = W - (int)bg;
  if (gy[1] > H - bg) gy[1] = H - (int)bg;
  const int a = gx[1] - gx[0] + 1, b = gy[1] - gy[0] + 1;
  ALDIC_CHECK(a >= 2 && b >= 2, E_ARG, "multigrid search: the ROI is empty after the border trim");
  int P1 = 1, P2 = 1, l1 = 0, l2 = 0;
  while (P1 < 2 * a - 1) { P1 <<= 1; l1++; }
  while (P2 < 2 * b - 1) { P2 <<= 1; l2++; }
  ALDIC_CHECK(P1 <= kMaxFFT && P2 <= kMaxFFT, E_ARG,
              "multigrid search: the ROI is wider than 4096 px");
  if (P1 < 2) { P1 = 2; l1 = 1; }
  if (P2 < 2) { P2 = 2; l2 = 1; }
  if ((rc = w.fft.ensure(sizeof(double2) * 2 * (size_t)P1 * P2))) return rc;
  if ((rc = w.tw.ensure(sizeof(double2) * (size_t)(P1 + P2)))) return rc;
  double2 *Z0 = w.fft.as<double2>(), *Z1 = Z0 + (size_t)P1 * P2;
  double2 *tw1 = w.tw.as<double2>(), *tw2 = tw1 + P1;
  k_fft_twiddle<<<(P1 + 255) / 256, 256, 0, st>>>(tw1, P1);
  k_fft_twiddle<<<(P2 + 255) / 256, 256, 0, st>>>(tw2, P2);
  const size_t sm1 = sizeof(double2) * P1, sm2 = sizeof(double2) * P2;
  const size_t smx = std::max(sm1, sm2);
  ALDIC_CUDA(cudaFuncSetAttribute(k_fft_pack_rows<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
  ALDIC_CUDA(cudaFuncSetAttribute(k_fft_rows<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
  ALDIC_CUDA(cudaFuncSetAttribute(k_fft_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smx));
  const int fth = 512;
  // rows: [y][x] (P2 rows of P1)
  k_fft_pack_rows<P><<<P2, fth, sm1, st>>>(f, g, W, H, gx[0], gy[0], a, b, sat, mu_g, Z0, P1, l1, tw1);
  k_transpose_c<<<dim3((P1 + 31) / 32, (P2 + 31) / 32), dim3(32, 8), 0, st>>>(Z0, Z1, P2, P1);
  k_fft_rows<false><<<P1, fth, sm2, st>>>(Z1, P2, l2, tw2, 0, 0);               // [kx][ky]
  k_mg_spectrum<<<1184, 256, 0, st>>>(Z1, Z0, P1, P2);
  k_fft_rows<true><<<P1, fth, sm2, st>>>(Z0, P2, l2, tw2, 0, 0);                // [kx][oy]
  k_transpose_c<<<dim3((P2 + 31) / 32, (P1 + 31) / 32), dim3(32, 8), 0, st>>>(Z0, Z1, P1, P2);
  // [oy][kx]: only rows oy in [-(b-1), b-1] (mod P2) are read
  k_fft_rows<true><<<P2, fth, sm1, st>>>(Z1, P1, l1, tw1, b, P2 - (b - 1));      // [oy][ox]
  ALDIC_CUDA(cudaGetLastError());
  L1Args<MgT<P>::integer, S> L1;
  L1.sat = sat;
  L1.W1 = (int)W1;
  L1.gx0 = gx[0] - 1;
  L1.gy0 = gy[0] - 1;
  L1.a = a;
  L1.b = b;
  L1.mn = (long long)a * b;
  L1.c = Z1;
  L1.P1 = P1;
  L1.P2 = P2;
  L1.inv = 1.0 / ((double)P1 * (double)P2);
  // template sums and mu on the host (two small reads)
  S sums[4];
  {
    S c4[2][4];
    const S *sf = sat, *sf2 = sat + plane;
    const long long xo0 = gx[0] - 1, yo0 = gy[0] - 1;
    const long long idx[4] = {yo0 * W1 + xo0, yo0 * W1 + xo0 + a, (yo0 + b) * W1 + xo0,
                              (yo0 + b) * W1 + xo0 + a};
    for (int k = 0; k < 4; ++k) {
      ALDIC_CUDA(cudaMemcpyAsync(&c4[0][k], sf + idx[k], sizeof(S), cudaMemcpyDeviceToHost, st));
      ALDIC_CUDA(cudaMemcpyAsync(&c4[1][k], sf2 + idx[k], sizeof(S), cudaMemcpyDeviceToHost, st));
    }
    double mu_h = 0;
    ALDIC_CUDA(cudaMemcpyAsync(&mu_h, mu_g, sizeof(double), cudaMemcpyDeviceToHost, st));
    ALDIC_CUDA(cudaStreamSynchronize(st));
    for (int q = 0; q < 2; ++q) sums[q] = c4[q][3] - c4[q][1] - c4[q][2] + c4[q][0];
    L1.mu = mu_h;
  }
  L1.st = sums[0];
  L1.st2 = sums[1];
  bool flat;
  if constexpr (MgT<P>::integer)
    flat = ((__int128)L1.mn * (long long)L1.st2 - (__int128)(long long)L1.st * (long long)L1.st) == 0;
  else
    flat = !((double)L1.mn * (double)L1.st2 - (double)L1.st * (double)L1.st > 0.0);
  ALDIC_CHECK(!flat, E_ARG, "multigrid search: the ROI of the reference image is constant");
  const int nblk = 148 * 8;
  if ((rc = w.part.ensure((sizeof(double) + sizeof(long long)) * nblk + 64))) return rc;
  double *pv = w.part.as<double>();
  long long *pi = (long long *)(pv + nblk);
  double *peak = (double *)(pi + nblk);
  k_mg_l1_argmax<MgT<P>::integer, S><<<nblk, 256, 0, st>>>(L1, sat + 2 * plane, sat + 3 * plane, pv, pi);
  k_mg_l1_peak<MgT<P>::integer, S><<<1, 32, 0, st>>>(L1, sat + 2 * plane, sat + 3 * plane, pv, pi, nblk, peak);
  ALDIC_CUDA(cudaGetLastError());
  double pk3[3];
  ALDIC_CUDA(cudaMemcpyAsync(pk3, peak, sizeof(pk3), cudaMemcpyDeviceToHost, st));
  ALDIC_CUDA(cudaStreamSynchronize(st));
  const double ut = pk3[0] - a, vt = pk3[1] - b;
  out.l1_u = ut;
  out.l1_v = vt;
  out.l1_cc = pk3[2];
  lap(0);

  // ---- shift the g ROI, clamp, even widths (:23-48)
  Region r0;
  r0.xf[0] = gx[0]; r0.xf[1] = gx[1]; r0.yf[0] = gy[0]; r0.yf[1] = gy[1];
  r0.xg[0] = gx[0] + mceil(ut); r0.xg[1] = gx[1] + mceil(ut);
  r0.yg[0] = gy[0] + mceil(vt); r0.yg[1] = gy[1] + mceil(vt);
  clamp_region(r0, bg, W, H);
  make_even(r0);
  std::vector<Region> cur{r0};
  std::vector<double> ucur{mceil(ut)}, vcur{mceil(vt)};
  double wx = r0.xf[1] - r0.xf[0], wy = r0.yf[1] - r0.yf[0];
  double ratio = wx / wy;
  const double wsz = winsize;
  int levels = 1;
  for (;;) {
    // ---- split (:58-147)
    std::vector<Region> nw;
    std::vector<double> un, vn;
    const int mode = ratio > 2 ? 0 : (ratio < 0.5 ? 1 : 2);
    if (mode == 0) wx /= 2; else if (mode == 1) wy /= 2; else { wx /= 2; wy /= 2; }
    const int rep = mode == 2 ? 4 : 2;
    nw.reserve(cur.size() * rep);
    for (size_t t = 0; t < cur.size(); ++t) {
      const Region &q = cur[t];
      const bool sx = q.xf[1] - q.xf[0] > wsz, sy = q.yf[1] - q.yf[0] > wsz;
      const double mxf = 0.5 * (q.xf[0] + q.xf[1]), mxg = 0.5 * (q.xg[0] + q.xg[1]);
      const double myf = 0.5 * (q.yf[0] + q.yf[1]), myg = 0.5 * (q.yg[0] + q.yg[1]);
      if (mode == 0 && sx) {
        Region lo = q, hi = q;
        lo.xf[1] = mxf; lo.xg[1] = mxg; hi.xf[0] = mxf; hi.xg[0] = mxg;
        nw.push_back(lo); nw.push_back(hi);
      } else if (mode == 1 && sy) {
        Region lo = q, hi = q;
        lo.yf[1] = myf; lo.yg[1] = myg; hi.yf[0] = myf; hi.yg[0] = myg;
        nw.push_back(lo); nw.push_back(hi);
      } else if (mode == 2 && sx && sy) {
        for (int jy = 0; jy < 2; ++jy)
          for (int ix = 0; ix < 2; ++ix) {
            Region s = q;
            if (ix == 0) { s.xf[1] = mxf; s.xg[1] = mxg; } else { s.xf[0] = mxf; s.xg[0] = mxg; }
            if (jy == 0) { s.yf[1] = myf; s.yg[1] = myg; } else { s.yf[0] = myf; s.yg[0] = myg; }
            nw.push_back(s);
          }
      } else {
        for (int k = 0; k < rep; ++k) nw.push_back(q);
      }
      for (int k = 0; k < rep; ++k) { un.push_back(ucur[t]); vn.push_back(vcur[t]); }
    }
    const bool last = wx < wsz && wy < wsz;
    levels++;
    const int n = (int)nw.size();
    ALDIC_CHECK(n <= (1 << 24), E_ARG, "multigrid search: too many regions");
    // ---- correlate every region (:148-172)
    std::vector<MgReg> hr(n);
    int amax = 0, bmax = 0;
    for (int t = 0; t < n; ++t) {
      hr[t] = describe(nw[t], W, H);
      if (hr[t].valid) { amax = std::max(amax, hr[t].a); bmax = std::max(bmax, hr[t].b); }
    }
    if ((rc = w.regs.ensure(sizeof(MgReg) * n))) return rc;
    if ((rc = w.res.ensure(sizeof(double) * 8 * n))) return rc;
    ALDIC_CUDA(cudaMemcpyAsync(w.regs.p, hr.data(), sizeof(MgReg) * n, cudaMemcpyHostToDevice, st));
    MgReg *dr = w.regs.as<MgReg>();
    double *dres = w.res.as<double>();
    if (last && qfactors) {
      ALDIC_CHECK(amax <= kMaxFinal && bmax <= kMaxFinal, E_ARG,
                  "multigrid search: last-level regions larger than 80 px");
      const int dwm = amax + 10, dhm = bmax + 10;
      const size_t sm = sizeof(double) * (size_t)(amax + dwm - 1) * (bmax + dhm - 1) +
                        sizeof(typename MgT<P>::V) *
                            ((size_t)(amax + 8) * bmax + (size_t)dhm * (dwm + 2 * kStrip + 8)) + 16;
      ALDIC_CHECK(sm <= 200 * 1024, E_ARG, "multigrid search: last-level map too large for shared memory");
      ALDIC_CUDA(cudaFuncSetAttribute(k_mg_full<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      if (amax > 0) k_mg_full<P><<<n, 256, sm, st>>>(f, g, W, H, dr, sat, mu_g, dres);
    } else {
      if ((rc = w.acc.ensure(sizeof(G) * (size_t)kCrop * n))) return rc;
      ALDIC_CUDA(cudaMemsetAsync(w.acc.p, 0, sizeof(G) * (size_t)kCrop * n, st));
      if (amax > 0) {
        constexpr int kTile = CropCfg<P>::TILE;
        const dim3 grid(n, (bmax + kBand - 1) / kBand, (amax + kTile - 1) / kTile);
        ALDIC_CHECK(grid.y <= 65535 && grid.z <= 65535, E_ARG, "multigrid search: region too large");
        k_mg_crop<P><<<grid, 224, 0, st>>>(f, g, W, dr, w.acc.as<G>());
        k_mg_crop_peak<P><<<n, 192, 0, st>>>(dr, W, H, sat, w.acc.as<G>(), mu_g, dres);
      }
    }
    ALDIC_CUDA(cudaGetLastError());
    std::vector<double> hres((size_t)8 * n, 0.0);
    ALDIC_CUDA(cudaMemcpyAsync(hres.data(), dres, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost, st));
    ALDIC_CUDA(cudaStreamSynchronize(st));
    lap(last ? 2 : 1);
    std::vector<double> phi(n, 0.0), q1(n, NAN), q2(n, NAN);
    int failed = 0;
    for (int t = 0; t < n; ++t) {
      const double *o = &hres[(size_t)8 * t];
      if (hr[t].valid && o[3] == 1.0) {
        un[t] += o[0];
        vn[t] += o[1];
        phi[t] = o[2];
        if (last && qfactors) { q1[t] = o[4]; q2[t] = o[5]; }
      } else {
        un[t] = vn[t] = NAN;
        phi[t] = 0.0;
        failed++;
      }
    }
    if (last) {
      // :173-178: q-factors normalised over the regions (NaN ignored)
      for (std::vector<double> *q : {&q1, &q2}) {
        double mn = INFINITY, mx = -INFINITY;
        for (double v : *q) if (!std::isnan(v) && v < mn) mn = v;
        for (double v : *q) if (!std::isnan(v) && v - mn > mx) mx = v - mn;
        for (double &v : *q) v = (v - mn) / mx;
      }
      out.tx.resize(n); out.ty.resize(n);
      for (int t = 0; t < n; ++t) {
        out.tx[t] = 0.5 * (nw[t].xf[0] + nw[t].xf[1]);
        out.ty[t] = 0.5 * (nw[t].yf[0] + nw[t].yf[1]);
      }
      out.u = un; out.v = vn; out.phi = phi; out.q1 = q1; out.q2 = q2;
      out.gridx[0] = gx[0]; out.gridx[1] = gx[1];
      out.gridy[0] = gy[0]; out.gridy[1] = gy[1];
      out.levels = levels;
      out.failed = failed;
      return OK;
    }
    // ---- next level's g regions (:179-209)
    for (int t = 0; t < n; ++t) {
      Region &q = nw[t];
      const double cu = mceil(un[t]), cv = mceil(vn[t]);
      q.xg[0] = q.xf[0] + cu; q.xg[1] = q.xf[1] + cu;
      q.yg[0] = q.yf[0] + cv; q.yg[1] = q.yf[1] + cv;
      clamp_region(q, bg, W, H);
    }
    for (auto &q : nw) make_even(q);
    ratio = wx / wy;
    cur.swap(nw);
    ucur.resize(n); vcur.resize(n);
    for (int t = 0; t < n; ++t) { ucur[t] = mceil(un[t]); vcur[t] = mceil(vn[t]); }
  }
}

}  // namespace

int search_mg_levels(MgWork &w, const void *f, const void *g, int dtype, int W, int H,
                     const double *mu_g, const int gridx[2], const int gridy[2], int winsize,
                     bool qfactors, MgData &out, cudaStream_t st) {
  ALDIC_CHECK(winsize > 0, E_ARG, "multigrid search: winsize must be positive");
  switch (dtype) {
    case 0: return run_levels<uint8_t>(w, (const uint8_t *)f, (const uint8_t *)g, W, H, mu_g, gridx, gridy, winsize, qfactors, out, st);
    case 1: return run_levels<uint16_t>(w, (const uint16_t *)f, (const uint16_t *)g, W, H, mu_g, gridx, gridy, winsize, qfactors, out, st);
    case 2: return run_levels<float>(w, (const float *)f, (const float *)g, W, H, mu_g, gridx, gridy, winsize, qfactors, out, st);
    default: return run_levels<double>(w, (const double *)f, (const double *)g, W, H, mu_g, gridx, gridy, winsize, qfactors, out, st);
  }
}

// funIntegerSearchMg.m:210-244: node grid from the borders of the extreme
// regions; returns false when the grid is empty.
bool search_mg_grid(const MgData &d, int winsize, int step, int W, int H, MgGrid &grid) {
  const int n = (int)d.tx.size();
  if (n == 0) return false;
  int ix1 = 0, ix2 = 0, iy1 = 0, iy2 = 0;
  for (int t = 1; t < n; ++t) {
    if (d.tx[t] < d.tx[ix1]) ix1 = t;
    if (d.tx[t] > d.tx[ix2]) ix2 = t;
    if (d.ty[t] < d.ty[iy1]) iy1 = t;
    if (d.ty[t] > d.ty[iy2]) iy2 = t;
  }
  const double bx1 = mceil(1 + 1.25 * winsize + d.u[ix1]), bx2 = mceil(1 + 1.25 * winsize + d.u[ix2]);
  const double by1 = mceil(1 + 1.25 * winsize + d.v[iy1]), by2 = mceil(1 + 1.25 * winsize + d.v[iy2]);
  double gx0 = d.gridx[0], gx1 = d.gridx[1], gy0 = d.gridy[0], gy1 = d.gridy[1];
  if (gx0 < bx1) gx0 = bx1;
  if (gy0 < by1) gy0 = by1;
  if (gx1 > W - bx2 + 1) gx1 = W - bx2 + 1;
  if (gy1 > H - by2 + 1) gy1 = H - by2 + 1;
  grid.x0 = gx0;
  grid.y0 = gy0;
  grid.nx = gx1 >= gx0 ? (int)std::floor((gx1 - gx0) / step) + 1 : 0;
  grid.ny = gy1 >= gy0 ? (int)std::floor((gy1 - gy0) / step) + 1 : 0;
  grid.step = step;
  return grid.nx >= 2 && grid.ny >= 2;
}

// gridfit(x, y, z, xList, yList, 'regularizer', 'springs') of u, v, Phi and
// the two q-factors (gridfit.m:328-596 with smoothness 1, triangle
// interpolation, autoscale on uniform nodes): the normal equations
// (A'A + (NA/NR)^2 Areg'Areg) z = A'data.  The springs part is the gridfit
// stencil of the grid PCG; A'A and A'z are gathered per node from the points
// of its four cells (k_mg_ata, points sorted by cell on the host: fixed
// order, no atomics); one solve per set of fields sharing a NaN pattern.
int search_mg_fit(GridWork &gw, MgWork &w, MgData &d, const MgGrid &grid, int nfields,
                  double *out, cudaStream_t st) {
  const auto t0 = std::chrono::steady_clock::now();
  struct Lap {
    MgData &d;
    std::chrono::steady_clock::time_point t0;
    ~Lap() {
      d.t_ms[3] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
  } lap{d, t0};
  const int nx = grid.nx, ny = grid.ny;
  const long long ng = (long long)nx * ny;
  const double h = grid.step;
  const double xmax = grid.x0 + (nx - 1) * h, ymax = grid.y0 + (ny - 1) * h;
  const int n = (int)d.tx.size();
  // data strictly inside the grid (funIntegerSearchMg.m:232-234)
  std::vector<int> sel;
  for (int t = 0; t < n; ++t)
    if (d.tx[t] > grid.x0 && d.tx[t] < xmax && d.ty[t] > grid.y0 && d.ty[t] < ymax) sel.push_back(t);
  const std::vector<double> *fields[5] = {&d.u, &d.v, &d.phi, &d.q1, &d.q2};
  const int nf = std::min(std::max(nfields, 1), 5);
  std::vector<int> group(nf, -1);
  std::vector<std::vector<int>> members;
  for (int fi = 0; fi < nf; ++fi) {
    if (group[fi] >= 0) continue;
    group[fi] = (int)members.size();
    members.push_back({fi});
    for (int fj = fi + 1; fj < nf; ++fj) {
      if (group[fj] >= 0) continue;
      bool same = true;
      for (int t : sel)
        if (std::isnan((*fields[fi])[t]) != std::isnan((*fields[fj])[t])) { same = false; break; }
      if (same) { group[fj] = group[fi]; members.back().push_back(fj); }
    }
  }
  double NR = 0;  // norm(Areg, 1)
  const double sq2 = 1.0 / std::sqrt(2.0);
  for (int j = 0; j < std::min(ny, 3); ++j)
    for (int i = 0; i < std::min(nx, 3); ++i) {
      double sreg = (i > 0) + (i < nx - 1) + (j > 0) + (j < ny - 1);
      sreg += sq2 * ((i > 0 && j > 0) + (i < nx - 1 && j > 0) + (i > 0 && j < ny - 1) +
                     (i < nx - 1 && j < ny - 1));
      NR = std::max(NR, sreg);
    }
  const long long ncell = (long long)(nx - 1) * (ny - 1);
  int rc;
  for (const auto &mem : members) {
    const int nr = (int)mem.size();
    std::vector<int> pts;
    for (int t : sel)
      if (!std::isnan((*fields[mem[0]])[t])) pts.push_back(t);
    const long long np = (long long)pts.size();
    ALDIC_CHECK(np >= 3, E_ARG, "multigrid search: gridfit has fewer than 3 data points");
    // histc cells (the last node belongs to the last cell), counting sort by
    // cell (stable: region order inside a cell), column sums of A for NA
    std::vector<int> cell(np), start(ncell + 1, 0);
    std::vector<double> colsum(ng, 0.0);
    for (long long q = 0; q < np; ++q) {
      const double x = d.tx[pts[q]], y = d.ty[pts[q]];
      int ix = (int)std::floor((x - grid.x0) / h), iy = (int)std::floor((y - grid.y0) / h);
      ix = std::min(std::max(ix, 0), nx - 2);
      iy = std::min(std::max(iy, 0), ny - 2);
      cell[q] = iy * (nx - 1) + ix;
      start[cell[q] + 1]++;
      const double tx = std::min(1.0, std::max(0.0, (x - (grid.x0 + ix * h)) / h));
      const double ty = std::min(1.0, std::max(0.0, (y - (grid.y0 + iy * h)) / h));
      const double t1 = std::min(tx, ty), t2 = std::max(tx, ty);
      const long long k0 = (long long)iy * nx + ix;
      colsum[k0] += 1 - t2;
      colsum[k0 + nx + 1] += t1;
      colsum[tx > ty ? k0 + 1 : k0 + nx] += t2 - t1;
    }
    double NA = 0;
    for (double c : colsum) NA = std::max(NA, c);
    for (long long c = 0; c < ncell; ++c) start[c + 1] += start[c];
    std::vector<int> fill(start.begin(), start.end() - 1);
    std::vector<double> hp((size_t)(2 + nr) * np);  // x | y | values (point-major)
    for (long long q = 0; q < np; ++q) {
      const long long o = fill[cell[q]]++;
      hp[o] = d.tx[pts[q]];
      hp[np + o] = d.ty[pts[q]];
      for (int m = 0; m < nr; ++m) hp[2 * np + o * nr + m] = (*fields[mem[m]])[pts[q]];
    }
    const size_t bytes = sizeof(int) * (ncell + 1) + sizeof(double) * hp.size() + sizeof(double) * 9 * ng + 64;
    if ((rc = w.csr.ensure(bytes))) return rc;
    int *dstart = w.csr.as<int>();
    double *dp = (double *)(((uintptr_t)(dstart + ncell + 1) + 15) & ~(uintptr_t)15);
    double *data = dp + hp.size();
    ALDIC_CUDA(cudaMemcpyAsync(dstart, start.data(), sizeof(int) * (ncell + 1), cudaMemcpyHostToDevice, st));
    ALDIC_CUDA(cudaMemcpyAsync(dp, hp.data(), sizeof(double) * hp.size(), cudaMemcpyHostToDevice, st));
    k_mg_ata<<<(unsigned)std::min<long long>((ng + 255) / 256, 148 * 16), 256, 0, st>>>(
        nx, ny, grid.x0, grid.y0, h, dstart, dp, dp + np, dp + 2 * np, nr, data, gw.b);
    ALDIC_CUDA(cudaGetLastError());
    ALDIC_CUDA(cudaMemsetAsync(gw.x, 0, sizeof(double) * nr * ng, st));
    ALDIC_CUDA(cudaMemsetAsync(gw.mask, 1, (size_t)nr * ng, st));
    const double lam2 = (NA / NR) * (NA / NR);
    if ((rc = grid_pcg(gw, OP_GRIDFIT, nx, ny, nr, 0.0, 0.0, 1.0, lam2, 1e-13, 20000, st, nullptr,
                       nullptr, data)))
      return rc;
    for (int m = 0; m < nr; ++m)
      ALDIC_CUDA(cudaMemcpyAsync(out + (size_t)mem[m] * ng, gw.x + (size_t)m * ng, sizeof(double) * ng,
                                 cudaMemcpyDeviceToDevice, st));
    ALDIC_CUDA(cudaStreamSynchronize(st));  // host vectors above are reused next group
  }
  return OK;
}

}  // namespace aldic
