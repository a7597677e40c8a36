// k_icgn.cu -- local IC-GN (funICGN.m) and the ADMM local step
// (funICGN_Subpb1.m) for every subset of a frame in one persistent launch.
//
// Mapping: one warp per subset; warps pull subset indices from a global
// atomic counter, so subsets that converge early free their warp at once
// (per-subset early exit with load balance).  Each lane owns pixels
// lane, lane+32, ... of the (w+1)^2 subset.  Per iteration a lane samples the
// deformed image at its warped pixels (Keys bicubic, a = -1/2, as
// ba_interp2.cpp) and accumulates 8 residual sums in the working precision;
// the warp reduces them in FP64 in one transposed butterfly (warp_sum_t:
// lane 4q ends with sum q, then every lane reads all eight, so control flow
// stays warp-uniform), and every lane then forms b, the convergence test and
// dP = -H\b with the FP64 Cholesky factor of H, and applies the
// inverse-compositional update in FP64.  State every lane holds alike (P,
// the subset's constants, the evaluation's inputs) lives in the warp's
// shared scratch rather than in registers.
//
// FP32 sampling reads the row-cubic coefficients of the deformed image
// (row_cubic: per pixel the Keys cubic of its row around that floor column,
// one 16-byte load): a sample is four Horner rules over tu on its four
// stencil rows and one cubic over tv.  Lanes map to subset columns: lane l
// walks column l (then l + 32, ...) down the rows, so X is fixed per lane and
// Y uniform per row -- u and v are one FMA each from per-lane bases, the
// terms weighted by X are summed unweighted and multiplied by X once -- and
// a lane keeps its last four stencil rows in registers: the next row of the
// column usually sits one image row lower on the same floor column
// (F12, F22 small), so it loads one new stencil row instead of four.  The
// columns past the last full 32 (one for a 33-pixel window) are spread over
// the lanes by pixel.  FP64 keeps the plain stencil over the image, pixel per
// lane.
//
// ZNSSD residual (funICGN.m:238): r = (f - fbar)/bf - (g - gbar)/bg.  With
// sd_k the steepest-descent images,
//   b2_k = S_fk/bf - (T_k - gm S_k)/bg,
// where S_fk = sum sd_k (f - fbar), S_k = sum sd_k are fixed per subset and
// T_k = sum sd_k (g - c), gm = mean(g) - c are accumulated per iteration with
// the shift c = fbar (which keeps the one-pass variance well conditioned).
#include <climits>
#include <map>
#include <mutex>
#include <vector>

#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {

namespace {


struct Args {
  IcgnImages im;
  const double *coords;
  long long n;
  const double *U0;     // IC-GN: U0; Subpb1: UOld
  const double *F0;     // IC-GN: initial deformation gradient [F11 F21 F12 F22] per subset, or null (0)
  const double *FOld;   // Subpb1
  const double *vdual;  // Subpb1
  const double *H21in;  // Subpb1
  const int *wins;
  int w;
  double tol, mu;
  double *U, *F, *H21out;
  int *iters;
  unsigned int *queue;
  // per-subset setup constants (IC-GN writes, Subpb1 reads; may be null):
  // [mean f, bf, S_f5, S_f6, S_5, S_6, w after growth, status 0/102/-1]
  double *cache;
};

__device__ __forceinline__ double nan64() { return __longlong_as_double(0x7ff8000000000000ll); }

// Subset bounds of funICGN.m:34-50: integral, Df index x-3 in [1, W-6].
__device__ __forceinline__ bool subset_ok(const IcgnImages &im, double x0, double y0, int w,
                                          int *xl, int *yl) {
  const double a = x0 - 0.5 * w, b = y0 - 0.5 * w;
  if (a != floor(a) || b != floor(b)) return false;
  *xl = (int)a;
  *yl = (int)b;
  return *xl >= 4 && *yl >= 4 && *xl + w <= im.W - 3 && *yl + w <= im.H - 3;
}

template <typename Real> struct Img;
template <> struct Img<float> {
  static __device__ __forceinline__ const float *f(const IcgnImages &m) { return m.f32; }
};
template <> struct Img<double> {
  static __device__ __forceinline__ const double *f(const IcgnImages &m) { return m.f64; }
};

// The FP64 reference gradients of a pixel (the FP32 path reads the (gx, gy)
// pairs of IcgnImages::gxy).
struct Grad64 {
  const double *x, *y;
  __device__ __forceinline__ explicit Grad64(const IcgnImages &m) : x(m.gx64), y(m.gy64) {}
  __device__ __forceinline__ void at(int k, double *fx, double *fy) const {
    *fx = x[k];
    *fy = y[k];
  }
};

// Cholesky of the 6x6 SPD matrix (lower, packed row-wise in L[21]); inv[i]
// = 1 / L(i,i), so that the solves multiply instead of dividing.
__device__ bool chol6(const double H[36], double L[21], double inv[6]) {
  int idx = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = H[i * 6 + j];
      for (int k = 0; k < j; ++k) s -= L[i * (i + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
      if (i == j) {
        if (!(s > 0.0)) return false;
        L[idx++] = sqrt(s);
        inv[i] = 1.0 / L[idx - 1];
      } else {
        L[idx++] = s * inv[j];
      }
    }
  return true;
}

__device__ void chol6_solve(const double *L, const double *inv, const double b[6], double x[6]) {
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double t = b[i];
#pragma unroll
    for (int k = 0; k < i; ++k) t -= L[i * (i + 1) / 2 + k] * y[k];
    y[i] = t * inv[i];
  }
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
#pragma unroll
    for (int k = i + 1; k < 6; ++k) t -= L[k * (k + 1) / 2 + i] * x[k];
    x[i] = t * inv[i];
  }
}

// inverse-compositional update of funICGN.m:268-286
__device__ __forceinline__ bool ic_compose(double P[6], const double d[6]) {
  const double det = (1 + d[0]) * (1 + d[3]) - d[1] * d[2];
  if (!(det != 0.0)) return false;
  const double id = 1.0 / det;
  const double t1 = (-d[0] - d[0] * d[3] + d[1] * d[2]) * id;
  const double t2 = -d[1] * id;
  const double t3 = -d[2] * id;
  const double t4 = (-d[3] - d[0] * d[3] + d[1] * d[2]) * id;
  const double t5 = (-d[4] - d[3] * d[4] + d[2] * d[5]) * id;
  const double t6 = (-d[5] - d[0] * d[5] + d[1] * d[4]) * id;
  const double a11 = 1 + P[0], a12 = P[2], a13 = P[4];
  const double a21 = P[1], a22 = 1 + P[3], a23 = P[5];
  P[0] = a11 * (1 + t1) + a12 * t2 - 1;
  P[1] = a21 * (1 + t1) + a22 * t2;
  P[2] = a11 * t3 + a12 * (1 + t4);
  P[3] = a21 * t3 + a22 * (1 + t4) - 1;
  P[4] = a11 * t5 + a12 * t6 + a13;
  P[5] = a21 * t5 + a22 * t6 + a23;
  return true;
}

// Keys bicubic sample of img (W wide) around the 0-based floor corner
// (cx, cy) with fractional parts (tu, tv).
template <typename Real>
__device__ __forceinline__ Real sample(const Real *__restrict__ img, int W, int cx, int cy,
                                       Real tu, Real tv) {
  Real wu[4], wv[4];
  keys_w(tu, wu);
  keys_w(tv, wv);
  const Real *p = img + ((cy - 1) * W + (cx - 1));
  Real acc = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const Real *q = p + r * W;
    Real s = wu[0] * __ldg(q) + wu[1] * __ldg(q + 1) + wu[2] * __ldg(q + 2) + wu[3] * __ldg(q + 3);
    acc += wv[r] * s;
  }
  return acc;
}

__device__ __forceinline__ double sample_minus(const double *img, int W, int cx, int cy,
                                               double tu, double tv, double c) {
  return sample<double>(img, W, cx, cy, tu, tv) - c;
}

// floor(x) and the same value as an int, for |x| < 2^22: x + 1.5 * 2^23
// rounded toward -infinity lands on the float grid of spacing 1, so it holds
// floor(x) + 1.5 * 2^23 exactly and floor(x) sits in its low mantissa bits
// (magic-number rounding).  Equal to floorf / (int) bit for bit, on the FP32
// and integer pipes instead of the conversion unit.  The sampled positions
// lie inside the image (the out-of-image test runs first), far below 2^22.
__device__ __forceinline__ float floor_i(float x, int *i) {
  const float t = __fadd_rd(x, 12582912.0f);
  *i = __float_as_int(t) - 0x4B400000;
  return t - 12582912.0f;
}

// Transposed butterfly over the warp: NV partial sums a lane (NV a power of
// two up to 32).  At each level a lane keeps the half of its values that its
// partner gives away and adds the partner's copy of that half, so NV sums
// take NV - 1 exchanges (then plain butterfly levels once a lane holds one)
// instead of NV butterflies of five.  Afterwards v[0] of lane l holds the
// total of value l >> (5 - log2 NV).  Each total is formed from the same
// pairs in the same order as warp_sum's (own partial + partner's), so the
// values are bit-identical to NV warp_sum calls.
template <int NV>
__device__ __forceinline__ double warp_sum_t(double (&v)[NV], int lane) {
#pragma unroll
  for (int lvl = 0; lvl < 5; ++lvl) {
    const int o = 16 >> lvl;
    const int m = NV >> lvl;  // values a lane still holds
    if (m > 1) {
      const bool hi = (lane & o) != 0;
#pragma unroll
      for (int i = 0; i < m / 2; ++i) {
        const double lo_v = v[i], hi_v = v[i + m / 2];
        const double send = hi ? lo_v : hi_v, keep = hi ? hi_v : lo_v;
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
    }
  }
  return v[0];
}

// Packed (two-lane) FP32 arithmetic of sm_100: two IEEE single-precision
// operations per instruction.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// FP32 bicubic from the four stencil rows' cubic coefficients (r0 .. r3 =
// image rows floor - 1 .. floor + 2) at fractions (tu, tv): each row's cubic
// at tu, then the Keys cubic over the four row values at tv (the same
// polynomial form as row_cubic, applied down the column).
__device__ __forceinline__ float horner3(const float4 &a, float t) {
  return fmaf(fmaf(fmaf(a.w, t, a.z), t, a.y), t, a.x);
}
__device__ __forceinline__ float cubic_rows(const float4 &r0, const float4 &r1, const float4 &r2,
                                           const float4 &r3, float tu, float tv) {
  const float h0 = horner3(r0, tu), h1 = horner3(r1, tu), h2 = horner3(r2, tu),
              h3 = horner3(r3, tu);
  const float c1 = 0.5f * (h2 - h0);
  const float c2 = fmaf(-0.5f, h3, fmaf(2.0f, h2, fmaf(-2.5f, h1, h0)));
  const float c3 = fmaf(1.5f, h1 - h2, 0.5f * (h3 - h0));
  return fmaf(fmaf(fmaf(c3, tv, c2), tv, c1), tv, h1);
}

// Pixel p of a block of nw-wide rows (x fastest): its column and row as
// exact small integers in Real, and its offset row * W + column.
// Branch-free, so the lanes of a warp (which wrap to the next row at
// different p) stay converged.  row = floor((p + 1/2) / nw) is exact:
// (p + 1/2) / nw lies at least 1/(2 nw) from an integer, and the two FP32
// roundings err by at most (p / nw) 2^-23, far less for p < 2^20.
template <typename Real> struct PixelMap {
  Real fnw, inw;
  int W;
  __device__ __forceinline__ PixelMap(int nw, int W_)
      : fnw((Real)nw), inw((Real)1 / (Real)nw), W(W_) {}
  __device__ __forceinline__ int at(int p, Real *col, Real *row) const {
    const Real fp = (Real)p;
    const Real r = floor((fp + (Real)0.5) * inw);
    const Real c = fp - r * fnw;
    *col = c;
    *row = r;
    return (int)r * W + (int)c;
  }
};

// One FP32 evaluation of the residual sums over an nw x nw subset whose
// top-left pixel is `base` and whose pixel (0, 0) sits at (ox, oy) from the
// subset centre: u = a11 X + a12 Y + c4, v = a21 X + a22 Y + c5 relative to
// the floor corner (xb, yb) of the centre (c4, c5 carry the centre's
// fraction).  Per lane: o = [sum d, sum d^2, sum X fx d, sum X fy d,
// sum Y fx d, sum Y fy d, sum fx d, sum fy d], d = g(warped) - cg
// (SUB: only o[0], o[1], o[6], o[7]).
struct Eval32 {
  const float4 *rc;   // row_cubic at (floor corner x of the centre - 1, its y - 2)
  const float2 *gxy;  // reference gradients at the subset's top-left pixel
  int W, nw;
  float ox, oy, a11, a12, a21, a22, c4, c5, cg;
};

// Packed partial sums of an evaluation: (sum d, sum d^2), (sum fx d, sum fy d)
// and their X- and Y-weighted versions.
struct Acc32 {
  float2 S, T, TX, TY;
};

// One row of a lane's column: u, v at Y; the stencil rows slide down by one
// when the floor corner moved one row down the same column, else all four
// reload.  Slot (K + j) & 3 of R holds stencil row j (K = row index mod 4,
// fixed by the unrolled caller), so sliding moves no registers.
template <bool SUB, int K>
__device__ __forceinline__ void col_row(const Eval32 &e, float4 (&R)[4], int &pcx, int &pcy,
                                        float bu, float bv, float Y, const float2 *gp, float2 &C,
                                        Acc32 &a) {
  const int W = e.W;
  const float ru = fmaf(e.a12, Y, bu), rv = fmaf(e.a22, Y, bv);
  int icx, icy;
  const float fu = floor_i(ru, &icx), fv = floor_i(rv, &icy);
  const float4 *q = e.rc + (icy + 3) * W + icx;  // stencil row 3
  const bool slide = icx == pcx && icy == pcy + 1;
  R[(K + 3) & 3] = __ldg(q);
  if (!slide) {
    R[K & 3] = __ldg(q - 3 * W);
    R[(K + 1) & 3] = __ldg(q - 2 * W);
    R[(K + 2) & 3] = __ldg(q - W);
  }
  pcx = icx;
  pcy = icy;
  const float d = cubic_rows(R[K & 3], R[(K + 1) & 3], R[(K + 2) & 3], R[(K + 3) & 3], ru - fu,
                             rv - fv) - e.cg;
  const float2 G = __ldg(gp);
  const float2 D = f2(d);
  a.S = __ffma2_rn(D, f2(1.f, d), a.S);
  const float2 A = __fmul2_rn(G, D);
  C = __fadd2_rn(C, A);
  if (!SUB) a.TY = __ffma2_rn(A, f2(Y), a.TY);
}

// One row of a lane's column under a pure translation (a11 = a22 = 1,
// a12 = a21 = 0): the fractions (tu, tv) are the same at every pixel and
// the floor corner moves down exactly one image row per subset row, so the
// window holds each stencil row's cubic at tu, formed once as the row
// enters (slot (K + 3) & 3, as in col_row), and the sample is the Keys
// weights at tv over the four values.
template <bool SUB, int K>
__device__ __forceinline__ void shift_row(float (&H)[4], const float4 *&q, int W, float tu,
                                          const float4 &wv, float cg, float Y, const float2 *gp,
                                          float2 &C, Acc32 &a) {
  H[(K + 3) & 3] = horner3(__ldg(q), tu);
  q += W;
  const float d = fmaf(wv.w, H[(K + 3) & 3],
                       fmaf(wv.z, H[(K + 2) & 3], fmaf(wv.y, H[(K + 1) & 3], fmaf(wv.x, H[K & 3], -cg))));
  const float2 G = __ldg(gp);
  const float2 D = f2(d);
  a.S = __ffma2_rn(D, f2(1.f, d), a.S);
  const float2 A = __fmul2_rn(G, D);
  C = __fadd2_rn(C, A);
  if (!SUB) a.TY = __ffma2_rn(A, f2(Y), a.TY);
}

// One FP32 evaluation of the residual sums over an nw x nw subset whose
// top-left pixel is `base` and whose pixel (0, 0) sits at (ox, oy) from the
// subset centre: u = a11 X + a12 Y + c4, v = a21 X + a22 Y + c5 relative to
// the floor corner (xb, yb) of the centre (c4, c5 carry the centre's
// fraction).  Per lane: o = [sum d, sum d^2, sum X fx d, sum X fy d,
// sum Y fx d, sum Y fy d, sum fx d, sum fy d], d = g(warped) - cg
// (SUB: only o[0], o[1], o[6], o[7]).
template <bool SUB>
__device__ __forceinline__ void eval32(const Eval32 &e, int lane, float o[8]) {
  const int W = e.W, nw = e.nw;
  Acc32 a;
  a.S = a.T = a.TX = a.TY = f2(0.f);
  // full 32-column blocks: lane = column, rows in order
  const int nch = nw >> 5;
  const bool shift = e.a11 == 1.f && e.a22 == 1.f && e.a12 == 0.f && e.a21 == 0.f;  // warp-uniform
  if (shift) {
    // v at row 0 (the general path's fmaf(1, Y, c5)); tv and the Keys
    // weights (a = -1/2) at it hold for every row
    const float rv0 = e.oy + e.c5, fv0 = floorf(rv0), tv = rv0 - fv0;
    const float t2 = tv * tv, t3 = t2 * tv;
    const float4 wv = make_float4(fmaf(-0.5f, t3, fmaf(-0.5f, tv, t2)),
                                  fmaf(1.5f, t3, fmaf(-2.5f, t2, 1.f)),
                                  fmaf(-1.5f, t3, fmaf(0.5f, tv, 2.f * t2)),
                                  0.5f * (t3 - t2));
    const int icy0 = (int)fv0;
    for (int ch = 0; ch < nch; ++ch) {
      const int col = (ch << 5) + lane;
      const float X = e.ox + (float)col;
      const float ru = X + e.c4, fu = floorf(ru), tu = ru - fu;
      const float4 *q = e.rc + icy0 * W + (int)fu;  // stencil row 0 of subset row 0
      const float2 *gp = e.gxy + col;
      float2 C = f2(0.f);
      float H[4];
      H[0] = horner3(__ldg(q), tu);
      H[1] = horner3(__ldg(q + W), tu);
      H[2] = horner3(__ldg(q + 2 * W), tu);
      q += 3 * W;
      float Y = e.oy;
      for (int r = 0; r < nw; r += 4, Y += 4.f, gp += 4 * W) {
        shift_row<SUB, 0>(H, q, W, tu, wv, e.cg, Y, gp, C, a);
        if (r + 1 < nw) shift_row<SUB, 1>(H, q, W, tu, wv, e.cg, Y + 1.f, gp + W, C, a);
        if (r + 2 < nw) shift_row<SUB, 2>(H, q, W, tu, wv, e.cg, Y + 2.f, gp + 2 * W, C, a);
        if (r + 3 < nw) shift_row<SUB, 3>(H, q, W, tu, wv, e.cg, Y + 3.f, gp + 3 * W, C, a);
      }
      a.T = __fadd2_rn(a.T, C);
      if (!SUB) a.TX = __ffma2_rn(C, f2(X), a.TX);
    }
  } else {
    for (int ch = 0; ch < nch; ++ch) {
      const int col = (ch << 5) + lane;
      const float X = e.ox + (float)col;
      const float bu = fmaf(e.a11, X, e.c4), bv = fmaf(e.a21, X, e.c5);
      const float2 *gp = e.gxy + col;
      float2 C = f2(0.f);
      float4 R[4];
      int pcx = INT_MIN, pcy = 0;
      float Y = e.oy;
      for (int r = 0; r < nw; r += 4, Y += 4.f, gp += 4 * W) {
        col_row<SUB, 0>(e, R, pcx, pcy, bu, bv, Y, gp, C, a);
        if (r + 1 < nw) col_row<SUB, 1>(e, R, pcx, pcy, bu, bv, Y + 1.f, gp + W, C, a);
        if (r + 2 < nw) col_row<SUB, 2>(e, R, pcx, pcy, bu, bv, Y + 2.f, gp + 2 * W, C, a);
        if (r + 3 < nw) col_row<SUB, 3>(e, R, pcx, pcy, bu, bv, Y + 3.f, gp + 3 * W, C, a);
      }
      a.T = __fadd2_rn(a.T, C);
      if (!SUB) a.TX = __ffma2_rn(C, f2(X), a.TX);
    }
  }
  // the remaining columns (one for a 33-pixel window), pixel per lane
  const int c0 = nch << 5, rem = nw - c0;
  if (rem) {
    const PixelMap<float> pm(rem, W);
    const int np = rem * nw;
    for (int p = lane; p < np; p += 32) {
      float rcol, rrow;
      const int k = c0 + pm.at(p, &rcol, &rrow);
      const float X = e.ox + (float)c0 + rcol, Y = e.oy + rrow;
      const float ru = fmaf(e.a11, X, fmaf(e.a12, Y, e.c4));
      const float rv = fmaf(e.a21, X, fmaf(e.a22, Y, e.c5));
      int iu, iv;
      const float fu = floor_i(ru, &iu), fv = floor_i(rv, &iv);
      const float4 *q = e.rc + iv * W + iu;
      const float d = cubic_rows(__ldg(q), __ldg(q + W), __ldg(q + 2 * W), __ldg(q + 3 * W),
                                 ru - fu, rv - fv) - e.cg;
      const float2 G = __ldg(e.gxy + k);
      const float2 D = f2(d);
      a.S = __ffma2_rn(D, f2(1.f, d), a.S);
      const float2 A = __fmul2_rn(G, D);
      a.T = __fadd2_rn(a.T, A);
      if (!SUB) {
        a.TX = __ffma2_rn(A, f2(X), a.TX);
        a.TY = __ffma2_rn(A, f2(Y), a.TY);
      }
    }
  }
  o[0] = a.S.x; o[1] = a.S.y; o[2] = a.TX.x; o[3] = a.TX.y;
  o[4] = a.TY.x; o[5] = a.TY.y; o[6] = a.T.x; o[7] = a.T.y;
}

// The FP32 setup sums of one subset (c the centre pixel's value): the
// zero-gradient count, a1 = sum (f - c), a2 = sum (f - c)^2, sk = sum sd_k,
// sfk = sum sd_k (f - c) with sd = [fx X, fy X, fx Y, fy Y, fx, fy], and the
// 18 distinct Hessian sums hh (index map in process()); lanes take columns
// as in eval32, the X weights applied once per column.
template <bool SUB>
__device__ __forceinline__ void setup32(const float *fI, const float2 *gxy, int W, int nw,
                                        int base, float ox, float oy, float c, int lane,
                                        int *cnt_out, float *a1o, float *a2o, float sk[6],
                                        float sfk[6], float hh[18]) {
  int cnt = 0;
  float a1 = 0.f, a2 = 0.f;
#pragma unroll
  for (int q = 0; q < 6; ++q) sk[q] = sfk[q] = 0.f;
#pragma unroll
  for (int q = 0; q < 18; ++q) hh[q] = 0.f;
  const int nch = nw >> 5;
  for (int ch = 0; ch < nch; ++ch) {
    const int col = (ch << 5) + lane;
    const float X = ox + (float)col;
    const float *fp = fI + base + col;
    const float2 *gp = gxy + base + col;
    // column sums, packed in pairs: (sum d, sum d^2), (sum fx, sum fy),
    // (sum fx d, sum fy d), their Y-weighted versions, and sum, sum Y,
    // sum Y^2 of (fxx, fxy) and of fyy
    float2 AD = f2(0.f), SG = f2(0.f), FD = f2(0.f), SGY = f2(0.f), FDY = f2(0.f);
    float2 H1 = f2(0.f), HY = f2(0.f), HYY = f2(0.f);
    float h1yy = 0.f, hYyy = 0.f, hYYyy = 0.f;
    float Y = oy;
#pragma unroll 4
    for (int r = 0; r < nw; ++r, Y += 1.f, fp += W, gp += W) {
      const float2 G = __ldg(gp);
      const float d = __ldg(fp) - c;
      cnt += G.x == 0.f;
      const float2 D = f2(d);
      AD = __ffma2_rn(D, f2(1.f, d), AD);
      SG = __fadd2_rn(SG, G);
      const float2 A = __fmul2_rn(G, D);
      FD = __fadd2_rn(FD, A);
      if (!SUB) {
        const float2 YP = f2(Y);
        SGY = __ffma2_rn(G, YP, SGY);
        FDY = __ffma2_rn(A, YP, FDY);
        const float2 FX = __fmul2_rn(f2(G.x), G);  // (fxx, fxy)
        const float fyy = G.y * G.y, YY = Y * Y;
        H1 = __fadd2_rn(H1, FX);
        HY = __ffma2_rn(YP, FX, HY);
        HYY = __ffma2_rn(f2(YY), FX, HYY);
        h1yy += fyy;
        hYyy = fmaf(Y, fyy, hYyy);
        hYYyy = fmaf(YY, fyy, hYYyy);
      }
    }
    a1 += AD.x;
    a2 += AD.y;
    sk[4] += SG.x;
    sk[5] += SG.y;
    sfk[4] += FD.x;
    sfk[5] += FD.y;
    if (!SUB) {
      const float XX = X * X;
      sk[0] = fmaf(X, SG.x, sk[0]);
      sk[1] = fmaf(X, SG.y, sk[1]);
      sk[2] += SGY.x;
      sk[3] += SGY.y;
      sfk[0] = fmaf(X, FD.x, sfk[0]);
      sfk[1] = fmaf(X, FD.y, sfk[1]);
      sfk[2] += FDY.x;
      sfk[3] += FDY.y;
      hh[0] = fmaf(XX, H1.x, hh[0]);
      hh[1] = fmaf(XX, H1.y, hh[1]);
      hh[2] = fmaf(X, HY.x, hh[2]);
      hh[3] = fmaf(X, HY.y, hh[3]);
      hh[4] = fmaf(X, H1.x, hh[4]);
      hh[5] = fmaf(X, H1.y, hh[5]);
      hh[6] = fmaf(XX, h1yy, hh[6]);
      hh[7] = fmaf(X, hYyy, hh[7]);
      hh[8] = fmaf(X, h1yy, hh[8]);
      hh[9] += HYY.x;
      hh[10] += HYY.y;
      hh[11] += HY.x;
      hh[12] += HY.y;
      hh[13] += hYYyy;
      hh[14] += hYyy;
      hh[15] += H1.x;
      hh[16] += H1.y;
      hh[17] += h1yy;
    }
  }
  const int c0 = nch << 5, rem = nw - c0;
  if (rem) {
    const PixelMap<float> pm(rem, W);
    const int np = rem * nw;
    for (int p = lane; p < np; p += 32) {
      float rc, rr;
      const int k = base + c0 + pm.at(p, &rc, &rr);
      const float2 G = __ldg(gxy + k);
      const float d = __ldg(fI + k) - c;
      cnt += G.x == 0.f;
      a1 += d;
      a2 = fmaf(d, d, a2);
      if (SUB) {
        sk[4] += G.x;
        sk[5] += G.y;
        sfk[4] = fmaf(G.x, d, sfk[4]);
        sfk[5] = fmaf(G.y, d, sfk[5]);
      } else {
        const float X = ox + (float)c0 + rc, Y = oy + rr;
        const float sd[6] = {G.x * X, G.y * X, G.x * Y, G.y * Y, G.x, G.y};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          sk[q] += sd[q];
          sfk[q] = fmaf(sd[q], d, sfk[q]);
        }
        const float fxx = G.x * G.x, fyy = G.y * G.y, fxy = G.x * G.y;
        const float XX = X * X, YY = Y * Y, XY = X * Y;
        hh[0] = fmaf(XX, fxx, hh[0]);  hh[1] = fmaf(XX, fxy, hh[1]);
        hh[2] = fmaf(XY, fxx, hh[2]);  hh[3] = fmaf(XY, fxy, hh[3]);
        hh[4] = fmaf(X, fxx, hh[4]);   hh[5] = fmaf(X, fxy, hh[5]);
        hh[6] = fmaf(XX, fyy, hh[6]);  hh[7] = fmaf(XY, fyy, hh[7]);
        hh[8] = fmaf(X, fyy, hh[8]);   hh[9] = fmaf(YY, fxx, hh[9]);
        hh[10] = fmaf(YY, fxy, hh[10]); hh[11] = fmaf(Y, fxx, hh[11]);
        hh[12] = fmaf(Y, fxy, hh[12]); hh[13] = fmaf(YY, fyy, hh[13]);
        hh[14] = fmaf(Y, fyy, hh[14]); hh[15] += fxx;
        hh[16] += fxy;                 hh[17] += fyy;
      }
    }
  }
  *cnt_out = cnt;
  *a1o = a1;
  *a2o = a2;
}

// MATLAB's catch branch (LocalICGN.m:75-80, Subpb1.m:89-92): -1 and NaN
template <bool SUB>
__device__ __forceinline__ void fail_minus1(const Args &a, long long s, int lane) {
  if (lane == 0) {
    if (!SUB && a.cache) a.cache[kIcgnCache * s + 7] = -1.0;
    a.iters[s] = -1;
    a.U[2 * s] = nan64();
    a.U[2 * s + 1] = nan64();
    if (!SUB) {
      for (int q = 0; q < 4; ++q) a.F[4 * s + q] = nan64();
      for (int q = 0; q < 21; ++q) a.H21out[(long long)q * a.n + s] = 0.0;
    }
  }
}

// more than half of the subset masked (funICGN.m:309-313): 102, P unchanged
template <bool SUB>
__device__ __forceinline__ void done_102(const Args &a, long long s, int lane) {
  if (lane == 0) {
    if (!SUB && a.cache) a.cache[kIcgnCache * s + 7] = 102.0;
    a.iters[s] = 102;
    a.U[2 * s] = a.U0[2 * s];
    a.U[2 * s + 1] = a.U0[2 * s + 1];
    if (!SUB) {
      for (int q = 0; q < 4; ++q) a.F[4 * s + q] = 0.0;
      for (int q = 0; q < 21; ++q) a.H21out[(long long)q * a.n + s] = 0.0;
    }
  }
}


// What one launch of the IC-GN kernel does for a subset: everything
// (MODE_FULL), the setup only -- status, window, sums and the Cholesky factor
// of H written to the per-subset cache record, H21 to its output --
// (MODE_SETUP), or the iterations from that record (MODE_ITER).  Splitting
// the FP32 LocalICGN in two leaves each launch fewer live registers, so more
// warps stay resident to hide the gathers' latency.
enum { MODE_FULL = 0, MODE_SETUP = 1, MODE_ITER = 2 };

// ws: per-warp shared scratch, H[36] at 0, its Cholesky factor L[21] at 36,
// S_f[6] at 57, S[6] at 63, 1 / diag(L) at 69, the warp parameters P[6] at 76
// and per-subset constants at 82 (x0, y0, the window's top-left offsets,
// bf, Subpb1's 2x2 factor, the first gradient norm), at 92 the FP32
// evaluation's fixed inputs (EvalBase) and at 98 the Eval32 block of the
// current evaluation, which eval32 reads from there -- values every lane
// holds alike,
// kept out of registers so that the evaluation's column loop has them to
// itself (fewer spills) and more warps stay resident
constexpr int WS = 108;

// the per-subset inputs of eval32 that stay fixed over the iterations
struct EvalBase {
  const float4 *rc;
  const float2 *gxy;
  int nw, w;
  float ox, oy, fx0, fy0, cg, pad;
};
static_assert(sizeof(EvalBase) <= 6 * sizeof(double), "EvalBase fits its scratch slots");
static_assert(sizeof(Eval32) <= 10 * sizeof(double), "Eval32 fits its scratch slots");

template <typename Real, bool SUB, int MODE>
__device__ void process(const Args &a, long long s, int lane, double *ws) {
  double *Lsh = ws + 36, *Sfs = ws + 57, *Sks = ws + 63, *Linv = ws + 69;
  const IcgnImages &im = a.im;
  const double x0 = a.coords[s], y0 = a.coords[a.n + s];
  int w = a.wins ? a.wins[s] : a.w;
  int xl, yl;
  const bool cached = (SUB && a.cache) || MODE == MODE_ITER;
  if (cached) {
    // the IC-GN launch of this frame already ran the setup on the same
    // reference image and window
    const double stc = a.cache[kIcgnCache * s + 7];
    if (stc == -1.0) {
      fail_minus1<SUB>(a, s, lane);
      return;
    }
    if (stc == 102.0) {
      done_102<SUB>(a, s, lane);
      return;
    }
    w = (int)a.cache[kIcgnCache * s + 6];
  }
  bool ok = subset_ok(im, x0, y0, w, &xl, &yl);
  if (!ok) {
    fail_minus1<SUB>(a, s, lane);
    return;
  }
  const Real *fI = Img<Real>::f(im);
  const int W = im.W;
  // One fused pass over the subset: the masked-pixel count of funICGN.m:54,
  // the Hessian sums of :67-79, and -- with a shift c (the subset's centre
  // pixel, keeping the one-pass variance well conditioned) -- sum(f - c),
  // sum(f - c)^2, S_k = sum sd_k and sum sd_k (f - c).  A 10-50 % masked
  // subset grows (funICGN.m:57-65) and the pass runs again on the new window.
  int nw, npx, base;
  Real ox, oy;
  double oxd, oyd, c0 = 0, A1 = 0, A2 = 0;
  double meanf, ssf;
  if (cached) {
    nw = w + 1;
    npx = nw * nw;
    oxd = (double)xl - x0;
    oyd = (double)yl - y0;
    ox = (Real)oxd;
    oy = (Real)oyd;
    base = (yl - 1) * W + (xl - 1);
    meanf = a.cache[kIcgnCache * s + 0];
    const double bfc = a.cache[kIcgnCache * s + 1];
    ssf = bfc * bfc;
    if (lane == 0) {
      Sfs[4] = a.cache[kIcgnCache * s + 2];
      Sfs[5] = a.cache[kIcgnCache * s + 3];
      Sks[4] = a.cache[kIcgnCache * s + 4];
      Sks[5] = a.cache[kIcgnCache * s + 5];
    }
    if (!SUB && MODE == MODE_ITER) {
      // the rest of the setup record: S_f0..3, S_0..3, L, 1 / diag(L)
      const double *cc = a.cache + kIcgnCache * s;
      for (int k = lane; k < 35; k += 32) {
        double *dst = k < 4 ? Sfs + k : (k < 8 ? Sks + (k - 4) : (k < 29 ? Lsh + (k - 8) : Linv + (k - 29)));
        *dst = cc[8 + k];
      }
    }
  } else {
  for (int attempt = 0;; ++attempt) {
    nw = w + 1;
    npx = nw * nw;
    oxd = (double)xl - x0;
    oyd = (double)yl - y0;
    ox = (Real)oxd;
    oy = (Real)oyd;
    base = (yl - 1) * W + (xl - 1);  // subset top-left, 0-based
    const Real c = fI[base + (nw / 2) * W + nw / 2];
    c0 = (double)c;
    int cnt = 0;
    Real a1 = 0, a2 = 0, sk[6], sfk[6], hh[18];
#pragma unroll
    for (int q = 0; q < 6; ++q) sk[q] = sfk[q] = 0;
#pragma unroll
    for (int q = 0; q < 18; ++q) hh[q] = 0;
    if constexpr (sizeof(Real) == 4) {
      setup32<SUB>(fI, im.gxy, W, nw, base, ox, oy, c, lane, &cnt, &a1, &a2, sk, sfk, hh);
    } else {
      const Grad64 grad(im);
      const PixelMap<Real> pm(nw, W);
      for (int p = lane; p < npx; p += 32) {
        Real rx, ry;
        const int k = base + pm.at(p, &rx, &ry);
        Real fx, fy;
        grad.at(k, &fx, &fy);
        const Real d = fI[k] - c;
        cnt += fx == (Real)0;
        a1 += d;
        a2 += d * d;
        if (SUB) {
          sk[4] += fx; sk[5] += fy;
          sfk[4] += fx * d; sfk[5] += fy * d;
        } else {
          const Real X = ox + rx, Y = oy + ry;
          const Real sd[6] = {fx * X, fy * X, fx * Y, fy * Y, fx, fy};
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            sk[q] += sd[q];
            sfk[q] += sd[q] * d;
          }
          const Real fxx = fx * fx, fyy = fy * fy, fxy = fx * fy;
          const Real XX = X * X, YY = Y * Y, XY = X * Y;
          hh[0] += XX * fxx;  hh[1] += XX * fxy;  hh[2] += XY * fxx;  hh[3] += XY * fxy;
          hh[4] += X * fxx;   hh[5] += X * fxy;   hh[6] += XX * fyy;  hh[7] += XY * fyy;
          hh[8] += X * fyy;   hh[9] += YY * fxx;  hh[10] += YY * fxy; hh[11] += Y * fxx;
          hh[12] += Y * fxy;  hh[13] += YY * fyy; hh[14] += Y * fyy;  hh[15] += fxx;
          hh[16] += fxy;      hh[17] += fyy;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    const double nn = (double)npx;
    if (attempt == 0) {
      if (!((double)cnt < 0.5 * nn)) {
        done_102<SUB>(a, s, lane);
        return;
      }
      if ((double)cnt > 0.1 * nn) {
        w = (int)round(sqrt(2.0) * w);
        if (!subset_ok(im, x0, y0, w, &xl, &yl)) {
          fail_minus1<SUB>(a, s, lane);
          return;
        }
        continue;
      }
    }
    {
      // the 32 sums in one transposed butterfly: lane l ends with sum l of
      // [a1, a2, S_k (6), sum sd_k (f - c) (6, corrected to f - mean f
      // below), the 18 distinct Hessian sums (staged in ws[0..17] until H is
      // expanded in place below)]
      double v[32];
      v[0] = (double)a1;
      v[1] = (double)a2;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        v[2 + q] = (double)sk[q];
        v[8 + q] = (double)sfk[q];
      }
#pragma unroll
      for (int q = 0; q < 18; ++q) v[14 + q] = (double)hh[q];
      const double t = warp_sum_t<32>(v, lane);
      A1 = __shfl_sync(0xffffffffu, t, 0);
      A2 = __shfl_sync(0xffffffffu, t, 1);
      if (lane >= 2 && lane < 8) Sks[lane - 2] = (SUB && lane < 6) ? 0.0 : t;
      else if (lane >= 8 && lane < 14) Sfs[lane - 8] = (SUB && lane < 12) ? 0.0 : t;
      else if (!SUB && lane >= 14) ws[lane - 14] = t;
      __syncwarp();
    }
    break;
  }
  const double dmc = A1 / (double)npx;  // mean(f) - c
  meanf = c0 + dmc;
  ssf = A2 - A1 * dmc;                  // sum (f - mean f)^2
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < 6; ++q) Sfs[q] -= dmc * Sks[q];  // sum sd_k (f - mean f)
    if (!SUB && a.cache) {
      double *cc = a.cache + kIcgnCache * s;
      cc[0] = meanf;
      cc[1] = sqrt(ssf);
      cc[2] = Sfs[4];
      cc[3] = Sfs[5];
      cc[4] = Sks[4];
      cc[5] = Sks[5];
      cc[6] = (double)w;
      cc[7] = 0.0;
      if (MODE == MODE_SETUP) {
        for (int q = 0; q < 4; ++q) {
          cc[8 + q] = Sfs[q];
          cc[12 + q] = Sks[q];
        }
      }
    }
  }
  }  // setup pass
  // P and the subset's constants in the warp's scratch (written by lane 0;
  // funICGN.m:39 starts from P = [0 0 0 0 u v], an external guess may give
  // the gradient terms too)
  double *const Pw = ws + 76, *const Gw = ws + 82;
  const double bf = sqrt(ssf);
  __syncwarp();
  if (lane == 0) {
    for (int q = 0; q < 4; ++q) Pw[q] = SUB ? a.FOld[4 * s + q] : (a.F0 ? a.F0[4 * s + q] : 0.0);
    Pw[4] = a.U0[2 * s];
    Pw[5] = a.U0[2 * s + 1];
    Gw[0] = x0;
    Gw[1] = y0;
    Gw[2] = oxd;
    Gw[3] = oyd;
    Gw[4] = bf;
  }

  // ---- Hessian factor (IC-GN) or the damped 2x2 system (Subpb1)
  double *Hm = ws;
  bool spd = true;
  double s2 = 0, l11i = 0, l21 = 0, l22i = 0;
  if (!SUB && MODE == MODE_ITER) {
    spd = a.cache[kIcgnCache * s + 43] != 0.0;
    __syncwarp();
  } else if (!SUB) {
    if (lane == 0) {
      // H of funICGN.m:67-79 from its 18 distinct sums (index map)
      const unsigned char map[36] = {0, 1, 2, 3, 4, 5,   1, 6, 3, 7, 5, 8,
                                     2, 3, 9, 10, 11, 12, 3, 7, 10, 13, 12, 14,
                                     4, 5, 11, 12, 15, 16, 5, 8, 12, 14, 16, 17};
      double q[18];
      for (int k = 0; k < 18; ++k) q[k] = ws[k];
      for (int k = 0; k < 36; ++k) Hm[k] = q[map[k]];
      spd = chol6(Hm, Lsh, Linv);
    }
    spd = __shfl_sync(0xffffffffu, (int)spd, 0);
    __syncwarp();
    if (MODE == MODE_SETUP) {
      // the record for the iteration launch, and H21 (funICGN.m:320)
      if (lane == 0) {
        double *cc = a.cache + kIcgnCache * s;
        for (int k = 0; k < 21; ++k) cc[16 + k] = Lsh[k];
        for (int k = 0; k < 6; ++k) cc[37 + k] = Linv[k];
        cc[43] = spd ? 1.0 : 0.0;
        int idx = 0;
        for (int c = 0; c < 6; ++c)
          for (int r = c; r < 6; ++r) a.H21out[(long long)(idx++) * a.n + s] = Hm[r * 6 + c];
      }
      return;
    }
  } else {
    __syncwarp();
    // funICGN_Subpb1.m:73,281-283
    s2 = 2.0 / (bf * bf);
    const double h55 = a.H21in[18 * a.n + s], h65 = a.H21in[19 * a.n + s],
                 h66 = a.H21in[20 * a.n + s];
    const double H2a = h55 * s2 + a.mu, H2b = h65 * s2, H2d = h66 * s2 + a.mu;
    const double dmax = H2a > H2d ? H2a : H2d;
    // the damped 2x2 matrix is fixed for the subset: factor it once
    const double Ha = H2a + 1e-3 * dmax, Hd = H2d + 1e-3 * dmax;
    const double l11 = sqrt(Ha);
    l11i = 1.0 / l11;
    l21 = H2b * l11i;
    l22i = 1.0 / sqrt(Hd - l21 * l21);
    if (lane == 0) {
      Gw[5] = s2;
      Gw[6] = l11i;
      Gw[7] = l21;
      Gw[8] = l22i;
    }
  }
  __syncwarp();

  // ---- iterations (funICGN.m:107-294 / funICGN_Subpb1.m:94-337)
  const double tol = a.tol;
  double normNew = 1, normAbs = 1;
  int step = 0;
  const Real cg = (Real)meanf;
  // u22 = x0 + ru: split x0 into its floor xb and fraction (0 or 1/2)
  const double xbd = floor(x0), ybd = floor(y0);
  const int xb = (int)xbd, yb = (int)ybd;
  const Real fx0 = (Real)(x0 - xbd), fy0 = (Real)(y0 - ybd);
  EvalBase *const eb = reinterpret_cast<EvalBase *>(ws + 92);
  if (sizeof(Real) == 4 && lane == 0) {
    eb->rc = im.gc + ((long long)(yb - 2) * W + (xb - 1));
    eb->gxy = im.gxy + base;
    eb->nw = nw;
    eb->w = w;
    eb->ox = (float)ox;
    eb->oy = (float)oy;
    eb->fx0 = (float)fx0;
    eb->fy0 = (float)fy0;
    eb->cg = (float)cg;
  }
  __syncwarp();
  while (step <= 100 && normNew > tol && normAbs > tol) {
    step++;
    double P[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) P[q] = Pw[q];
    // out-of-image test (funICGN.m:118): an affine map takes its extremes at
    // the subset corners
    bool out = false;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int wv = sizeof(Real) == 4 ? eb->w : w;
      const double X = (c & 1) ? Gw[2] + wv : Gw[2], Y = (c & 2) ? Gw[3] + wv : Gw[3];
      const double u22 = (1 + P[0]) * X + P[2] * Y + (Gw[0] + P[4]);
      const double v22 = P[1] * X + (1 + P[3]) * Y + (Gw[1] + P[5]);
      out |= (u22 < 3 || u22 > W - 2 || v22 < 3 || v22 > im.H - 2);
    }
    if (out) {
      normNew = 1e6;
      break;
    }
    bool pfin = true;
#pragma unroll
    for (int q = 0; q < 6; ++q) pfin &= isfinite(P[q]);
    double sums[8];
    if (!pfin) {
#pragma unroll
      for (int q = 0; q < 8; ++q) sums[q] = nan64();
    } else if constexpr (sizeof(Real) == 4) {
      Eval32 *const ep = reinterpret_cast<Eval32 *>(ws + 98);
      if (lane == 0) {
        Eval32 e;
        e.rc = eb->rc;
        e.gxy = eb->gxy;
        e.W = W; e.nw = eb->nw;
        e.ox = eb->ox; e.oy = eb->oy;
        e.a11 = (float)(1 + P[0]); e.a12 = (float)P[2]; e.a21 = (float)P[1]; e.a22 = (float)(1 + P[3]);
        e.c4 = (float)P[4] + eb->fx0; e.c5 = (float)P[5] + eb->fy0; e.cg = eb->cg;
        *ep = e;
      }
      __syncwarp();
      float o[8];
      eval32<SUB>(*ep, lane, o);
      if (SUB) {  // o[0], o[1], o[6], o[7]: totals at lanes 0, 8, 16, 24
        double v[4] = {(double)o[0], (double)o[1], (double)o[6], (double)o[7]};
        const double t = warp_sum_t<4>(v, lane);
        sums[0] = __shfl_sync(0xffffffffu, t, 0);
        sums[1] = __shfl_sync(0xffffffffu, t, 8);
        sums[6] = __shfl_sync(0xffffffffu, t, 16);
        sums[7] = __shfl_sync(0xffffffffu, t, 24);
        sums[2] = sums[3] = sums[4] = sums[5] = 0.0;
      } else {  // totals at lanes 0, 4, .., 28
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = (double)o[q];
        const double t = warp_sum_t<8>(v, lane);
#pragma unroll
        for (int q = 0; q < 8; ++q) sums[q] = __shfl_sync(0xffffffffu, t, 4 * q);
      }
    } else {
      const Real *gI = im.g64;
      const Grad64 grad(im);
      const Real a11 = (Real)(1 + P[0]), a12 = (Real)P[2], a21 = (Real)P[1],
                 a22 = (Real)(1 + P[3]), p4 = (Real)P[4], p5 = (Real)P[5];
      Real s1 = 0, s2r = 0, t[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) t[q] = 0;
      const PixelMap<Real> pm(nw, W);
      const Real c4 = p4 + fx0, c5 = p5 + fy0;
      // two pixels per trip pay off in the lighter Subpb1 loop only
      constexpr int kUnroll = SUB ? 2 : 1;
#pragma unroll kUnroll
      for (int p = lane; p < npx; p += 32) {
        Real rx, ry;
        const int k = base + pm.at(p, &rx, &ry);
        const Real X = ox + rx, Y = oy + ry;
        const Real ru = a11 * X + (a12 * Y + c4);
        const Real rv = a21 * X + (a22 * Y + c5);
        const Real fu = floor(ru), fv = floor(rv);
        const int cx = xb + (int)fu - 1, cy = yb + (int)fv - 1;  // 0-based floor corner
        const Real d = sample_minus(gI, W, cx, cy, ru - fu, rv - fv, cg);
        s1 += d;
        s2r += d * d;
        Real fx, fy;
        grad.at(k, &fx, &fy);
        const Real ax = fx * d, ay = fy * d;
        t[4] += ax;
        t[5] += ay;
        if (!SUB) {
          t[0] += ax * X;
          t[1] += ay * X;
          t[2] += ax * Y;
          t[3] += ay * Y;
        }
      }
      sums[0] = warp_sum((double)s1);
      sums[1] = warp_sum((double)s2r);
#pragma unroll
      for (int q = 0; q < 6; ++q) sums[2 + q] = (SUB && q < 4) ? 0.0 : warp_sum((double)t[q]);
    }
    __syncwarp();  // (P and the constants are read again from the scratch)
    const double n = sizeof(Real) == 4 ? (double)(eb->nw * eb->nw) : (double)npx;
    const double gm = sums[0] / n;                 // mean(g) - c
    const double ssg = sums[1] - sums[0] * gm;     // sum (g - gbar)^2
    const double bg = sqrt(ssg);
    // b_k = bf (S_fk / bf - (T_k - gm S_k) / bg) = S_fk - (bf / bg)(T_k - gm S_k)
    // (a flat reference subset, bf = 0, stays NaN as the division gives it)
    const double bfw = Gw[4];
    const double rfg = bfw > 0.0 ? bfw / bg : nan64();
    double b[6], nb = 0;
    if (!SUB) {
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        b[q] = Sfs[q] - rfg * (sums[2 + q] - gm * Sks[q]);
        nb += b[q] * b[q];
      }
    } else {
      const double b5 = Sfs[4] - rfg * (sums[6] - gm * Sks[4]);
      const double b6 = Sfs[5] - rfg * (sums[7] - gm * Sks[5]);
      const double s2w = Gw[5];
      b[4] = b5 * s2w + a.mu * (Pw[4] - a.U0[2 * s] - a.vdual[2 * s]);
      b[5] = b6 * s2w + a.mu * (Pw[5] - a.U0[2 * s + 1] - a.vdual[2 * s + 1]);
      nb = b[4] * b[4] + b[5] * b[5];
    }
    normNew = sqrt(nb);
    normAbs = normNew;
    const double normInit = step == 1 ? normNew : Gw[9];
    if (step == 1 && lane == 0) Gw[9] = normNew;
    if (normInit > tol) normNew = normNew / normInit;
    else normNew = 0;
    if (normNew < tol || normAbs < tol) break;
    double dP[6] = {0, 0, 0, 0, 0, 0};
    if (!SUB) {
      if (spd) {
        chol6_solve(Lsh, Linv, b, dP);
#pragma unroll
        for (int q = 0; q < 6; ++q) dP[q] = -dP[q];
      } else {
#pragma unroll
        for (int q = 0; q < 6; ++q) dP[q] = nan64();
      }
    } else {
      // 2x2 SPD solve with the Cholesky factor of the damped matrix
      const double f11i = Gw[6], f21 = Gw[7], f22i = Gw[8];
      const double y1 = b[4] * f11i, y2 = (b[5] - f21 * y1) * f22i;
      const double x2 = y2 * f22i, x1 = (y1 - f21 * x2) * f11i;
      dP[4] = -x1;
      dP[5] = -x2;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) P[q] = Pw[q];
    if (!ic_compose(P, dP)) break;
    __syncwarp();
    if (lane == 0)
      for (int q = 0; q < 6; ++q) Pw[q] = P[q];
    __syncwarp();
  }
  __syncwarp();
  if (!(normNew < tol || normAbs < tol)) step = 101;
  if (isnan(normNew)) step = 101;
  if (lane == 0) {
    a.iters[s] = step;
    a.U[2 * s] = Pw[4];
    a.U[2 * s + 1] = Pw[5];
    if (!SUB) {
      for (int q = 0; q < 4; ++q) a.F[4 * s + q] = Pw[q];
      if (MODE == MODE_FULL) {
        int idx = 0;
        for (int c = 0; c < 6; ++c)
          for (int r = c; r < 6; ++r) a.H21out[(long long)(idx++) * a.n + s] = Hm[r * 6 + c];
      }
    }
  }
}

// Launch shapes the autotuner chooses from: NW warps per CTA and MINB
// resident CTAs per SM in the launch bounds (NW * 32 * MINB threads share
// the SM's 64 K registers, so MINB sets the register cap: 8 x 4 and 4 x 8 ->
// 64 registers, 8 x 3 -> 80, 8 x 2 -> 128, 4 x 6 -> 80, 16 x 2 -> 64,
// 4 x 5 -> 96 (rounded to the allocation unit); FP64: 8 x 2 -> 128, 4 x 3 ->
// 168).  Every shape runs the same per-subset code,
// so the results are bit-identical and only the time differs.
template <typename Real, bool SUB, int MODE, int NW, int MINB>
__global__ void __launch_bounds__(NW * 32, MINB) k_icgn(Args a) {
  __shared__ double Lsh[NW][WS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned int s = 0;
  if (lane == 0) s = atomicAdd(a.queue, 1u);
  s = __shfl_sync(0xffffffffu, s, 0);
  while ((long long)s < a.n) {
    // the next subset's index is requested before this one is processed, so
    // the atomic's round trip overlaps the work
    unsigned int next = 0;
    if (lane == 0) next = atomicAdd(a.queue, 1u);
    process<Real, SUB, MODE>(a, (long long)s, lane, Lsh[wid]);
    __syncwarp();
    s = __shfl_sync(0xffffffffu, next, 0);
  }
}

struct Shape {
  int nw, minb;
  const void *fn;
};

template <typename Real, bool SUB, int MODE>
std::vector<Shape> make_shapes() {
  if constexpr (sizeof(Real) == 4)
    return {{8, 4, (const void *)k_icgn<Real, SUB, MODE, 8, 4>},
            {8, 3, (const void *)k_icgn<Real, SUB, MODE, 8, 3>},
            {8, 2, (const void *)k_icgn<Real, SUB, MODE, 8, 2>},
            {4, 8, (const void *)k_icgn<Real, SUB, MODE, 4, 8>},
            {4, 6, (const void *)k_icgn<Real, SUB, MODE, 4, 6>},
            {16, 2, (const void *)k_icgn<Real, SUB, MODE, 16, 2>},
            {4, 5, (const void *)k_icgn<Real, SUB, MODE, 4, 5>}};
  else
    return {{8, 2, (const void *)k_icgn<Real, SUB, MODE, 8, 2>},
            {4, 3, (const void *)k_icgn<Real, SUB, MODE, 4, 3>}};
}

template <typename Real, bool SUB, int MODE>
const std::vector<Shape> &shapes() {
  static const std::vector<Shape> v = make_shapes<Real, SUB, MODE>();
  return v;
}

int launch_shape(const Shape &sh, const Args &a, cudaStream_t st) {
  int dev = 0, sms = 148, per = 1;
  ALDIC_CUDA(cudaGetDevice(&dev));
  ALDIC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  ALDIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sh.fn, sh.nw * 32, 0));
  if (per < 1) per = 1;
  long long blocks = (long long)sms * per;  // persistent: every resident CTA, one wave
  const long long need = (a.n + sh.nw - 1) / sh.nw;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  ALDIC_CUDA(cudaMemsetAsync(a.queue, 0, sizeof(unsigned int), st));
  Args arg = a;
  void *args[] = {&arg};
  ALDIC_CUDA(cudaLaunchKernel(sh.fn, dim3((unsigned)blocks), dim3(sh.nw * 32), args, 0, st));
  return OK;
}

// ---------------------------------------------------------------- autotuner
// The launch shape per (precision, instance, device, subset size, log2 of
// the subset count) is picked by timed trials on the first launch that may
// synchronise (not inside a stream capture): every shape runs twice on the
// call's own data and the faster second run wins.  The choice is kept for
// the process; a launch inside a capture before any trial uses shape 0.
struct TuneKey {
  int prec, sub, dev, w, nlog;
  bool operator<(const TuneKey &o) const {
    if (prec != o.prec) return prec < o.prec;
    if (sub != o.sub) return sub < o.sub;
    if (dev != o.dev) return dev < o.dev;
    if (w != o.w) return w < o.w;
    return nlog < o.nlog;
  }
};
struct TuneVal {
  int shape;
  float ms[8];
  int count;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;
bool g_tune_on = true;

// instance: 0 the LocalICGN iteration launch, 1 Subpb1, 2 the LocalICGN
// setup launch, 3 LocalICGN in one launch
int instance_of(bool sub, int mode) {
  return sub ? 1 : (mode == MODE_SETUP ? 2 : (mode == MODE_ITER ? 0 : 3));
}
TuneKey tune_key(int prec, int inst, int w, long long n) {
  int dev = 0;
  cudaGetDevice(&dev);
  int nl = 0;
  while ((1LL << (nl + 1)) <= n) ++nl;
  return TuneKey{prec, inst, dev, w, nl};
}

template <typename Real, bool SUB, int MODE>
int launch(const Args &a, cudaStream_t st) {
  const auto &sv = shapes<Real, SUB, MODE>();
  const TuneKey key = tune_key(sizeof(Real) == 8, instance_of(SUB, MODE), a.wins ? -1 : a.w, a.n);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return launch_shape(sv[it->second.shape], a, st);
    if (!g_tune_on) return launch_shape(sv[0], a, st);
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ALDIC_CUDA(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone || a.n < 2048) return launch_shape(sv[0], a, st);
  cudaEvent_t e0, e1;
  ALDIC_CUDA(cudaEventCreate(&e0));
  ALDIC_CUDA(cudaEventCreate(&e1));
  TuneVal tv{};
  tv.count = (int)sv.size();
  int rc = OK;
  for (size_t k = 0; k < sv.size() && rc == OK; ++k) {
    float ms = 0.f;
    for (int rep = 0; rep < 2 && rc == OK; ++rep) {
      cudaEventRecord(e0, st);
      rc = launch_shape(sv[k], a, st);
      cudaEventRecord(e1, st);
      if (rc == OK && (cudaEventSynchronize(e1) != cudaSuccess ||
                       cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)) {
        set_error("icgn autotune: timing failed");
        rc = E_CUDA;
      }
    }
    tv.ms[k] = ms;
    if (ms < tv.ms[tv.shape]) tv.shape = (int)k;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  // the outputs of the last trial stand (every shape computes the same)
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = tv;
  return OK;
}

}  // namespace

int icgn(const IcgnImages &im, const double *coords, long long n, const double *U0,
         const int *wins, int w, double tol, int precision, double *U, double *F, int *iters,
         double *H21, unsigned int *queue, cudaStream_t st, double *cache, const double *F0) {
  if (n <= 0) return OK;
  Args a{};
  a.cache = cache;
  a.F0 = F0;
  a.im = im; a.coords = coords; a.n = n; a.U0 = U0; a.wins = wins; a.w = w; a.tol = tol;
  a.U = U; a.F = F; a.H21out = H21; a.iters = iters; a.queue = queue;
  if (precision) return launch<double, false, MODE_FULL>(a, st);
  if (!cache) return launch<float, false, MODE_FULL>(a, st);
  // FP32 with a setup record: setup launch, then the iterations from it
  const int rc = launch<float, false, MODE_SETUP>(a, st);
  return rc ? rc : launch<float, false, MODE_ITER>(a, st);
}

bool icgn_tuned(int precision, bool sub, int w, long long n) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (!g_tune_on || n < 2048) return true;
  const int p = precision ? 1 : 0;
  if (sub) return g_tune.count(tune_key(p, 1, w, n)) != 0;
  if (precision) return g_tune.count(tune_key(p, 3, w, n)) != 0;
  return g_tune.count(tune_key(p, 0, w, n)) != 0 && g_tune.count(tune_key(p, 2, w, n)) != 0;
}

void icgn_autotune(bool on) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_on = on;
  if (!on) g_tune.clear();
}

int icgn_tuned_shape(int precision, int instance, int w, long long n, int *nwarps, int *minb,
                     float ms[8], int *count) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const int p = precision ? 1 : 0;
  auto it = g_tune.find(tune_key(p, instance, w, n));
  if (it == g_tune.end() && instance == 0) it = g_tune.find(tune_key(p, 3, w, n));
  if (it == g_tune.end()) return E_STATE;
  // every mode's shape table has the same (warps, CTAs) entries
  const auto &sv = precision ? (instance == 1 ? shapes<double, true, MODE_FULL>()
                                              : shapes<double, false, MODE_FULL>())
                             : (instance == 1 ? shapes<float, true, MODE_FULL>()
                                              : shapes<float, false, MODE_FULL>());
  const Shape &sh = sv[it->second.shape];
  if (nwarps) *nwarps = sh.nw;
  if (minb) *minb = sh.minb;
  if (count) *count = it->second.count;
  if (ms)
    for (int k = 0; k < 8; ++k) ms[k] = k < it->second.count ? it->second.ms[k] : 0.f;
  return OK;
}

int subpb1(const IcgnImages &im, const double *coords, long long n, const double *UOld,
           const double *FOld, const double *vdual, const double *H21, const int *wins, int w,
           double mu, double tol, int precision, double *U, int *iters, unsigned int *queue,
           cudaStream_t st, const double *cache) {
  if (n <= 0) return OK;
  Args a{};
  a.cache = const_cast<double *>(cache);
  a.im = im; a.coords = coords; a.n = n; a.U0 = UOld; a.FOld = FOld; a.vdual = vdual;
  a.H21in = H21; a.wins = wins; a.w = w; a.mu = mu; a.tol = tol; a.U = U; a.iters = iters;
  a.queue = queue;
  // with the LocalICGN record the setup is skipped: the iteration-only
  // instance, which carries no setup code (fewer registers)
  if (cache)
    return precision ? launch<double, true, MODE_ITER>(a, st) : launch<float, true, MODE_ITER>(a, st);
  return precision ? launch<double, true, MODE_FULL>(a, st) : launch<float, true, MODE_FULL>(a, st);
}

}  // namespace aldic
