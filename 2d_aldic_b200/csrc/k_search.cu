// k_search.cu -- whole-field integer search (funIntegerSearch.m:82-200,
// findpeak.m:26-66, compute_qFactor :211-264).
//
// One CTA per grid point.  The template C = f(ii:ii+w, jj:jj+w) and the
// region D = g(ii-s:ii+w+s, jj-s:jj+w+s) are staged in shared memory (D with
// a zero border), each thread owns a strip of KX horizontally adjacent
// shifts and slides the template over D with the strip held in registers.
// On 8-bit images every template row's partial correlation is an exact
// integer in FP32 (<= 65 * 255^2 < 2^24) and is flushed to a 64-bit integer,
// so the correlation maps are exact; 16-bit images use 32x32->64-bit integer
// multiply-adds.  The normalised cross-correlation is then formed from those
// integers with a fixed FP64 formula (explicit rounding, no contraction)
// shared with the CPU restatement, which makes argmax and the 1e-3-rounded
// sub-pixel peak bit-identical to it.
#include <algorithm>

#include "aldic_internal.cuh"
#include "kernels.cuh"
#include "ncc.cuh"

namespace aldic {

namespace {

constexpr int KX = 8;

template <typename T> struct SearchTraits;
template <> struct SearchTraits<uint8_t> {
  using V = float;           // shared-memory value type
  using RowAcc = float;      // exact per template row
  static __device__ __forceinline__ RowAcc mac(RowAcc a, V t, V d) { return fmaf(t, d, a); }
  static constexpr bool integer = true;
};
template <> struct SearchTraits<uint16_t> {
  using V = unsigned int;
  using RowAcc = unsigned long long;
  static __device__ __forceinline__ RowAcc mac(RowAcc a, V t, V d) {
    return a + (unsigned long long)(t * d);
  }
  static constexpr bool integer = true;
};
template <> struct SearchTraits<float> {
  using V = double;
  using RowAcc = double;
  static __device__ __forceinline__ RowAcc mac(RowAcc a, V t, V d) { return fma(t, d, a); }
  static constexpr bool integer = false;
};
template <> struct SearchTraits<double> : SearchTraits<float> {};

// S = integral sums type of the box sums
template <bool INT> struct SumT { using type = long long; };
template <> struct SumT<false> { using type = double; };

struct SearchGeom {
  int W, H;
  int gx1, gy1, nx, ny, step;
  int w, sx, sy;
  int tw, twp, dw, dh, cr, cc, nsx, dpw, dph;
  const double *mu;  // device pointer: ROI mean of the deformed image
};

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

// Shared-memory layout of the per-point kernel.  With big = true (search
// regions whose window row sums and correlation map exceed the 227 KB of
// shared memory a CTA may have) the row sums RS, RS2 and the map live in a
// per-CTA slot of global work memory instead (`slot` bytes each, offsets
// g_rs, g_rs2, g_map) and shared memory holds the template and the region.
template <typename V, typename S>
struct SmemLayout {
  size_t tp, dp, rs, rs2, colsum, rowsum, map, red, total;
  size_t g_rs, g_rs2, g_map, slot;
  __host__ __device__ SmemLayout(const SearchGeom &g, bool big = false) {
    size_t o = 0;
    tp = o; o = align16(o + sizeof(V) * g.tw * g.twp);
    dp = o; o = align16(o + sizeof(V) * g.dph * g.dpw);
    const size_t brs = align16(sizeof(S) * g.dph * g.cr), bmap = align16(sizeof(double) * g.cr * g.cc);
    g_rs = 0;
    g_rs2 = brs;
    g_map = 2 * brs;
    slot = (2 * brs + bmap + 255) & ~size_t(255);
    rs = rs2 = map = 0;
    if (!big) {
      rs = o; o += brs;
      rs2 = o; o += brs;
    }
    colsum = o; o = align16(o + sizeof(S) * g.tw);
    rowsum = o; o = align16(o + sizeof(S) * g.tw);
    if (!big) {
      map = o; o += bmap;
    }
    red = o; o = align16(o + (sizeof(double) + sizeof(int)) * 32 + 64);
    total = o;
  }
};

// Argmax of the cropped map (first maximum in column-major order, as
// MATLAB's max), the sub-pixel fit of findpeak.m and the outputs of
// funIntegerSearch.m:148-159.  Called by all threads of the block.
__device__ void peak_epilogue(const double *map, const SearchGeom &G, int ii, int jj,
                              long long out_idx, double *redv, int *redi, double *ox,
                              double *oy, double *ou, double *ov, double *occ) {
  const int tid = threadIdx.x, nth = blockDim.x;
  double best = -1e300;
  int bi = 0x7fffffff;
  const int nm = G.cr * G.cc;
  for (int i = tid; i < nm; i += nth) {
    const double v = map[i];
    if (v > best || (v == best && i < bi)) {
      best = v;
      bi = i;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  if ((tid & 31) == 0) {
    redv[tid >> 5] = best;
    redi[tid >> 5] = bi;
  }
  __syncthreads();
  if (tid == 0) {
    for (int k = 1; k < (nth + 31) / 32; ++k)
      if (redv[k] > best || (redv[k] == best && redi[k] < bi)) {
        best = redv[k];
        bi = redi[k];
      }
    double rpk, cpk, mf;
    findpeak_fit(map, G.cr, G.cc, bi, &rpk, &cpk, &mf);
    ox[out_idx] = (ii + ii + G.w) / 2.0;
    oy[out_idx] = (jj + jj + G.w) / 2.0;
    ou[out_idx] = __dsub_rn(rpk, (double)(G.sx + 2));
    ov[out_idx] = __dsub_rn(cpk, (double)(G.sy + 2));
    occ[out_idx] = mf;
  }
}

// Template pixels of a placement that fall into the padding: column t is
// outside when t + a - 1 lies outside [0, dw), row t when t + b - 1 lies
// outside [0, dh).  Returns their template sum and count.
template <typename S, typename TV>
__device__ __forceinline__ void pad_terms(const SearchGeom &G, int a, int b, const S *colsum,
                                          const S *rowsum, TV tpix, S *st_out, long long *n_out) {
  S so = 0;
  long long nco = 0, nro = 0;
  for (int t = 0; t < G.tw; ++t) {
    const int xo = t + a - 1, yo = t + b - 1;
    if (xo < 0 || xo >= G.dw) { so += colsum[t]; nco++; }
    if (yo < 0 || yo >= G.dh) { so += rowsum[t]; nro++; }
  }
  if (nco && nro) {
    for (int ty = 0; ty < G.tw; ++ty) {
      const int yo = ty + b - 1;
      if (!(yo < 0 || yo >= G.dh)) continue;
      for (int tx = 0; tx < G.tw; ++tx) {
        const int xo = tx + a - 1;
        if (xo < 0 || xo >= G.dw) so -= (S)tpix(ty, tx);
      }
    }
  }
  *st_out = so;
  *n_out = nco * G.tw + nro * G.tw - nco * nro;
}

// One CTA per grid point at a time, looping over the points (grid-stride):
// with BIG the row sums and the map of the CTA's current point are in its
// slot of the global work memory `work` (SmemLayout).
template <typename T, bool BIG>
__global__ void __launch_bounds__(512) k_search(const T *__restrict__ f, const T *__restrict__ g,
                                                SearchGeom G, double *__restrict__ ox,
                                                double *__restrict__ oy, double *__restrict__ ou,
                                                double *__restrict__ ov, double *__restrict__ occ,
                                                unsigned char *__restrict__ work) {
  using Tr = SearchTraits<T>;
  using V = typename Tr::V;
  using RowAcc = typename Tr::RowAcc;
  using S = typename SumT<Tr::integer>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout<V, S> L(G, BIG);
  unsigned char *wk = BIG ? work + (size_t)blockIdx.x * L.slot : nullptr;
  V *Tp = (V *)(smem + L.tp);
  V *Dp = (V *)(smem + L.dp);
  S *RS = BIG ? (S *)(wk + L.g_rs) : (S *)(smem + L.rs);
  S *RS2 = BIG ? (S *)(wk + L.g_rs2) : (S *)(smem + L.rs2);
  S *colsum = (S *)(smem + L.colsum);
  S *rowsum = (S *)(smem + L.rowsum);
  double *map = BIG ? (double *)(wk + L.g_map) : (double *)(smem + L.map);
  double *redv = (double *)(smem + L.red);
  int *redi = (int *)(redv + 32);
  __shared__ S s_st, s_st2;
  const double mu = *G.mu;

  for (int pt = blockIdx.x; pt < G.nx * G.ny; pt += gridDim.x) {
  const int ix = pt % G.nx, iy = pt / G.nx;
  const int ii = G.gx1 + ix * G.step, jj = G.gy1 + iy * G.step;  // 1-based
  const int tid = threadIdx.x, nth = blockDim.x;

  // ---- stage template (zero-padded to twp columns) and padded region
  for (int i = tid; i < G.tw * G.twp; i += nth) {
    const int ty = i / G.twp, tx = i % G.twp;
    V v = 0;
    if (tx < G.tw) v = (V)f[(long long)(jj - 1 + ty) * G.W + (ii - 1 + tx)];
    Tp[i] = v;
  }
  for (int i = tid; i < G.dph * G.dpw; i += nth) {
    const int y = i / G.dpw, x = i % G.dpw;
    V v = 0;
    if (y >= 1 && y <= G.dh && x >= 1 && x <= G.dw)
      v = (V)g[(long long)(jj - 1 - G.sy + y - 1) * G.W + (ii - 1 - G.sx + x - 1)];
    Dp[i] = v;
  }
  __syncthreads();
  // ---- template row/column sums, window row sums of D and D^2
  for (int i = tid; i < G.tw; i += nth) {
    S cs = 0, rs = 0;
    for (int k = 0; k < G.tw; ++k) {
      cs += (S)Tp[k * G.twp + i];
      rs += (S)Tp[i * G.twp + k];
    }
    colsum[i] = cs;
    rowsum[i] = rs;
  }
  for (int i = tid; i < G.dph * G.cr; i += nth) {
    const int y = i / G.cr, oxx = i % G.cr;
    S a = 0, a2 = 0;
    const V *row = Dp + y * G.dpw + oxx;
    for (int k = 0; k < G.tw; ++k) {
      const S v = (S)row[k];
      a += v;
      a2 += v * v;
    }
    RS[i] = a;
    RS2[i] = a2;
  }
  if (tid < 32) {
    S a = 0, a2 = 0;
    for (int i = tid; i < G.tw * G.twp; i += 32) {
      const S v = (S)Tp[i];
      a += v;
      a2 += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (tid == 0) {
      s_st = a;
      s_st2 = a2;
    }
  }
  __syncthreads();
  const S st = s_st, st2 = s_st2;
  const long long mn = (long long)G.tw * G.tw;
  bool flat;
  if (Tr::integer) flat = ((long long)mn * (long long)st2 - (long long)st * (long long)st) == 0;
  else flat = !((double)mn * (double)st2 - (double)st * (double)st > 0.0);
  const long long out_idx = (long long)iy + (long long)ix * G.ny;
  if (flat) {
    // normxcorr2 rejects a constant template: funIntegerSearch.m:153-157
    if (tid == 0) {
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      ox[out_idx] = (ii + ii + G.w) / 2.0;
      oy[out_idx] = (jj + jj + G.w) / 2.0;
      ou[out_idx] = nan;
      ov[out_idx] = nan;
      occ[out_idx] = nan;
    }
    __syncthreads();  // the next point restages the template
    continue;
  }

  // ---- correlation strips
  const int nstrips = G.cc * G.nsx;
  for (int sidx = tid; sidx < nstrips; sidx += nth) {
    const int b = sidx / G.nsx;          // window row start in padded coords
    const int a0 = (sidx % G.nsx) * KX;  // first window column
    S acc[KX];
#pragma unroll
    for (int k = 0; k < KX; ++k) acc[k] = 0;
    for (int ty = 0; ty < G.tw; ++ty) {
      const V *Drow = Dp + (b + ty) * G.dpw + a0;
      const V *Trow = Tp + ty * G.twp;
      RowAcc ra[KX];
      V win[KX];
#pragma unroll
      for (int k = 0; k < KX; ++k) ra[k] = 0;
#pragma unroll
      for (int k = 0; k < KX - 1; ++k) win[k] = Drow[k];
      for (int tx0 = 0; tx0 < G.twp; tx0 += KX) {
#pragma unroll
        for (int j = 0; j < KX; ++j) {
          win[(j + KX - 1) % KX] = Drow[tx0 + j + KX - 1];
          const V t = Trow[tx0 + j];
#pragma unroll
          for (int k = 0; k < KX; ++k) ra[k] = Tr::mac(ra[k], t, win[(j + k) % KX]);
        }
      }
#pragma unroll
      for (int k = 0; k < KX; ++k) acc[k] += (S)ra[k];
    }
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      const int a = a0 + k;
      if (a >= G.cr) break;
      S sd = 0, sd2 = 0;
      for (int ty = 0; ty < G.tw; ++ty) {
        sd += RS[(b + ty) * G.cr + a];
        sd2 += RS2[(b + ty) * G.cr + a];
      }
      S st_out;
      long long n_out;
      pad_terms<S>(G, a, b, colsum, rowsum, [&](int ty, int tx) { return Tp[ty * G.twp + tx]; },
                   &st_out, &n_out);
      double r;
      if (Tr::integer)
        r = ncc_combine(mn, (long long)st, (long long)st2, (long long)acc[k], (long long)sd,
                        (long long)sd2, (long long)st_out, n_out, mu);
      else
        r = ncc_combine_f((double)mn, (double)st, (double)st2, (double)acc[k], (double)sd,
                          (double)sd2, (double)st_out, (double)n_out, mu);
      map[b * G.cr + a] = r;
    }
  }
  __syncthreads();
  peak_epilogue(map, G, ii, jj, out_idx, redv, redi, ox, oy, ou, ov, occ);
  __syncthreads();  // the next point overwrites the staging and the map
  }
}

// ---- 8-bit images: byte-packed correlation with __dp4a (exact int32).
// The padded region is staged once as aligned 32-bit words (4 pixels each);
// the 4-pixel window starting at any column is one funnel shift of two
// neighbouring words, and the template row is packed 4 pixels per word.  A
// thread owns 8 consecutive shifts of one window row: per template word it
// loads one template word and one region word, forms 8 windows and issues 8
// dp4a -- 32 exact multiply-adds.
struct U8Layout {
  int tw4, dqw;  // template words per row, region words per row (odd pitch)
  size_t tb, dw, tq, rs, cs, map, red, total;
  __host__ __device__ U8Layout(const SearchGeom &g) {
    tw4 = (g.tw + 3) / 4;
    // words read: up to (nsx-1)*2 + tw4 + 1; the bytes must also hold the
    // padded region (dw + 2) and the row-sum window (cr + tw)
    int need = 2 * g.nsx + tw4 + 2;
    const int nb = (g.cr + g.tw + 3) / 4 + 1;
    if (need < nb) need = nb;
    dqw = need | 1;  // odd pitch: the rows a warp touches fall on different banks
    size_t o = 0;
    tb = o; o = align16(o + (size_t)g.tw * g.tw);
    dw = o; o = align16(o + sizeof(unsigned) * g.dph * dqw);
    tq = o; o = align16(o + sizeof(unsigned) * g.tw * tw4);
    // window row sums RS, RS2 (dph x cr each); dead once the box sums are
    // formed, after which the NCC map (cr x cc doubles) reuses the space
    rs = o;
    const size_t rsz = sizeof(int) * 2 * g.dph * g.cr, msz = sizeof(double) * g.cr * g.cc;
    o = align16(o + (rsz > msz ? rsz : msz));
    map = rs;
    cs = o; o = align16(o + sizeof(int) * 2 * g.cc * g.cr);  // box sums of D and D^2
    red = o; o = align16(o + (sizeof(double) + sizeof(int)) * 32 + 64);
    total = o;
  }
};

__device__ __forceinline__ void search_point_u8(const uint8_t *__restrict__ f,
                                                const uint8_t *__restrict__ g,
                                                const SearchGeom &G, const int pt,
                                                double *__restrict__ ox, double *__restrict__ oy,
                                                double *__restrict__ ou, double *__restrict__ ov,
                                                double *__restrict__ occ) {
  extern __shared__ __align__(16) unsigned char smem[];
  const U8Layout L(G);
  uint8_t *Tb = smem + L.tb;                 // template bytes, tw x tw
  unsigned *Dw = (unsigned *)(smem + L.dw);  // padded region, dph rows of dqw words
  const uint8_t *Db = (const uint8_t *)Dw;   // the same, as bytes (row pitch 4*dqw)
  unsigned *Tq = (unsigned *)(smem + L.tq);
  int *RS = (int *)(smem + L.rs);
  int *RS2 = RS + G.dph * G.cr;
  int *CS = (int *)(smem + L.cs);
  int *CS2 = CS + G.cc * G.cr;
  double *map = (double *)(smem + L.map);
  double *redv = (double *)(smem + L.red);
  int *redi = (int *)(redv + 32);
  __shared__ long long s_st, s_st2;
  __shared__ int colsum_s[72], rowsum_s[72];
  const double mu = *G.mu;
  const int ix = pt % G.nx, iy = pt / G.nx;
  const int ii = G.gx1 + ix * G.step, jj = G.gy1 + iy * G.step;  // 1-based
  const int tid = threadIdx.x, nth = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nwarp = nth >> 5;
  const uint8_t *trow0 = f + (long long)(jj - 1) * G.W + (ii - 1);
  const uint8_t *drow0 = g + (long long)(jj - 1 - G.sy) * G.W + (ii - 1 - G.sx);
  const int dbp = 4 * L.dqw;  // byte pitch
  // ---- stage template bytes and the padded region (warp per row, lanes over
  // columns; 1-pixel zero border at the top/left, zeros beyond the region)
  for (int ty = wid; ty < G.tw; ty += nwarp)
    for (int tx = lane; tx < G.tw; tx += 32) Tb[ty * G.tw + tx] = trow0[(long long)ty * G.W + tx];
  for (int y = wid; y < G.dph; y += nwarp) {
    const bool rin = y >= 1 && y <= G.dh;
    const uint8_t *src = drow0 + (long long)(y - 1) * G.W;
    for (int w4 = lane; w4 < L.dqw; w4 += 32) {
      unsigned v = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int x = 4 * w4 + k;
        if (rin && x >= 1 && x <= G.dw) v |= (unsigned)src[x - 1] << (8 * k);
      }
      Dw[y * L.dqw + w4] = v;
    }
  }
  __syncthreads();
  // ---- packed template words, window row sums, template sums
  for (int ty = wid; ty < G.tw; ty += nwarp)
    for (int w4 = lane; w4 < L.tw4; w4 += 32) {
      unsigned v = 0;
      for (int k = 0; k < 4; ++k) {
        const int tx = 4 * w4 + k;
        if (tx < G.tw) v |= (unsigned)Tb[ty * G.tw + tx] << (8 * k);
      }
      Tq[ty * L.tw4 + w4] = v;
    }
  for (int y = tid; y < G.dph; y += nth) {
    const uint8_t *row = Db + y * dbp;
    int s1 = 0, s2 = 0;
    for (int k = 0; k < G.tw; ++k) {
      const int v = row[k];
      s1 += v;
      s2 += v * v;
    }
    for (int a = 0; a < G.cr; ++a) {
      RS[y * G.cr + a] = s1;
      RS2[y * G.cr + a] = s2;
      const int vo = row[a], vi = row[a + G.tw];
      s1 += vi - vo;
      s2 += vi * vi - vo * vo;
    }
  }
  for (int i = tid; i < G.tw; i += nth) {
    int cs = 0, rsum = 0;
    for (int k = 0; k < G.tw; ++k) {
      cs += Tb[k * G.tw + i];
      rsum += Tb[i * G.tw + k];
    }
    colsum_s[i] = cs;
    rowsum_s[i] = rsum;
  }
  if (tid < 32) {
    long long a = 0, a2 = 0;
    for (int i = tid; i < G.tw * G.tw; i += 32) {
      const long long v = Tb[i];
      a += v;
      a2 += v * v;
    }
    a = warp_sum_ll(a);
    a2 = warp_sum_ll(a2);
    if (tid == 0) {
      s_st = a;
      s_st2 = a2;
    }
  }
  __syncthreads();
  // ---- box sums of D and D^2 over every window: slide the row sums down
  for (int a = tid; a < 2 * G.cr; a += nth) {
    const int col = a < G.cr ? a : a - G.cr;
    const int *R = a < G.cr ? RS : RS2;
    int *Cc = a < G.cr ? CS : CS2;
    int s1 = 0;
    for (int k = 0; k < G.tw; ++k) s1 += R[k * G.cr + col];
    for (int b = 0; b < G.cc; ++b) {
      Cc[b * G.cr + col] = s1;
      s1 += R[(b + G.tw) * G.cr + col] - R[b * G.cr + col];
    }
  }
  __syncthreads();  // RS is dead from here on; the map takes its place
  const long long st = s_st, st2 = s_st2;
  const long long mn = (long long)G.tw * G.tw;
  const long long out_idx = (long long)iy + (long long)ix * G.ny;
  if (mn * st2 - st * st == 0) {
    if (tid == 0) {
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      ox[out_idx] = (ii + ii + G.w) / 2.0;
      oy[out_idx] = (jj + jj + G.w) / 2.0;
      ou[out_idx] = nan;
      ov[out_idx] = nan;
      occ[out_idx] = nan;
    }
    return;
  }
  // ---- correlation strips: 8 shifts of one window row per thread
  const int nstrips = G.cc * G.nsx;
  for (int sidx = tid; sidx < nstrips; sidx += nth) {
    const int b = sidx / G.nsx;
    const int a0 = (sidx % G.nsx) * KX;  // multiple of 8
    unsigned acc[KX];
#pragma unroll
    for (int k = 0; k < KX; ++k) acc[k] = 0u;
    const int wbase = a0 >> 2;
    for (int ty = 0; ty < G.tw; ++ty) {
      const unsigned *trow = Tq + ty * L.tw4;
      const unsigned *dr = Dw + (b + ty) * L.dqw + wbase;
      // windows of the word pair (w0, w1) shifted by 1..3 bytes; each step
      // computes the shifts of (w1, w2) once and hands them to the next step
      unsigned w0 = dr[0], w1 = dr[1];
      unsigned s1 = __funnelshift_r(w0, w1, 8), s2 = __funnelshift_r(w0, w1, 16),
               s3 = __funnelshift_r(w0, w1, 24);
#pragma unroll 3
      for (int jw = 0; jw < L.tw4; ++jw) {
        const unsigned t = trow[jw];
        const unsigned w2 = dr[jw + 2];
        const unsigned n1 = __funnelshift_r(w1, w2, 8), n2 = __funnelshift_r(w1, w2, 16),
                       n3 = __funnelshift_r(w1, w2, 24);
        acc[0] = __dp4a(t, w0, acc[0]);
        acc[1] = __dp4a(t, s1, acc[1]);
        acc[2] = __dp4a(t, s2, acc[2]);
        acc[3] = __dp4a(t, s3, acc[3]);
        acc[4] = __dp4a(t, w1, acc[4]);
        acc[5] = __dp4a(t, n1, acc[5]);
        acc[6] = __dp4a(t, n2, acc[6]);
        acc[7] = __dp4a(t, n3, acc[7]);
        w0 = w1;
        w1 = w2;
        s1 = n1;
        s2 = n2;
        s3 = n3;
      }
    }
    const bool ring_b = (b == 0 || b == G.cc - 1);
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      const int a = a0 + k;
      if (a >= G.cr) break;
      const long long sd = CS[b * G.cr + a], sd2 = CS2[b * G.cr + a];
      // Only the outermost ring of the cropped map overhangs the region, by
      // one template column (a = 0: column 0; a = cr-1: column tw-1) and/or
      // one template row (b = 0 / cc-1), so the padded part is O(1).
      int st_out = 0;
      long long n_out = 0;
      if (ring_b || a == 0 || a == G.cr - 1) {
        const int oc = a == 0 ? 0 : (a == G.cr - 1 ? G.tw - 1 : -1);
        const int orow = b == 0 ? 0 : (b == G.cc - 1 ? G.tw - 1 : -1);
        if (oc >= 0) st_out += colsum_s[oc];
        if (orow >= 0) st_out += rowsum_s[orow];
        if (oc >= 0 && orow >= 0) st_out -= Tb[orow * G.tw + oc];
        const long long nco = oc >= 0, nro = orow >= 0;
        n_out = nco * G.tw + nro * G.tw - nco * nro;
      }
      map[b * G.cr + a] = ncc_combine(mn, st, st2, (long long)acc[k], sd, sd2, st_out, n_out, mu);
    }
  }
  __syncthreads();
  peak_epilogue(map, G, ii, jj, out_idx, redv, redi, ox, oy, ou, ov, occ);
}

// ---- 16-bit images: the same strips with __dp2a (16-bit x 8-bit, exact).
// The padded region is staged as two byte planes (high and low bytes of each
// pixel) in the word layout of the 8-bit path, the template as 16-bit pairs;
// with g = 256 gh + gl, sum t g = 256 sum t gh + sum t gl, and __dp2a_lo /
// __dp2a_hi take the pixel pair at bytes 0-1 / 2-3 of a plane word, so the
// words at byte offsets 2j, 2j+1, 2j+4, 2j+5 from a strip's first shift give
// all 8 shifts of template pair j.  Per template row the two 32-bit partial
// sums (at most 17 pairs of products below 2^25) are folded into a 64-bit
// total.
struct U16Layout {
  int tw4, tp, dqw;  // 4-pixel template groups per row, pair words per row, plane words per row
  size_t tb, dh, dl, tq, rs, rs2, cs, cs2, map, red, total;
  __host__ __device__ U16Layout(const SearchGeom &g) {
    tw4 = (g.tw + 3) / 4;
    tp = 2 * tw4;
    int need = 2 * g.nsx + tw4 + 2;
    const int nb = (g.cr + g.tw + 3) / 4 + 1;
    if (need < nb) need = nb;
    dqw = need | 1;
    size_t o = 0;
    tb = o; o = align16(o + sizeof(uint16_t) * g.tw * g.tw);
    dh = o; o = align16(o + sizeof(unsigned) * g.dph * dqw);
    dl = o; o = align16(o + sizeof(unsigned) * g.dph * dqw);
    tq = o; o = align16(o + sizeof(unsigned) * g.tw * tp);
    // window row sums (dead once the box sums are formed: the map reuses them)
    rs = o;
    const size_t rsz = (sizeof(int) + sizeof(long long)) * g.dph * g.cr + 16,
                 msz = sizeof(double) * g.cr * g.cc;
    rs2 = align16(rs + sizeof(int) * g.dph * g.cr);
    o = align16(o + (rsz > msz ? rsz : msz));
    map = rs;
    cs = o; o = align16(o + sizeof(int) * g.cc * g.cr);
    cs2 = o; o = align16(o + sizeof(long long) * g.cc * g.cr);
    red = o; o = align16(o + (sizeof(double) + sizeof(int)) * 32 + 64);
    total = o;
  }
};

__device__ __forceinline__ void search_point_u16(const uint16_t *__restrict__ f,
                                                 const uint16_t *__restrict__ g,
                                                 const SearchGeom &G, const int pt,
                                                 double *__restrict__ ox, double *__restrict__ oy,
                                                 double *__restrict__ ou, double *__restrict__ ov,
                                                 double *__restrict__ occ) {
  extern __shared__ __align__(16) unsigned char smem[];
  const U16Layout L(G);
  uint16_t *Tb = (uint16_t *)(smem + L.tb);   // template, tw x tw
  unsigned *Dh = (unsigned *)(smem + L.dh);   // padded region, high bytes, dph rows of dqw words
  unsigned *Dl = (unsigned *)(smem + L.dl);   // low bytes
  unsigned *Tq = (unsigned *)(smem + L.tq);   // template pairs, tp words per row
  int *RS = (int *)(smem + L.rs);
  long long *RS2 = (long long *)(smem + L.rs2);
  int *CS = (int *)(smem + L.cs);
  long long *CS2 = (long long *)(smem + L.cs2);
  double *map = (double *)(smem + L.map);
  double *redv = (double *)(smem + L.red);
  int *redi = (int *)(redv + 32);
  __shared__ long long s_st, s_st2;
  __shared__ int colsum_s[72], rowsum_s[72];
  const double mu = *G.mu;
  const int ix = pt % G.nx, iy = pt / G.nx;
  const int ii = G.gx1 + ix * G.step, jj = G.gy1 + iy * G.step;  // 1-based
  const int tid = threadIdx.x, nth = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nwarp = nth >> 5;
  const uint16_t *trow0 = f + (long long)(jj - 1) * G.W + (ii - 1);
  const uint16_t *drow0 = g + (long long)(jj - 1 - G.sy) * G.W + (ii - 1 - G.sx);
  // ---- stage the template and the region's byte planes (1-pixel zero
  // border at the top/left, zeros beyond the region)
  for (int ty = wid; ty < G.tw; ty += nwarp)
    for (int tx = lane; tx < G.tw; tx += 32) Tb[ty * G.tw + tx] = trow0[(long long)ty * G.W + tx];
  for (int y = wid; y < G.dph; y += nwarp) {
    const bool rin = y >= 1 && y <= G.dh;
    const uint16_t *src = drow0 + (long long)(y - 1) * G.W;
    for (int w4 = lane; w4 < L.dqw; w4 += 32) {
      unsigned vh = 0, vl = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int x = 4 * w4 + k;
        if (rin && x >= 1 && x <= G.dw) {
          const unsigned v = src[x - 1];
          vh |= (v >> 8) << (8 * k);
          vl |= (v & 0xFFu) << (8 * k);
        }
      }
      Dh[y * L.dqw + w4] = vh;
      Dl[y * L.dqw + w4] = vl;
    }
  }
  __syncthreads();
  // ---- template pair words, window row sums, template sums
  for (int ty = wid; ty < G.tw; ty += nwarp)
    for (int w = lane; w < L.tp; w += 32) {
      const int tx = 2 * w;
      const unsigned a = tx < G.tw ? Tb[ty * G.tw + tx] : 0u;
      const unsigned b = tx + 1 < G.tw ? Tb[ty * G.tw + tx + 1] : 0u;
      Tq[ty * L.tp + w] = a | (b << 16);
    }
  for (int y = tid; y < G.dph; y += nth) {
    const uint8_t *rh = (const uint8_t *)(Dh + y * L.dqw), *rl = (const uint8_t *)(Dl + y * L.dqw);
    int s1 = 0;
    long long s2 = 0;
    for (int k = 0; k < G.tw; ++k) {
      const long long v = 256 * rh[k] + rl[k];
      s1 += (int)v;
      s2 += v * v;
    }
    for (int a = 0; a < G.cr; ++a) {
      RS[y * G.cr + a] = s1;
      RS2[y * G.cr + a] = s2;
      const long long vo = 256 * rh[a] + rl[a], vi = 256 * rh[a + G.tw] + rl[a + G.tw];
      s1 += (int)(vi - vo);
      s2 += vi * vi - vo * vo;
    }
  }
  for (int i = tid; i < G.tw; i += nth) {
    int cs = 0, rsum = 0;
    for (int k = 0; k < G.tw; ++k) {
      cs += Tb[k * G.tw + i];
      rsum += Tb[i * G.tw + k];
    }
    colsum_s[i] = cs;
    rowsum_s[i] = rsum;
  }
  if (tid < 32) {
    long long a = 0, a2 = 0;
    for (int i = tid; i < G.tw * G.tw; i += 32) {
      const long long v = Tb[i];
      a += v;
      a2 += v * v;
    }
    a = warp_sum_ll(a);
    a2 = warp_sum_ll(a2);
    if (tid == 0) {
      s_st = a;
      s_st2 = a2;
    }
  }
  __syncthreads();
  // ---- box sums of D and D^2 over every window: slide the row sums down
  for (int a = tid; a < 2 * G.cr; a += nth) {
    const int col = a < G.cr ? a : a - G.cr;
    if (a < G.cr) {
      int s1 = 0;
      for (int k = 0; k < G.tw; ++k) s1 += RS[k * G.cr + col];
      for (int b = 0; b < G.cc; ++b) {
        CS[b * G.cr + col] = s1;
        s1 += RS[(b + G.tw) * G.cr + col] - RS[b * G.cr + col];
      }
    } else {
      long long s2 = 0;
      for (int k = 0; k < G.tw; ++k) s2 += RS2[k * G.cr + col];
      for (int b = 0; b < G.cc; ++b) {
        CS2[b * G.cr + col] = s2;
        s2 += RS2[(b + G.tw) * G.cr + col] - RS2[b * G.cr + col];
      }
    }
  }
  __syncthreads();  // RS is dead from here on; the map takes its place
  const long long st = s_st, st2 = s_st2;
  const long long mn = (long long)G.tw * G.tw;
  const long long out_idx = (long long)iy + (long long)ix * G.ny;
  if (mn * st2 - st * st == 0) {
    if (tid == 0) {
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      ox[out_idx] = (ii + ii + G.w) / 2.0;
      oy[out_idx] = (jj + jj + G.w) / 2.0;
      ou[out_idx] = nan;
      ov[out_idx] = nan;
      occ[out_idx] = nan;
    }
    return;
  }
  // ---- correlation strips: 8 shifts of one window row per thread
  const int nstrips = G.cc * G.nsx;
  for (int sidx = tid; sidx < nstrips; sidx += nth) {
    const int b = sidx / G.nsx;
    const int a0 = (sidx % G.nsx) * KX;  // multiple of 8
    unsigned long long acc[KX];
#pragma unroll
    for (int k = 0; k < KX; ++k) acc[k] = 0ull;
    const int wbase = a0 >> 2;
    for (int ty = 0; ty < G.tw; ++ty) {
      const unsigned *trow = Tq + ty * L.tp;
      const unsigned *dh = Dh + (b + ty) * L.dqw + wbase, *dl = Dl + (b + ty) * L.dqw + wbase;
      unsigned ah[KX], al[KX];
#pragma unroll
      for (int k = 0; k < KX; ++k) ah[k] = al[k] = 0u;
      // words w0, w1 of each plane and their 1-byte shift, carried along
      unsigned h0 = dh[0], h1 = dh[1], l0 = dl[0], l1 = dl[1];
      unsigned hs = __funnelshift_r(h0, h1, 8), ls = __funnelshift_r(l0, l1, 8);
#pragma unroll 2
      for (int m = 0; m < L.tw4; ++m) {
        const unsigned te = trow[2 * m], to = trow[2 * m + 1];  // template pairs 2m, 2m+1
        const unsigned h2 = dh[m + 2], l2 = dl[m + 2];
        const unsigned hn = __funnelshift_r(h1, h2, 8), ln = __funnelshift_r(l1, l2, 8);
        const unsigned h16 = __funnelshift_r(h0, h1, 16), h24 = __funnelshift_r(h0, h1, 24);
        const unsigned l16 = __funnelshift_r(l0, l1, 16), l24 = __funnelshift_r(l0, l1, 24);
        const unsigned h16n = __funnelshift_r(h1, h2, 16), h24n = __funnelshift_r(h1, h2, 24);
        const unsigned l16n = __funnelshift_r(l1, l2, 16), l24n = __funnelshift_r(l1, l2, 24);
        // pair 2m: byte offsets 4m + k; words at 4m (h0), 4m+1 (hs), 4m+4 (h1), 4m+5 (hn)
        ah[0] = __dp2a_lo(te, h0, ah[0]);  al[0] = __dp2a_lo(te, l0, al[0]);
        ah[2] = __dp2a_hi(te, h0, ah[2]);  al[2] = __dp2a_hi(te, l0, al[2]);
        ah[1] = __dp2a_lo(te, hs, ah[1]);  al[1] = __dp2a_lo(te, ls, al[1]);
        ah[3] = __dp2a_hi(te, hs, ah[3]);  al[3] = __dp2a_hi(te, ls, al[3]);
        ah[4] = __dp2a_lo(te, h1, ah[4]);  al[4] = __dp2a_lo(te, l1, al[4]);
        ah[6] = __dp2a_hi(te, h1, ah[6]);  al[6] = __dp2a_hi(te, l1, al[6]);
        ah[5] = __dp2a_lo(te, hn, ah[5]);  al[5] = __dp2a_lo(te, ln, al[5]);
        ah[7] = __dp2a_hi(te, hn, ah[7]);  al[7] = __dp2a_hi(te, ln, al[7]);
        // pair 2m+1: byte offsets 4m + 2 + k; words at 4m+2, 4m+3, 4m+6, 4m+7
        ah[0] = __dp2a_lo(to, h16, ah[0]);  al[0] = __dp2a_lo(to, l16, al[0]);
        ah[2] = __dp2a_hi(to, h16, ah[2]);  al[2] = __dp2a_hi(to, l16, al[2]);
        ah[1] = __dp2a_lo(to, h24, ah[1]);  al[1] = __dp2a_lo(to, l24, al[1]);
        ah[3] = __dp2a_hi(to, h24, ah[3]);  al[3] = __dp2a_hi(to, l24, al[3]);
        ah[4] = __dp2a_lo(to, h16n, ah[4]);  al[4] = __dp2a_lo(to, l16n, al[4]);
        ah[6] = __dp2a_hi(to, h16n, ah[6]);  al[6] = __dp2a_hi(to, l16n, al[6]);
        ah[5] = __dp2a_lo(to, h24n, ah[5]);  al[5] = __dp2a_lo(to, l24n, al[5]);
        ah[7] = __dp2a_hi(to, h24n, ah[7]);  al[7] = __dp2a_hi(to, l24n, al[7]);
        h0 = h1; h1 = h2; l0 = l1; l1 = l2; hs = hn; ls = ln;
      }
#pragma unroll
      for (int k = 0; k < KX; ++k) acc[k] += ((unsigned long long)ah[k] << 8) + al[k];
    }
    const bool ring_b = (b == 0 || b == G.cc - 1);
#pragma unroll
    for (int k = 0; k < KX; ++k) {
      const int a = a0 + k;
      if (a >= G.cr) break;
      const long long sd = CS[b * G.cr + a], sd2 = CS2[b * G.cr + a];
      int st_out = 0;
      long long n_out = 0;
      if (ring_b || a == 0 || a == G.cr - 1) {
        const int oc = a == 0 ? 0 : (a == G.cr - 1 ? G.tw - 1 : -1);
        const int orow = b == 0 ? 0 : (b == G.cc - 1 ? G.tw - 1 : -1);
        if (oc >= 0) st_out += colsum_s[oc];
        if (orow >= 0) st_out += rowsum_s[orow];
        if (oc >= 0 && orow >= 0) st_out -= Tb[orow * G.tw + oc];
        const long long nco = oc >= 0, nro = orow >= 0;
        n_out = nco * G.tw + nro * G.tw - nco * nro;
      }
      map[b * G.cr + a] = ncc_combine(mn, st, st2, (long long)acc[k], sd, sd2, st_out, n_out, mu);
    }
  }
  __syncthreads();
  peak_epilogue(map, G, ii, jj, out_idx, redv, redi, ox, oy, ou, ov, occ);
}

__global__ void __launch_bounds__(512) k_search_u16(const uint16_t *__restrict__ f,
                                                    const uint16_t *__restrict__ g, SearchGeom G,
                                                    double *__restrict__ ox,
                                                    double *__restrict__ oy,
                                                    double *__restrict__ ou,
                                                    double *__restrict__ ov,
                                                    double *__restrict__ occ) {
  for (int pt = blockIdx.x; pt < G.nx * G.ny; pt += gridDim.x) {
    search_point_u16(f, g, G, pt, ox, oy, ou, ov, occ);
    __syncthreads();  // the next point restages shared memory
  }
}

__global__ void __launch_bounds__(512) k_search_u8(const uint8_t *__restrict__ f,
                                                   const uint8_t *__restrict__ g, SearchGeom G,
                                                   double *__restrict__ ox,
                                                   double *__restrict__ oy,
                                                   double *__restrict__ ou,
                                                   double *__restrict__ ov,
                                                   double *__restrict__ occ) {
  search_point_u8(f, g, G, blockIdx.x, ox, oy, ou, ov, occ);
}

// The same over a device-side list of grid points (list[0] entries from
// list[1]): the points the tiled search hands back.
__global__ void __launch_bounds__(512) k_search_u8_list(const uint8_t *__restrict__ f,
                                                        const uint8_t *__restrict__ g,
                                                        SearchGeom G, const int *__restrict__ list,
                                                        double *__restrict__ ox,
                                                        double *__restrict__ oy,
                                                        double *__restrict__ ou,
                                                        double *__restrict__ ov,
                                                        double *__restrict__ occ) {
  const int n = list[0];
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    search_point_u8(f, g, G, list[1 + i], ox, oy, ou, ov, occ);
    __syncthreads();
  }
}

// ---- 8-bit images, tiled: step a multiple of 4 that divides the subset size.
// Neighbouring subsets overlap (step 8 of a 33 px window: every pixel lies in
// 16 windows), so the per-point kernel above recomputes each product
// f(q) g(q + d) up to 16 times.  Here one CTA takes a TSX x TSY tile of grid
// points and every shift d = (a, b) of the cropped map once: a thread walks
// the tile's rows for its shift, forms each 4-pixel group product once
// (dp4a on word-aligned views of g, no funnel shifts) and assembles the
// windows from step x step block sums:
//   window(ix, iy) = blocks iy .. iy+QB-1 (all rows) + row 0 of block iy+QB,
//   each block row = groups GS*ix .. GS*ix+Q-1 + the first pixel of group
//   GS*ix+Q,
// with the pixels whose partner lies beyond the search region (the outer
// ring of the map) left out exactly.  All sums are exact 32-bit integers, the
// same ones the per-point kernel forms.
//
// The exact sums of every shift go to a per-point map in global memory (a
// tile's maps, 64 points x (2s+3)^2 words, stay in L2 while the tile runs).
// Peak search without an FP64 division per entry: at the end a warp a point
// estimates each entry's NCC in FP32 from the exact integers (interior
// entries from the window sum and 1/sqrt of the window variance term, the
// outer ring from ncc_combine's own FP64 numerator and denominator), with
// |estimate - ncc_combine| < kTileEps.  A running bound T = max(estimate -
// eps) grows over the map; entries with estimate + eps >= T are queued and,
// once T is final, those still within reach are evaluated with ncc_combine
// (lanes in parallel), as is the 3 x 3 neighbourhood of the winner for
// findpeak.  Every entry that can be the maximum (or tie with it) is
// evaluated, so argmax and findpeak's fit are those of the full map.  A point
// with more than kTileQueue queued entries (near-ties, flat search regions),
// or whose evaluated maximum falls below T, is handed to the per-point kernel.
//
// The window sums of every shift of the tile live in shared memory: the
// full windows (sum, sum of squares, 1/sqrt(C0)) copied from a per-image
// table, the windows of the outer ring (one column and/or row left out)
// formed from the staged g.
constexpr float kTileEps = 1e-5f;
constexpr int kTileThreads = 512;
constexpr int kTileQueue = 64;  // queued entries a point (a warp's shared-memory queue)
constexpr int kTileTSX = 8;     // grid points per tile row

struct TileSub {
  int st, st2, cs0, csL, rs0, rsL, c00, cL0, c0L, cLL;
  float invT;     // 1 / sqrt(mn st2 - st^2)
  int state;      // 0 searched, 1 constant template (NaN), 2 beyond the grid
};

struct TileArgs {
  const uint8_t *f, *g;
  const uint4 *tab;  // W x H: (sum, sum of squares, bits of 1/sqrt(C0), 0) of full windows
  unsigned *cmap;    // exact correlation sums, cr * cc a point (b * cr + a), tile by tile
  TileSub *subs;     // template sums of every point, tile by tile
  uint2 *ringw;      // window sums of every point's outer ring, ring order
  int W, H, px1, py1, nx, ny, w, sx, sy, cr, cc;
  int tsy, ndy, nbatch, pitch, rows_g, pb, qxn, qyn;
  long long mn;
  int off_g, off_ti, off_ra, off_rb, off_rc, off_sub;
};

__device__ __forceinline__ unsigned fkey(float x) {  // order-preserving float -> unsigned
  const unsigned u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// template pixels of entry (a, b) whose partner lies beyond the search region
__device__ __forceinline__ void tile_pad(const TileSub &S, int a, int b, int cr, int cc, int tw,
                                         long long *st_out, long long *n_out) {
  const int nco = (a == 0) || (a == cr - 1), nro = (b == 0) || (b == cc - 1);
  long long so = 0;
  if (a == 0) so += S.cs0;
  if (a == cr - 1) so += S.csL;
  if (b == 0) so += S.rs0;
  if (b == cc - 1) so += S.rsL;
  if (nco && nro) so -= (b == 0) ? (a == 0 ? S.c00 : S.cL0) : (a == 0 ? S.c0L : S.cLL);
  *st_out = so;
  *n_out = (long long)nco * tw + (long long)nro * tw - (long long)nco * nro;
}

template <int STEP, int WS, int TSX>
struct TileShape {
  static constexpr int TW = WS + 1, Q = WS / 4, GS = STEP / 4, QB = WS / STEP;
  static constexpr int NG = GS * (TSX - 1) + Q + 1;  // 4-pixel groups of a tile row
  static constexpr int NE = TSX + QB;                // groups whose first pixel is kept apart
  static constexpr int NGP = (NG + 3) & ~3;          // words per staged f row
};

// shared-memory views of one tile
struct TileMem {
  const uint32_t *Fw, *Gw;
  const int *tis, *tis2;   // full windows at tile position (qxi, qyi): sums of g, g^2
  const uint2 *ra, *rb, *rc;
  int pitch, qxn, qyn, tsy;
};

// (sum g, sum g^2) over the part of entry (a, b)'s window inside the search region
template <int STEP>
__device__ __forceinline__ uint2 tile_wsum(const TileMem &M, int ix, int iy, int a, int b,
                                           int cr, int cc) {
  const bool ra = a == 0 || a == cr - 1, rb = b == 0 || b == cc - 1;
  const int qxi = ix * STEP + a, qyi = iy * STEP + b;
  if (!ra && !rb) {
    const int i = qyi * M.qxn + qxi;
    return make_uint2((unsigned)M.tis[i], (unsigned)M.tis2[i]);
  }
  if (!rb) return M.ra[((a != 0) * kTileTSX + ix) * M.qyn + qyi];
  if (!ra) return M.rb[((b != 0) * M.tsy + iy) * M.qxn + qxi];
  return M.rc[(iy * kTileTSX + ix) * 4 + (a != 0) + 2 * (b != 0)];
}

// the outer ring of the cropped map, r in [0, 2 (cr + cc) - 4): columns a = 0
// and cr-1 (all b), then rows b = 0 and cc-1 (a = 1 .. cr-2)
__device__ __forceinline__ void ring_pos(int r, int cr, int cc, int *a, int *b) {
  if (r < 2 * cc) {
    *a = r < cc ? 0 : cr - 1;
    *b = r < cc ? r : r - cc;
  } else {
    const int m = r - 2 * cc;
    *a = 1 + (m < cr - 2 ? m : m - (cr - 2));
    *b = m < cr - 2 ? 0 : cc - 1;
  }
}
__device__ __forceinline__ int ring_index(int a, int b, int cr, int cc) {
  if (a == 0) return b;
  if (a == cr - 1) return cc + b;
  return 2 * cc + (a - 1) + (b == 0 ? 0 : cr - 2);
}

// one tile row for shift (a, b): group products into acc, first pixels into accE
template <int STEP, int WS, int TSX>
__device__ __forceinline__ void tile_row(const uint32_t *__restrict__ frow,
                                         const uint32_t *__restrict__ grow,
                                         unsigned (&acc)[TileShape<STEP, WS, TSX>::NG],
                                         unsigned (&accE)[TileShape<STEP, WS, TSX>::NE]) {
  using T = TileShape<STEP, WS, TSX>;
  uint32_t fw[T::NGP];
#pragma unroll
  for (int k4 = 0; k4 < T::NGP / 4; ++k4) {
    const uint4 v = reinterpret_cast<const uint4 *>(frow)[k4];
    fw[4 * k4] = v.x;
    fw[4 * k4 + 1] = v.y;
    fw[4 * k4 + 2] = v.z;
    fw[4 * k4 + 3] = v.w;
  }
#pragma unroll
  for (int k = 0; k < T::NG; ++k) {
    const uint32_t gw = grow[4 * k];
    if (k < T::NG - 1) acc[k] = __dp4a(fw[k], gw, acc[k]);
    if (k % T::GS == 0) accE[k / T::GS] = __dp4a(fw[k] & 0xFFu, gw, accE[k / T::GS]);
  }
}

// the TSX horizontal window sums of the rows accumulated in acc / accE
template <int STEP, int WS, int TSX>
__device__ __forceinline__ void tile_hsum(const unsigned (&acc)[TileShape<STEP, WS, TSX>::NG],
                                          const unsigned (&accE)[TileShape<STEP, WS, TSX>::NE],
                                          unsigned cF, unsigned cL, unsigned (&S)[TSX]) {
  using T = TileShape<STEP, WS, TSX>;
  unsigned run = 0;
#pragma unroll
  for (int k = 0; k < T::Q; ++k) run += acc[k];
#pragma unroll
  for (int ix = 0; ix < TSX; ++ix) {
    S[ix] = run + cL * accE[ix + T::QB] - cF * accE[ix];
    if (ix + 1 < TSX) {
#pragma unroll
      for (int k = 0; k < T::GS; ++k) run += acc[T::GS * ix + T::Q + k] - acc[T::GS * ix + k];
    }
  }
}

template <int STEP, int WS, int TSX>
__global__ void __launch_bounds__(kTileThreads, 1) k_search_tile(const TileArgs A) {
  using T = TileShape<STEP, WS, TSX>;
  constexpr int TW = T::TW, NG = T::NG, NE = T::NE, NGP = T::NGP, QB = T::QB;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t *Fw = reinterpret_cast<uint32_t *>(smem);
  uint32_t *Gw = reinterpret_cast<uint32_t *>(smem + A.off_g);
  int *tis = reinterpret_cast<int *>(smem + A.off_ti);
  int *tis2 = tis + A.qxn * A.qyn;
  uint2 *ra = reinterpret_cast<uint2 *>(smem + A.off_ra);
  uint2 *rb = reinterpret_cast<uint2 *>(smem + A.off_rb);
  uint2 *rc = reinterpret_cast<uint2 *>(smem + A.off_rc);
  TileSub *sub = reinterpret_cast<TileSub *>(smem + A.off_sub);
  uint8_t *tmp = smem + A.off_ti;  // g bytes while staging (the window tables come later)
  const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nth >> 5;
  const int TSY = A.tsy, NS = TSX * TSY, RYf = (TSY - 1) * STEP + TW;
  const int cr = A.cr, cc = A.cc, pitch = A.pitch, qxn = A.qxn, qyn = A.qyn;
  const int tx0 = blockIdx.x * TSX, ty0 = blockIdx.y * TSY;       // first grid point
  const int px0 = A.px1 + tx0 * STEP, py0 = A.py1 + ty0 * STEP;   // its 0-based corner
  const int gx0 = px0 - A.sx - 1, gy0 = py0 - A.sy - 1;           // corner of the g tile
  const TileMem M{Fw, Gw, tis, tis2, ra, rb, rc, pitch, qxn, qyn, TSY};
  const int nmap = cr * cc;
  unsigned *cmap = A.cmap + (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * NS * nmap;

  // ---- stage f (4 pixels a word) and g (word m of a row = bytes m .. m+3)
  for (int i = tid; i < RYf * NGP; i += nth) {
    const int y = i / NGP, k = i - y * NGP;
    unsigned v = 0;
    if (py0 + y < A.H) {
      const uint8_t *row = A.f + (long long)(py0 + y) * A.W;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int x = px0 + 4 * k + j;
        if (x < A.W) v |= (unsigned)row[x] << (8 * j);
      }
    }
    Fw[i] = v;
  }
  for (int i = tid; i < A.rows_g * A.pb; i += nth) {
    const int r = i / A.pb, x = i - r * A.pb;
    const int yy = gy0 + r, xx = gx0 + x;
    tmp[i] = (yy < A.H && xx < A.W) ? A.g[(long long)yy * A.W + xx] : (uint8_t)0;
  }
  __syncthreads();
  for (int i = tid; i < A.rows_g * pitch; i += nth) {
    const int r = i / pitch, m = i - r * pitch;
    const uint32_t *tw = reinterpret_cast<const uint32_t *>(tmp + r * A.pb);
    Gw[i] = __funnelshift_r(tw[m >> 2], tw[(m >> 2) + 1], 8 * (m & 3));
  }
  __syncthreads();
  // ---- full windows at every tile position (positions beyond the image: 0)
  const int tabw = A.W - TW, tabh = A.H - TW;
  for (int i = tid; i < qxn * qyn; i += nth) {
    const int qyi = i / qxn, qxi = i - qyi * qxn;
    const int xx = gx0 + qxi, yy = gy0 + qyi;
    uint4 e = make_uint4(0, 0, 0, 0);
    if (xx <= tabw && yy <= tabh) e = A.tab[(long long)yy * A.W + xx];
    tis[i] = (int)e.x;
    tis2[i] = (int)e.y;
  }
  __syncthreads();
  // ---- the outer ring's windows: full window minus a column and/or a row
  const uint8_t *gb = reinterpret_cast<const uint8_t *>(Gw);  // byte 0 of word c = g(c)
  auto colsum = [&](int col, int r0, unsigned &s1, unsigned &s2) {
    s1 = s2 = 0;
    for (int r = r0; r < r0 + TW; ++r) {
      const unsigned v = gb[(r * pitch + col) * 4];
      s1 += v;
      s2 += v * v;
    }
  };
  auto rowsum = [&](int row, int c0, unsigned &s1, unsigned &s2) {
    const uint32_t *w = Gw + row * pitch + c0;
    s1 = s2 = 0;
#pragma unroll
    for (int k = 0; k < T::Q; ++k) {
      s1 = __dp4a(w[4 * k], 0x01010101u, s1);
      s2 = __dp4a(w[4 * k], w[4 * k], s2);
    }
    const unsigned v = w[4 * T::Q] & 0xFFu;
    s1 += v;
    s2 += v * v;
  };
  for (int i = tid; i < 2 * TSX * qyn; i += nth) {
    const int side = i / (TSX * qyn), r = i - side * TSX * qyn, ix = r / qyn, qyi = r - ix * qyn;
    const int qxi = ix * STEP + (side ? cr - 1 : 0), col = side ? qxi + TW - 1 : qxi;
    unsigned c1, c2;
    colsum(col, qyi, c1, c2);
    const int j = qyi * qxn + qxi;
    ra[i] = make_uint2((unsigned)tis[j] - c1, (unsigned)tis2[j] - c2);
  }
  for (int i = tid; i < 2 * TSY * qxn; i += nth) {
    const int side = i / (TSY * qxn), r = i - side * TSY * qxn, iy = r / qxn, qxi = r - iy * qxn;
    const int qyi = iy * STEP + (side ? cc - 1 : 0), row = side ? qyi + TW - 1 : qyi;
    unsigned r1, r2;
    rowsum(row, qxi, r1, r2);
    const int j = qyi * qxn + qxi;
    rb[i] = make_uint2((unsigned)tis[j] - r1, (unsigned)tis2[j] - r2);
  }
  for (int i = tid; i < NS * 4; i += nth) {
    const int s = i >> 2, as = i & 1, bs = (i >> 1) & 1, ix = s % TSX, iy = s / TSX;
    const int qxi = ix * STEP + (as ? cr - 1 : 0), qyi = iy * STEP + (bs ? cc - 1 : 0);
    const int col = as ? qxi + TW - 1 : qxi, row = bs ? qyi + TW - 1 : qyi;
    unsigned c1, c2, r1, r2;
    colsum(col, qyi, c1, c2);
    rowsum(row, qxi, r1, r2);
    const unsigned v = gb[(row * pitch + col) * 4];
    const int j = qyi * qxn + qxi;
    rc[i] = make_uint2((unsigned)tis[j] - c1 - r1 + v, (unsigned)tis2[j] - c2 - r2 + v * v);
  }
  // ---- template sums of every point (a warp per point, lanes over rows)
  for (int s = wid; s < NS; s += nw) {
    const int ix = s % TSX, iy = s / TSX;
    const bool valid = tx0 + ix < A.nx && ty0 + iy < A.ny;
    int v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // st st2 cs0 csL rs0 rsL c00 cL0 c0L cLL
    if (valid)
      for (int ty = lane; ty < TW; ty += 32) {
        const uint32_t *fr = Fw + (iy * STEP + ty) * NGP + T::GS * ix;
        unsigned rs = 0, rq = 0;
#pragma unroll
        for (int k = 0; k < T::Q; ++k) {
          rs = __dp4a(fr[k], 0x01010101u, rs);
          rq = __dp4a(fr[k], fr[k], rq);
        }
        const int first = fr[0] & 0xFF, last = fr[T::Q] & 0xFF;
        rs += last;
        rq += last * last;
        v[0] += rs;
        v[1] += rq;
        v[2] += first;
        v[3] += last;
        if (ty == 0) { v[4] = rs; v[6] = first; v[7] = last; }
        if (ty == TW - 1) { v[5] = rs; v[8] = first; v[9] = last; }
      }
#pragma unroll
    for (int k = 0; k < 10; ++k) v[k] = __reduce_add_sync(0xffffffffu, v[k]);
    if (lane == 0) {
      TileSub &S = sub[s];
      S.st = v[0]; S.st2 = v[1]; S.cs0 = v[2]; S.csL = v[3]; S.rs0 = v[4]; S.rsL = v[5];
      S.c00 = v[6]; S.cL0 = v[7]; S.c0L = v[8]; S.cLL = v[9];
      const long long denT = A.mn * v[1] - (long long)v[0] * v[0];
      S.state = !valid ? 2 : (denT == 0 ? 1 : 0);
      S.invT = denT > 0 ? (float)(1.0 / sqrt((double)denT)) : 0.f;
    }
  }
  __syncthreads();

  // ---- every shift of the cropped map, ndy map columns per batch; the two
  // ring shifts (a = 0, cr-1) of each column take the first lanes, so the
  // interior shifts of a warp run along a in one bank sequence
  for (int bt = 0; bt < A.nbatch; ++bt) {
    const int b0 = bt * A.ndy, nbr = min(A.ndy, cc - b0);
    int a, b;
    bool active;
    if (tid < 2 * nbr) {
      a = (tid & 1) ? cr - 1 : 0;
      b = b0 + (tid >> 1);
      active = true;
    } else {
      const int u = tid - 2 * nbr;
      a = 1 + u % (cr - 2);
      b = b0 + u / (cr - 2);
      active = b < b0 + nbr;
      if (!active) {  // in-bounds work whose results are dropped
        a = 1;
        b = b0;
      }
    }
    const unsigned cF = (a == 0), cL = (a != cr - 1), cRF = (b == 0), cRL = (b != cc - 1);
    const uint32_t *gbase = Gw + b * pitch + a;
    unsigned win[QB][TSX];
    unsigned acc[NG], accE[NE], S[TSX];
    for (int j0 = 0; j0 < TSY + QB; j0 += QB) {
#pragma unroll
      for (int sl = 0; sl < QB; ++sl) {
        const int j = j0 + sl;
        if (j >= TSY + QB) break;
#pragma unroll
        for (int k = 0; k < NG; ++k) acc[k] = 0;
#pragma unroll
        for (int k = 0; k < NE; ++k) accE[k] = 0;
        tile_row<STEP, WS, TSX>(Fw + j * STEP * NGP, gbase + j * STEP * pitch, acc, accE);
        tile_hsum<STEP, WS, TSX>(acc, accE, cF, cL, S);
        if (j >= QB) {
          // ---- the windows of point row iy are complete: to the maps
          const int iy = j - QB;
#pragma unroll
          for (int ix = 0; ix < TSX; ++ix) {
            const int s = iy * TSX + ix;
            if (active && sub[s].state == 0) cmap[(size_t)s * nmap + b * cr + a] = win[sl][ix] + cRL * S[ix];
          }
        }
        if (j < TSY) {
#pragma unroll
          for (int ix = 0; ix < TSX; ++ix) win[sl][ix] = 0u - cRF * S[ix];
        }
        if (j < TSY + QB - 1) {
          for (int rr = 1; rr < STEP; ++rr)
            tile_row<STEP, WS, TSX>(Fw + (j * STEP + rr) * NGP, gbase + (j * STEP + rr) * pitch,
                                    acc, accE);
          tile_hsum<STEP, WS, TSX>(acc, accE, cF, cL, S);
          // the open windows: point rows j-QB+1 .. j, one per slot
#pragma unroll
          for (int s2 = 0; s2 < QB; ++s2) {
            const int iy = j - ((sl - s2 + QB) % QB);
            if (iy >= 0 && iy < TSY) {
#pragma unroll
              for (int ix = 0; ix < TSX; ++ix) win[s2][ix] += S[ix];
            }
          }
        }
      }
    }
  }
  __syncthreads();

  // ---- export: each point's template sums and the window sums of its outer
  // ring (the peak kernel reads them with the maps)
  const size_t tile0 = (size_t)(blockIdx.y * gridDim.x + blockIdx.x) * NS;
  const int nring = 2 * (cr + cc) - 4;
  for (int s = wid; s < NS; s += nw) {
    if (lane == 0) A.subs[tile0 + s] = sub[s];
    if (sub[s].state != 0) continue;
    const int ix = s % TSX, iy = s / TSX;
    uint2 *rw = A.ringw + (tile0 + s) * nring;
    for (int r = lane; r < nring; r += 32) {
      int ra, rb;
      ring_pos(r, cr, cc, &ra, &rb);
      rw[r] = tile_wsum<STEP>(M, ix, iy, ra, rb, cr, cc);
    }
  }
}

// ---- per-image table of the full tw x tw windows of g: (sum, sum of
// squares, 1/sqrt(mn sum^2 - sum^2) or 0) at every top-left corner in
// [x0, x1] x [y0, y1].  A block per kTabX x kTabY corners: the bytes in
// shared memory, vertical sums per column, a prefix sum per row.
constexpr int kTabX = 128, kTabY = 32;

__global__ void __launch_bounds__(256) k_box_tab(const uint8_t *__restrict__ g, int W, int H,
                                                 int tw, long long mn, int x0, int x1, int y0,
                                                 int y1, uint4 *__restrict__ tab) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int bx = x0 + blockIdx.x * kTabX, by = y0 + blockIdx.y * kTabY;
  const int nc = kTabX + tw - 1, nr = kTabY + tw - 1, np = nc + 1;
  uint8_t *G = sm;
  unsigned *P1 = reinterpret_cast<unsigned *>(sm + align16((size_t)nr * nc));
  unsigned *P2 = P1 + kTabY * np;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int i = tid; i < nr * nc; i += 256) {
    const int r = i / nc, c = i - r * nc, yy = by + r, xx = bx + c;
    G[i] = (yy < H && xx < W) ? g[(long long)yy * W + xx] : (uint8_t)0;
  }
  __syncthreads();
  for (int c = tid; c < nc; c += 256) {  // vertical sums, column c, rows oy .. oy+tw-1
    unsigned s1 = 0, s2 = 0;
    for (int r = 0; r < tw; ++r) {
      const unsigned v = G[r * nc + c];
      s1 += v;
      s2 += v * v;
    }
    for (int oy = 0; oy < kTabY; ++oy) {
      P1[oy * np + c + 1] = s1;
      P2[oy * np + c + 1] = s2;
      if (oy + 1 < kTabY) {
        const unsigned vo = G[oy * nc + c], vi = G[(oy + tw) * nc + c];
        s1 += vi - vo;
        s2 += vi * vi - vo * vo;
      }
    }
  }
  __syncthreads();
  for (int oy = wid; oy < kTabY; oy += 8) {  // prefix sums along each row, a warp a row
    unsigned *q1 = P1 + oy * np, *q2 = P2 + oy * np;
    if (lane == 0) q1[0] = q2[0] = 0;
    unsigned c1 = 0, c2 = 0;
    for (int c0 = 1; c0 <= nc; c0 += 32) {
      const int c = c0 + lane;
      unsigned v1 = c <= nc ? q1[c] : 0u, v2 = c <= nc ? q2[c] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t1 = __shfl_up_sync(0xffffffffu, v1, o), t2 = __shfl_up_sync(0xffffffffu, v2, o);
        if (lane >= o) {
          v1 += t1;
          v2 += t2;
        }
      }
      if (c <= nc) {
        q1[c] = c1 + v1;
        q2[c] = c2 + v2;
      }
      c1 += __shfl_sync(0xffffffffu, v1, 31);
      c2 += __shfl_sync(0xffffffffu, v2, 31);
    }
  }
  __syncthreads();
  for (int i = tid; i < kTabX * kTabY; i += 256) {
    const int oy = i / kTabX, ox = i - oy * kTabX, x = bx + ox, y = by + oy;
    if (x > x1 || y > y1) continue;
    const unsigned s1 = P1[oy * np + ox + tw] - P1[oy * np + ox];
    const unsigned s2 = P2[oy * np + ox + tw] - P2[oy * np + ox];
    const long long c0 = mn * (long long)s2 - (long long)s1 * s1;
    tab[(long long)y * W + x] =
        make_uint4(s1, s2, c0 > 0 ? __float_as_uint(rsqrtf((float)c0)) : 0u, 0u);
  }
}

// ---- peak search of every grid point from its exact correlation map (a
// warp a point, full occupancy): FP32 estimates over the map, the entries
// within reach of the running bound T = max(estimate - eps) queued in shared
// memory, ncc_combine on those still within reach of the final T (lanes in
// parallel), argmax (first in map order on ties), findpeak's 3 x 3 fit from
// the neighbours' exact values; outputs of funIntegerSearch.m:148-159.
constexpr int kPeakWarps = 8;
constexpr int kPeakUnroll = 4;  // map entries a lane has in flight
constexpr int kRingUnroll = 5;  // outer-ring entries a lane takes a round (136 for s = 16: one round)

struct PeakArgs {
  const unsigned *cmap;   // exact correlation sums, tile by tile
  const uint2 *ringw;     // window sums of the outer ring, ring order
  const TileSub *subs;    // template sums
  const uint4 *tab;       // W x H full-window table (sum, sum of squares, 1/sqrt(C0))
  const double *mu;
  double *ox, *oy, *ou, *ov, *occ;
  int *fb;                // fb[0] count, fb[1 ..] grid points for the per-point kernel
  int W, px1, py1, nx, ny, step, w, tw, sx, sy, cr, cc, tsy, tiles_x;
  long long mn;
};

__global__ void __launch_bounds__(kPeakWarps * 32, 4) k_search_peak(const PeakArgs A) {
  __shared__ uint3 qbuf[kPeakWarps][kTileQueue];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint3 *queue = qbuf[wid];
  const double mu = *A.mu;
  const int cr = A.cr, cc = A.cc, ci = cr - 2, ni = ci * (cc - 2), nring = 2 * (cr + cc) - 4;
  const int nmap = cr * cc, NS = kTileTSX * A.tsy;
  const long long npts = (long long)A.nx * A.ny;
  for (long long pt = (long long)blockIdx.x * kPeakWarps + wid; pt < npts;
       pt += (long long)gridDim.x * kPeakWarps) {
    const int gix = (int)(pt % A.nx), giy = (int)(pt / A.nx);
    const size_t ps = (size_t)((giy / A.tsy) * A.tiles_x + gix / kTileTSX) * NS +
                      (giy % A.tsy) * kTileTSX + gix % kTileTSX;
    const TileSub &P = A.subs[ps];  // fields loaded where used (L1), not held in registers
    const long long out_idx = (long long)giy + (long long)gix * A.ny;
    const int px = A.px1 + gix * A.step, py = A.py1 + giy * A.step;
    const int ii = px + 1, jj = py + 1;  // 1-based
    if (P.state != 0) {  // constant template: normxcorr2 raises (funIntegerSearch.m:153-157)
      if (lane == 0) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        A.ox[out_idx] = (ii + ii + A.w) / 2.0;
        A.oy[out_idx] = (jj + jj + A.w) / 2.0;
        A.ou[out_idx] = nan;
        A.ov[out_idx] = nan;
        A.occ[out_idx] = nan;
      }
      continue;
    }
    const unsigned *cm = A.cmap + ps * nmap;
    const uint2 *rw = A.ringw + ps * nring;
    const uint4 *tb = A.tab + (long long)(py - 1 - A.sy) * A.W + (px - 1 - A.sx);  // entry (a, b): tb[b W + a]
    auto exact = [&](int a, int b, unsigned C) -> double {
      uint2 w;
      if (a == 0 || a == cr - 1 || b == 0 || b == cc - 1) {
        w = rw[ring_index(a, b, cr, cc)];
      } else {
        const uint4 t = tb[(long long)b * A.W + a];
        w = make_uint2(t.x, t.y);
      }
      long long st_out, n_out;
      tile_pad(P, a, b, cr, cc, A.tw, &st_out, &n_out);
      return ncc_combine(A.mn, P.st, P.st2, (long long)C, (long long)w.x, (long long)w.y, st_out,
                         n_out, mu);
    };
    unsigned tkey = 0u;  // ordered key of the running bound
    int nq = 0;          // queued entries (the same in every lane)
    // kPeakUnroll entries a lane at a time: the loads first, one bound update,
    // then the queue (ballot order keeps it dense)
    // (rounds where no lane keeps an entry -- most, once the bound is near
    // the peak -- skip the queue bookkeeping)
    auto screen = [&](auto const &valid, auto const &k, auto const &C, auto const &e) {
      constexpr int U = sizeof(e) / sizeof(float);
      float mx = -INFINITY;
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (valid[j]) mx = fmaxf(mx, e[j] - kTileEps);
      tkey = max(tkey, __reduce_max_sync(0xffffffffu, fkey(mx)));
      bool keep[U], any = false;
#pragma unroll
      for (int j = 0; j < U; ++j) {
        keep[j] = valid[j] && fkey(e[j] + kTileEps) >= tkey;
        any |= keep[j];
      }
      if (!__any_sync(0xffffffffu, any)) return;
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const unsigned bal = __ballot_sync(0xffffffffu, keep[j]);
        if (keep[j]) {
          const int pos = nq + __popc(bal & ((1u << lane) - 1u));
          if (pos < kTileQueue) queue[pos] = make_uint3((unsigned)k[j], C[j], __float_as_uint(e[j]));
        }
        nq += __popc(bal);
      }
    };
    // interior entries (a, b in 1 .. cr-2, 1 .. cc-2), lanes along a; the
    // lane's map index and table entry advance with it
    int a = 1 + lane, b = 1;
    while (a > ci) {
      a -= ci;
      ++b;
    }
    int km = b * cr + a;
    const uint4 *tp = tb + (long long)b * A.W + a;
    for (int k0 = 0; k0 < ni; k0 += 32 * kPeakUnroll) {
      bool valid[kPeakUnroll];
      int k[kPeakUnroll];
      unsigned C[kPeakUnroll];
      uint4 t[kPeakUnroll];
      float e[kPeakUnroll];
#pragma unroll
      for (int j = 0; j < kPeakUnroll; ++j) {
        valid[j] = k0 + 32 * j + lane < ni;
        k[j] = km;
        C[j] = 0u;
        t[j] = make_uint4(0, 0, 0, 0);
        if (valid[j]) {
          C[j] = cm[km];
          t[j] = *tp;
        }
        a += 32;
        km += 32;
        tp += 32;
        while (a > ci) {
          a -= ci;
          km += cr - ci;
          tp += A.W - ci;
        }
      }
#pragma unroll
      for (int j = 0; j < kPeakUnroll; ++j) {
        const long long num = A.mn * (long long)C[j] - (long long)P.st * (int)t[j].x;
        e[j] = (float)num * P.invT * __uint_as_float(t[j].z);
      }
      screen(valid, k, C, e);
    }
    // the outer ring, from ncc_combine's own FP64 numerator and denominator
    for (int k0 = 0; k0 < nring; k0 += 32 * kRingUnroll) {
      bool valid[kRingUnroll];
      int k[kRingUnroll], ra[kRingUnroll], rb[kRingUnroll];
      unsigned C[kRingUnroll];
      uint2 w[kRingUnroll];
      float e[kRingUnroll];
#pragma unroll
      for (int j = 0; j < kRingUnroll; ++j) {
        const int r = k0 + 32 * j + lane;
        valid[j] = r < nring;
        ring_pos(valid[j] ? r : 0, cr, cc, &ra[j], &rb[j]);
        k[j] = rb[j] * cr + ra[j];
        C[j] = valid[j] ? cm[k[j]] : 0u;
        w[j] = valid[j] ? rw[r] : make_uint2(0, 0);
      }
#pragma unroll
      for (int j = 0; j < kRingUnroll; ++j) {
        e[j] = 0.f;
        if (valid[j]) {
          long long st_out, n_out;
          tile_pad(P, ra[j], rb[j], cr, cc, A.tw, &st_out, &n_out);
          double num, den;
          ncc_parts(A.mn, P.st, (long long)C[j], (long long)w[j].x, (long long)w[j].y, st_out,
                    n_out, mu, &num, &den);
          e[j] = den > 0.0 ? (float)num * P.invT * rsqrtf((float)den) : 0.f;
        }
      }
      screen(valid, k, C, e);
    }
    __syncwarp();
    bool hand_back = nq > kTileQueue;
    double best = -INFINITY;
    int bi = 0x7fffffff;
    if (!hand_back) {
      for (int q = lane; q < nq; q += 32) {
        const uint3 e = queue[q];
        if (fkey(__uint_as_float(e.z) + kTileEps) >= tkey) {
          const double r = exact((int)e.x % cr, (int)e.x / cr, e.y);
          if (r > best || (r == best && (int)e.x < bi)) {
            best = r;
            bi = (int)e.x;
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      // the bound must hold for the evaluated maximum (it can only fail where
      // an estimate met ncc_combine's clamp of |r| > 1)
      hand_back = !(best >= (double)fkey_inv(tkey));
    }
    __syncwarp();  // the queue is the next point's
    if (hand_back) {
      if (lane == 0) {
        const int pos = atomicAdd(A.fb, 1);
        A.fb[1 + pos] = giy * A.nx + gix;
      }
      continue;
    }
    const int am = bi % cr, bm = bi / cr;
    double rpk = am + 1, cpk = bm + 1, mf = best;
    if (am > 0 && am < cr - 1 && bm > 0 && bm < cc - 1) {
      // the 3 x 3 neighbourhood, lane k = (dc + 1) * 3 + dr + 1
      double r = best;
      if (lane < 9 && lane != 4) {
        const int na = am + lane % 3 - 1, nb = bm + lane / 3 - 1;
        r = exact(na, nb, cm[nb * cr + na]);
      }
      double u9[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) u9[k] = __shfl_sync(0xffffffffu, r, k);
      if (lane == 0) findpeak_fit9(u9, am, bm, &rpk, &cpk, &mf);
    }
    if (lane == 0) {
      A.ox[out_idx] = (ii + ii + A.w) / 2.0;
      A.oy[out_idx] = (jj + jj + A.w) / 2.0;
      A.ou[out_idx] = __dsub_rn(rpk, (double)(A.sx + 2));
      A.ov[out_idx] = __dsub_rn(cpk, (double)(A.sy + 2));
      A.occ[out_idx] = mf;
    }
  }
}

struct TilePlan {
  int tsy = 0, ndy = 0, nbatch = 0, pitch = 0, rows_g = 0, pb = 0, qxn = 0, qyn = 0;
  int off_g = 0, off_ti = 0, off_ra = 0, off_rb = 0, off_rc = 0, off_sub = 0;
  int total = 0;
};

// tile rows, thread batches and the shared-memory layout: the largest tile
// (up to 8 point rows) that fits one CTA per SM
template <int STEP, int WS>
bool tile_plan(int sx, int sy, TilePlan &P) {
  using T = TileShape<STEP, WS, kTileTSX>;
  const int cr = 2 * sx + 3, cc = 2 * sy + 3;
  if (cr > kTileThreads) return false;
  P.nbatch = (cc + kTileThreads / cr - 1) / (kTileThreads / cr);
  P.ndy = (cc + P.nbatch - 1) / P.nbatch;
  // the interior lanes of a warp continue the bank sequence across rows
  const int minp = cr + 4 * T::NG - 4;
  P.pitch = minp + (((cr - 2 - minp) % 32) + 32) % 32;
  P.pb = (int)align16(4 * ((P.pitch - 1) / 4 + 2));
  P.qxn = (kTileTSX - 1) * STEP + cr;
  for (int tsy = 8; tsy >= 1; --tsy) {
    const int ryf = (tsy - 1) * STEP + T::TW, rows_g = ryf + cc - 1, ns = kTileTSX * tsy;
    const int qyn = (tsy - 1) * STEP + cc;
    size_t o = align16((size_t)ryf * T::NGP * 4);
    const size_t og = o;
    o += align16((size_t)rows_g * P.pitch * 4);
    const size_t oti = o;
    o += align16(std::max((size_t)2 * P.qxn * qyn * 4, (size_t)rows_g * P.pb));
    const size_t ora = o;
    o += align16((size_t)2 * kTileTSX * qyn * sizeof(uint2));
    const size_t orb = o;
    o += align16((size_t)2 * tsy * P.qxn * sizeof(uint2));
    const size_t orc = o;
    o += align16((size_t)ns * 4 * sizeof(uint2));
    const size_t os = o;
    o += align16((size_t)ns * sizeof(TileSub));
    if (o <= (size_t)227 * 1024) {
      P.tsy = tsy;
      P.rows_g = rows_g;
      P.qyn = qyn;
      P.off_g = (int)og;
      P.off_ti = (int)oti;
      P.off_ra = (int)ora;
      P.off_rb = (int)orb;
      P.off_rc = (int)orc;
      P.off_sub = (int)os;
      P.total = (int)o;
      return true;
    }
  }
  return false;
}

template <int STEP, int WS>
int tile_launch(TileArgs A, const TilePlan &P, cudaStream_t st) {
  A.tsy = P.tsy; A.ndy = P.ndy; A.nbatch = P.nbatch; A.pitch = P.pitch;
  A.rows_g = P.rows_g; A.pb = P.pb; A.qxn = P.qxn; A.qyn = P.qyn;
  A.off_g = P.off_g; A.off_ti = P.off_ti; A.off_ra = P.off_ra; A.off_rb = P.off_rb;
  A.off_rc = P.off_rc; A.off_sub = P.off_sub;
  auto kern = k_search_tile<STEP, WS, kTileTSX>;
  ALDIC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, P.total));
  const dim3 grid((A.nx + kTileTSX - 1) / kTileTSX, (A.ny + P.tsy - 1) / P.tsy);
  kern<<<grid, kTileThreads, P.total, st>>>(A);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// (step, winsize) pairs with a tiled kernel
#define ALDIC_TILE_SHAPES(X) X(4, 16) X(8, 16) X(8, 24) X(8, 32) X(16, 32)

bool tile_shape(int step, int w, int sx, int sy, TilePlan &P) {
#define ALDIC_TILE_PLAN(S, Wd) \
  if (step == S && w == Wd) return tile_plan<S, Wd>(sx, sy, P);
  ALDIC_TILE_SHAPES(ALDIC_TILE_PLAN)
#undef ALDIC_TILE_PLAN
  return false;
}

int tile_dispatch(const TileArgs &A, const TilePlan &P, int step, cudaStream_t st) {
#define ALDIC_TILE_GO(S, Wd) \
  if (step == S && A.w == Wd) return tile_launch<S, Wd>(A, P, st);
  ALDIC_TILE_SHAPES(ALDIC_TILE_GO)
#undef ALDIC_TILE_GO
  return E_ARG;
}

// work slab: the window table (16 B per pixel), the hand-back list, then
// per tile point (tiles hold at most 8 x 8 points, so (nx + 7) (ny + 7)
// bounds them) the correlation map (4 B per entry of the (2s+3)^2 map), the
// template sums and the outer ring's window sums
struct TileBufs {
  uint4 *tab;
  int *fb;
  unsigned *cmap;
  TileSub *subs;
  uint2 *ringw;
  size_t bytes;
};
TileBufs tile_bufs(char *base, int W, int H, int nx, int ny, const int search[2]) {
  const size_t cr = 2 * search[0] + 3, cc = 2 * search[1] + 3, slots = (size_t)(nx + 7) * (ny + 7);
  TileBufs B;
  size_t o = 0;
  B.tab = reinterpret_cast<uint4 *>(base + o);
  o += align16((size_t)W * H * sizeof(uint4));
  B.fb = reinterpret_cast<int *>(base + o);
  o += align16((size_t)((long long)nx * ny + 1) * sizeof(int));
  B.cmap = reinterpret_cast<unsigned *>(base + o);
  o += align16(slots * cr * cc * sizeof(unsigned));
  B.subs = reinterpret_cast<TileSub *>(base + o);
  o += align16(slots * sizeof(TileSub));
  B.ringw = reinterpret_cast<uint2 *>(base + o);
  o += align16(slots * (2 * (cr + cc) - 4) * sizeof(uint2));
  B.bytes = o;
  return B;
}

// tiled 8-bit search; false in *used when the geometry has no tiled kernel
int tile_search(const uint8_t *f, const uint8_t *g, const SearchGeom &G, SearchWork &sw,
                double *x, double *y, double *u, double *v, double *cc, int threads_pt,
                size_t smem_pt, cudaStream_t st, bool *used) {
  *used = false;
  TilePlan P;
  if (G.step % 4 || G.w % G.step || !tile_shape(G.step, G.w, G.sx, G.sy, P)) return OK;
  const int px1 = G.gx1 - 1, py1 = G.gy1 - 1;
  if (px1 - G.sx - 1 < 0 || py1 - G.sy - 1 < 0) return OK;
  const long long npts = (long long)G.nx * G.ny;
  const int srch[2] = {G.sx, G.sy};
  int rc = search_work_ensure(sw, G.W, G.H, G.nx, G.ny, srch);
  if (rc) return rc;
  const TileBufs B = tile_bufs(sw.buf.as<char>(), G.W, G.H, G.nx, G.ny, srch);
  uint4 *tab = B.tab;
  int *fb = B.fb;
  const long long mn = (long long)G.tw * G.tw;
  // full windows of every shift of every point (outer ring included)
  const int x0 = px1 - G.sx - 1, x1 = px1 + (G.nx - 1) * G.step + G.sx + 1;
  const int y0 = py1 - G.sy - 1, y1 = py1 + (G.ny - 1) * G.step + G.sy + 1;
  const size_t smt = align16((size_t)(kTabY + G.tw - 1) * (kTabX + G.tw - 1)) +
                     2 * sizeof(unsigned) * kTabY * (kTabX + G.tw);
  ALDIC_CUDA(cudaFuncSetAttribute(k_box_tab, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smt));
  k_box_tab<<<dim3((x1 - x0 + kTabX) / kTabX, (y1 - y0 + kTabY) / kTabY), 256, smt, st>>>(
      g, G.W, G.H, G.tw, mn, x0, x1, y0, y1, tab);
  ALDIC_CUDA(cudaMemsetAsync(fb, 0, sizeof(int), st));
  TileArgs A{};
  A.f = f; A.g = g; A.tab = tab; A.cmap = B.cmap; A.subs = B.subs; A.ringw = B.ringw;
  A.W = G.W; A.H = G.H; A.px1 = px1; A.py1 = py1; A.nx = G.nx; A.ny = G.ny; A.w = G.w;
  A.sx = G.sx; A.sy = G.sy; A.cr = G.cr; A.cc = G.cc; A.mn = mn;
  if ((rc = tile_dispatch(A, P, G.step, st))) return rc;
  PeakArgs K{};
  K.cmap = B.cmap; K.ringw = B.ringw; K.subs = B.subs; K.tab = tab; K.mu = G.mu;
  K.ox = x; K.oy = y; K.ou = u; K.ov = v; K.occ = cc; K.fb = fb;
  K.W = G.W; K.px1 = px1; K.py1 = py1; K.nx = G.nx; K.ny = G.ny; K.step = G.step; K.w = G.w;
  K.tw = G.tw; K.sx = G.sx; K.sy = G.sy; K.cr = G.cr; K.cc = G.cc; K.tsy = P.tsy;
  K.tiles_x = (G.nx + kTileTSX - 1) / kTileTSX; K.mn = mn;
  const int pb = (int)std::min<long long>((npts + kPeakWarps - 1) / kPeakWarps, 148 * 16);
  k_search_peak<<<pb, kPeakWarps * 32, 0, st>>>(K);
  ALDIC_CUDA(cudaGetLastError());
  // the points handed back: per-point kernel over the device-side list
  const int nb = (int)std::min<long long>(npts, 296);
  k_search_u8_list<<<nb, threads_pt, smem_pt, st>>>(f, g, G, fb, x, y, u, v, cc);
  ALDIC_CUDA(cudaGetLastError());
  *used = true;
  return OK;
}

// ---- q-factors over the full (2w+2s+1)^2 map (optional, direct sums)
template <typename T>
__global__ void k_qfactor(const T *__restrict__ f, const T *__restrict__ g, SearchGeom G,
                          double *__restrict__ pce, double *__restrict__ ppe) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int fr = 2 * G.w + 2 * G.sx + 1, fc = 2 * G.w + 2 * G.sy + 1;
  double *full = (double *)smem;
  double *Tq = full + fr * fc;
  double *Dq = Tq + G.tw * G.tw;
  __shared__ double red[64];
  __shared__ int hist[30];
  const int pt = blockIdx.x;
  const int ix = pt % G.nx, iy = pt / G.nx;
  const int ii = G.gx1 + ix * G.step, jj = G.gy1 + iy * G.step;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int i = tid; i < G.tw * G.tw; i += nth)
    Tq[i] = (double)f[(long long)(jj - 1 + i / G.tw) * G.W + (ii - 1 + i % G.tw)];
  for (int i = tid; i < G.dw * G.dh; i += nth)
    Dq[i] = (double)g[(long long)(jj - 1 - G.sy + i / G.dw) * G.W + (ii - 1 - G.sx + i % G.dw)];
  if (tid < 30) hist[tid] = 0;
  __syncthreads();
  double st = 0, st2 = 0;
  for (int i = 0; i < G.tw * G.tw; ++i) {
    st += Tq[i];
    st2 += Tq[i] * Tq[i];
  }
  const double mn = (double)G.tw * G.tw;
  const bool flat = !(mn * st2 - st * st > 0);
  if (flat) {
    if (tid == 0) {
      pce[pt] = __longlong_as_double(0x7ff0000000000000ll);
      ppe[pt] = __longlong_as_double(0x7ff0000000000000ll);
    }
    return;
  }
  for (int e = tid; e < fr * fc; e += nth) {
    const int a = e % fr, b = e / fr;
    const int ox0 = a - G.w, oy0 = b - G.w;  // template offset in D
    const int x0 = ox0 < 0 ? -ox0 : 0, y0 = oy0 < 0 ? -oy0 : 0;
    int x1 = G.tw, y1 = G.tw;
    if (ox0 + x1 > G.dw) x1 = G.dw - ox0;
    if (oy0 + y1 > G.dh) y1 = G.dh - oy0;
    double r = 0.0;
    if (x1 > x0 && y1 > y0) {
      double sd = 0, sd2 = 0, stdv = 0, st_in = 0;
      for (int ty = y0; ty < y1; ++ty)
        for (int tx = x0; tx < x1; ++tx) {
          const double d = Dq[(ty + oy0) * G.dw + tx + ox0], t = Tq[ty * G.tw + tx];
          sd += d;
          sd2 += d * d;
          stdv += t * d;
          st_in += t;
        }
      const double n_pad = mn - (double)(x1 - x0) * (y1 - y0);
      r = ncc_combine_f(mn, st, st2, stdv, sd, sd2, st - st_in, n_pad, *G.mu);
    }
    full[e] = r;
  }
  __syncthreads();
  // min, then sum of squares and max of cc - min, then histogram
  double mnv = 1e300;
  for (int e = tid; e < fr * fc; e += nth) mnv = fmin(mnv, full[e]);
  for (int o = 16; o > 0; o >>= 1) mnv = fmin(mnv, __shfl_xor_sync(0xffffffffu, mnv, o));
  if ((tid & 31) == 0) red[tid >> 5] = mnv;
  __syncthreads();
  if (tid == 0) {
    for (int k = 1; k < (nth + 31) / 32; ++k) mnv = fmin(mnv, red[k]);
    red[32] = mnv;
  }
  __syncthreads();
  mnv = red[32];
  double pk = 0, ss = 0;
  for (int e = tid; e < fr * fc; e += nth) {
    const double v = full[e] - mnv;
    pk = fmax(pk, v);
    ss += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    pk = fmax(pk, __shfl_xor_sync(0xffffffffu, pk, o));
    ss += __shfl_xor_sync(0xffffffffu, ss, o);
  }
  __syncthreads();
  if ((tid & 31) == 0) {
    red[tid >> 5] = pk;
    red[32 + (tid >> 5)] = ss;
  }
  __syncthreads();
  if (tid == 0) {
    double P = 0, Sq = 0;
    for (int k = 0; k < (nth + 31) / 32; ++k) {
      P = fmax(P, red[k]);
      Sq += red[32 + k];
    }
    red[0] = P;
    red[1] = Sq;
  }
  __syncthreads();
  const double peak = red[0], sumsq = red[1];
  for (int e = tid; e < fr * fc; e += nth) {
    const double v = full[e] - mnv;
    int bb = peak > 0 ? (int)floor(v / peak * 30.0) : 0;
    bb = bb > 29 ? 29 : (bb < 0 ? 0 : bb);
    atomicAdd(&hist[bb], 1);
  }
  __syncthreads();
  if (tid == 0) {
    const double n = (double)(fr * fc);
    pce[pt] = (peak * peak) / (sumsq / n);
    double ent = 0;
    for (int k = 0; k < 30; ++k) {
      const double p = hist[k] / n;
      if (p > 0) ent += p * log(1.0 / p);
    }
    ppe[pt] = 1.0 / ent;
  }
}

constexpr size_t kSmemMax = 227 * 1024;
constexpr int kBigBlocks = 296;  // CTAs (and global work slots) of the big-region search

// Search regions too large for shared memory: the per-point kernel with its
// row sums and map in global work slots, one per CTA, kBigBlocks CTAs
// looping over the points.  The slots are in SearchWork::big, sized before
// any capture by search_work_ensure (or here, outside a capture).
template <typename T>
int launch_big(const void *f, const void *g, const SearchGeom &G, double *x, double *y, double *u,
               double *v, double *cc, cudaStream_t st, SearchWork *sw) {
  using Tr = SearchTraits<T>;
  using V = typename Tr::V;
  using S = typename SumT<Tr::integer>::type;
  const SmemLayout<V, S> L(G, true);
  ALDIC_CHECK(L.total <= kSmemMax, E_ARG,
              "integer search: window/search size too large even with the map in global memory");
  const int npts = G.nx * G.ny;
  const int blocks = npts < kBigBlocks ? npts : kBigBlocks;
  const size_t need = L.slot * (size_t)blocks;
  ALDIC_CHECK(sw != nullptr, E_ARG, "integer search: this search region needs the context's work memory");
  if (sw->big.cap < need) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    ALDIC_CUDA(cudaStreamIsCapturing(st, &cs));
    ALDIC_CHECK(cs == cudaStreamCaptureStatusNone, E_STATE,
                "integer search: work memory for this search region was not set up before capture");
    int rc = sw->big.ensure(need);
    if (rc) return rc;
  }
  int threads = ((G.cc * G.nsx + 31) / 32) * 32;
  if (threads < 64) threads = 64;
  if (threads > 512) threads = 512;
  ALDIC_CUDA(cudaFuncSetAttribute(k_search<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)L.total));
  k_search<T, true><<<blocks, threads, L.total, st>>>((const T *)f, (const T *)g, G, x, y, u, v, cc,
                                                      sw->big.as<unsigned char>());
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

template <typename T>
int launch_search(const void *f, const void *g, const SearchGeom &G, double *x, double *y,
                  double *u, double *v, double *cc, double *pce, double *ppe, cudaStream_t st,
                  SearchWork *sw) {
  using Tr = SearchTraits<T>;
  using V = typename Tr::V;
  using S = typename SumT<Tr::integer>::type;
  const int nstrips = G.cc * G.nsx;
  int threads = ((nstrips + 31) / 32) * 32;
  if (threads < 64) threads = 64;
  if (threads > 512) threads = 512;
  const int npts = G.nx * G.ny;
  if (npts == 0) return OK;
  if (sizeof(T) == 1 && !(U8Layout(G).total <= kSmemMax && G.tw <= 72)) {
    const int rc = launch_big<T>(f, g, G, x, y, u, v, cc, st, sw);
    if (rc) return rc;
  } else if (sizeof(T) == 1) {
    U8Layout L(G);
    ALDIC_CUDA(cudaFuncSetAttribute(k_search_u8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)L.total));
    ALDIC_CUDA(cudaFuncSetAttribute(k_search_u8_list,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    bool tiled = false;
    if (sw) {
      const int rc = tile_search((const uint8_t *)f, (const uint8_t *)g, G, *sw, x, y, u, v, cc,
                                 threads, L.total, st, &tiled);
      if (rc) return rc;
    }
    if (!tiled)
      k_search_u8<<<npts, threads, L.total, st>>>((const uint8_t *)f, (const uint8_t *)g, G, x,
                                                   y, u, v, cc);
  } else if (sizeof(T) == 2 && U16Layout(G).total <= kSmemMax && G.tw <= 72) {
    const U16Layout L(G);
    ALDIC_CUDA(cudaFuncSetAttribute(k_search_u16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)L.total));
    k_search_u16<<<npts, threads, L.total, st>>>((const uint16_t *)f, (const uint16_t *)g, G, x, y,
                                                  u, v, cc);
  } else {
    SmemLayout<V, S> L(G);
    if (L.total > kSmemMax) {
      const int rc = launch_big<T>(f, g, G, x, y, u, v, cc, st, sw);
      if (rc) return rc;
    } else {
      ALDIC_CUDA(cudaFuncSetAttribute(k_search<T, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
      k_search<T, false><<<npts, threads, L.total, st>>>((const T *)f, (const T *)g, G, x, y, u, v,
                                                         cc, nullptr);
    }
  }
  ALDIC_CUDA(cudaGetLastError());
  if (pce) {
    const int fr = 2 * G.w + 2 * G.sx + 1, fc = 2 * G.w + 2 * G.sy + 1;
    const size_t sm = sizeof(double) * ((size_t)fr * fc + (size_t)G.tw * G.tw + (size_t)G.dw * G.dh);
    ALDIC_CHECK(sm <= 227 * 1024, E_ARG, "q-factors: full correlation map too large for shared memory");
    ALDIC_CUDA(cudaFuncSetAttribute(k_qfactor<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_qfactor<T><<<npts, 256, sm, st>>>((const T *)f, (const T *)g, G, pce, ppe);
    ALDIC_CUDA(cudaGetLastError());
  }
  return OK;
}

}  // namespace

int search_dims(int W, int H, const int gridx[2], const int gridy[2], int winsize, int step,
                const int search[2], int *nx, int *ny, int *gx1o, int *gy1o) {
  // funIntegerSearch.m:14-25 and :90-91
  if (step <= 0 || winsize <= 0 || search[0] < 0 || search[1] < 0) return E_ARG;
  int gx1 = gridx[0], gx2 = gridx[1], gy1 = gridy[0], gy2 = gridy[1];
  const double hw = 0.5 * winsize, w15 = 1.5 * winsize;
  while (gx1 - search[0] - hw < 1) gx1++;
  while (gy1 - search[1] - hw < 1) gy1++;
  while (gx2 + w15 + search[0] > W) gx2--;
  while (gy2 + w15 + search[1] > H) gy2--;
  *nx = (gx2 - step >= gx1) ? (gx2 - step - gx1) / step + 1 : 0;
  *ny = (gy2 - step >= gy1) ? (gy2 - step - gy1) / step + 1 : 0;
  if (gx1o) *gx1o = gx1;
  if (gy1o) *gy1o = gy1;
  return OK;
}

// the window / region / map extents of a search geometry (funIntegerSearch.m:121-134)
void geom_sizes(SearchGeom &G, int winsize, const int search[2]) {
  G.w = winsize; G.sx = search[0]; G.sy = search[1];
  G.tw = winsize + 1;
  G.twp = (G.tw + KX - 1) / KX * KX;
  G.dw = G.tw + 2 * G.sx;
  G.dh = G.tw + 2 * G.sy;
  G.cr = 2 * G.sx + 3;
  G.cc = 2 * G.sy + 3;
  G.nsx = (G.cr + KX - 1) / KX;
  G.dpw = G.nsx * KX + G.twp - 1;
  if (G.dpw < G.dw + 2) G.dpw = G.dw + 2;
  G.dph = G.dh + 2;
}

template <typename T>
size_t big_bytes(const SearchGeom &G) {
  using Tr = SearchTraits<T>;
  using S = typename SumT<Tr::integer>::type;
  const bool small = sizeof(T) == 1 ? (U8Layout(G).total <= kSmemMax && G.tw <= 72)
                                    : ((sizeof(T) == 2 && U16Layout(G).total <= kSmemMax && G.tw <= 72) ||
                                       SmemLayout<typename Tr::V, S>(G).total <= kSmemMax);
  if (small) return 0;
  const int npts = G.nx * G.ny;
  return SmemLayout<typename Tr::V, S>(G, true).slot * (size_t)(npts < kBigBlocks ? npts : kBigBlocks);
}

int search_work_ensure(SearchWork &w, int W, int H, int nx, int ny, const int search[2], int winsize,
                       int dtype) {
  int rc = w.buf.ensure(tile_bufs(nullptr, W, H, nx, ny, search).bytes);
  if (rc || winsize <= 0) return rc;
  SearchGeom G{};
  G.nx = nx;
  G.ny = ny;
  geom_sizes(G, winsize, search);
  const size_t b = dtype == 0 ? big_bytes<uint8_t>(G) : dtype == 1 ? big_bytes<uint16_t>(G)
                 : dtype == 2 ? big_bytes<float>(G) : big_bytes<double>(G);
  return b ? w.big.ensure(b) : OK;
}

int int_search(const void *f_raw, const void *g_raw, int dtype, int W, int H, const double *mu_g,
               const int gridx[2], const int gridy[2], int winsize, int step,
               const int search[2], double *x, double *y, double *u, double *v, double *cc,
               double *pce, double *ppe, cudaStream_t st, SearchWork *sw) {
  SearchGeom G;
  int rc = search_dims(W, H, gridx, gridy, winsize, step, search, &G.nx, &G.ny, &G.gx1, &G.gy1);
  if (rc) return rc;
  G.W = W; G.H = H; G.step = step;
  geom_sizes(G, winsize, search);
  G.mu = mu_g;
  switch (dtype) {
    case 0: return launch_search<uint8_t>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st, sw);
    case 1: return launch_search<uint16_t>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st, sw);
    case 2: return launch_search<float>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st, sw);
    default: return launch_search<double>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st, sw);
  }
}

}  // namespace aldic
