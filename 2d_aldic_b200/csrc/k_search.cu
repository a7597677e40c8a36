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

template <typename V, typename S>
struct SmemLayout {
  size_t tp, dp, rs, rs2, colsum, rowsum, map, red, total;
  __host__ __device__ SmemLayout(const SearchGeom &g) {
    size_t o = 0;
    tp = o; o = align16(o + sizeof(V) * g.tw * g.twp);
    dp = o; o = align16(o + sizeof(V) * g.dph * g.dpw);
    rs = o; o = align16(o + sizeof(S) * g.dph * g.cr);
    rs2 = o; o = align16(o + sizeof(S) * g.dph * g.cr);
    colsum = o; o = align16(o + sizeof(S) * g.tw);
    rowsum = o; o = align16(o + sizeof(S) * g.tw);
    map = o; o = align16(o + sizeof(double) * g.cr * g.cc);
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

template <typename T>
__global__ void __launch_bounds__(512) k_search(const T *__restrict__ f, const T *__restrict__ g,
                                                SearchGeom G, double *__restrict__ ox,
                                                double *__restrict__ oy, double *__restrict__ ou,
                                                double *__restrict__ ov, double *__restrict__ occ) {
  using Tr = SearchTraits<T>;
  using V = typename Tr::V;
  using RowAcc = typename Tr::RowAcc;
  using S = typename SumT<Tr::integer>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout<V, S> L(G);
  V *Tp = (V *)(smem + L.tp);
  V *Dp = (V *)(smem + L.dp);
  S *RS = (S *)(smem + L.rs);
  S *RS2 = (S *)(smem + L.rs2);
  S *colsum = (S *)(smem + L.colsum);
  S *rowsum = (S *)(smem + L.rowsum);
  double *map = (double *)(smem + L.map);
  double *redv = (double *)(smem + L.red);
  int *redi = (int *)(redv + 32);
  __shared__ S s_st, s_st2;
  const double mu = *G.mu;

  const int pt = blockIdx.x;
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
    return;
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

__global__ void __launch_bounds__(512) k_search_u8(const uint8_t *__restrict__ f,
                                                   const uint8_t *__restrict__ g, SearchGeom G,
                                                   double *__restrict__ ox,
                                                   double *__restrict__ oy,
                                                   double *__restrict__ ou,
                                                   double *__restrict__ ov,
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
  const int pt = blockIdx.x;
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

template <typename T>
int launch_search(const void *f, const void *g, const SearchGeom &G, double *x, double *y,
                  double *u, double *v, double *cc, double *pce, double *ppe, cudaStream_t st) {
  using Tr = SearchTraits<T>;
  using V = typename Tr::V;
  using S = typename SumT<Tr::integer>::type;
  const int nstrips = G.cc * G.nsx;
  int threads = ((nstrips + 31) / 32) * 32;
  if (threads < 64) threads = 64;
  if (threads > 512) threads = 512;
  const int npts = G.nx * G.ny;
  if (npts == 0) return OK;
  if (sizeof(T) == 1) {
    U8Layout L(G);
    ALDIC_CHECK(L.total <= 227 * 1024 && G.tw <= 72, E_ARG,
                "integer search: window/search size too large for shared memory");
    ALDIC_CUDA(cudaFuncSetAttribute(k_search_u8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)L.total));
    k_search_u8<<<npts, threads, L.total, st>>>((const uint8_t *)f, (const uint8_t *)g, G, x, y,
                                                 u, v, cc);
  } else {
    SmemLayout<V, S> L(G);
    ALDIC_CHECK(L.total <= 227 * 1024, E_ARG,
                "integer search: window/search size too large for shared memory");
    ALDIC_CUDA(cudaFuncSetAttribute(k_search<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)L.total));
    k_search<T><<<npts, threads, L.total, st>>>((const T *)f, (const T *)g, G, x, y, u, v, cc);
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

int int_search(const void *f_raw, const void *g_raw, int dtype, int W, int H, const double *mu_g,
               const int gridx[2], const int gridy[2], int winsize, int step,
               const int search[2], double *x, double *y, double *u, double *v, double *cc,
               double *pce, double *ppe, cudaStream_t st) {
  SearchGeom G;
  int rc = search_dims(W, H, gridx, gridy, winsize, step, search, &G.nx, &G.ny, &G.gx1, &G.gy1);
  if (rc) return rc;
  G.W = W; G.H = H; G.step = step; G.w = winsize; G.sx = search[0]; G.sy = search[1];
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
  G.mu = mu_g;
  switch (dtype) {
    case 0: return launch_search<uint8_t>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st);
    case 1: return launch_search<uint16_t>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st);
    case 2: return launch_search<float>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st);
    default: return launch_search<double>(f_raw, g_raw, G, x, y, u, v, cc, pce, ppe, st);
  }
}

}  // namespace aldic
