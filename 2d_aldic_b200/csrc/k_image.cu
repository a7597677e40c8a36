// k_image.cu -- image preparation (a1 normalisation, a2 gradients) and the
// standalone bicubic sampler (a3, ba_interp2).
//
// Normalisation follows funNormalizeImg.m:22-39; for integer images the ROI
// sums are exact (integer atomics), so mean/std match the CPU restatement bit
// for bit.  Gradients follow funImgGradient.m:53-78 with the symmetric taps
// paired; the FP64 arithmetic is written with explicit round-to-nearest
// intrinsics so no FMA contraction changes the result.
#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {

// ------------------------------------------------------------------ ROI stats
template <typename T>
__global__ void k_roi_sums_int(const T *__restrict__ img, int W, int x0, int x1, int y0,
                               int y1, unsigned long long *__restrict__ sums) {
  const int rw = x1 - x0 + 1;
  const long long n = (long long)rw * (y1 - y0 + 1);
  unsigned long long s1 = 0, s2 = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = y0 + (int)(i / rw), x = x0 + (int)(i % rw);
    const unsigned long long v = img[(long long)(y - 1) * W + (x - 1)];
    s1 += v;
    s2 += v * v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], s1);
    atomicAdd(&sums[1], s2);
  }
}

// deterministic per-block partials of sum(v - m)^p, p in {1,2}
template <typename T>
__global__ void k_roi_partials(const T *__restrict__ img, int W, int x0, int x1, int y0,
                               int y1, const double *__restrict__ mean, int pw,
                               double *__restrict__ part) {
  const int rw = x1 - x0 + 1;
  const long long n = (long long)rw * (y1 - y0 + 1);
  const double m = pw == 2 ? *mean : 0.0;
  double s = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = y0 + (int)(i / rw), x = x0 + (int)(i % rw);
    const double v = (double)img[(long long)(y - 1) * W + (x - 1)] - m;
    s += pw == 2 ? v * v : v;
  }
  s = warp_sum(s);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    part[blockIdx.x] = t;
  }
}

__global__ void k_stats_int_final(const unsigned long long *sums, long long n, double *out) {
  const double m = (double)sums[0] / (double)n;
  const double ssd = __dsub_rn((double)sums[1], __dmul_rn(m, (double)sums[0]));
  out[0] = m;
  out[1] = sqrt(ssd / (double)(n - 1));
}

__global__ void k_sum_partials(const double *part, int np, long long n, int pw, double *out) {
  double t = 0;
  for (int k = 0; k < np; ++k) t += part[k];
  if (pw == 1) out[0] = t / (double)n;
  else out[1] = sqrt(t / (double)(n - 1));
}

int roi_stats(const void *img, int dtype, int W, const int roi[4], double *d_stats,
              unsigned long long *d_isums, double *d_part, cudaStream_t st) {
  const long long n = (long long)(roi[1] - roi[0] + 1) * (roi[3] - roi[2] + 1);
  const int blocks = 296, threads = 256;
  if (dtype == 0 || dtype == 1) {
    ALDIC_CUDA(cudaMemsetAsync(d_isums, 0, 2 * sizeof(unsigned long long), st));
    if (dtype == 0)
      k_roi_sums_int<uint8_t><<<blocks, threads, 0, st>>>((const uint8_t *)img, W, roi[0],
                                                          roi[1], roi[2], roi[3], d_isums);
    else
      k_roi_sums_int<uint16_t><<<blocks, threads, 0, st>>>((const uint16_t *)img, W, roi[0],
                                                           roi[1], roi[2], roi[3], d_isums);
    k_stats_int_final<<<1, 1, 0, st>>>(d_isums, n, d_stats);
  } else {
    for (int pw = 1; pw <= 2; ++pw) {
      if (dtype == 2)
        k_roi_partials<float><<<blocks, threads, 0, st>>>((const float *)img, W, roi[0], roi[1],
                                                          roi[2], roi[3], d_stats, pw, d_part);
      else
        k_roi_partials<double><<<blocks, threads, 0, st>>>((const double *)img, W, roi[0],
                                                           roi[1], roi[2], roi[3], d_stats, pw,
                                                           d_part);
      k_sum_partials<<<1, 1, 0, st>>>(d_part, blocks, n, pw, d_stats);
    }
  }
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------------------ normalise
template <typename T>
__global__ void k_normalize(const T *__restrict__ img, long long n,
                            const double *__restrict__ stats, double *__restrict__ o64,
                            float *__restrict__ o32) {
  const double m = stats[0], s = stats[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = __ddiv_rn(__dsub_rn((double)img[i], m), s);
    o64[i] = v;
    o32[i] = __double2float_rn(v);
  }
}

int normalize(const void *img, int dtype, long long n, const double *d_stats, double *o64,
              float *o32, cudaStream_t st) {
  const int blocks = 1184, threads = 256;
  switch (dtype) {
    case 0: k_normalize<uint8_t><<<blocks, threads, 0, st>>>((const uint8_t *)img, n, d_stats, o64, o32); break;
    case 1: k_normalize<uint16_t><<<blocks, threads, 0, st>>>((const uint16_t *)img, n, d_stats, o64, o32); break;
    case 2: k_normalize<float><<<blocks, threads, 0, st>>>((const float *)img, n, d_stats, o64, o32); break;
    default: k_normalize<double><<<blocks, threads, 0, st>>>((const double *)img, n, d_stats, o64, o32); break;
  }
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// ---------------------------------------------------- row-cubic coefficients
// The Keys cubic (a = -1/2) of ba_interp2.cpp along one row as a polynomial:
// with taps g_k (k = 0..3 at offsets -1..2 from the floor column) and
// fraction t, sum_k w_k(t) g_k = a0 + a1 t + a2 t^2 + a3 t^3, where row p of
// the 4 x 4 matrix behind keys_rows holds the t^p coefficients of the four
// Keys weights.  q[y W + x] = (a0, a1, a2, a3) of row y with floor column x,
// from the FP64 image and rounded once to FP32 (zeros where the stencil
// leaves the row: the IC-GN out-of-image test keeps every sampled floor
// column in [2, W-3]).  A bicubic sample is then four Horner rules over tu
// on consecutive rows and one cubic over tv -- and consecutive rows of a
// subset column share three of their four stencil rows.
__device__ __forceinline__ void keys_rows(const double g[4], double a[4]) {
  a[0] = g[1];
  a[1] = 0.5 * (g[2] - g[0]);
  a[2] = g[0] - 2.5 * g[1] + 2.0 * g[2] - 0.5 * g[3];
  a[3] = 0.5 * (g[3] - g[0]) + 1.5 * (g[1] - g[2]);
}

__global__ void k_row_cubic(const double *__restrict__ g, int W, long long n,
                            float4 *__restrict__ q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % W);
    if (x < 1 || x > W - 3) {
      q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      continue;
    }
    const double t[4] = {__ldg(g + i - 1), __ldg(g + i), __ldg(g + i + 1), __ldg(g + i + 2)};
    double a[4];
    keys_rows(t, a);
    q[i] = make_float4((float)a[0], (float)a[1], (float)a[2], (float)a[3]);
  }
}

int row_cubic(const double *g, int W, int H, float4 *q, cudaStream_t st) {
  k_row_cubic<<<1184, 256, 0, st>>>(g, W, (long long)W * H, q);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// q[i] = (gx[i], gy[i]): the two FP32 gradients of a pixel in one 8-byte load
__global__ void k_pair(const float *__restrict__ gx, const float *__restrict__ gy, long long n,
                       float2 *__restrict__ q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    q[i] = make_float2(gx[i], gy[i]);
}

int grad_pairs(const float *gx, const float *gy, long long n, float2 *q, cudaStream_t st) {
  k_pair<<<1184, 256, 0, st>>>(gx, gy, n, q);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}


// ------------------------------------------------------------------ gradient
__device__ __forceinline__ double grad7(const double *f, long long i, long long s) {
  const double c1 = 0.75, c2 = 3.0 / 20.0, c3 = 1.0 / 60.0;
  const double a = __dmul_rn(c1, __dsub_rn(f[i + s], f[i - s]));
  const double b = __dmul_rn(c2, __dsub_rn(f[i + 2 * s], f[i - 2 * s]));
  const double c = __dmul_rn(c3, __dsub_rn(f[i + 3 * s], f[i - 3 * s]));
  return __dadd_rn(__dsub_rn(a, b), c);
}

__global__ void k_gradient(const double *__restrict__ f, const double *__restrict__ mask, int W,
                           int H, double *__restrict__ gx64, double *__restrict__ gy64,
                           float *__restrict__ gx32, float *__restrict__ gy32) {
  const long long n = (long long)W * H;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / W), x = (int)(i % W);
    double tx = 0.0, ty = 0.0;
    if (x >= 3 && x < W - 3 && y >= 3 && y < H - 3) {
      const double m = mask ? mask[i] : 1.0;
      tx = __dmul_rn(grad7(f, i, 1), m);
      ty = __dmul_rn(grad7(f, i, W), m);
    }
    gx64[i] = tx;
    gy64[i] = ty;
    gx32[i] = __double2float_rn(tx);
    gy32[i] = __double2float_rn(ty);
  }
}

int gradient(const double *f, const double *mask, int W, int H, double *gx64, double *gy64,
             float *gx32, float *gy32, cudaStream_t st) {
  k_gradient<<<1184, 256, 0, st>>>(f, mask, W, H, gx64, gy64, gx32, gy32);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// ------------------------------------------------------------------ ba_interp2
// ba_interp2.cpp:133-182 restated with explicit rounding so both precisions
// reproduce the reference's compiled results bit for bit.
__device__ __forceinline__ long long corner_index(double cf, long long extent) {
  const double lo = -4.0, hi = (double)extent + 4.0;
  const double c = cf < lo ? lo : (cf > hi ? hi : cf);
  return (long long)(c - 1.0);
}
__device__ __forceinline__ long long clampll(long long v, long long lo, long long hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

__device__ __forceinline__ void weights_f64(double d, double w[4]) {
  const double d2 = __dmul_rn(d, d), d3 = __dmul_rn(d2, d);
  w[0] = __dmul_rn(0.5, __dsub_rn(__dadd_rn(-d, __dmul_rn(2.0, d2)), d3));
  w[1] = __dmul_rn(0.5, __dadd_rn(__dsub_rn(2.0, __dmul_rn(5.0, d2)), __dmul_rn(3.0, d3)));
  w[2] = __dmul_rn(0.5, __dsub_rn(__dadd_rn(d, __dmul_rn(4.0, d2)), __dmul_rn(3.0, d3)));
  w[3] = __dmul_rn(0.5, __dadd_rn(-d2, d3));
}

// float inputs: the weight polynomials run in double from float powers
__device__ __forceinline__ void weights_f32(float d, float w[4]) {
  const float d2 = __fmul_rn(d, d), d3 = __fmul_rn(d2, d);
  const double D = d, D2 = d2, D3 = d3;
  w[0] = __double2float_rn(__dmul_rn(0.5, __dsub_rn(__dadd_rn((double)(-d), __dmul_rn(2.0, D2)), D3)));
  w[1] = __double2float_rn(__dmul_rn(0.5, __dadd_rn(__dsub_rn(2.0, __dmul_rn(5.0, D2)), __dmul_rn(3.0, D3))));
  w[2] = __double2float_rn(__dmul_rn(0.5, __dsub_rn(__dadd_rn(D, __dmul_rn(4.0, D2)), __dmul_rn(3.0, D3))));
  w[3] = __double2float_rn(__dmul_rn(0.5, (double)__fadd_rn(-d2, d3)));
}

__global__ void k_interp_f64(const double *__restrict__ F, long long M, long long N, long long P,
                             const double *__restrict__ X, const double *__restrict__ Y,
                             long long n, double *__restrict__ Z) {
  const long long LO = M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double x = X[i], y = Y[i];
    if (!isfinite(x) || !isfinite(y)) {
      for (long long j = 0; j < P; ++j) Z[i + j * n] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    const double xf = floor(x), yf = floor(y);
    double wx[4], wy[4];
    weights_f64(__dsub_rn(x, xf), wx);
    weights_f64(__dsub_rn(y, yf), wy);
    const long long xc = corner_index(xf, N), yc = corner_index(yf, M);
    long long c[4], r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c[k] = clampll(xc - 1 + k, 0, N - 1) * M;
      r[k] = clampll(yc - 1 + k, 0, M - 1);
    }
    for (long long j = 0; j < P; ++j) {
      const double *Fj = F + j * LO;
      double acc = 0.0;
#pragma unroll
      for (int rr = 0; rr < 4; ++rr) {
        double s = __dmul_rn(wx[0], Fj[c[0] + r[rr]]);
        s = __dadd_rn(s, __dmul_rn(wx[1], Fj[c[1] + r[rr]]));
        s = __dadd_rn(s, __dmul_rn(wx[2], Fj[c[2] + r[rr]]));
        s = __dadd_rn(s, __dmul_rn(wx[3], Fj[c[3] + r[rr]]));
        acc = rr == 0 ? __dmul_rn(wy[0], s) : __dadd_rn(acc, __dmul_rn(wy[rr], s));
      }
      Z[i + j * n] = acc;
    }
  }
}

__global__ void k_interp_f32(const float *__restrict__ F, long long M, long long N, long long P,
                             const float *__restrict__ X, const float *__restrict__ Y,
                             long long n, float *__restrict__ Z) {
  const long long LO = M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float x = X[i], y = Y[i];
    if (!isfinite(x) || !isfinite(y)) {
      for (long long j = 0; j < P; ++j) Z[i + j * n] = __int_as_float(0x7fc00000);
      continue;
    }
    const float xf = floorf(x), yf = floorf(y);
    float wx[4], wy[4];
    weights_f32(__fsub_rn(x, xf), wx);
    weights_f32(__fsub_rn(y, yf), wy);
    const long long xc = corner_index((double)xf, N), yc = corner_index((double)yf, M);
    long long c[4], r[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c[k] = clampll(xc - 1 + k, 0, N - 1) * M;
      r[k] = clampll(yc - 1 + k, 0, M - 1);
    }
    for (long long j = 0; j < P; ++j) {
      const float *Fj = F + j * LO;
      float acc = 0.0f;
#pragma unroll
      for (int rr = 0; rr < 4; ++rr) {
        float s = __fmul_rn(wx[0], Fj[c[0] + r[rr]]);
        s = __fadd_rn(s, __fmul_rn(wx[1], Fj[c[1] + r[rr]]));
        s = __fadd_rn(s, __fmul_rn(wx[2], Fj[c[2] + r[rr]]));
        s = __fadd_rn(s, __fmul_rn(wx[3], Fj[c[3] + r[rr]]));
        acc = rr == 0 ? __fmul_rn(wy[0], s) : __fadd_rn(acc, __fmul_rn(wy[rr], s));
      }
      Z[i + j * n] = acc;
    }
  }
}

int interp_f64(const double *F, long long M, long long N, long long P, const double *X,
               const double *Y, long long n, double *Z, cudaStream_t st) {
  if (n <= 0) return OK;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_interp_f64<<<(int)blocks, 256, 0, st>>>(F, M, N, P, X, Y, n, Z);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int interp_f32(const float *F, long long M, long long N, long long P, const float *X,
               const float *Y, long long n, float *Z, cudaStream_t st) {
  if (n <= 0) return OK;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_interp_f32<<<(int)blocks, 256, 0, st>>>(F, M, N, P, X, Y, n, Z);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

}  // namespace aldic
