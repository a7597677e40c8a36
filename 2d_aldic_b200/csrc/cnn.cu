// cnn.cu -- the learned initial guess: a Siamese patch network that maps a
// reference / deformed 64 x 64 patch pair to the six affine warp parameters
// of the subset at its centre plus a confidence logit.  No counterpart in the
// reference (its data-driven guess is POD-GPR over earlier frames).
//
//   x   [2B, 64, 64, 1]  the B reference patches, then the B deformed ones,
//                        each normalised to zero mean and unit deviation
//   E1  8x8 patches -> 128 (K = 64), ReLU      e1 [2B, 8, 8, 128]
//   E2  1x1 -> 128 (linear)                    e2 [2B, 8, 8, 128]
//   C   all-pairs cell correlation of the two patches' features,
//       corr[b][i][j] = e2_f[b][i] . e2_g[b][j] / sqrt(128)   [B, 64 x 64]
//   L3  dense 4096 -> 256, ReLU                y3 [B, 256]
//   L4  dense 256 -> 8 (FP32)                  out [B, 8]: u/16, v/16,
//        20 du/dx, 20 dv/dx, 20 du/dy, 20 dv/dy, confidence logit, 0
// E1, E2, C and L3 run on the tcgen05 GEMM (bf16 operands, FP32
// accumulation; C as B independent 64 x 64 x 128 products); their backward
// products are the same GEMM with transposed operands.  The encoder sees
// both patches as one batch of 2B, so its weight gradients sum over both.
// Parameters are FP32 masters updated by Adam; bf16 copies feed the GEMMs.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <random>
#include <vector>

#include "../../include/aldic_b200.h"
#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {
namespace cnn {

constexpr int P = 64, PS = 8, CELLS = (P / PS) * (P / PS), C1 = 128, C2 = 128, F3 = 256, NOUT = 8;
constexpr int K1 = PS * PS, K2 = C1, K3 = CELLS * CELLS, K5 = F3;
constexpr float TSCALE = 16.f, GSCALE = 20.f;
constexpr int NL = 4;
// parameter blocks: W1 b1 W2 b2 W3 b3 W4 b4 (E1, E2, L3, L4)
constexpr long long NW[NL] = {(long long)C1 * K1, (long long)C2 * K2, (long long)F3 * K3,
                              (long long)NOUT * K5};
constexpr long long NB[NL] = {C1, C2, F3, NOUT};

long long n_params() {
  long long s = 0;
  for (int l = 0; l < NL; ++l) s += NW[l] + NB[l];
  return s;
}

}  // namespace cnn

namespace {

using bf16 = __nv_bfloat16;

__global__ void k_patches(const float *__restrict__ f, const float *__restrict__ g, int W, int H,
                          const double *__restrict__ coords, long long n, bf16 *__restrict__ outb,
                          float *__restrict__ outf) {
  const long long p = blockIdx.x;
  if (p >= n) return;
  const int x0 = (int)floor(coords[p] + 0.5), y0 = (int)floor(coords[n + p] + 0.5);
  __shared__ float sh[2][cnn::P * cnn::P];
  __shared__ double red[4][32];
  double s[4] = {0, 0, 0, 0};
  for (int q = threadIdx.x; q < cnn::P * cnn::P; q += blockDim.x) {
    const int r = q / cnn::P, c = q - r * cnn::P;
    int x = x0 - cnn::P / 2 + c, y = y0 - cnn::P / 2 + r;  // 1-based pixel
    x = x < 1 ? 1 : (x > W ? W : x);
    y = y < 1 ? 1 : (y > H ? H : y);
    const long long o = (long long)(y - 1) * W + (x - 1);
    const float a = f[o], b = g[o];
    sh[0][q] = a;
    sh[1][q] = b;
    s[0] += a; s[1] += (double)a * a; s[2] += b; s[3] += (double)b * b;
  }
  for (int k = 0; k < 4; ++k) {
    double v = warp_sum(s[k]);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  __shared__ float mean[2], inv[2];
  if (threadIdx.x < 2) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red[2 * threadIdx.x][w];
      b += red[2 * threadIdx.x + 1][w];
    }
    const double m = a / (cnn::P * cnn::P), var = b / (cnn::P * cnn::P) - m * m;
    mean[threadIdx.x] = (float)m;
    inv[threadIdx.x] = var > 1e-12 ? (float)(1.0 / sqrt(var)) : 0.f;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < cnn::P * cnn::P; q += blockDim.x)
    for (int ch = 0; ch < 2; ++ch) {
      const float v = (sh[ch][q] - mean[ch]) * inv[ch];
      const long long o = (p * cnn::P * cnn::P + q) * 2 + ch;
      if (outb) outb[o] = __float2bfloat16_rn(v);
      if (outf) outf[o] = v;
    }
}

// pairs [B, 64, 64, 2] -> the encoder batch [2B, 64, 64]: reference patches
// first, deformed patches after them
__global__ void k_split(const bf16 *__restrict__ pairs, long long B, bf16 *__restrict__ x) {
  const long long n = B * cnn::P * cnn::P;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    x[k] = pairs[2 * k];
    x[n + k] = pairs[2 * k + 1];
  }
}

__global__ void k_f2bf(const float *__restrict__ a, bf16 *__restrict__ b, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    b[k] = __float2bfloat16_rn(a[k]);
}

// out[b][o] = y[b] . W[o] + bias[o] (the FP32 output layer)
__global__ void k_fc5(const bf16 *__restrict__ y4, const float *__restrict__ W5,
                      const float *__restrict__ b5, float *__restrict__ out, int B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= B * cnn::NOUT) return;
  const int b = t / cnn::NOUT, o = t - b * cnn::NOUT;
  float s = b5[o];
  for (int k = 0; k < cnn::K5; ++k) s += __bfloat162float(y4[(long long)b * cnn::K5 + k]) * W5[o * cnn::K5 + k];
  out[t] = s;
}

// loss = mean over the batch of sum_i (o_i - t_i)^2 (i < 6) + BCE of the
// confidence against "translation within 0.5 px"; dout = d loss / d out
__global__ void k_loss(const float *__restrict__ out, const float *__restrict__ tgt, int B,
                       float *__restrict__ dout, double *__restrict__ loss) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (b < B) {
    const float *o = out + (long long)b * cnn::NOUT;
    const float *t = tgt + (long long)b * 6;
    float *d = dout + (long long)b * cnn::NOUT;
    for (int i = 0; i < 6; ++i) {
      const float e = o[i] - t[i];
      l += (double)e * e;
      d[i] = 2.f * e / B;
    }
    const float err = fmaxf(fabsf(o[0] - t[0]), fabsf(o[1] - t[1])) * cnn::TSCALE;
    const float c = err < 0.5f ? 1.f : 0.f;
    const float z = o[6];
    const float pz = 1.f / (1.f + expf(-z));
    l += (double)(fmaxf(z, 0.f) - z * c + log1pf(expf(-fabsf(z))));
    d[6] = (pz - c) / B;
    d[7] = 0.f;
  }
  l = warp_sum(l);
  if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l / B);
}

// output-layer backward: dW, db (thread per (o, k) / o), dz = (dout . W) * (y > 0)
__global__ void k_fc5_back(const float *__restrict__ dout, const bf16 *__restrict__ y4,
                           const float *__restrict__ W5, int B, float *__restrict__ gW5,
                           float *__restrict__ gb5, bf16 *__restrict__ dz4) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nW = (long long)cnn::NOUT * cnn::K5;
  if (t < nW) {
    const int o = (int)(t / cnn::K5), k = (int)(t - (long long)o * cnn::K5);
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += dout[b * cnn::NOUT + o] * __bfloat162float(y4[(long long)b * cnn::K5 + k]);
    gW5[t] = s;
  } else if (t < nW + cnn::NOUT) {
    const int o = (int)(t - nW);
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += dout[b * cnn::NOUT + o];
    gb5[o] = s;
  } else if (t < nW + cnn::NOUT + (long long)B * cnn::K5) {
    const long long q = t - nW - cnn::NOUT;
    const int b = (int)(q / cnn::K5), k = (int)(q - (long long)b * cnn::K5);
    float s = 0.f;
    for (int o = 0; o < cnn::NOUT; ++o) s += dout[b * cnn::NOUT + o] * W5[o * cnn::K5 + k];
    dz4[q] = __float2bfloat16_rn(__bfloat162float(y4[q]) > 0.f ? s : 0.f);
  }
}

// column sums of a rows x cols bf16 matrix (bias gradients), fixed order
__global__ void k_colsum(const bf16 *__restrict__ a, long long rows, int cols, float *__restrict__ out) {
  const int c = blockIdx.x;
  __shared__ float red[32];
  float s = 0.f;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) s += __bfloat162float(a[r * cols + c]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    out[c] = t;
  }
}

__global__ void k_splitk_sum(const float *__restrict__ part, int splits, long long n, float *__restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int z = 0; z < splits; ++z) s += part[(long long)z * n + k];
    out[k] = s;
  }
}

// the split-K partials of a forward layer summed in split order, + bias,
// ReLU, rounded to bf16 (the epilogue the unsplit product applies)
__global__ void k_splitk_relu(const float *__restrict__ part, int splits, long long n, int N,
                              const float *__restrict__ bias, bf16 *__restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int z = 0; z < splits; ++z) s += part[(long long)z * n + k];
    s += bias[k % N];
    out[k] = __float2bfloat16_rn(s > 0.f ? s : 0.f);
  }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on an FP32 block; optional bf16 copy
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, long long n, float lr, float c1, float c2,
                       bf16 *__restrict__ wb) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const float gk = g[k];
    const float mk = 0.9f * m[k] + 0.1f * gk, vk = 0.999f * v[k] + 0.001f * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk * c1) / (sqrtf(vk * c2) + 1e-8f);
    w[k] = wk;
    if (wb) wb[k] = __float2bfloat16_rn(wk);
  }
}

// U0, F0 and confidence from the network output
__global__ void k_to_init(const float *__restrict__ out, long long n, double *__restrict__ U0,
                          double *__restrict__ F0, float *__restrict__ conf) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float *o = out + k * cnn::NOUT;
  if (U0) {
    U0[2 * k] = (double)o[0] * cnn::TSCALE;
    U0[2 * k + 1] = (double)o[1] * cnn::TSCALE;
  }
  if (F0)
    for (int i = 0; i < 4; ++i) F0[4 * k + i] = (double)o[2 + i] / cnn::GSCALE;
  if (conf) conf[k] = 1.f / (1.f + expf(-o[6]));
}

inline unsigned nblk(long long n, int t = 256) {
  long long b = (n + t - 1) / t;
  return (unsigned)(b > 4096 ? 4096 : (b < 1 ? 1 : b));
}

}  // namespace
}  // namespace aldic

using namespace aldic;

struct aldic_cnn {
  int device = 0;
  int maxB = 0;
  long long steps = 0;
  DevBuf prm, grad, adm, adv, wbf;  // packed FP32 parameters, gradients, Adam moments; bf16 W1-W3
  DevBuf xin, x0, e1, e2, corr, y3, out, dout, dz3, dcorr, de2, dz1, part, err, loss, tgt;
  float *W(int l) const { return prm.as<float>() + off_w(l); }
  float *Bv(int l) const { return prm.as<float>() + off_w(l) + cnn::NW[l]; }
  float *gW(int l) const { return grad.as<float>() + off_w(l); }
  float *gB(int l) const { return grad.as<float>() + off_w(l) + cnn::NW[l]; }
  bf16 *Wb(int l) const {
    long long o = 0;
    for (int i = 0; i < l; ++i) o += cnn::NW[i];
    return wbf.as<bf16>() + o;
  }
  static long long off_w(int l) {
    long long o = 0;
    for (int i = 0; i < l; ++i) o += cnn::NW[i] + cnn::NB[i];
    return o;
  }
};

namespace aldic {
namespace {

GemmSrc src(const void *p, int mode, long long rows, long long kdim, long long ld, int Hin = 0,
            int Win = 0, int C = 0, int ps = 0, long long bstride = 0) {
  GemmSrc s;
  s.p = (const bf16 *)p; s.mode = mode; s.rows = rows; s.kdim = kdim; s.ld = ld;
  s.Hin = Hin; s.Win = Win; s.C = C; s.ps = ps; s.bstride = bstride;
  return s;
}

GemmDst dst(void *p, long long M, long long N, long long ld, int fp32, const float *bias, int relu,
            int mode = GEMM_ROW, const void *mask = nullptr) {
  GemmDst d;
  d.p = p; d.M = M; d.N = N; d.ld = ld; d.fp32 = fp32; d.bias = bias; d.relu = relu; d.mode = mode;
  d.mask = (const bf16 *)mask; d.Hin = d.Win = d.C = d.ps = 0; d.split_stride = 0;
  return d;
}

int ensure(aldic_cnn *c, int B) {
  if (B <= c->maxB) return OK;
  const long long b = B, cells = 2 * b * cnn::CELLS;
  int rc;
  if ((rc = c->xin.ensure(2 * b * cnn::P * cnn::P * 2)) || (rc = c->x0.ensure(2 * 2 * b * cnn::P * cnn::P)) ||
      (rc = c->e1.ensure(2 * cells * cnn::C1)) || (rc = c->e2.ensure(2 * cells * cnn::C2)) ||
      (rc = c->corr.ensure(2 * b * cnn::K3)) || (rc = c->y3.ensure(2 * b * cnn::F3)) ||
      (rc = c->out.ensure(4 * b * cnn::NOUT)) || (rc = c->dout.ensure(4 * b * cnn::NOUT)) ||
      (rc = c->dz3.ensure(2 * b * cnn::F3)) || (rc = c->dcorr.ensure(2 * b * cnn::K3)) ||
      (rc = c->de2.ensure(2 * cells * cnn::C2)) || (rc = c->dz1.ensure(2 * cells * cnn::C1)) ||
      (rc = c->tgt.ensure(4 * b * 6)))
    return rc;
  c->maxB = B;
  return OK;
}

constexpr float kCorrScale = 0.08838834764831845f;  // 1 / sqrt(128)

int forward(aldic_cnn *c, int B, cudaStream_t st) {
  int *err = c->err.as<int>();
  int rc;
  const long long b = B, cells = 2 * b * cnn::CELLS, fs = (long long)cnn::CELLS * cnn::C2;
  k_split<<<nblk(b * cnn::P * cnn::P), 256, 0, st>>>(c->xin.as<bf16>(), b, c->x0.as<bf16>());
  ALDIC_CUDA(cudaGetLastError());
  // E1: 8x8 patch embedding of both patches
  if ((rc = gemm_bf16(src(c->x0.p, GEMM_PATCH, cells, cnn::K1, 0, cnn::P, cnn::P, 1, cnn::PS),
                      src(c->Wb(0), GEMM_ROW, cnn::C1, cnn::K1, cnn::K1),
                      dst(c->e1.p, cells, cnn::C1, cnn::C1, 0, c->Bv(0), 1), 1, err, st)))
    return rc;
  // E2: 1x1 (linear)
  if ((rc = gemm_bf16(src(c->e1.p, GEMM_ROW, cells, cnn::K2, cnn::C1),
                      src(c->Wb(1), GEMM_ROW, cnn::C2, cnn::K2, cnn::K2),
                      dst(c->e2.p, cells, cnn::C2, cnn::C2, 0, c->Bv(1), 0), 1, err, st)))
    return rc;
  // C: per pair, reference cells x deformed cells
  GemmDst dc = dst(c->corr.p, cnn::CELLS, cnn::CELLS, cnn::CELLS, 0, nullptr, 0);
  dc.scale = kCorrScale;
  dc.bstride = cnn::K3;
  if ((rc = gemm_bf16(src(c->e2.p, GEMM_ROW, cnn::CELLS, cnn::C2, cnn::C2, 0, 0, 0, 0, fs),
                      src(c->e2.as<bf16>() + b * fs, GEMM_ROW, cnn::CELLS, cnn::C2, cnn::C2, 0, 0, 0, 0, fs),
                      dc, 1, err, st, B)))
    return rc;
  // L3: K = 4096 on only b / 128 row tiles -- split K eight ways into FP32
  // partials, then sum, bias and ReLU in one pass
  {
    constexpr int kL3Split = 8;
    const long long n3 = b * cnn::F3;
    if ((rc = c->part.ensure(sizeof(float) * n3 * kL3Split))) return rc;
    GemmDst d3 = dst(c->part.p, b, cnn::F3, cnn::F3, 1, nullptr, 0);
    d3.split_stride = n3;
    if ((rc = gemm_bf16(src(c->corr.p, GEMM_ROW, b, cnn::K3, cnn::K3),
                        src(c->Wb(2), GEMM_ROW, cnn::F3, cnn::K3, cnn::K3), d3, kL3Split, err, st)))
      return rc;
    k_splitk_relu<<<nblk(n3), 256, 0, st>>>(c->part.as<float>(), kL3Split, n3, cnn::F3, c->Bv(2),
                                            c->y3.as<bf16>());
    ALDIC_CUDA(cudaGetLastError());
  }
  k_fc5<<<nblk(b * cnn::NOUT), 256, 0, st>>>(c->y3.as<bf16>(), c->W(3), c->Bv(3), c->out.as<float>(), B);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// dW = A . B^T product with split-K, summed into g
int weight_grad(aldic_cnn *c, const GemmSrc &A, const GemmSrc &Bm, float *g, cudaStream_t st) {
  const long long kt = (A.kdim + 63) / 64;
  int splits = (int)(kt / 8);
  splits = splits < 1 ? 1 : (splits > 64 ? 64 : splits);
  const long long n = A.rows * Bm.rows;
  int rc;
  if ((rc = c->part.ensure(sizeof(float) * n * splits))) return rc;
  GemmDst d = dst(c->part.p, A.rows, Bm.rows, Bm.rows, 1, nullptr, 0);
  d.split_stride = n;
  if ((rc = gemm_bf16(A, Bm, d, splits, c->err.as<int>(), st))) return rc;
  k_splitk_sum<<<nblk(n), 256, 0, st>>>(c->part.as<float>(), splits, n, g);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int backward(aldic_cnn *c, int B, cudaStream_t st) {
  int *err = c->err.as<int>();
  const long long b = B, cells = 2 * b * cnn::CELLS, fs = (long long)cnn::CELLS * cnn::C2;
  int rc;
  const long long t5 = (long long)cnn::NOUT * cnn::K5 + cnn::NOUT + b * cnn::K5;
  k_fc5_back<<<(unsigned)((t5 + 255) / 256), 256, 0, st>>>(c->dout.as<float>(), c->y3.as<bf16>(),
                                                           c->W(3), B, c->gW(3), c->gB(3),
                                                           c->dz3.as<bf16>());
  ALDIC_CUDA(cudaGetLastError());
  // L3
  if ((rc = weight_grad(c, src(c->dz3.p, GEMM_TRANS, cnn::F3, b, cnn::F3),
                        src(c->corr.p, GEMM_TRANS, cnn::K3, b, cnn::K3), c->gW(2), st)))
    return rc;
  k_colsum<<<cnn::F3, 256, 0, st>>>(c->dz3.as<bf16>(), b, cnn::F3, c->gB(2));
  if ((rc = gemm_bf16(src(c->dz3.p, GEMM_ROW, b, cnn::F3, cnn::F3),
                      src(c->Wb(2), GEMM_TRANS, cnn::K3, cnn::F3, cnn::K3),
                      dst(c->dcorr.p, b, cnn::K3, cnn::K3, 0, nullptr, 0), 1, err, st)))
    return rc;
  // C: d e2_f = s dcorr . e2_g,  d e2_g = s dcorr^T . e2_f  (one product per pair)
  GemmDst df = dst(c->de2.p, cnn::CELLS, cnn::C2, cnn::C2, 0, nullptr, 0);
  df.scale = kCorrScale;
  df.bstride = fs;
  if ((rc = gemm_bf16(src(c->dcorr.p, GEMM_ROW, cnn::CELLS, cnn::CELLS, cnn::CELLS, 0, 0, 0, 0, cnn::K3),
                      src(c->e2.as<bf16>() + b * fs, GEMM_TRANS, cnn::C2, cnn::CELLS, cnn::C2, 0, 0, 0, 0, fs),
                      df, 1, err, st, B)))
    return rc;
  GemmDst dg = df;
  dg.p = c->de2.as<bf16>() + b * fs;
  if ((rc = gemm_bf16(src(c->dcorr.p, GEMM_TRANS, cnn::CELLS, cnn::CELLS, cnn::CELLS, 0, 0, 0, 0, cnn::K3),
                      src(c->e2.p, GEMM_TRANS, cnn::C2, cnn::CELLS, cnn::C2, 0, 0, 0, 0, fs),
                      dg, 1, err, st, B)))
    return rc;
  // E2 (linear)
  if ((rc = weight_grad(c, src(c->de2.p, GEMM_TRANS, cnn::C2, cells, cnn::C2),
                        src(c->e1.p, GEMM_TRANS, cnn::K2, cells, cnn::C1), c->gW(1), st)))
    return rc;
  k_colsum<<<cnn::C2, 256, 0, st>>>(c->de2.as<bf16>(), cells, cnn::C2, c->gB(1));
  if ((rc = gemm_bf16(src(c->de2.p, GEMM_ROW, cells, cnn::C2, cnn::C2),
                      src(c->Wb(1), GEMM_TRANS, cnn::K2, cnn::C2, cnn::K2),
                      dst(c->dz1.p, cells, cnn::C1, cnn::C1, 0, nullptr, 0, GEMM_ROW, c->e1.p), 1, err,
                      st)))
    return rc;
  // E1
  if ((rc = weight_grad(c, src(c->dz1.p, GEMM_TRANS, cnn::C1, cells, cnn::C1),
                        src(c->x0.p, GEMM_PATCHT, cnn::K1, cells, 0, cnn::P, cnn::P, 1, cnn::PS),
                        c->gW(0), st)))
    return rc;
  k_colsum<<<cnn::C1, 256, 0, st>>>(c->dz1.as<bf16>(), cells, cnn::C1, c->gB(0));
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int adam(aldic_cnn *c, float lr, cudaStream_t st) {
  c->steps++;
  const float c1 = 1.f / (1.f - powf(0.9f, (float)c->steps));
  const float c2 = 1.f / (1.f - powf(0.999f, (float)c->steps));
  for (int l = 0; l < cnn::NL; ++l) {
    const long long o = aldic_cnn::off_w(l), n = cnn::NW[l] + cnn::NB[l];
    float *w = c->prm.as<float>() + o;
    // weights (bf16 copy for the tensor-core layers), then biases
    k_adam<<<nblk(cnn::NW[l]), 256, 0, st>>>(w, c->grad.as<float>() + o, c->adm.as<float>() + o,
                                             c->adv.as<float>() + o, cnn::NW[l], lr, c1, c2,
                                             l < cnn::NL - 1 ? c->Wb(l) : nullptr);
    k_adam<<<1, 256, 0, st>>>(w + cnn::NW[l], c->grad.as<float>() + o + cnn::NW[l],
                              c->adm.as<float>() + o + cnn::NW[l], c->adv.as<float>() + o + cnn::NW[l],
                              n - cnn::NW[l], lr, c1, c2, nullptr);
  }
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int sync_bf16(aldic_cnn *c, cudaStream_t st) {
  for (int l = 0; l < cnn::NL - 1; ++l)
    k_f2bf<<<nblk(cnn::NW[l]), 256, 0, st>>>(c->W(l), c->Wb(l), cnn::NW[l]);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int check_err(aldic_cnn *c, cudaStream_t st) {
  int e = 0;
  ALDIC_CUDA(cudaMemcpyAsync(&e, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  ALDIC_CUDA(cudaStreamSynchronize(st));
  if (e) {
    cudaMemsetAsync(c->err.p, 0, sizeof(int), st);
    set_error("cnn: a tensor-core wait timed out");
    return E_TIMEOUT;
  }
  return OK;
}

// network input: fp32 (host or device) or bf16 (device) patches
int load_input(aldic_cnn *c, const void *x, int x_bf16, int B, cudaStream_t st) {
  const long long n = (long long)B * cnn::P * cnn::P * 2;
  if (x_bf16) {
    ALDIC_CUDA(cudaMemcpyAsync(c->xin.p, x, 2 * n, cudaMemcpyDefault, st));
    return OK;
  }
  DevBuf tmp;
  const float *xd = (const float *)x;
  cudaPointerAttributes at;
  const bool dev = cudaPointerGetAttributes(&at, x) == cudaSuccess &&
                   (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  if (!dev) {
    int rc;
    if ((rc = tmp.ensure(4 * n))) return rc;
    ALDIC_CUDA(cudaMemcpyAsync(tmp.p, x, 4 * n, cudaMemcpyHostToDevice, st));
    xd = tmp.as<float>();
  }
  k_f2bf<<<nblk(n), 256, 0, st>>>(xd, c->xin.as<bf16>(), n);
  ALDIC_CUDA(cudaGetLastError());
  if (!dev) {
    ALDIC_CUDA(cudaStreamSynchronize(st));
    tmp.release();
  }
  return OK;
}

}  // namespace
}  // namespace aldic

extern "C" {

int aldic_cnn_create(int device, unsigned long long seed, aldic_cnn **out) {
  ALDIC_CHECK(out, E_ARG, "cnn_create: null output");
  *out = nullptr;
  int prev = 0;
  cudaGetDevice(&prev);
  ALDIC_CUDA(cudaSetDevice(device));
  auto *c = new aldic_cnn();
  c->device = device;
  const long long np = cnn::n_params();
  long long nwb = 0;
  for (int l = 0; l < cnn::NL - 1; ++l) nwb += cnn::NW[l];
  int rc;
  if ((rc = c->prm.ensure(4 * np)) || (rc = c->grad.ensure(4 * np)) || (rc = c->adm.ensure(4 * np)) ||
      (rc = c->adv.ensure(4 * np)) || (rc = c->wbf.ensure(2 * nwb)) || (rc = c->err.ensure(64)) ||
      (rc = c->loss.ensure(64))) {
    delete c;
    cudaSetDevice(prev);
    return rc;
  }
  // He-normal weights (std sqrt(2 / fan_in)), zero biases, seeded
  std::vector<float> h(np, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < cnn::NL; ++l) {
    const long long fan_in = cnn::NW[l] / cnn::NB[l];
    std::normal_distribution<float> nd(0.f, l == 1 || l == cnn::NL - 1 ? (float)std::sqrt(1.0 / fan_in)
                                                                       : (float)std::sqrt(2.0 / fan_in));
    float *w = h.data() + aldic_cnn::off_w(l);
    for (long long k = 0; k < cnn::NW[l]; ++k) w[k] = nd(rng);
  }
  cudaMemcpy(c->prm.p, h.data(), 4 * np, cudaMemcpyHostToDevice);
  cudaMemset(c->adm.p, 0, 4 * np);
  cudaMemset(c->adv.p, 0, 4 * np);
  cudaMemset(c->err.p, 0, 64);
  sync_bf16(c, 0);
  const cudaError_t e = cudaDeviceSynchronize();
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    delete c;
    set_error(std::string("cnn_create: ") + cudaGetErrorString(e));
    return E_CUDA;
  }
  *out = c;
  return OK;
}

int aldic_cnn_destroy(aldic_cnn *c) {
  if (!c) return OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  DevBuf *b[] = {&c->prm, &c->grad, &c->adm, &c->adv, &c->wbf, &c->xin, &c->x0, &c->e1, &c->e2,
                 &c->corr, &c->y3, &c->out, &c->dout, &c->dz3, &c->dcorr, &c->de2, &c->dz1,
                 &c->part, &c->err, &c->loss, &c->tgt};
  for (auto *x : b) x->release();
  cudaSetDevice(prev);
  delete c;
  return OK;
}

long long aldic_cnn_num_params(void) { return cnn::n_params(); }

int aldic_cnn_get_params(aldic_cnn *c, float *params) {
  ALDIC_CHECK(c && params, E_ARG, "cnn_get_params: null argument");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  const cudaError_t e = cudaMemcpy(params, c->prm.p, 4 * cnn::n_params(), cudaMemcpyDefault);
  cudaSetDevice(prev);
  ALDIC_CHECK(e == cudaSuccess, E_CUDA, "cnn_get_params: copy failed");
  return OK;
}

int aldic_cnn_set_params(aldic_cnn *c, const float *params) {
  ALDIC_CHECK(c && params, E_ARG, "cnn_set_params: null argument");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaError_t e = cudaMemcpy(c->prm.p, params, 4 * cnn::n_params(), cudaMemcpyDefault);
  if (e == cudaSuccess) {
    sync_bf16(c, 0);
    e = cudaDeviceSynchronize();
  }
  cudaSetDevice(prev);
  ALDIC_CHECK(e == cudaSuccess, E_CUDA, "cnn_set_params: copy failed");
  return OK;
}

// forward + loss + backward (+ Adam step when lr > 0); grads (optional,
// n_params floats) receive the gradients, out (optional, B x 8) the outputs
int aldic_cnn_train_step(aldic_cnn *c, const void *x, int x_bf16, const float *targets, int B,
                         float lr, void *stream, double *loss, float *grads, float *out) {
  ALDIC_CHECK(c && x && targets && B >= 1, E_ARG, "cnn_train_step: bad arguments");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure(c, B);
  if (!rc) rc = load_input(c, x, x_bf16, B, st);
  if (!rc && cudaMemcpyAsync(c->tgt.p, targets, sizeof(float) * 6 * B, cudaMemcpyDefault, st) != cudaSuccess) {
    set_error("cnn_train_step: target copy failed");
    rc = E_CUDA;
  }
  if (!rc) rc = forward(c, B, st);
  if (!rc) {
    cudaMemsetAsync(c->loss.p, 0, sizeof(double), st);
    k_loss<<<(B + 255) / 256, 256, 0, st>>>(c->out.as<float>(), c->tgt.as<float>(), B,
                                           c->dout.as<float>(), c->loss.as<double>());
    rc = backward(c, B, st);
  }
  if (!rc && lr > 0) rc = adam(c, lr, st);
  if (!rc && grads)
    if (cudaMemcpyAsync(grads, c->grad.p, 4 * cnn::n_params(), cudaMemcpyDefault, st) != cudaSuccess) rc = E_CUDA;
  if (!rc && out)
    if (cudaMemcpyAsync(out, c->out.p, 4LL * B * cnn::NOUT, cudaMemcpyDefault, st) != cudaSuccess) rc = E_CUDA;
  if (!rc && loss)
    if (cudaMemcpyAsync(loss, c->loss.p, sizeof(double), cudaMemcpyDefault, st) != cudaSuccess) rc = E_CUDA;
  if (!rc) rc = check_err(c, st);
  cudaSetDevice(prev);
  return rc;
}

int aldic_cnn_predict(aldic_cnn *c, const void *x, int x_bf16, int B, void *stream, float *out) {
  ALDIC_CHECK(c && x && out && B >= 1, E_ARG, "cnn_predict: bad arguments");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure(c, B);
  if (!rc) rc = load_input(c, x, x_bf16, B, st);
  if (!rc) rc = forward(c, B, st);
  if (!rc && cudaMemcpyAsync(out, c->out.p, 4LL * B * cnn::NOUT, cudaMemcpyDefault, st) != cudaSuccess)
    rc = E_CUDA;
  if (!rc) rc = check_err(c, st);
  cudaSetDevice(prev);
  return rc;
}

}  // extern "C"

namespace aldic {

int cnn_patches(const float *f, const float *g, int W, int H, const double *coords, long long n,
                void *bf16_out, float *f32_out, cudaStream_t st) {
  if (n <= 0) return OK;
  k_patches<<<(unsigned)n, 256, 0, st>>>(f, g, W, H, coords, n, (bf16 *)bf16_out, f32_out);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int cnn_to_init(const float *out, long long n, double *U0, double *F0, float *conf, cudaStream_t st) {
  if (n <= 0) return OK;
  k_to_init<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, U0, F0, conf);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

}  // namespace aldic
