// fdm.cu -- direct solve of the uniform-mesh Subproblem 2 by fast
// diagonalisation (Lynch, Rice and Thomas, "Direct solution of partial
// difference equations by tensor product methods", Numer. Math. 6, 1964).
//
// On the M x N node grid of MeshSetUp.m both Subproblem 2 operators are
// Kronecker sums of 1-D operators, one per grid direction:
//
//   FE (Subpb2.m:100-195, bilinear squares of side h, 3x3 Gauss -- exact for
//   these integrands, natural boundaries):
//       A = beta (Kx (x) My + Mx (x) Ky) + mu Mx (x) My
//   with the 1-D linear-element stiffness K = (1/h) tridiag(-1, 2, -1)
//   (corner entries 1) and mass M = (h/6) tridiag(1, 4, 1) (corner entries 2);
//
//   FD (funDerivativeOp.m on the (M-2) x (N-2) interior, main_ALDIC.m:243-259):
//       A = beta (I (x) Gx + Gy (x) I) + mu I
//   with G = d'd, d the 1-D difference of funDerivativeOp (central / 2h inside,
//   one-sided with doubled weights at the two ends).
//
// With the generalised eigenbases K V = M V Lambda, V' M V = I of each
// direction, A^-1 = (Vx (x) Vy) D^-1 (Vx (x) Vy)', D = beta (lx_p + ly_q) + mu,
// so a solve is four dense products per field (two per direction) and a
// diagonal scale: C = Vy' B Vx, C ./= D, X = Vy C Vx'.  The 1-D bases are
// computed once per geometry on the host in FP64 (Cholesky M = L L',
// Householder tridiagonalisation and implicit symmetric QR steps with
// Wilkinson shifts of L^-1 K L^-T -- Golub and Van Loan, Matrix
// Computations, 4th ed., algorithms 8.3.1 and 8.3.2) and kept on the device;
// the products run as FP64 CUDA-core tiles.  The solution is exact up to
// rounding (about 1e-13 relative), where an iterative solve stops at a
// residual of 1e-11.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/aldic_b200.h"
#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {

namespace {

// ---------------------------------------------------------------- host: 1-D operators
// assembled 1-D linear-element stiffness K and mass M of n nodes at spacing h
// (natural boundaries), dense row-major
void fe_stiffness_mass(int n, double h, std::vector<double> &K, std::vector<double> &Mm) {
  K.assign((size_t)n * n, 0.0);
  Mm.assign((size_t)n * n, 0.0);
  for (int e = 0; e + 1 < n; ++e) {  // element (e, e+1)
    const int a = e, b = e + 1;
    K[(size_t)a * n + a] += 1.0 / h;
    K[(size_t)b * n + b] += 1.0 / h;
    K[(size_t)a * n + b] -= 1.0 / h;
    K[(size_t)b * n + a] -= 1.0 / h;
    Mm[(size_t)a * n + a] += 2.0 * h / 6.0;
    Mm[(size_t)b * n + b] += 2.0 * h / 6.0;
    Mm[(size_t)a * n + b] += h / 6.0;
    Mm[(size_t)b * n + a] += h / 6.0;
  }
}

// G = d'd with d the n x n difference of funDerivativeOp.m:25-35 along one line
void fd_gram(int n, double h, std::vector<double> &G) {
  std::vector<double> d((size_t)n * n, 0.0);
  const double s = 1.0 / (2.0 * h);
  for (int t = 0; t < n && n > 1; ++t) {
    if (t == 0) {
      d[(size_t)t * n + 1] += 2 * s;
      d[(size_t)t * n + 0] -= 2 * s;
    } else if (t == n - 1) {
      d[(size_t)t * n + n - 1] += 2 * s;
      d[(size_t)t * n + n - 2] -= 2 * s;
    } else {
      d[(size_t)t * n + t + 1] += s;
      d[(size_t)t * n + t - 1] -= s;
    }
  }
  G.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = std::max(0, i - 2); j <= std::min(n - 1, i + 2); ++j) {
      double v = 0.0;
      for (int t = std::max(0, i - 1); t <= std::min(n - 1, i + 1); ++t)
        v += d[(size_t)t * n + i] * d[(size_t)t * n + j];
      G[(size_t)i * n + j] = v;
    }
}

// ---------------------------------------------------------------- host: symmetric eigenproblem
// Householder reduction of the symmetric A (n x n, row-major, destroyed) to
// tridiagonal form T = Q' A Q: diag d, sub-diagonal e (e[k] = T[k+1][k]);
// returns Qt = Q' (row k of Qt is column k of Q).
void tridiagonalise(int n, std::vector<double> &A, std::vector<double> &d, std::vector<double> &e,
                    std::vector<double> &Qt) {
  d.assign(n, 0.0);
  e.assign(n > 1 ? n - 1 : 0, 0.0);
  Qt.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Qt[(size_t)i * n + i] = 1.0;
  std::vector<double> v(n), p(n), w(n), sc(n);
  for (int k = 0; k + 2 < n; ++k) {
    // x = A[k+1:, k]
    const int m = n - k - 1;
    double sig = 0.0;
    for (int i = 1; i < m; ++i) sig += A[(size_t)(k + 1 + i) * n + k] * A[(size_t)(k + 1 + i) * n + k];
    const double x0 = A[(size_t)(k + 1) * n + k];
    if (sig == 0.0) {  // already tridiagonal in this column
      e[k] = x0;
      continue;
    }
    const double nx = std::sqrt(x0 * x0 + sig);
    const double alpha = x0 >= 0 ? -nx : nx;  // H x = alpha e1
    // v = x - alpha e1, H = I - tau v v', tau = 2 / v'v
    v[0] = x0 - alpha;
    for (int i = 1; i < m; ++i) v[i] = A[(size_t)(k + 1 + i) * n + k];
    const double tau = 2.0 / (v[0] * v[0] + sig);
    // p = tau A22 v ; w = p - (tau p'v / 2) v ; A22 -= v w' + w v'
    for (int i = 0; i < m; ++i) {
      const double *row = &A[(size_t)(k + 1 + i) * n + k + 1];
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += row[j] * v[j];
      p[i] = tau * s;
    }
    double pv = 0.0;
    for (int i = 0; i < m; ++i) pv += p[i] * v[i];
    const double kk = 0.5 * tau * pv;
    for (int i = 0; i < m; ++i) w[i] = p[i] - kk * v[i];
    for (int i = 0; i < m; ++i) {
      double *row = &A[(size_t)(k + 1 + i) * n + k + 1];
      for (int j = 0; j < m; ++j) row[j] -= v[i] * w[j] + w[i] * v[j];
    }
    e[k] = alpha;
    // Q <- Q H on columns k+1..: Qt rows k+1.. <- H Qt rows (H symmetric),
    // as row sweeps: sc = v' Qt[k+1:], then Qt[k+1+i] -= tau v_i sc
    std::fill(sc.begin(), sc.end(), 0.0);
    for (int i = 0; i < m; ++i) {
      const double *row = &Qt[(size_t)(k + 1 + i) * n];
      const double vi = v[i];
      for (int c = 0; c < n; ++c) sc[c] += vi * row[c];
    }
    for (int i = 0; i < m; ++i) {
      double *row = &Qt[(size_t)(k + 1 + i) * n];
      const double tv = tau * v[i];
      for (int c = 0; c < n; ++c) row[c] -= tv * sc[c];
    }
  }
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i];
  if (n >= 2) e[n - 2] = A[(size_t)(n - 1) * n + n - 2];
}

// implicit symmetric QR steps with Wilkinson shifts on (d, e) until every
// off-diagonal is negligible; each rotation R of rows k, k+1 (T <- R T R')
// is applied to rows k, k+1 of Qt as well, so with Qt = Q' from
// tridiagonalise the original matrix is Qt' diag(d) Qt on return: row p of
// Qt is the eigenvector of eigenvalue d[p].
int tridiagonal_qr(int n, std::vector<double> &d, std::vector<double> &e, std::vector<double> &Qt) {
  const double eps = 2.220446049250313e-16;
  int hi = n - 1, sweeps = 0;
  while (hi > 0) {
    if (std::fabs(e[hi - 1]) <= eps * (std::fabs(d[hi - 1]) + std::fabs(d[hi]))) {
      e[hi - 1] = 0.0;
      --hi;
      continue;
    }
    int lo = hi - 1;
    while (lo > 0 && std::fabs(e[lo - 1]) > eps * (std::fabs(d[lo - 1]) + std::fabs(d[lo]))) --lo;
    if (++sweeps > 60 * n) return E_STATE;
    // Wilkinson shift from the trailing 2 x 2 block
    const double dd = 0.5 * (d[hi - 1] - d[hi]);
    const double eh = e[hi - 1];
    const double den = dd + (dd >= 0 ? 1.0 : -1.0) * std::hypot(dd, eh);
    const double shift = d[hi] - eh * eh / den;
    double x = d[lo] - shift, z = e[lo];
    for (int k = lo; k < hi; ++k) {
      // rotation R (rows k, k+1): [c s; -s c] (x, z)' = (r, 0)'
      const double r = std::hypot(x, z);
      const double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : z / r;
      if (k > lo) e[k - 1] = r;
      const double a = d[k], b = e[k], dn = d[k + 1];
      d[k] = c * c * a + 2 * c * s * b + s * s * dn;
      d[k + 1] = s * s * a - 2 * c * s * b + c * c * dn;
      e[k] = c * s * (dn - a) + (c * c - s * s) * b;
      if (k + 1 < hi) {  // the bulge moves to (k+2, k)
        const double f = e[k + 1];
        x = e[k];
        z = s * f;
        e[k + 1] = c * f;
      }
      double *qa = &Qt[(size_t)k * n], *qb = &Qt[(size_t)(k + 1) * n];
      for (int j = 0; j < n; ++j) {
        const double u = qa[j], w = qb[j];
        qa[j] = c * u + s * w;
        qb[j] = -s * u + c * w;
      }
    }
  }
  return OK;
}

// ---------------------------------------------------------------- device: FP64 products
// 64 x 64 outputs per 256-thread CTA, 4 x 4 per thread taken strided (rows
// ty + 16 i, columns tx + 16 j), so a warp's shared-memory reads of a k row
// are 16 consecutive doubles (one wavefront, broadcast to the two row
// groups) and each thread does 16 FMA per 8 loads.  The operand tiles of
// 32-wide K chunks go to shared memory by cp.async (no register round trip),
// double-buffered so that chunk c + 1 arrives while chunk c is multiplied.
constexpr int TR = 64, TC = 64, KC = 32, GT = 256, LDT = TR + 1;
// Products with fewer tiles than SMs (the 2-field solves: 32 tiles at 243^2)
// split K into up to kMaxSplit slices written to a partial buffer and summed
// in a fixed order by k_fdm_reduce (deterministic, no atomics).
constexpr int kMaxSplit = 4, kFdmPart = 8;  // partial capacity: kFdmPart fields of M N
constexpr int kBuf = 2 * KC * LDT;                              // doubles per buffer (A + B)
constexpr int kSmem = 2 * kBuf * (int)sizeof(double);           // two buffers: 66 560 B

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

struct GemmArgs {
  const double *A, *B;
  double *C;
  long long sab, sar, sak;  // element (r, k) of batch b of A at A[b sab + r sar + k sak]
  long long sbb, sbk, sbc;  // element (k, c) of batch b of B
  long long scb, scr, scc;  // element (r, c) of batch b of C
  int R, Cn, K;
  // epilogue 1: C /= beta_b (lr[r] + lc[c]) + mu
  int scale;
  const double *lr, *lc;
  double mu;
  double beta[12];
  const double *beta_ptr;  // if set, beta = *beta_ptr for every batch entry
  // split K: slice s of batch entry b writes P[(s batch + b) R Cn + r Cn + c]
  int splits;
  double *P;
};

// stage K chunk [k0, k0 + KC) of the A and B tiles into buffer `buf`
// (zeros outside the operands)
__device__ __forceinline__ void stage_chunk(const GemmArgs &g, const double *A, const double *B,
                                            int r0, int c0, int k0, double *buf, bool a_rfast,
                                            bool b_cfast) {
  double *As = buf, *Bs = buf + KC * LDT;
#pragma unroll 4
  for (int e = threadIdx.x; e < TR * KC; e += GT) {
    const int rr = a_rfast ? (e & (TR - 1)) : (e >> 5), kk = a_rfast ? (e >> 6) : (e & (KC - 1));
    const int r = r0 + rr, k = k0 + kk;
    double *d = As + kk * LDT + rr;
    if (r < g.R && k < g.K) cp_async8(d, A + (long long)r * g.sar + (long long)k * g.sak);
    else *d = 0.0;
  }
#pragma unroll 4
  for (int e = threadIdx.x; e < TC * KC; e += GT) {
    const int cc = b_cfast ? (e & (TC - 1)) : (e >> 5), kk = b_cfast ? (e >> 6) : (e & (KC - 1));
    const int c = c0 + cc, k = k0 + kk;
    double *d = Bs + kk * LDT + cc;
    if (c < g.Cn && k < g.K) cp_async8(d, B + (long long)k * g.sbk + (long long)c * g.sbc);
    else *d = 0.0;
  }
  cp_async_commit();
}

__global__ void __launch_bounds__(GT) k_fdm_gemm(GemmArgs g) {
  extern __shared__ double sm[];
  const int nb = gridDim.z / g.splits;
  const int b = blockIdx.z % nb, sp = blockIdx.z / nb;
  const int r0 = blockIdx.y * TR, c0 = blockIdx.x * TC;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const double *A = g.A + (long long)b * g.sab;
  const double *B = g.B + (long long)b * g.sbb;
  double acc[4][4] = {};
  const bool a_rfast = g.sar <= g.sak, b_cfast = g.sbc <= g.sbk;
  // this slice's K range, in whole chunks
  const int nall = (g.K + KC - 1) / KC, per = (nall + g.splits - 1) / g.splits;
  const int ch0 = sp * per, ch1 = ch0 + per < nall ? ch0 + per : nall;
  if (ch0 < ch1) stage_chunk(g, A, B, r0, c0, ch0 * KC, sm, a_rfast, b_cfast);
  for (int ch = ch0; ch < ch1; ++ch) {
    if (ch + 1 < ch1) {
      stage_chunk(g, A, B, r0, c0, (ch + 1) * KC, sm + ((ch + 1 - ch0) & 1) * kBuf, a_rfast,
                  b_cfast);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double *As = sm + ((ch - ch0) & 1) * kBuf, *Bs = As + KC * LDT;
    const int kc = g.K - ch * KC < KC ? g.K - ch * KC : KC;
#pragma unroll 8
    for (int kk = 0; kk < kc; ++kk) {
      const double *ar = As + kk * LDT + ty, *br = Bs + kk * LDT + tx;
      double a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = ar[16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bb[j] = br[16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
    __syncthreads();  // this buffer is restaged by the next round
  }
  if (g.splits > 1) {
    double *P = g.P + ((long long)sp * nb + b) * g.R * g.Cn;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = r0 + ty + 16 * i;
      if (r >= g.R) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = c0 + tx + 16 * j;
        if (c < g.Cn) P[(long long)r * g.Cn + c] = acc[i][j];
      }
    }
    return;
  }
  const double beta = g.beta_ptr ? *g.beta_ptr : g.beta[b < 12 ? b : 11];
  double *C = g.C + (long long)b * g.scb;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = r0 + ty + 16 * i;
    if (r >= g.R) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + tx + 16 * j;
      if (c >= g.Cn) continue;
      double v = acc[i][j];
      if (g.scale) v /= beta * (g.lr[r] + g.lc[c]) + g.mu;
      C[(long long)r * g.scr + (long long)c * g.scc] = v;
    }
  }
}

// the kernel's dynamic shared memory (above the 48 KB default) on the current
// device; set by fdm_ensure, ahead of any stream capture
int gemm_setup() {
  ALDIC_CUDA(cudaFuncSetAttribute(k_fdm_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem));
  return OK;
}

// the split-K slices of every output summed in slice order, then the epilogue
__global__ void k_fdm_reduce(GemmArgs g, int batch) {
  const long long rc = (long long)g.R * g.Cn, n = rc * batch;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / rc);
    const long long e = i - (long long)b * rc;
    const int r = (int)(e / g.Cn), c = (int)(e - (long long)r * g.Cn);
    double v = 0.0;
    for (int s = 0; s < g.splits; ++s) v += g.P[((long long)s * batch + b) * rc + e];
    if (g.scale) {
      const double beta = g.beta_ptr ? *g.beta_ptr : g.beta[b < 12 ? b : 11];
      v /= beta * (g.lr[r] + g.lc[c]) + g.mu;
    }
    g.C[(long long)b * g.scb + (long long)r * g.scr + (long long)c * g.scc] = v;
  }
}

int gemm(GemmArgs g, int batch, double *part, cudaStream_t st) {
  const int tiles = ((g.Cn + TC - 1) / TC) * ((g.R + TR - 1) / TR) * batch;
  int sp = 1;
  while (sp < kMaxSplit && tiles * sp < 148 && (sp + 1) * batch <= kFdmPart) ++sp;
  g.splits = sp;
  g.P = part;
  dim3 grid((unsigned)((g.Cn + TC - 1) / TC), (unsigned)((g.R + TR - 1) / TR), (unsigned)(batch * sp));
  k_fdm_gemm<<<grid, GT, kSmem, st>>>(g);
  ALDIC_CUDA(cudaGetLastError());
  if (sp > 1) {
    const long long n = (long long)g.R * g.Cn * batch;
    k_fdm_reduce<<<(unsigned)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184), 256, 0, st>>>(g, batch);
    ALDIC_CUDA(cudaGetLastError());
  }
  return OK;
}

}  // namespace

// V (n x n row-major, column p = eigenvector p) and lam (n) of the 1-D
// pencil (K, M) of `type` (FDM_FE: linear-element stiffness and mass;
// FDM_FD: funDerivativeOp's d'd with M = I), V' M V = I.
int fdm_basis_1d(int type, int n, double h, double *V, double *lam) {
  ALDIC_CHECK(n >= 1 && n <= 16384 && h > 0 && V && lam && (type == FDM_FE || type == FDM_FD), E_ARG,
              "fdm basis: bad arguments");
  std::vector<double> K, Mm;
  if (type == FDM_FE) {
    fe_stiffness_mass(n, h, K, Mm);
  } else {
    fd_gram(n, h, K);
  }
  if (n == 1) {  // a single node: K = 0 (FE) / G = 0 (FD)
    lam[0] = 0.0;
    V[0] = type == FDM_FE ? 1.0 / std::sqrt(Mm[0] > 0 ? Mm[0] : 1.0) : 1.0;
    return OK;
  }
  // C = L^-1 K L^-T with M = L L' (L lower bidiagonal: diag l, sub m); FD: L = I
  std::vector<double> l(n, 1.0), m(n, 0.0);
  std::vector<double> C = K;
  if (type == FDM_FE) {
    for (int i = 0; i < n; ++i) {
      const double t = Mm[(size_t)i * n + i] - (i ? m[i] * m[i] : 0.0);
      ALDIC_CHECK(t > 0, E_STATE, "fdm basis: mass matrix not positive definite");
      l[i] = std::sqrt(t);
      if (i + 1 < n) m[i + 1] = Mm[(size_t)(i + 1) * n + i] / l[i];
    }
    // X = L^-1 K (rows), then C = L^-1 X' (= L^-1 K L^-T, K symmetric)
    std::vector<double> X((size_t)n * n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        X[(size_t)i * n + j] = (K[(size_t)i * n + j] - (i ? m[i] * X[(size_t)(i - 1) * n + j] : 0.0)) / l[i];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        C[(size_t)i * n + j] = (X[(size_t)j * n + i] - (i ? m[i] * C[(size_t)(i - 1) * n + j] : 0.0)) / l[i];
    for (int i = 0; i < n; ++i)  // symmetrise the rounding
      for (int j = 0; j < i; ++j) {
        const double s = 0.5 * (C[(size_t)i * n + j] + C[(size_t)j * n + i]);
        C[(size_t)i * n + j] = C[(size_t)j * n + i] = s;
      }
  }
  std::vector<double> d, e, Qt;
  tridiagonalise(n, C, d, e, Qt);
  const int rc = tridiagonal_qr(n, d, e, Qt);
  ALDIC_CHECK(rc == OK, E_STATE, "fdm basis: the QR iteration did not converge");
  // V = L^-T Q: back substitution L' V = Q, Q[i][p] = Qt[p][i]
  for (int i = n - 1; i >= 0; --i)
    for (int p = 0; p < n; ++p) {
      double q = Qt[(size_t)p * n + i];
      if (i + 1 < n) q -= m[i + 1] * V[(size_t)(i + 1) * n + p];
      V[(size_t)i * n + p] = q / l[i];
    }
  for (int p = 0; p < n; ++p) lam[p] = d[p];
  return OK;
}

int fdm_ensure(FdmBasis &B, int type, int M, int N, double h, cudaStream_t st) {
  int rc0 = gemm_setup();
  if (rc0) return rc0;
  if (B.type == type && B.M == M && B.N == N && B.h == h && B.buf.p) return OK;
  ALDIC_CHECK(M >= 1 && N >= 1, E_ARG, "fdm: empty grid");
  std::vector<double> host((size_t)M * M + (size_t)N * N + M + N);
  double *Vx = host.data(), *Vy = Vx + (size_t)M * M, *lx = Vy + (size_t)N * N, *ly = lx + M;
  int rc;
  if ((rc = fdm_basis_1d(type, M, h, Vx, lx))) return rc;
  if ((rc = fdm_basis_1d(type, N, h, Vy, ly))) return rc;
  B.type = -1;
  const size_t nbasis = host.size();
  if ((rc = B.buf.ensure(sizeof(double) * (nbasis + (size_t)kFdmPart * M * N)))) return rc;
  ALDIC_CUDA(cudaMemcpyAsync(B.buf.p, host.data(), sizeof(double) * host.size(),
                             cudaMemcpyHostToDevice, st));
  ALDIC_CUDA(cudaStreamSynchronize(st));  // the host vector goes out of scope
  double *d = B.buf.as<double>();
  B.Vx = d;
  B.Vy = d + (size_t)M * M;
  B.lx = B.Vy + (size_t)N * N;
  B.ly = B.lx + M;
  B.part = d + nbasis;
  B.type = type;
  B.M = M;
  B.N = N;
  B.h = h;
  return OK;
}

int fdm_solve(const FdmBasis &B, int nrhs, const double *b, double *x, double *tmp, double mu,
              double beta, const double *beta_each, const double *beta_ptr, cudaStream_t st) {
  ALDIC_CHECK(B.buf.p && nrhs >= 1 && nrhs <= 12, E_ARG, "fdm solve: bad arguments");
  const int M = B.M, N = B.N;
  const long long n = (long long)M * N;
  GemmArgs g{};
  g.mu = mu;
  for (int f = 0; f < 12; ++f) g.beta[f] = (beta_each && f < nrhs) ? beta_each[f] : beta;
  g.beta_ptr = beta_ptr;
  int rc;
  // field f as an N x M matrix (row j = node row y, column i = x): B_f[j][i] = b[f n + j M + i]
  // 1. T = B_f Vx  -> tmp
  g.A = b; g.sab = n; g.sar = M; g.sak = 1;
  g.B = B.Vx; g.sbb = 0; g.sbk = M; g.sbc = 1;
  g.C = tmp; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = M; g.scale = 0;
  if ((rc = gemm(g, nrhs, B.part, st))) return rc;
  // 2. C = Vy' T, C[q][p] /= beta (ly[q] + lx[p]) + mu  -> x
  g.A = B.Vy; g.sab = 0; g.sar = 1; g.sak = N;
  g.B = tmp; g.sbb = n; g.sbk = M; g.sbc = 1;
  g.C = x; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = N; g.scale = 1; g.lr = B.ly; g.lc = B.lx;
  if ((rc = gemm(g, nrhs, B.part, st))) return rc;
  // 3. S = C Vx'  -> tmp
  g.A = x; g.sab = n; g.sar = M; g.sak = 1;
  g.B = B.Vx; g.sbb = 0; g.sbk = 1; g.sbc = M;
  g.C = tmp; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = M; g.scale = 0;
  if ((rc = gemm(g, nrhs, B.part, st))) return rc;
  // 4. X = Vy S  -> x
  g.A = B.Vy; g.sab = 0; g.sar = N; g.sak = 1;
  g.B = tmp; g.sbb = n; g.sbk = M; g.sbc = 1;
  g.C = x; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = N; g.scale = 0;
  return gemm(g, nrhs, B.part, st);
}

// The beta sweep's eigen-domain solutions from the two transformed
// right-hand-side parts C4 (fields 0-1 beta part, 2-3 mu part; entry
// (q, p) at q M + p): X field 2k + c = (beta_k F_c + mu U_c) /
// (beta_k (ly[q] + lx[p]) + mu), the divisor of the one-system epilogue.
struct SweepBetas {
  double v[6];
};
__global__ void k_fdm_sweep_combine(int M, int N, const double *__restrict__ ly,
                                    const double *__restrict__ lx, SweepBetas be, double mu,
                                    const double *__restrict__ C4, double *__restrict__ X) {
  const long long n = (long long)M * N;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(idx / M), p = (int)(idx - (long long)q * M);
    const double lam = ly[q] + lx[p];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double F = C4[c * n + idx], U = C4[(2 + c) * n + idx];
#pragma unroll
      for (int k = 0; k < 6; ++k)
        X[(2 * k + c) * n + idx] = (be.v[k] * F + mu * U) / (be.v[k] * lam + mu);
    }
  }
}

int fdm_solve_sweep(const FdmBasis &B, const double beta[6], const double *b, double *x,
                    double *tmp, double mu, cudaStream_t st) {
  ALDIC_CHECK(B.buf.p, E_ARG, "fdm sweep: no basis");
  const int M = B.M, N = B.N;
  const long long n = (long long)M * N;
  GemmArgs g{};
  g.mu = mu;
  int rc;
  // 1. T = B_f Vx for the two parts (4 fields) -> tmp fields 0-3
  g.A = b; g.sab = n; g.sar = M; g.sak = 1;
  g.B = B.Vx; g.sbb = 0; g.sbk = M; g.sbc = 1;
  g.C = tmp; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = M; g.scale = 0;
  if ((rc = gemm(g, 4, B.part, st))) return rc;
  // 2. C = Vy' T, unscaled -> tmp fields 4-7
  g.A = B.Vy; g.sab = 0; g.sar = 1; g.sak = N;
  g.B = tmp; g.sbb = n; g.sbk = M; g.sbc = 1;
  g.C = tmp + 4 * n; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = N; g.scale = 0;
  if ((rc = gemm(g, 4, B.part, st))) return rc;
  // the six systems' scaled eigen-domain solutions -> x fields 0-11
  SweepBetas be;
  for (int k = 0; k < 6; ++k) be.v[k] = beta[k];
  const long long nb = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
  k_fdm_sweep_combine<<<(unsigned)nb, 256, 0, st>>>(M, N, B.ly, B.lx, be, mu, tmp + 4 * n, x);
  ALDIC_CUDA(cudaGetLastError());
  // 3. S = C Vx' -> tmp (12 fields)
  g.A = x; g.sab = n; g.sar = M; g.sak = 1;
  g.B = B.Vx; g.sbb = 0; g.sbk = 1; g.sbc = M;
  g.C = tmp; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = M; g.scale = 0;
  if ((rc = gemm(g, 12, B.part, st))) return rc;
  // 4. X = Vy S -> x
  g.A = B.Vy; g.sab = 0; g.sar = N; g.sak = 1;
  g.B = tmp; g.sbb = n; g.sbk = M; g.sbc = 1;
  g.C = x; g.scb = n; g.scr = M; g.scc = 1;
  g.R = N; g.Cn = M; g.K = N; g.scale = 0;
  return gemm(g, 12, B.part, st);
}

}  // namespace aldic

extern "C" ALDIC_API int aldic_fdm_basis(int type, int n, double h, double *V, double *lam) {
  return aldic::fdm_basis_1d(type, n, h, V, lam);
}
