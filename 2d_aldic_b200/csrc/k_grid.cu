// k_grid.cu -- solvers and field kernels on the M x N node grid of the
// uniform Q4 mesh (MeshSetUp.m): Subproblem 2 (Subpb2.m), nodal strain
// (funGlobal_NodalStrainAvg.m), gridfit 'springs' (gridfit.m), spring
// inpainting (inpaint_nans.m method 4), the bad-subset flags of LocalICGN.m /
// Subpb1.m and the 3x3 Gaussian nanconv of funSmoothDisp.m.
//
// All systems are SPD and solved by Jacobi-preconditioned CG in FP64 inside
// ONE cooperative persistent launch: blocks meet at a bounded grid barrier
// (two per iteration -- the search direction p = z + beta*p_prev is formed on
// the fly from ping-pong buffers, so no barrier separates its update from the
// next mat-vec).  Dot products are per-block partials summed in block order
// by every block, so all blocks take identical convergence decisions and the
// result is bit-reproducible.  Several right-hand sides (u and v, or the four
// components of F) share the operator and are solved in the same launch.
#include <cooperative_groups.h>

#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {

namespace {

constexpr int PCG_THREADS = 512;
constexpr int MAXRHS = 12;

struct PcgArgs {
  double *x, *r, *z, *p0, *p1, *q, *b, *diag, *part;
  double *zz, *qq, *ss, *pp;  // pipelined-CG directions
  const unsigned char *mask;
  int M, N, nrhs, maxit, blocks;
  double mu, h, lam2, rtol;
  double beta[MAXRHS];     // FE: beta per right-hand side
  const double *beta_ptr;  // if set, every right-hand side uses *beta_ptr
  GridSync gs;
  int *iters_out;
  CsrOp csr;               // OP_CSR
  const double *ata;       // OP_GRIDFIT with scattered data: A'A, 9 coefficients per node
};

// Scalar Q4 element matrices on a square element of size h with local nodes
// (-,-), (+,-), (+,+), (-,+) -- the 3x3 Gauss rule of Subpb2.m:100-101
// integrates them exactly: stiffness (1/6)[4 -1 -2 -1; ...] (Laplacian of
// u and v separately, beta*DN'DN) and mass (h^2/36)[4 2 1 2; ...]
// (mu*N'N).  Their node-pair sums give the 9-point stencil below.

// local node index -> (di, dj) offset from the element's first node
__device__ __forceinline__ int lx(int a) { return (a == 1 || a == 2) ? 1 : 0; }
__device__ __forceinline__ int ly(int a) { return (a >= 2) ? 1 : 0; }

// FE stencil weights on a square-element grid: the element matrices above
// summed over the elements two nodes share.  kap[0] centre, [1] axial, [2]
// diagonal; the coefficient of neighbour (di, dj) of node (i, j) is
// cnt(i, di) * cnt(j, dj) * kap[|di| + |dj|], cnt counting the element
// columns (rows) adjacent to both nodes.
__device__ __forceinline__ int ecnt(int i, int di, int M) {
  return di == 0 ? (i >= 1) + (i <= M - 2) : (di > 0 ? (i <= M - 2) : (i >= 1));
}

// funDerivativeOp.m:25-35 along one line of n nodes: 2h times the weight of
// x_s in the difference at t (central inside, one-sided doubled at the ends)
__device__ __forceinline__ double fdc(int t, int s, int n) {
  if (t == 0) return s == 1 ? 2.0 : (s == 0 ? -2.0 : 0.0);
  if (t == n - 1) return s == n - 1 ? 2.0 : (s == n - 2 ? -2.0 : 0.0);
  return s == t + 1 ? 1.0 : (s == t - 1 ? -1.0 : 0.0);
}

// (D'D v) along one line through node index c of a line with n nodes,
// stride st between line neighbours (scaled by 4 h^2)
__device__ __forceinline__ double fd_dtd(const double *__restrict__ v, long long k, int c, int n,
                                         long long st) {
  double y = 0.0;
#pragma unroll
  for (int dt = -1; dt <= 1; ++dt) {
    const int t = c + dt;
    if (t < 0 || t >= n) continue;
    const double w = fdc(t, c, n);
    if (w == 0.0) continue;
    double d = 0.0;
#pragma unroll
    for (int ds = -1; ds <= 1; ++ds) {
      const int s = t + ds;
      if (s < 0 || s >= n) continue;
      const double ws = fdc(t, s, n);
      if (ws != 0.0) d += ws * v[k + (long long)(s - c) * st];
    }
    y += w * d;
  }
  return y;
}

__device__ __forceinline__ double fd_diag1(int c, int n) {
  double y = 0.0;
  for (int t = c - 1; t <= c + 1; ++t)
    if (t >= 0 && t < n) {
      const double w = fdc(t, c, n);
      y += w * w;
    }
  return y;
}

template <int OP>
__device__ __forceinline__ double op_diag(const PcgArgs &A, double beta, int i, int j,
                                          long long k, int f) {
  const int M = A.M, N = A.N;
  if (OP == OP_FE) {
    const double kc = beta * (4.0 / 6.0) + A.mu * A.h * A.h * (4.0 / 36.0);
    return ecnt(i, 0, M) * ecnt(j, 0, N) * kc;
  } else if (OP == OP_FD) {
    return beta * (fd_diag1(i, M) + fd_diag1(j, N)) / (4.0 * A.h * A.h) + A.mu;
  } else if (OP == OP_CSR) {
    if (!A.mask[(long long)f * M * N + k]) return 1.0;
    return A.csr.valM ? beta * A.csr.diag[k] + A.mu * A.csr.diagM[k] : A.csr.diag[k];
  } else if (OP == OP_GRIDFIT) {
    const double w = A.ata ? A.ata[9 * k + 4] : (A.mask[(long long)f * M * N + k] ? 1.0 : 0.0);
    const int na = (i > 0) + (i < M - 1) + (j > 0) + (j < N - 1);
    const int nd = (i > 0 && j > 0) + (i < M - 1 && j > 0) + (i > 0 && j < N - 1) +
                   (i < M - 1 && j < N - 1);
    return w + A.lam2 * (na + 0.5 * nd);
  } else {
    if (!A.mask[(long long)f * M * N + k]) return 1.0;
    return (double)((i > 0) + (i < M - 1) + (j > 0) + (j < N - 1));
  }
}

// y = op(v)_k, v = one field (M*N values)
template <int OP>
__device__ __forceinline__ double op_apply(const PcgArgs &A, double beta, int i, int j,
                                           long long k, int f, const double *__restrict__ v) {
  const int M = A.M, N = A.N;
  if (OP == OP_FE) {
    const double km = A.mu * A.h * A.h;
    const double kap[3] = {beta * (4.0 / 6.0) + km * (4.0 / 36.0),
                           beta * (-1.0 / 6.0) + km * (2.0 / 36.0),
                           beta * (-2.0 / 6.0) + km * (1.0 / 36.0)};
    double y = 0.0;
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
      const int cj = ecnt(j, dj, N);
      if (!cj) continue;
#pragma unroll
      for (int di = -1; di <= 1; ++di) {
        const int ci = ecnt(i, di, M);
        if (!ci) continue;
        const int t = (di != 0) + (dj != 0);
        y += (double)(ci * cj) * kap[t] * v[k + di + (long long)dj * M];
      }
    }
    return y;
  } else if (OP == OP_FD) {
    return beta * (fd_dtd(v, k, i, M, 1) + fd_dtd(v, k, j, N, M)) / (4.0 * A.h * A.h) + A.mu * v[k];
  } else if (OP == OP_CSR) {
    const unsigned char *fr = A.mask + (long long)f * M * N;
    if (!fr[k]) return v[k];
    double y = 0.0;
    const int p1 = A.csr.row[k + 1];
    if (A.csr.valM) {
      for (int p = A.csr.row[k]; p < p1; ++p) {
        const int c = A.csr.col[p];
        if (fr[c]) y += (beta * A.csr.val[p] + A.mu * A.csr.valM[p]) * v[c];
      }
    } else {
      for (int p = A.csr.row[k]; p < p1; ++p) {
        const int c = A.csr.col[p];
        if (fr[c]) y += A.csr.val[p] * v[c];
      }
    }
    return y;
  } else if (OP == OP_GRIDFIT) {
    const double xk = v[k];
    double s = 0.0, sd = 0.0;
    if (i > 0) s += xk - v[k - 1];
    if (i < M - 1) s += xk - v[k + 1];
    if (j > 0) s += xk - v[k - M];
    if (j < N - 1) s += xk - v[k + M];
    if (i > 0 && j > 0) sd += xk - v[k - M - 1];
    if (i < M - 1 && j > 0) sd += xk - v[k - M + 1];
    if (i > 0 && j < N - 1) sd += xk - v[k + M - 1];
    if (i < M - 1 && j < N - 1) sd += xk - v[k + M + 1];
    double dterm;
    if (A.ata) {  // scattered data: the 9-point A'A stencil of the triangle interpolation
      const double *c = A.ata + 9 * k;
      dterm = c[4] * xk;
      if (i > 0) dterm += c[3] * v[k - 1];
      if (i < M - 1) dterm += c[5] * v[k + 1];
      if (j > 0) {
        dterm += c[1] * v[k - M];
        if (i > 0) dterm += c[0] * v[k - M - 1];
        if (i < M - 1) dterm += c[2] * v[k - M + 1];
      }
      if (j < N - 1) {
        dterm += c[7] * v[k + M];
        if (i > 0) dterm += c[6] * v[k + M - 1];
        if (i < M - 1) dterm += c[8] * v[k + M + 1];
      }
    } else {
      dterm = (A.mask[(long long)f * M * N + k] ? 1.0 : 0.0) * xk;
    }
    return dterm + A.lam2 * (s + 0.5 * sd);
  } else {
    const unsigned char *unk = A.mask + (long long)f * M * N;
    const double xk = v[k];
    if (!unk[k]) return xk;
    double s = 0.0;
    if (i > 0) s += xk - (unk[k - 1] ? v[k - 1] : 0.0);
    if (i < M - 1) s += xk - (unk[k + 1] ? v[k + 1] : 0.0);
    if (j > 0) s += xk - (unk[k - M] ? v[k - M] : 0.0);
    if (j < N - 1) s += xk - (unk[k + M] ? v[k + M] : 0.0);
    return s;
  }
}

// The operator on a direction vector of the iteration sweep, at an unknown
// entry.  Inpainting and CSR (masked) systems: directions are 0 at every
// known entry (both m buffers are cleared at set-up and only unknown entries
// are ever written), so the neighbour terms need no mask -- the same value
// as op_apply without its mask loads.
template <int OP>
__device__ __forceinline__ double op_apply_dir(const PcgArgs &A, double beta, int i, int j,
                                               long long k, int f, const double *__restrict__ v) {
  if (OP == OP_CSR) {
    double y = 0.0;
    const int p1 = A.csr.row[k + 1];
    if (A.csr.valM) {
      for (int p = A.csr.row[k]; p < p1; ++p)
        y += (beta * A.csr.val[p] + A.mu * A.csr.valM[p]) * v[A.csr.col[p]];
    } else {
      for (int p = A.csr.row[k]; p < p1; ++p) y += A.csr.val[p] * v[A.csr.col[p]];
    }
    return y;
  }
  if (OP == OP_INPAINT) {
    const int M = A.M, N = A.N;
    const double xk = v[k];
    double s = 0.0;
    if (i > 0) s += xk - v[k - 1];
    if (i < M - 1) s += xk - v[k + 1];
    if (j > 0) s += xk - v[k - M];
    if (j < N - 1) s += xk - v[k + M];
    return s;
  }
  return op_apply<OP>(A, beta, i, j, k, f, v);
}

// Per-warp partials staged in shared memory: sh[warp][slot]; a warp adds
// its butterfly-reduced values for `cnt` slots starting at s0.
struct PcgShared {
  double warp_part[PCG_THREADS / 32][4 * MAXRHS];
  double gsum[4 * MAXRHS];
  double alpha[MAXRHS], beta[MAXRHS], gam[MAXRHS], bb[MAXRHS];
  int done[MAXRHS];
};

__device__ __forceinline__ void warp_stage(PcgShared &S, int slot, double v) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) S.warp_part[threadIdx.x >> 5][slot] = v;
}

// block partial of slots [0, cnt) -> part[slot][blockIdx]
__device__ __forceinline__ void block_partials(PcgShared &S, int cnt, double *part, int blocks) {
  __syncthreads();
  if (threadIdx.x < cnt) {
    double t = 0.0;
    for (int w = 0; w < PCG_THREADS / 32; ++w) t += S.warp_part[w][threadIdx.x];
    part[(long long)threadIdx.x * blocks + blockIdx.x] = t;
  }
}

// Global sums of slots [0, cnt) after a grid barrier: warp w of every block
// reduces slots w, w+16, ... over the block partials (independent loads, then
// a fixed-order butterfly), so every block obtains bit-identical totals.
__device__ void global_sums(PcgShared &S, const double *part, int cnt, int blocks) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = wid; c < cnt; c += PCG_THREADS / 32) {
    const double *pp = part + (long long)c * blocks;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int b = lane + 32 * q;
      v[q] = b < blocks ? pp[b] : 0.0;
    }
    double t = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
    for (int b = lane + 256; b < blocks; b += 32) t += pp[b];
    t = warp_sum(t);
    if (lane == 0) S.gsum[c] = t;
  }
  __syncthreads();
}

// Pipelined preconditioned CG (Ghysels and Vanroose, "Hiding global
// synchronization latency in the preconditioned Conjugate Gradient
// algorithm", Parallel Computing 40, 2014): with u = M^-1 r, w = A u,
// m = M^-1 w, n = A m the recurrences
//   z = n + beta z, q = m + beta q, s = w + beta s, p = u + beta p,
//   x += alpha p, r -= alpha s, u -= alpha q, w -= alpha z
// need the dot products (r,u), (w,u) of the current vectors and one mat-vec
// n = A m, so an iteration is ONE sweep (the mat-vec and updates of a node,
// then its next dot-product terms and m = w / diag) and ONE grid barrier
// (the dot products' block partials, and every m, complete).  m and the
// partials alternate between two buffers, so a block that runs ahead never
// overwrites what a slower block still reads.  Jacobi preconditioner M =
// diag(A); convergence on the recursive residual, |r| <= rtol |b|.
// Buffers: x, r, u (= z slot), w (= q slot), m (p0 / p1), the directions
// zz, qq, ss, pp, 1/diag.
template <int OP, int NR>
__global__ void __launch_bounds__(PCG_THREADS) k_pcg(PcgArgs A) {
  __shared__ PcgShared S;
  if (A.beta_ptr) {
    const double bv = *A.beta_ptr;
#pragma unroll
    for (int f = 0; f < NR; ++f) A.beta[f] = bv;
  }
  const long long n = (long long)A.M * A.N;
  const int M = A.M;
  const long long tid0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  double *const X = A.x, *const R = A.r, *const Uv = A.z, *const Wv = A.q, *const Di = A.diag;
  double *const Zd = A.zz, *const Qd = A.qq, *const Sd = A.ss, *const Pd = A.pp;
  double *Mv[2] = {A.p0, A.p1};
  const long long pstride = (long long)4 * MAXRHS * A.blocks;  // second partials buffer
  // ---- r = b - A x, u = D^-1 r, directions 0
#pragma unroll 1
  for (int f = 0; f < NR; ++f) {
    const double bt = A.beta[f];
    for (long long k = tid0; k < n; k += stride) {
      const int j = (int)k / M, i = (int)k - j * M;  // n < 2^31 (checked at launch)
      const long long o = f * n + k;
      const double rv = A.b[o] - op_apply<OP>(A, bt, i, j, k, f, X + f * n);
      const double dinv = 1.0 / op_diag<OP>(A, bt, i, j, k, f);
      R[o] = rv;
      Uv[o] = rv * dinv;
      Di[o] = dinv;
      Zd[o] = 0.0;
      Qd[o] = 0.0;
      Sd[o] = 0.0;
      Pd[o] = 0.0;
    }
  }
  if (!grid_sync(A.gs, A.blocks)) return;
  // ---- w = A u, m = D^-1 w; partials (r,u) (w,u) (r,r) (b,b)
#pragma unroll 1
  for (int f = 0; f < NR; ++f) {
    const double bt = A.beta[f];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    for (long long k = tid0; k < n; k += stride) {
      const int j = (int)k / M, i = (int)k - j * M;  // n < 2^31 (checked at launch)
      const long long o = f * n + k;
      const double wv = op_apply<OP>(A, bt, i, j, k, f, Uv + f * n);
      Wv[o] = wv;
      Mv[0][o] = wv * Di[o];
      Mv[1][o] = 0.0;  // known inpainting entries are never written again
      const double rv = R[o], uv = Uv[o], bv = A.b[o];
      a0 += rv * uv;
      a1 += wv * uv;
      a2 += rv * rv;
      a3 += bv * bv;
    }
    warp_stage(S, f, a0);
    warp_stage(S, NR + f, a1);
    warp_stage(S, 2 * NR + f, a2);
    warp_stage(S, 3 * NR + f, a3);
  }
  block_partials(S, 4 * NR, A.part, A.blocks);
  if (!grid_sync(A.gs, A.blocks)) return;
  global_sums(S, A.part, 4 * NR, A.blocks);
  if (threadIdx.x < NR) {
    const int f = threadIdx.x;
    S.gam[f] = S.gsum[f];
    S.alpha[f] = S.gsum[f] / S.gsum[NR + f];
    S.beta[f] = 0.0;
    S.bb[f] = S.gsum[3 * NR + f];
    S.done[f] = !(S.gsum[2 * NR + f] > A.rtol * A.rtol * S.bb[f]);
  }
  __syncthreads();
  int it = 0;
  for (; it < A.maxit; ++it) {
    bool all = true;
#pragma unroll
    for (int f = 0; f < NR; ++f) all &= (S.done[f] != 0);
    if (all) break;
    const double *Mo = Mv[it & 1];
    double *Mn = Mv[(it + 1) & 1];
    double *part = A.part + ((it + 1) & 1) * pstride;
    // ---- n = A m; directions and iterates; next partials and m.  Fields
    // go in groups (pairs; threes for inpainting, whose sweep is a few
    // dependent loads a node), every load of a group before any store, so
    // the fields' memory round trips overlap.
    constexpr int G2 = ((OP == OP_INPAINT || OP == OP_CSR) && NR % 3 == 0) ? 3 : (NR >= 2 ? 2 : 1);
#pragma unroll 1
    for (int f0 = 0; f0 < NR; f0 += G2) {
      double a0[G2], a1[G2], a2[G2], al[G2], be[G2], bt[G2];
      bool live[G2], anylive = false;
#pragma unroll
      for (int q = 0; q < G2; ++q) {
        a0[q] = a1[q] = a2[q] = 0.0;
        const int f = f0 + q;
        live[q] = f < NR && !S.done[f];
        anylive |= live[q];
        bt[q] = f < NR ? A.beta[f] : 0.0;
        al[q] = f < NR ? S.alpha[f] : 0.0;
        be[q] = f < NR ? S.beta[f] : 0.0;
      }
      if (anylive) {
        for (long long k = tid0; k < n; k += stride) {
          const int j = (int)k / M, i = (int)k - j * M;  // n < 2^31 (checked at launch)
          double nv[G2], zo[G2], qo[G2], so[G2], po[G2], mo[G2], wo[G2], uo[G2], ro[G2], xo[G2],
              di[G2];
          // inpainting and CSR: a known entry is an identity row whose r, u,
          // w, m and directions are 0 after the set-up sweeps and stay 0, and
          // no unknown row reads it -- skip it (its dot-product terms are 0)
          constexpr bool kMasked = OP == OP_INPAINT || OP == OP_CSR;
          bool act[G2];
#pragma unroll
          for (int q = 0; q < G2; ++q)
            act[q] = live[q] && (!kMasked || A.mask[(long long)(f0 + q) * n + k]);
#pragma unroll
          for (int q = 0; q < G2; ++q) {
            if (!act[q]) continue;
            const int f = f0 + q;
            const long long o = f * n + k;
            nv[q] = op_apply_dir<OP>(A, bt[q], i, j, k, f, Mo + f * n);
            zo[q] = Zd[o]; qo[q] = Qd[o]; so[q] = Sd[o]; po[q] = Pd[o];
            mo[q] = Mo[o]; wo[q] = Wv[o]; uo[q] = Uv[o]; ro[q] = R[o]; xo[q] = X[o]; di[q] = Di[o];
          }
#pragma unroll
          for (int q = 0; q < G2; ++q) {
            if (!act[q]) continue;
            const long long o = (f0 + q) * n + k;
            const double zv = nv[q] + be[q] * zo[q];
            const double qv = mo[q] + be[q] * qo[q];
            const double sv = wo[q] + be[q] * so[q];
            const double pv = uo[q] + be[q] * po[q];
            Zd[o] = zv;
            Qd[o] = qv;
            Sd[o] = sv;
            Pd[o] = pv;
            X[o] = xo[q] + al[q] * pv;
            const double rv = ro[q] - al[q] * sv;
            const double uv = uo[q] - al[q] * qv;
            const double wv = wo[q] - al[q] * zv;
            R[o] = rv;
            Uv[o] = uv;
            Wv[o] = wv;
            Mn[o] = wv * di[q];
            a0[q] += rv * uv;
            a1[q] += wv * uv;
            a2[q] += rv * rv;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < G2; ++q) {
        const int f = f0 + q;
        if (f < NR) {
          warp_stage(S, f, a0[q]);
          warp_stage(S, NR + f, a1[q]);
          warp_stage(S, 2 * NR + f, a2[q]);
        }
      }
    }
    block_partials(S, 3 * NR, part, A.blocks);
    if (!grid_sync(A.gs, A.blocks)) return;
    global_sums(S, part, 3 * NR, A.blocks);
    if (threadIdx.x < NR) {
      const int f = threadIdx.x;
      if (!S.done[f]) {
        const double gn = S.gsum[f], dl = S.gsum[NR + f];
        const double be = gn / S.gam[f];
        S.beta[f] = be;
        S.alpha[f] = gn / (dl - be * gn / S.alpha[f]);
        S.gam[f] = gn;
        S.done[f] = !(S.gsum[2 * NR + f] > A.rtol * A.rtol * S.bb[f]);
      }
    }
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *A.iters_out = it > *A.iters_out ? it : *A.iters_out;
    bool all = true;
    for (int f = 0; f < NR; ++f) all &= (S.done[f] != 0);
    if (!all) atomicExch(A.gs.err, 2);  // not converged within maxit
  }
}

// ------------------------------------------------------------------ Subpb2 RHS
// Subpb2.m:88-149 per node, gathered from its (up to 4) elements.
// NB right-hand sides at once (the beta sweep: one per beta, the same
// operations for each as a single one), and the solve's start x = U with every
// entry unknown: fields (2q, 2q + 1) of b and x for beta[q].
struct FeBetas {
  double v[6], m[6];  // beta and mu of each right-hand side
};
template <int NB>
__global__ void k_fe_rhs(int M, int N, double h, FeBetas be, const double *beta_ptr,
                         const double *__restrict__ U, const double *__restrict__ F,
                         const double *__restrict__ ud, const double *__restrict__ vd,
                         double *__restrict__ b, double *__restrict__ x,
                         unsigned char *__restrict__ mask) {
  if (beta_ptr) be.v[0] = *beta_ptr;
  const long long n = (long long)M * N;
  const double gp[3] = {-0.7745966692414834, 0.0, 0.7745966692414834};  // sqrt(3/5)
  const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    // F - W with the column order [4a-3, 4a-1, 4a-2, 4a] of Subpb2.m:88-91
    const double fw0 = F[4 * k + 0] - ud[4 * k + 0];
    const double fw1 = F[4 * k + 2] - ud[4 * k + 2];
    const double fw2 = F[4 * k + 1] - ud[4 * k + 1];
    const double fw3 = F[4 * k + 3] - ud[4 * k + 3];
    double bu[NB], bv[NB];
#pragma unroll
    for (int q = 0; q < NB; ++q) bu[q] = bv[q] = 0.0;
    for (int ej = j - 1; ej <= j; ++ej)
      for (int ei = i - 1; ei <= i; ++ei) {
        if (ei < 0 || ei >= M - 1 || ej < 0 || ej >= N - 1) continue;
        const int la = (i - ei) + (j - ej) * 3 - 2 * (i - ei) * (j - ej);
        double uvu[4], uvv[4];
        for (int lb = 0; lb < 4; ++lb) {
          const long long q = (long long)(ej + ly(lb)) * M + (ei + lx(lb));
          uvu[lb] = U[2 * q] - vd[2 * q];
          uvv[lb] = U[2 * q + 1] - vd[2 * q + 1];
        }
        for (int ti = 0; ti < 3; ++ti)
          for (int tj = 0; tj < 3; ++tj) {
            const double ksi = gp[ti], eta = gp[tj];
            const double Nn[4] = {(1 - ksi) * (1 - eta) * 0.25, (1 + ksi) * (1 - eta) * 0.25,
                                  (1 + ksi) * (1 + eta) * 0.25, (1 - ksi) * (1 + eta) * 0.25};
            const double dks[4] = {-(1 - eta) / 4, (1 - eta) / 4, (1 + eta) / 4, -(1 + eta) / 4};
            const double det_[4] = {-(1 - ksi) / 4, -(1 + ksi) / 4, (1 + ksi) / 4, (1 - ksi) / 4};
            const double s = (0.25 * h * h) * (gw[ti] * gw[tj]);
            const double gx = (2.0 / h) * dks[la], gy = (2.0 / h) * det_[la];
            double nu = 0.0, nv = 0.0;
            for (int lb = 0; lb < 4; ++lb) {
              nu += Nn[lb] * uvu[lb];
              nv += Nn[lb] * uvv[lb];
            }
#pragma unroll
            for (int q = 0; q < NB; ++q) {
              bu[q] += s * (be.v[q] * (gx * fw0 + gy * fw1) + be.m[q] * Nn[la] * nu);
              bv[q] += s * (be.v[q] * (gx * fw2 + gy * fw3) + be.m[q] * Nn[la] * nv);
            }
          }
      }
    const double u0 = U[2 * k], v0 = U[2 * k + 1];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      b[2 * q * n + k] = bu[q];
      b[(2 * q + 1) * n + k] = bv[q];
      x[2 * q * n + k] = u0;
      x[(2 * q + 1) * n + k] = v0;
      mask[2 * q * n + k] = 1;
      mask[(2 * q + 1) * n + k] = 1;
    }
  }
}

// beta D'a + mu b on the interior grid (Mi = M - 2, Ni = N - 2); a = F - udual,
// b = U - vdual at the interior nodes of the full M x N grid; x starts at U
__global__ void k_fd_rhs(int M, int N, double h, double beta, const double *beta_ptr, double mu,
                         const double *__restrict__ U, const double *__restrict__ F,
                         const double *__restrict__ ud, const double *__restrict__ vd,
                         double *__restrict__ b, double *__restrict__ x,
                         unsigned char *__restrict__ mask) {
  if (beta_ptr) beta = *beta_ptr;
  const int Mi = M - 2, Ni = N - 2;
  const long long ni = (long long)Mi * Ni;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ni;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % Mi), j = (int)(k / Mi);
    // D' a: x-differences of the F11 / F21 slots, y-differences of F12 / F22
    double au = 0.0, av = 0.0;
    for (int t = i - 1; t <= i + 1; ++t) {
      if (t < 0 || t >= Mi) continue;
      const double w = fdc(t, i, Mi);
      if (w == 0.0) continue;
      const long long q = (long long)(j + 1) * M + (t + 1);
      au += w * (F[4 * q + 0] - ud[4 * q + 0]);
      av += w * (F[4 * q + 1] - ud[4 * q + 1]);
    }
    for (int t = j - 1; t <= j + 1; ++t) {
      if (t < 0 || t >= Ni) continue;
      const double w = fdc(t, j, Ni);
      if (w == 0.0) continue;
      const long long q = (long long)(t + 1) * M + (i + 1);
      au += w * (F[4 * q + 2] - ud[4 * q + 2]);
      av += w * (F[4 * q + 3] - ud[4 * q + 3]);
    }
    const long long q = (long long)(j + 1) * M + (i + 1);
    b[k] = beta * au / (2.0 * h) + mu * (U[2 * q] - vd[2 * q]);
    b[ni + k] = beta * av / (2.0 * h) + mu * (U[2 * q + 1] - vd[2 * q + 1]);
    x[k] = U[2 * q];
    x[ni + k] = U[2 * q + 1];
    mask[k] = 1;
    mask[ni + k] = 1;
  }
}

__global__ void k_fd_store(int M, int N, const double *__restrict__ x, const double *__restrict__ U1,
                           double *__restrict__ U2) {
  const long long n = (long long)M * N, ni = (long long)(M - 2) * (N - 2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    if (i >= 1 && i <= M - 2 && j >= 1 && j <= N - 2) {
      const long long q = (long long)(j - 1) * (M - 2) + (i - 1);
      U2[2 * k] = x[q];
      U2[2 * k + 1] = x[ni + q];
    } else {
      U2[2 * k] = U1[2 * k];
      U2[2 * k + 1] = U1[2 * k + 1];
    }
  }
}

// F = D2 U (funDerivativeOp(M, N, h) * U): [du/dx dv/dx du/dy dv/dy]
__global__ void k_fd_strain(int M, int N, double h, const double *__restrict__ U,
                            double *__restrict__ F) {
  const long long n = (long long)M * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    double ux = 0, vx = 0, uy = 0, vy = 0;
    for (int s = i - 1; s <= i + 1; ++s) {
      if (s < 0 || s >= M) continue;
      const double w = fdc(i, s, M);
      if (w == 0.0) continue;
      const long long q = (long long)j * M + s;
      ux += w * U[2 * q];
      vx += w * U[2 * q + 1];
    }
    for (int s = j - 1; s <= j + 1; ++s) {
      if (s < 0 || s >= N) continue;
      const double w = fdc(j, s, N);
      if (w == 0.0) continue;
      const long long q = (long long)s * M + i;
      uy += w * U[2 * q];
      vy += w * U[2 * q + 1];
    }
    const double c = 1.0 / (2.0 * h);
    F[4 * k + 0] = ux * c;
    F[4 * k + 1] = vx * c;
    F[4 * k + 2] = uy * c;
    F[4 * k + 3] = vy * c;
  }
}

__global__ void k_fd_dual(int M, int N, const double *__restrict__ F2, const double *__restrict__ F1,
                          const double *__restrict__ U2, const double *__restrict__ U1,
                          double *__restrict__ ud, double *__restrict__ vd, int accumulate) {
  const long long n = (long long)M * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    const bool in = i >= 1 && i <= M - 2 && j >= 1 && j <= N - 2;
    for (int c = 0; c < 4; ++c) {
      const double d = in ? F2[4 * k + c] - F1[4 * k + c] : 0.0;
      ud[4 * k + c] = accumulate ? ud[4 * k + c] + d : d;
    }
    for (int c = 0; c < 2; ++c) {
      const double d = in ? U2[2 * k + c] - U1[2 * k + c] : 0.0;
      vd[2 * k + c] = accumulate ? vd[2 * k + c] + d : d;
    }
  }
}

__global__ void k_fe_store(long long n, const double *__restrict__ x, double *__restrict__ U) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    U[2 * k] = x[k];
    U[2 * k + 1] = x[n + k];
  }
}

// ------------------------------------------------------------------ nodal strain
// funGlobal_NodalStrainAvg.m:51-144: per element, DN*U at the 2x2 Gauss points
// in the order (-,-), (+,-), (+,+), (-,+); extrapolated to the corners with
// the matrix of :105-108; averaged over the elements sharing a node.  Output
// slots per node are [du/dx, du/dy, dv/dx, dv/dy] as written at :123-137.
// The nodal strain of node (i, j); ld(q, &u, &v) reads the displacement of
// node q.
template <class Load>
__device__ __forceinline__ void nodal_strain_node(int M, int N, double h, int i, int j,
                                                  const Load &ld, double out[4]) {
  const double r3 = 0.5773502691896257;  // 1/sqrt(3)
  const double s3 = 1.7320508075688772;
  const double gks[4] = {-r3, r3, r3, -r3}, get_[4] = {-r3, -r3, r3, r3};
  const double E[4][4] = {{1 + 0.5 * s3, -0.5, 1 - 0.5 * s3, -0.5},
                          {-0.5, 1 + 0.5 * s3, -0.5, 1 - 0.5 * s3},
                          {1 - 0.5 * s3, -0.5, 1 + 0.5 * s3, -0.5},
                          {-0.5, 1 - 0.5 * s3, -0.5, 1 + 0.5 * s3}};
  double acc[4] = {0, 0, 0, 0};
  int cnt = 0;
  for (int ej = j - 1; ej <= j; ++ej)
    for (int ei = i - 1; ei <= i; ++ei) {
      if (ei < 0 || ei >= M - 1 || ej < 0 || ej >= N - 1) continue;
      const int la = (i - ei) + (j - ej) * 3 - 2 * (i - ei) * (j - ej);
      double ue[8];
      for (int lb = 0; lb < 4; ++lb) {
        const long long q = (long long)(ej + ly(lb)) * M + (ei + lx(lb));
        ld(q, &ue[2 * lb], &ue[2 * lb + 1]);
      }
      double G[4][4];
      for (int g = 0; g < 4; ++g) {
        const double ksi = gks[g], eta = get_[g];
        const double dks[4] = {-(1 - eta) / 4, (1 - eta) / 4, (1 + eta) / 4, -(1 + eta) / 4};
        const double det_[4] = {-(1 - ksi) / 4, -(1 + ksi) / 4, (1 + ksi) / 4, (1 - ksi) / 4};
        double v[4] = {0, 0, 0, 0};
        for (int a = 0; a < 4; ++a) {
          const double gx = (2.0 / h) * dks[a], gy = (2.0 / h) * det_[a];
          v[0] += gx * ue[2 * a];
          v[1] += gy * ue[2 * a];
          v[2] += gx * ue[2 * a + 1];
          v[3] += gy * ue[2 * a + 1];
        }
        for (int c = 0; c < 4; ++c) G[g][c] = v[c];
      }
      for (int c = 0; c < 4; ++c) {
        double s = 0.0;
        for (int g = 0; g < 4; ++g) s += E[la][g] * G[g][c];
        acc[c] += s;
      }
      cnt++;
    }
  for (int c = 0; c < 4; ++c) out[c] = acc[c] / cnt;
}

__global__ void k_nodal_strain(int M, int N, double h, const double *__restrict__ U,
                               double *__restrict__ F) {
  const long long n = (long long)M * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    double out[4];
    nodal_strain_node(M, N, h, i, j,
                      [&](long long q, double *u, double *v) {
                        *u = U[2 * q];
                        *v = U[2 * q + 1];
                      },
                      out);
    for (int c = 0; c < 4; ++c) F[4 * k + c] = out[c];
  }
}

// ------------------------------------------------------------------ beta sweep errors
// The beta sweep of Subproblem 2 (main_ALDIC.m:206-230) stores each
// candidate solution, forms its nodal strain and takes |U1 - U2| and
// |F1 - F2|; only those two norms outlive the sweep.  One pass over the
// nodes forms both for every candidate c (fields 2c, 2c + 1 of the solver's
// x, node order) without writing the candidates out: block partials go to
// part[s * gridDim.x + block], s = c for the displacement norm and
// kSweepMax + c for the strain norm.
constexpr int kSweepMax = 6;
constexpr int kSweepThreads = 256;
__global__ void __launch_bounds__(kSweepThreads) k_sweep_err(int M, int N, int nc, double h,
                                                             const double *__restrict__ x,
                                                             const double *__restrict__ U1,
                                                             const double *__restrict__ F1,
                                                             double *__restrict__ part) {
  const long long n = (long long)M * N;
  double su[kSweepMax], sf[kSweepMax];
#pragma unroll
  for (int c = 0; c < kSweepMax; ++c) su[c] = sf[c] = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    const double u1 = U1[2 * k], v1 = U1[2 * k + 1];
    double f1[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) f1[m] = F1[4 * k + m];
#pragma unroll
    for (int c = 0; c < kSweepMax; ++c) {
      if (c >= nc) break;
      const double *xu = x + 2 * c * n, *xv = xu + n;
      const double du = u1 - xu[k], dv = v1 - xv[k];
      su[c] += du * du + dv * dv;
      double fn[4];
      nodal_strain_node(M, N, h, i, j,
                        [&](long long q, double *u, double *v) {
                          *u = xu[q];
                          *v = xv[q];
                        },
                        fn);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const double d = f1[m] - fn[m];
        sf[c] += d * d;
      }
    }
  }
  __shared__ double sh[2 * kSweepMax][kSweepThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < kSweepMax; ++c) {
    const double a = warp_sum(su[c]), b = warp_sum(sf[c]);
    if (lane == 0) {
      sh[c][wid] = a;
      sh[kSweepMax + c][wid] = b;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * kSweepMax) {
    double t = 0.0;
    for (int w = 0; w < kSweepThreads / 32; ++w) t += sh[threadIdx.x][w];
    part[threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
}

// err[c] = |U1 - U2_c|, err[kSweepMax + c] = |F1 - F2_c|: one warp per norm,
// fixed summation order
__global__ void k_sweep_err_final(const double *__restrict__ part, int nb, int nc,
                                  double *__restrict__ err) {
  const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = s % kSweepMax;
  if (c >= nc) return;
  double t = 0.0;
  for (int b = lane; b < nb; b += 32) t += part[s * nb + b];
  t = warp_sum(t);
  if (lane == 0) err[s] = sqrt(t);
}

// ------------------------------------------------------------------ loaders
__global__ void k_gridfit_load(int M, int N, int nf, const double *__restrict__ vals, int stride,
                               const int *__restrict__ iters, const double *__restrict__ guess,
                               double *__restrict__ b, double *__restrict__ x,
                               unsigned char *__restrict__ mask) {
  const long long n = (long long)M * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const bool bad = iters && (iters[k] < 0 || iters[k] > 99);
    for (int f = 0; f < nf; ++f) {
      const double v = vals[k * stride + f];
      const bool ok = !bad && !isnan(v);
      mask[f * n + k] = ok;
      b[f * n + k] = ok ? v : 0.0;
      x[f * n + k] = ok ? v : (guess ? guess[k * stride + f] : 0.0);
    }
  }
}


__global__ void k_grid_store(int M, int N, int nf, const double *__restrict__ x,
                             double *__restrict__ vals, int stride) {
  const long long n = (long long)M * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    for (int f = 0; f < nf; ++f) vals[k * stride + f] = x[f * n + k];
}

__global__ void k_inpaint_load(int M, int N, int nf, const double *__restrict__ vals, int stride,
                               const unsigned char *__restrict__ badmask,
                               double *__restrict__ b, double *__restrict__ x,
                               unsigned char *__restrict__ mask) {
  // fields [0, nf) of vals land in slots f0.. of the work vectors (the
  // caller offsets b, x, mask by f0 * n)
  const long long n = (long long)M * N;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    for (int f = 0; f < nf; ++f) {
      auto known = [&](long long q) {
        return !(badmask && badmask[q]) && !isnan(vals[q * stride + f]);
      };
      const bool kn = known(k);
      mask[f * n + k] = !kn;
      double bv;
      int kc = 0;  // known neighbours of an unknown entry
      if (kn) {
        bv = vals[k * stride + f];
      } else {
        bv = 0.0;
        if (i > 0 && known(k - 1)) { bv += vals[(k - 1) * stride + f]; ++kc; }
        if (i < M - 1 && known(k + 1)) { bv += vals[(k + 1) * stride + f]; ++kc; }
        if (j > 0 && known(k - M)) { bv += vals[(k - M) * stride + f]; ++kc; }
        if (j < N - 1 && known(k + M)) { bv += vals[(k + M) * stride + f]; ++kc; }
      }
      b[f * n + k] = bv;
      // an unknown entry starts from the mean of its known neighbours (the
      // solution itself for an isolated one), else from 0
      x[f * n + k] = kn ? bv : (kc > 0 ? bv / kc : 0.0);
    }
  }
}

// ------------------------------------------------------------------ flags
__global__ void k_icgn_flags(long long n, const int *__restrict__ it,
                             unsigned char *__restrict__ bad, int *badnum, double *meanit,
                             int *nconv, double floor) {
  __shared__ long long sh[32][3];
  __shared__ double shd[32];
  __shared__ double s_mean, s_thr;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long cb = 0, c102 = 0, sg = 0, ng = 0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    const int v = it[k];
    const bool b1 = v < 0 || v > 99;
    cb += b1;
    c102 += (v == 102);
    if (!b1) {
      sg += v;
      ng++;
    }
  }
  cb = warp_sum_ll(cb); c102 = warp_sum_ll(c102); sg = warp_sum_ll(sg); ng = warp_sum_ll(ng);
  if (lane == 0) { sh[wid][0] = cb; sh[wid][1] = c102; sh[wid][2] = sg; shd[wid] = (double)ng; }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long a = 0, b = 0, c = 0, d = 0;
    for (int w = 0; w < nw; ++w) { a += sh[w][0]; b += sh[w][1]; c += sh[w][2]; d += (long long)shd[w]; }
    *badnum = (int)(a - b);
    *nconv = (int)d;
    s_mean = d ? (double)c / (double)d : __longlong_as_double(0x7ff8000000000000ll);
    *meanit = s_mean;
    sh[0][0] = d;
  }
  __syncthreads();
  const long long ngood = sh[0][0];
  const double m = s_mean;
  double ss = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    const int v = it[k];
    if (!(v < 0 || v > 99)) ss += (v - m) * (v - m);
  }
  ss = warp_sum(ss);
  __syncthreads();
  if (lane == 0) shd[wid] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += shd[w];
    const double sd = ngood > 1 ? sqrt(t / (double)(ngood - 1))
                                : (ngood == 1 ? 0.0 : __longlong_as_double(0x7ff8000000000000ll));
    // Subpb1Quadtree.m:180 raises the threshold to at least `floor`
    // (MATLAB's max ignores a NaN); NaN floor = LocalICGN.m:128-131
    s_thr = isnan(floor) ? m + 0.15 * sd : fmax(m + 0.15 * sd, floor);
  }
  __syncthreads();
  const double thr = s_thr;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    const int v = it[k];
    bad[k] = (v < 0 || v > 99 || (double)v > thr) ? 1 : 0;
  }
}

__global__ void k_subpb1_flags(long long n, const int *__restrict__ it,
                               unsigned char *__restrict__ bad, int *badnum) {
  __shared__ long long sh[32];
  long long c = 0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) {
    const bool b = it[k] < 0 || it[k] > 99;
    bad[k] = b;
    c += b;
  }
  c = warp_sum_ll(c);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    *badnum = (int)t;
  }
}

// nanconv(z, fspecial('gaussian',3,0.5), 'edge', 'nanout') with no NaN input
__global__ void k_nanconv3(int M, int N, int nf, const double *__restrict__ in,
                           double *__restrict__ out) {
  const long long n = (long long)M * N;
  const double e1 = 0.1353352832366127;   // exp(-2)
  const double e2 = 0.01831563888873418;  // exp(-4)
  const double ks = 1.0 + 4.0 * e1 + 4.0 * e2;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n * nf;
       k += (long long)gridDim.x * blockDim.x) {
    const long long kk = k % n, f = k / n;
    const int i = (int)(kk % M), j = (int)(kk / M);
    double s = 0.0, w = 0.0;
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        const int ii = i + di, jj = j + dj;
        if (ii < 0 || ii >= M || jj < 0 || jj >= N) continue;
        const int d2 = di * di + dj * dj;
        const double kv = (d2 == 0 ? 1.0 : (d2 == 1 ? e1 : e2)) / ks;
        s += kv * in[f * n + (long long)jj * M + ii];
        w += kv;
      }
    out[k] = s / w;
  }
}

__global__ void k_vsub(const double *a, const double *b, double *o, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    o[k] = a[k] - b[k];
}

// o1 = a1 - b1 (n1 entries) and o2 = a2 - b2 (n2) in one launch
__global__ void k_vsub2(const double *a1, const double *b1, double *o1, long long n1,
                        const double *a2, const double *b2, double *o2, long long n2) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n1 + n2;
       k += (long long)gridDim.x * blockDim.x) {
    if (k < n1) o1[k] = a1[k] - b1[k];
    else o2[k - n1] = a2[k - n1] - b2[k - n1];
  }
}

// block partials of |a - b|^2; with copy, a <- b as it goes (the caller's
// "old" vector refreshed in the same pass)
__global__ void k_diffnorm_part(double *a, const double *b, long long n, double *part, bool copy) {
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const double bk = b[k];
    const double d = a[k] - bk;
    s += d * d;
    if (copy) a[k] = bk;
  }
  s = warp_sum(s);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

// one 256-thread block: strided partial sums, then a fixed-order tree;
// res = sqrt(sum) * scale
__global__ void k_diffnorm_final(const double *part, int np, double *res, double scale) {
  double t = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) t += part[k];
  t = warp_sum(t);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) u += sh[w];
    *res = sqrt(u) * scale;
  }
}

inline int blocks_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 8) b = 148 * 8;
  return b < 1 ? 1 : (int)b;
}

}  // namespace

int grid_pcg(GridWork &w, int op, int M, int N, int nrhs, double beta, double mu, double h,
             double lam2, double rtol, int maxit, cudaStream_t st, const double *beta_ptr,
             const double *beta_each, const double *ata) {
  ALDIC_CHECK(nrhs >= 1 && nrhs <= MAXRHS, E_ARG, "grid_pcg: 1..12 right-hand sides");
  const long long n = (long long)M * N;
  ALDIC_CHECK(n < (1LL << 31), E_ARG, "grid_pcg: more than 2^31 nodes");
  int dev = 0, sms = 148, per = 1;
  ALDIC_CUDA(cudaGetDevice(&dev));
  ALDIC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  void *fn = nullptr;
#define ALDIC_PCG_FN(OPV)                                                         \
  switch (nrhs) {                                                                 \
    case 1: fn = (void *)k_pcg<OPV, 1>; break;                                    \
    case 2: fn = (void *)k_pcg<OPV, 2>; break;                                    \
    case 3: case 4: fn = (void *)k_pcg<OPV, 4>; break;                            \
    case 5: case 6: fn = (void *)k_pcg<OPV, 6>; break;                            \
    default: fn = (void *)k_pcg<OPV, 12>; break;                                  \
  }
  if (op == OP_FE) { ALDIC_PCG_FN(OP_FE) }
  else if (op == OP_FD) { ALDIC_PCG_FN(OP_FD) }
  else if (op == OP_GRIDFIT) { ALDIC_PCG_FN(OP_GRIDFIT) }
  else { ALDIC_PCG_FN(OP_INPAINT) }
#undef ALDIC_PCG_FN
  const int nr_pad = nrhs <= 2 ? nrhs : (nrhs <= 4 ? 4 : (nrhs <= 6 ? 6 : 12));
  ALDIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, PCG_THREADS, 0));
  // one block per SM at most: fewer partials and cheaper barriers, while the
  // grid-stride loops still cover every node
  long long blocks = (long long)sms * (per < 1 ? 1 : (per > 1 ? 1 : per));
  const long long need = (n + PCG_THREADS - 1) / PCG_THREADS;
  if (blocks > need) blocks = need;
  if (blocks > w.max_blocks) blocks = w.max_blocks;
  if (blocks < 1) blocks = 1;
  PcgArgs A;
  A.x = w.x; A.r = w.r; A.z = w.z; A.p0 = w.p; A.p1 = w.p + MAXRHS * n; A.q = w.q; A.b = w.b;
  A.diag = w.diag; A.part = w.part; A.mask = w.mask;
  A.zz = w.zz; A.qq = w.qq; A.ss = w.ss; A.pp = w.pp;
  if (nr_pad > nrhs) {  // padded right-hand sides: b = x = 0 converge at once
    ALDIC_CUDA(cudaMemsetAsync(w.b + nrhs * n, 0, sizeof(double) * (nr_pad - nrhs) * n, st));
    ALDIC_CUDA(cudaMemsetAsync(w.x + nrhs * n, 0, sizeof(double) * (nr_pad - nrhs) * n, st));
    ALDIC_CUDA(cudaMemsetAsync(w.mask + nrhs * n, 0, (size_t)(nr_pad - nrhs) * n, st));
  }
  A.M = M; A.N = N; A.nrhs = nr_pad; A.maxit = maxit; A.blocks = (int)blocks;
  for (int f = 0; f < MAXRHS; ++f) A.beta[f] = (beta_each && f < nrhs) ? beta_each[f] : beta;
  A.mu = mu; A.h = h; A.lam2 = lam2; A.rtol = rtol;
  A.gs.count = w.bar; A.gs.gen = w.bar + 1; A.gs.err = w.err;
  A.iters_out = w.iters_out;
  A.beta_ptr = beta_ptr;
  A.csr = CsrOp{};
  A.ata = op == OP_GRIDFIT ? ata : nullptr;
  ALDIC_CUDA(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned int), st));
  void *args[] = {&A};
  ALDIC_CUDA(cudaLaunchCooperativeKernel(fn, dim3((unsigned)blocks), dim3(PCG_THREADS), args, 0, st));
  return OK;
}

int csr_pcg(GridWork &w, const CsrOp &op, long long n, int nrhs, double rtol, int maxit,
            cudaStream_t st, const double *beta_each, double mu) {
  ALDIC_CHECK(nrhs >= 1 && nrhs <= 6, E_ARG, "csr_pcg: 1..6 right-hand sides");
  ALDIC_CHECK(n >= 1 && n < (1LL << 31), E_ARG, "csr_pcg: bad size");
  int dev = 0, sms = 148;
  ALDIC_CUDA(cudaGetDevice(&dev));
  ALDIC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  void *fn = nullptr;
  switch (nrhs) {
    case 1: fn = (void *)k_pcg<OP_CSR, 1>; break;
    case 2: fn = (void *)k_pcg<OP_CSR, 2>; break;
    case 3: case 4: fn = (void *)k_pcg<OP_CSR, 4>; break;
    default: fn = (void *)k_pcg<OP_CSR, 6>; break;
  }
  const int nr_pad = nrhs <= 2 ? nrhs : (nrhs <= 4 ? 4 : 6);
  long long blocks = sms;
  const long long need = (n + PCG_THREADS - 1) / PCG_THREADS;
  if (blocks > need) blocks = need;
  if (blocks > w.max_blocks) blocks = w.max_blocks;
  if (blocks < 1) blocks = 1;
  PcgArgs A;
  A.x = w.x; A.r = w.r; A.z = w.z; A.p0 = w.p; A.p1 = w.p + MAXRHS * n; A.q = w.q; A.b = w.b;
  A.diag = w.diag; A.part = w.part; A.mask = w.mask;
  A.zz = w.zz; A.qq = w.qq; A.ss = w.ss; A.pp = w.pp;
  if (nr_pad > nrhs) {
    ALDIC_CUDA(cudaMemsetAsync(w.b + nrhs * n, 0, sizeof(double) * (nr_pad - nrhs) * n, st));
    ALDIC_CUDA(cudaMemsetAsync(w.x + nrhs * n, 0, sizeof(double) * (nr_pad - nrhs) * n, st));
    ALDIC_CUDA(cudaMemsetAsync(w.mask + nrhs * n, 0, (size_t)(nr_pad - nrhs) * n, st));
  }
  A.M = (int)n; A.N = 1; A.nrhs = nr_pad; A.maxit = maxit; A.blocks = (int)blocks;
  for (int f = 0; f < MAXRHS; ++f) A.beta[f] = (beta_each && f < nrhs) ? beta_each[f] : 0.0;
  A.mu = mu; A.h = 1; A.lam2 = 0; A.rtol = rtol;
  A.gs.count = w.bar; A.gs.gen = w.bar + 1; A.gs.err = w.err;
  A.iters_out = w.iters_out;
  A.beta_ptr = nullptr;
  A.csr = op;
  A.ata = nullptr;
  ALDIC_CUDA(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned int), st));
  void *args[] = {&A};
  ALDIC_CUDA(cudaLaunchCooperativeKernel(fn, dim3((unsigned)blocks), dim3(PCG_THREADS), args, 0, st));
  return OK;
}

int fe_rhs(GridWork &w, int M, int N, double h, double beta, double mu, const double *U,
           const double *F, const double *udual, const double *vdual, cudaStream_t st,
           const double *beta_ptr, int f0) {
  const long long n = (long long)M * N;
  FeBetas be{};
  be.v[0] = beta;
  be.m[0] = mu;
  k_fe_rhs<1><<<blocks_for(n), 256, 0, st>>>(M, N, h, be, beta_ptr, U, F, udual, vdual,
                                             w.b + f0 * n, w.x + f0 * n, w.mask + f0 * n);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int fe_rhs_parts(GridWork &w, int M, int N, double h, const double *U, const double *F,
                 const double *udual, const double *vdual, cudaStream_t st) {
  const long long n = (long long)M * N;
  FeBetas be{};
  be.v[0] = 1.0;  // fields 0-1: the beta part (beta 1, mu 0)
  be.m[1] = 1.0;  // fields 2-3: the mu part (beta 0, mu 1)
  k_fe_rhs<2><<<blocks_for(n), 256, 0, st>>>(M, N, h, be, nullptr, U, F, udual, vdual, w.b,
                                             w.x, w.mask);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int fd_rhs(GridWork &w, int M, int N, double h, double beta, double mu, const double *U,
           const double *F, const double *udual, const double *vdual, cudaStream_t st,
           const double *beta_ptr, int f0) {
  ALDIC_CHECK(M >= 4 && N >= 4, E_ARG, "FD Subpb2: the node grid needs at least 4 x 4 nodes");
  const long long ni = (long long)(M - 2) * (N - 2);
  k_fd_rhs<<<blocks_for(ni), 256, 0, st>>>(M, N, h, beta, beta_ptr, mu, U, F, udual, vdual,
                                          w.b + f0 * ni, w.x + f0 * ni, w.mask + f0 * ni);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int fd_store(const GridWork &w, int M, int N, const double *U1, double *U2, cudaStream_t st, int f0) {
  const long long ni = (long long)(M - 2) * (N - 2);
  k_fd_store<<<blocks_for((long long)M * N), 256, 0, st>>>(M, N, w.x + f0 * ni, U1, U2);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int fd_strain(int M, int N, double h, const double *U, double *F, cudaStream_t st) {
  k_fd_strain<<<blocks_for((long long)M * N), 256, 0, st>>>(M, N, h, U, F);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int fd_dual(int M, int N, const double *F2, const double *F1, const double *U2, const double *U1,
            double *udual, double *vdual, int accumulate, cudaStream_t st) {
  k_fd_dual<<<blocks_for((long long)M * N), 256, 0, st>>>(M, N, F2, F1, U2, U1, udual, vdual,
                                                         accumulate);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

// PlaneFit2.m on the symmetric (2 rad + 1)^2 window: the least-squares plane
// a + b (i h) + c (j h) has b = sum(i u) / (h (2r+1) sum i^2) and c likewise
// (the window's sums of i, j and i j vanish)
__global__ void k_plane_fit(int M, int N, double h, int rad, const double *__restrict__ U,
                            double *__restrict__ F) {
  const long long n = (long long)M * N;
  double s2 = 0.0;
  for (int t = -rad; t <= rad; ++t) s2 += (double)t * t;
  const double den = h * (2 * rad + 1) * s2;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % M), j = (int)(k / M);
    if (i < rad || i >= M - rad || j < rad || j >= N - rad) continue;
    double ux = 0, vx = 0, uy = 0, vy = 0;
    for (int tj = -rad; tj <= rad; ++tj)
      for (int ti = -rad; ti <= rad; ++ti) {
        const long long q = (long long)(j + tj) * M + (i + ti);
        const double u = U[2 * q], v = U[2 * q + 1];
        ux += ti * u;
        vx += ti * v;
        uy += tj * u;
        vy += tj * v;
      }
    F[4 * k + 0] = ux / den;
    F[4 * k + 1] = vx / den;
    F[4 * k + 2] = uy / den;
    F[4 * k + 3] = vy / den;
  }
}

// ComputeStrain.m:105-129 on [du/dx dv/dx du/dy dv/dy] per node
__global__ void k_finite_strain(long long n, int type, const double *__restrict__ F,
                                double *__restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const double ux = F[4 * k], vx = F[4 * k + 1], uy = F[4 * k + 2], vy = F[4 * k + 3];
    double o0 = ux, o1 = vx, o2 = uy, o3 = vy;
    if (type == 1) {         // Eulerian
      o0 = 1.0 / (1.0 - ux) - 1.0;
      o3 = 1.0 / (1.0 - vy) - 1.0;
      o2 = uy / (1.0 - vy);
      o1 = vx / (1.0 - ux);
    } else if (type == 2) {  // Green-Lagrangian, E = (C - I) / 2
      o0 = 0.5 * (ux * 2 - ux * ux - vx * vx);
      o3 = 0.5 * (vy * 2 - uy * uy - vy * vy);
      o2 = 0.5 * (uy + vx - ux * uy - vx * vy);
      o1 = 0.5 * (vx + uy - uy * ux - vy * vx);
    }
    out[4 * k] = o0;
    out[4 * k + 1] = o1;
    out[4 * k + 2] = o2;
    out[4 * k + 3] = o3;
  }
}

int plane_fit(int M, int N, double h, int rad, const double *U, double *F, cudaStream_t st) {
  k_plane_fit<<<blocks_for((long long)M * N), 256, 0, st>>>(M, N, h, rad, U, F);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int finite_strain(long long n, int type, const double *F, double *out, cudaStream_t st) {
  k_finite_strain<<<blocks_for(n), 256, 0, st>>>(n, type, F, out);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int fe_store(const GridWork &w, int M, int N, double *Uhat, cudaStream_t st, int f0) {
  const long long n = (long long)M * N;
  k_fe_store<<<blocks_for(n), 256, 0, st>>>(n, w.x + f0 * n, Uhat);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int nodal_strain(int M, int N, double h, const double *U, double *F, cudaStream_t st) {
  const long long n = (long long)M * N;
  k_nodal_strain<<<blocks_for(n), 256, 0, st>>>(M, N, h, U, F);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int gridfit_load(GridWork &w, int M, int N, int nf, const double *vals, int stride,
                 const int *bad_iters, cudaStream_t st, int f0, const double *guess) {
  const long long n = (long long)M * N;
  k_gridfit_load<<<blocks_for(n), 256, 0, st>>>(M, N, nf, vals, stride, bad_iters, guess,
                                                w.b + f0 * n, w.x + f0 * n, w.mask + f0 * n);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int grid_store(const GridWork &w, int M, int N, int nf, double *vals, int stride,
               cudaStream_t st, int f0) {
  const long long n = (long long)M * N;
  k_grid_store<<<blocks_for(n), 256, 0, st>>>(M, N, nf, w.x + f0 * n, vals, stride);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int inpaint_load(GridWork &w, int M, int N, int nf, const double *vals, int stride,
                 const unsigned char *badmask, cudaStream_t st, int f0) {
  const long long n = (long long)M * N;
  k_inpaint_load<<<blocks_for(n), 256, 0, st>>>(M, N, nf, vals, stride, badmask, w.b + f0 * n,
                                                w.x + f0 * n, w.mask + f0 * n);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int inpaint_store(const GridWork &w, int M, int N, int nf, double *vals, int stride,
                  cudaStream_t st, int f0) {
  return grid_store(w, M, N, nf, vals, stride, st, f0);
}

int icgn_flags(int M, int N, const int *iters, unsigned char *badmask, int *d_badnum,
               double *d_meaniters, int *d_nconv, cudaStream_t st, double floor) {
  k_icgn_flags<<<1, 1024, 0, st>>>((long long)M * N, iters, badmask, d_badnum, d_meaniters,
                                   d_nconv, floor);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int subpb1_flags(int n, const int *iters, unsigned char *badmask, int *d_badnum,
                 cudaStream_t st) {
  k_subpb1_flags<<<1, 1024, 0, st>>>(n, iters, badmask, d_badnum);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int nanconv3(GridWork &w, int M, int N, int nf, cudaStream_t st) {
  const long long n = (long long)M * N;
  k_nanconv3<<<blocks_for(n * nf), 256, 0, st>>>(M, N, nf, w.x, w.r);
  ALDIC_CUDA(cudaMemcpyAsync(w.x, w.r, sizeof(double) * n * nf, cudaMemcpyDeviceToDevice, st));
  return OK;
}

int vsub(const double *a, const double *b, double *out, long long n, cudaStream_t st) {
  k_vsub<<<blocks_for(n), 256, 0, st>>>(a, b, out, n);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int sweep_err(int M, int N, int nc, double h, const double *x, const double *U1,
              const double *F1, double *part, int npart, double *err, cudaStream_t st) {
  ALDIC_CHECK(nc >= 1 && nc <= kSweepMax, E_ARG, "sweep_err: 1..6 candidates");
  const long long n = (long long)M * N;
  int nb = npart / (2 * kSweepMax);
  if (nb > 148) nb = 148;
  if ((long long)nb * kSweepThreads > n) nb = (int)((n + kSweepThreads - 1) / kSweepThreads);
  ALDIC_CHECK(nb >= 1, E_ARG, "sweep_err: partials buffer too small");
  k_sweep_err<<<nb, kSweepThreads, 0, st>>>(M, N, nc, h, x, U1, F1, part);
  k_sweep_err_final<<<1, 2 * kSweepMax * 32, 0, st>>>(part, nb, nc, err);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int vsub2(const double *a1, const double *b1, double *o1, long long n1, const double *a2,
          const double *b2, double *o2, long long n2, cudaStream_t st) {
  k_vsub2<<<blocks_for(n1 + n2), 256, 0, st>>>(a1, b1, o1, n1, a2, b2, o2, n2);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int vdiffnorm(const double *a, const double *b, long long n, double *part, double *res,
              cudaStream_t st) {
  const int nb = 148;
  k_diffnorm_part<<<nb, 256, 0, st>>>(const_cast<double *>(a), b, n, part, false);
  k_diffnorm_final<<<1, 256, 0, st>>>(part, nb, res, 1.0);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

int diffnorm_update(double *old, const double *cur, long long n, double *part, double *res,
                    double scale, cudaStream_t st) {
  const int nb = 148;
  k_diffnorm_part<<<nb, 256, 0, st>>>(old, cur, n, part, true);
  k_diffnorm_final<<<1, 256, 0, st>>>(part, nb, res, scale);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

}  // namespace aldic
