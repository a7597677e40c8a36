// kernels.cuh -- launchers of the sm_100a kernels (called by capi.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace aldic {

// ---- k_image.cu
int roi_stats(const void *img, int dtype, int W, const int roi[4], double *d_stats,
              unsigned long long *d_isums, double *d_part, cudaStream_t st);
int normalize(const void *img, int dtype, long long n, const double *d_stats, double *o64,
              float *o32, cudaStream_t st);
int gradient(const double *f, const double *mask, int W, int H, double *gx64, double *gy64,
             float *gx32, float *gy32, cudaStream_t st);
// row-cubic coefficients of the FP64 image g: W H float4, q[y W + x] =
// (a0, a1, a2, a3) of row y's Keys cubic on floor column x
int row_cubic(const double *g, int W, int H, float4 *q, cudaStream_t st);
// q[i] = (gx[i], gy[i]), n float2
int grad_pairs(const float *gx, const float *gy, long long n, float2 *q, cudaStream_t st);
int interp_f64(const double *F, long long M, long long N, long long P, const double *X,
               const double *Y, long long n, double *Z, cudaStream_t st);
int interp_f32(const float *F, long long M, long long N, long long P, const float *X,
               const float *Y, long long n, float *Z, cudaStream_t st);

// ---- k_search.cu
// work of the tiled 8-bit search: the window table of the deformed image, the
// list of points handed to the per-point kernel and the correlation maps
struct SearchWork {
  DevBuf buf;
  DevBuf big;  // per-CTA row sums and maps of search regions too large for shared memory
  void release() {
    buf.release();
    big.release();
  }
};
// work memory of a search geometry (with winsize > 0 and the image dtype also
// the big-region slots), allocated ahead of any stream capture
int search_work_ensure(SearchWork &w, int W, int H, int nx, int ny, const int search[2],
                       int winsize = 0, int dtype = -1);
int search_dims(int W, int H, const int gridx[2], const int gridy[2], int winsize, int step,
                const int search[2], int *nx, int *ny, int *gx1, int *gy1);
int int_search(const void *f_raw, const void *g_raw, int dtype, int W, int H, const double *mu_g,
               const int gridx[2], const int gridy[2], int winsize, int step,
               const int search[2], double *x, double *y, double *u, double *v, double *cc,
               double *pce, double *ppe, cudaStream_t st, SearchWork *sw = nullptr);

// ---- k_icgn.cu
// doubles per subset of the IC-GN setup record (the cache argument of icgn
// and subpb1): [mean f, bf, S_f5, S_f6, S_5, S_6, w, status], then S_f0..3,
// S_0..3, the Cholesky factor of H (21), 1 / diag (6), SPD flag
constexpr int kIcgnCache = 44;
struct IcgnImages {
  const float *f32, *g32, *gx32, *gy32;
  const float4 *gc;   // row-cubic coefficients of g (row_cubic): the FP32 sampler's
  const float2 *gxy;  // (gx32, gy32) pairs (grad_pairs) read by the FP32 IC-GN
  const double *f64, *g64, *gx64, *gy64;
  int W, H;
};
int icgn(const IcgnImages &im, const double *coords, long long n, const double *U0,
         const int *wins, int w, double tol, int precision, double *U, double *F, int *iters,
         double *H21, unsigned int *queue, cudaStream_t st, double *cache = nullptr,
         const double *F0 = nullptr);
// launch-shape autotuner of the IC-GN / Subpb1 kernels (k_icgn.cu)
bool icgn_tuned(int precision, bool sub, int w, long long n);
void icgn_autotune(bool on);
// instance 0 LocalICGN (its iteration launch when the setup runs apart), 1
// Subpb1, 2 the LocalICGN setup launch
int icgn_tuned_shape(int precision, int instance, int w, long long n, int *nwarps, int *minb,
                     float ms[8], int *count);
int subpb1(const IcgnImages &im, const double *coords, long long n, const double *UOld,
           const double *FOld, const double *vdual, const double *H21, const int *wins, int w,
           double mu, double tol, int precision, double *U, int *iters, unsigned int *queue,
           cudaStream_t st, const double *cache = nullptr);

// ---- k_grid.cu: node-grid solvers and field kernels on the M x N mesh
struct GridWork {
  // PCG vectors for up to 12 right-hand sides of M*N (x fastest) each; p is
  // two vectors (the second 12*M*N after the first)
  double *x, *r, *z, *p, *q, *b, *diag;
  double *zz, *qq, *ss, *pp;  // pipelined-CG directions
  double *part;          // per-block partial sums: 2 buffers of [4][nrhs][blocks]
  unsigned char *mask;   // per node flags (data present / unknown)
  unsigned int *bar;     // grid barrier {count, gen}
  int *err;              // barrier / solver error flag
  int *iters_out;        // PCG iterations used
  int max_blocks;
};
enum GridOp { OP_FE = 0, OP_GRIDFIT = 1, OP_INPAINT = 2, OP_CSR = 3, OP_FD = 4 };

// ---- fdm.cu: direct Subproblem 2 solves on the uniform node grid by fast
// diagonalisation (the FE and FD operators are Kronecker sums of 1-D ones)
enum { FDM_FE = 0, FDM_FD = 1 };
struct FdmBasis {
  int type = -1, M = 0, N = 0;
  double h = 0.0;
  DevBuf buf;  // Vx (M x M), Vy (N x N), lx (M), ly (N), split-K partials (kFdmPart M N)
  double *Vx = nullptr, *Vy = nullptr, *lx = nullptr, *ly = nullptr, *part = nullptr;
  void release() {
    buf.release();
    type = -1;
  }
};
// 1-D eigenbasis (row-major V, column p = eigenvector p, V' M V = I) and
// eigenvalues of the FE (stiffness, mass) or FD (d'd, I) pencil of n nodes
int fdm_basis_1d(int type, int n, double h, double *V, double *lam);
// the bases of an M x N grid on the device (host work once per geometry;
// synchronises the stream, so never inside a capture)
int fdm_ensure(FdmBasis &B, int type, int M, int N, double h, cudaStream_t st);
// x_f = A_f^-1 b_f for the nrhs fields of M*N values (x fastest) at b, x;
// A_f = beta_f (Kx (+) Ky) + mu Mx (x) My with beta_f = *beta_ptr if given,
// else beta_each[f] if given, else beta; tmp: nrhs*M*N doubles
int fdm_solve(const FdmBasis &B, int nrhs, const double *b, double *x, double *tmp, double mu,
              double beta, const double *beta_each, const double *beta_ptr, cudaStream_t st);
// the beta sweep's six systems at once from the two right-hand-side parts
// (b fields 0-1: beta part, 2-3: mu part): x fields 2q, 2q + 1 solve
// (beta[q] K + mu M) x = beta[q] b_beta + mu b_mu; tmp holds 12 fields
int fdm_solve_sweep(const FdmBasis &B, const double beta[6], const double *b, double *x,
                    double *tmp, double mu, cudaStream_t st);

// Finite-difference Subproblem 2 (funDerivativeOp.m, main_ALDIC.m:243-278):
// (beta D'D + mu I) x = beta D' a + mu b on the interior (M-2) x (N-2) nodes,
// D central differences with the reference's one-sided borders.
int fd_rhs(GridWork &w, int M, int N, double h, double beta, double mu, const double *U,
           const double *F, const double *udual, const double *vdual, cudaStream_t st,
           const double *beta_ptr = nullptr, int f0 = 0);
// U2 = U1 with the interior replaced by the solution of fields f0, f0 + 1
int fd_store(const GridWork &w, int M, int N, const double *U1, double *U2, cudaStream_t st,
             int f0 = 0);
// F = D2 U on the full M x N grid, slots [du/dx dv/dx du/dy dv/dy]
int fd_strain(int M, int N, double h, const double *U, double *F, cudaStream_t st);
// FD dual update on the interior nodes (main_ALDIC.m:334-338, 434-438):
// reset (accumulate = 0: zero elsewhere) or accumulate
int fd_dual(int M, int N, const double *F2, const double *F1, const double *U2, const double *U1,
            double *udual, double *vdual, int accumulate, cudaStream_t st);
// ComputeStrain.m: plane-fit gradients on the interior (PlaneFit2.m, window
// (2 rad + 1)^2) written over F; finite-strain conversion of F (type 1
// Eulerian, 2 Green-Lagrangian) into out
int plane_fit(int M, int N, double h, int rad, const double *U, double *F, cudaStream_t st);
int finite_strain(long long n, int type, const double *F, double *out, cudaStream_t st);

// A symmetric sparse operator for the PCG: CSR rows of n nodes (sorted
// columns), its diagonal, shared by every field.  Rows whose field mask is 0
// are identity rows; columns whose mask is 0 are skipped (their values were
// moved to the right-hand side).
// A CSR operator; with valM / diagM set, field f's matrix is
// beta[f] val + mu valM (a stiffness and a mass part on one pattern)
struct CsrOp {
  const int *row, *col;
  const double *val, *diag;
  const double *valM = nullptr, *diagM = nullptr;
};
int csr_pcg(GridWork &w, const CsrOp &op, long long n, int nrhs, double rtol, int maxit,
            cudaStream_t st, const double *beta_each = nullptr, double mu = 0.0);

// ---- BF16 tensor-core GEMM (k_gemm.cu): D = A . B^T over K
enum GemmMode { GEMM_ROW = 0, GEMM_PATCH = 1, GEMM_TRANS = 2, GEMM_PATCHT = 3 };
// An operand of `rows` x `kdim` bf16 values read from p:
//   ROW    (r, k) at p[r * ld + k]
//   PATCH  (r, k) = im2col of an NHWC tensor [*, Hin, Win, C] with
//          non-overlapping ps x ps patches: r = (b, i, j) output position,
//          k = (di, dj, c) in that order
//   TRANS  (r, k) at p[k * ld + r]          (a ROW source read transposed)
//   PATCHT (r, k) = PATCH element (k, r)    (im2col read transposed)
struct GemmSrc {
  const __nv_bfloat16 *p;
  long long ld;
  int mode;
  long long rows, kdim;
  int Hin, Win, C, ps;
  long long bstride = 0;   // elements between the operands of a batch of products
};
// Output: ROW (m, n) at p[m * ld + n], or PATCH scatter of (m, n) into the
// NHWC tensor the PATCH operand reads; x = acc (+ bias[n]) (ReLU) and zeroed
// where mask (same layout as the output, bf16) is not positive.
struct GemmDst {
  void *p;
  long long ld;
  int mode;
  int fp32;
  const float *bias;
  int relu;
  const __nv_bfloat16 *mask;
  int Hin, Win, C, ps;
  long long M, N;
  long long split_stride;  // elements between the partial products of split-K
  float scale = 1.f;       // x = scale * acc (+ bias ...)
  long long bstride = 0;   // elements between the outputs of a batch of products
};
// splits > 1: split-K; batches > 1: independent products (operand and output
// strides bstride), one per grid z
int gemm_bf16(const GemmSrc &A, const GemmSrc &B, const GemmDst &D, int splits, int *err,
              cudaStream_t st, int batches = 1);
// learned initial guess (cnn.cu)
int cnn_patches(const float *f, const float *g, int W, int H, const double *coords, long long n,
                void *bf16_out, float *f32_out, cudaStream_t st);
int cnn_to_init(const float *out, long long n, double *U0, double *F0, float *conf, cudaStream_t st);

// solve op(x) = b for nrhs fields; b and x live in w.b / w.x (field-major)
// ata (OP_GRIDFIT only, may be NULL): scattered-data A'A as 9 coefficients per
// node (offsets (di, dj) in row-major 3 x 3 order); the mask is then unused
int grid_pcg(GridWork &w, int op, int M, int N, int nrhs, double beta, double mu, double h,
             double lam2, double rtol, int maxit, cudaStream_t st,
             const double *beta_ptr = nullptr, const double *beta_each = nullptr,
             const double *ata = nullptr);
// Subpb2 right-hand side (Subpb2.m:76-159) into w.b (2 fields: u, v)
int fe_rhs(GridWork &w, int M, int N, double h, double beta, double mu, const double *U,
           const double *F, const double *udual, const double *vdual, cudaStream_t st,
           const double *beta_ptr = nullptr, int f0 = 0);
// the two parts of the Subpb2 right-hand side, linear in beta and mu: the
// beta part into fields 0-1, the mu part into 2-3 (for the beta sweep)
int fe_rhs_parts(GridWork &w, int M, int N, double h, const double *U, const double *F,
                 const double *udual, const double *vdual, cudaStream_t st);
// interleave w.x (2 fields from slot f0) into Uhat
int fe_store(const GridWork &w, int M, int N, double *Uhat, cudaStream_t st, int f0 = 0);
// nodal strain (funGlobal_NodalStrainAvg.m)
int nodal_strain(int M, int N, double h, const double *U, double *F, cudaStream_t st);
// gridfit springs: load nf interleaved (stride, offset) fields, NaN = no data;
// the solve starts from the data and, at nodes without data, from guess (the
// same layout as vals; 0 where null) -- the solution does not depend on it
int gridfit_load(GridWork &w, int M, int N, int nf, const double *vals, int stride,
                 const int *bad_iters, cudaStream_t st, int f0 = 0,
                 const double *guess = nullptr);
int grid_store(const GridWork &w, int M, int N, int nf, double *vals, int stride,
               cudaStream_t st, int f0 = 0);
// inpaint springs: load nf fields, nodes flagged (NaN or bad) are unknown
int inpaint_load(GridWork &w, int M, int N, int nf, const double *vals, int stride,
                 const unsigned char *badmask, cudaStream_t st, int f0 = 0);
int inpaint_store(const GridWork &w, int M, int N, int nf, double *vals, int stride,
                  cudaStream_t st, int f0 = 0);
// LocalICGN.m:117-131 flags; writes badmask and the bad count to d_badnum
int icgn_flags(int M, int N, const int *iters, unsigned char *badmask, int *d_badnum,
               double *d_meaniters, int *d_nconv, cudaStream_t st, double floor = __builtin_nan(""));
// Subpb1.m:167-169 flags
int subpb1_flags(int n, const int *iters, unsigned char *badmask, int *d_badnum,
                 cudaStream_t st);
// 3x3 Gaussian nanconv with edge normalisation on nf fields (in w.x)
int nanconv3(GridWork &w, int M, int N, int nf, cudaStream_t st);
// out = a - b (n elements)
int vsub(const double *a, const double *b, double *out, long long n, cudaStream_t st);
// o1 = a1 - b1, o2 = a2 - b2 in one launch
int vsub2(const double *a1, const double *b1, double *o1, long long n1, const double *a2,
          const double *b2, double *o2, long long n2, cudaStream_t st);
// ||a - b||_2 into *res (deterministic)
// the beta sweep's errors |U1 - U2_c| -> err[c], |F1 - F2_c| -> err[6 + c] for
// the nc <= 6 FE candidates in fields (2c, 2c + 1) of x; part holds npart doubles
int sweep_err(int M, int N, int nc, double h, const double *x, const double *U1,
              const double *F1, double *part, int npart, double *err, cudaStream_t st);
int vdiffnorm(const double *a, const double *b, long long n, double *part, double *res,
              cudaStream_t st);
// res = |old - cur| * scale (part: 148 doubles), and old <- cur in the same pass
int diffnorm_update(double *old, const double *cur, long long n, double *part, double *res,
                    double scale, cudaStream_t st);

// ---- multigrid integer search (k_searchmg.cu, funIntegerSearchMg.m)
struct MgWork {
  DevBuf sat, tot;         // summed-area tables of f, f^2, g, g^2 and column-chunk totals
  DevBuf fft, tw, part;    // level-1 transforms, twiddles, argmax partials
  DevBuf regs, acc, res;   // per-level region descriptors, crop products, results
  DevBuf csr;              // gridfit normal equations
  void release() {
    for (DevBuf *b : {&sat, &tot, &fft, &tw, &part, &regs, &acc, &res, &csr}) b->release();
  }
};
// last level of the search: region centres and their results (NaN where the
// correlation raised; Phi 0 there), normalised q-factors, the trimmed ROI
struct MgData {
  std::vector<double> tx, ty, u, v, phi, q1, q2;
  int gridx[2] = {0, 0}, gridy[2] = {0, 0};
  int levels = 0, failed = 0;
  double l1_u = 0, l1_v = 0, l1_cc = 0;  // level-1 (whole ROI) shift and peak
  double t_ms[4] = {0, 0, 0, 0};         // host time: tables + level 1, levels 2.., last level, fit
};
struct MgGrid {
  double x0 = 0, y0 = 0;  // first node (xList(1), yList(1))
  int nx = 0, ny = 0, step = 1;
};
// qfactors: compute the last level's full maps and compute_qFactor (else
// only the 13 x 14 crops, q1/q2 NaN)
int search_mg_levels(MgWork &w, const void *f, const void *g, int dtype, int W, int H,
                     const double *mu_g, const int gridx[2], const int gridy[2], int winsize,
                     bool qfactors, MgData &out, cudaStream_t st);
bool search_mg_grid(const MgData &d, int winsize, int step, int W, int H, MgGrid &grid);
// out: the first nfields of (u v Phi q1 q2), nx*ny values each, x fastest;
// gw sized for nx*ny
int search_mg_fit(GridWork &gw, MgWork &w, MgData &d, const MgGrid &grid, int nfields,
                  double *out, cudaStream_t st);

}  // namespace aldic
