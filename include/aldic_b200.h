/*
 * aldic_b200.h -- C ABI of libaldic_b200.so, the B200 (sm_100a) AL-DIC hot path.
 *
 * The entry points replace, one for one, the calls of the reference's frame
 * loop (jyang526843/2D_ALDIC, main_ALDIC.m Sections 2-6) that a MEX gateway
 * would bind.  Each declaration names the reference interface it replaces.
 *
 * Conventions (identical to the reference after ReadImage's transpose):
 *   - an image is W x H, Img(x, y), x = image column, 1-based coordinates,
 *     stored x-fastest (MATLAB's column-major W x H array);
 *   - node order x-fastest; U interleaved [u1 v1 u2 v2 ...]; F per node
 *     [F11 F21 F12 F22]; coords n x 2 column-major ([x1..xn y1..yn]);
 *   - H21 is n x 21 column-major (entry k of node j at k*n + j): the packing
 *     of funICGN.m:320, i.e. HtempPar of LocalICGN.m:46 / HPar of Subpb1.m;
 *   - status codes in iters: 1..100 converged after that many evaluations,
 *     101 not converged / left the image / NaN, 102 more than half the subset
 *     masked, -1 subset outside the valid area (MATLAB's catch branch).
 *
 * Memory: every array argument may point to host memory or to device memory
 * of the context's GPU; the library detects which.  Host arrays are staged
 * through the context's device buffers and the call returns after the copy
 * back; device arrays are used in place and the call is stream-ordered on
 * the context stream (no host synchronisation).  The caller owns all arrays.
 *
 * Errors: every function returns ALDIC_OK (0) or a negative code; the text of
 * the last error of the calling thread is returned by aldic_last_error().
 * No function aborts the process or longjmps across CUDA frames.
 */
#ifndef ALDIC_B200_H
#define ALDIC_B200_H
#include <stdint.h>

#if defined(__GNUC__)
#define ALDIC_API __attribute__((visibility("default")))
#else
#define ALDIC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ALDIC_OK 0
#define ALDIC_E_ARG (-1)
#define ALDIC_E_STATE (-2)
#define ALDIC_E_CUDA (-3)
#define ALDIC_E_TIMEOUT (-4)
#define ALDIC_E_NOMEM (-5)

#define ALDIC_U8 0
#define ALDIC_U16 1
#define ALDIC_F32 2
#define ALDIC_F64 3

#define ALDIC_FP32 0 /* FP32 sampling/residuals, FP64 sums and 6x6 solve */
#define ALDIC_FP64 1 /* FP64 throughout */

typedef struct aldic_ctx aldic_ctx;

ALDIC_API int aldic_version(void);
ALDIC_API const char *aldic_last_error(void);

/* Z = ba_interp2(F, X, Y[, method]) -- ba_interp2.cpp:318-335.
 * F: M x N x P column-major; X indexes columns (N), Y rows (M), 1-based;
 * Z: n x P.  Bit-identical to the reference in both precisions.
 * stream: cudaStream_t (NULL = default stream). */
ALDIC_API int aldic_ba_interp2_f64(const double *F, int64_t M, int64_t N, int64_t P,
                         const double *X, const double *Y, int64_t n, double *Z,
                         void *stream);
ALDIC_API int aldic_ba_interp2_f32(const float *F, int64_t M, int64_t N, int64_t P,
                         const float *X, const float *Y, int64_t n, float *Z,
                         void *stream);

/* Context: device-resident images, gradients and work buffers that persist
 * across calls (the MEX side keeps one per MATLAB session: mexLock/mexAtExit).
 * Its own stream is a blocking stream (ordered with the legacy default
 * stream); callers that produce or consume device arrays on other streams
 * pass their stream with aldic_ctx_set_stream. */
ALDIC_API int aldic_ctx_create(int device, aldic_ctx **out);
ALDIC_API int aldic_ctx_destroy(aldic_ctx *ctx);
ALDIC_API int aldic_ctx_set_stream(aldic_ctx *ctx, void *stream);

/* Reference image: funNormalizeImg.m:1 (ROI mean/std normalisation) and
 * funImgGradient.m:1 (7-tap gradients times the mask, DfCropWidth = 3).
 * roi = {gx1, gx2, gy1, gy2} (gridxyROIRange) or NULL for the whole image;
 * mask: W*H doubles (ImgRefMask) or NULL. */
ALDIC_API int aldic_set_ref(aldic_ctx *ctx, const void *img, int dtype, int W, int H,
                  const int roi[4], const double *mask);
/* Deformed image: funNormalizeImg.m:1 with the reference image's ROI. */
ALDIC_API int aldic_set_def(aldic_ctx *ctx, const void *img, int dtype);
/* funNormalizeImg.m:1 for one image: out = (img - mean_ROI) / std_ROI (W x H
 * doubles); stats receives {mean, std}.  Stateless apart from scratch. */
ALDIC_API int aldic_normalize(aldic_ctx *ctx, const void *img, int dtype, int W, int H,
                              const int roi[4], double *out, double stats[2]);
/* funImgGradient.m:1 for a normalised image f (W x H doubles): dfdx, dfdy are
 * W x H with a zero 3-pixel border (Df.DfDx is the interior), times mask
 * (W x H doubles, or NULL). */
ALDIC_API int aldic_gradient(aldic_ctx *ctx, const double *f, int W, int H, const double *mask,
                             double *dfdx, double *dfdy);

/* Prepared fields as the reference's functions receive them: normalised
 * ImgRef/ImgDef (W x H doubles) and Df.DfDx/Df.DfDy expanded to W x H with a
 * zero 3-pixel border.  Any pointer may be NULL to keep the current field
 * (f, dfdx and dfdy are required on the first call).  The integer search then
 * runs on the normalised doubles (padding value 0). */
ALDIC_API int aldic_set_fields(aldic_ctx *ctx, const double *f, const double *g,
                               const double *dfdx, const double *dfdy, int W, int H);
/* Export the prepared fields (any pointer may be NULL).  dfdx/dfdy are W x H
 * with a zero 3-pixel border: Df.DfDx of the reference is the interior
 * (x, y in [4, W-3] x [4, H-3]).  stats = {mean_f, std_f, mean_g, std_g}. */
ALDIC_API int aldic_get_images(aldic_ctx *ctx, double *f, double *g, double *dfdx,
                     double *dfdy, double stats[4]);

/* Normalisation statistics given from outside instead of the ROI of the
 * images held (funNormalizeImg.m's mean and sample standard deviation of
 * the ROI, {mean_f, std_f, mean_g, std_g}): for a context that holds only a
 * band of the images (a frame split across GPUs), whose ROI statistics are
 * summed over the ranks.  Renormalises both images and the gradients; a
 * later aldic_set_ref/aldic_set_def or aldic_frame takes the statistics from
 * the ROI again. */
ALDIC_API int aldic_set_stats(aldic_ctx *ctx, const double stats[4]);

/* Integer search -- funIntegerSearch.m:3 (whole field, tempNoOfInitPt = 0):
 * grid trimming of :14-25, then per grid point the normalised cross-
 * correlation of the (w+1)^2 template against the (w+1+2s)^2 region and the
 * sub-pixel peak of findpeak.m.  Outputs are ny x nx column-major (MATLAB's
 * x, y, u, v, cc.max); qfactors (n x 2, cc.qfactors) may be NULL to skip.
 * On integer images the correlation maps are exact and the peaks match the
 * project's CPU restatement bit for bit. */
ALDIC_API int aldic_search_dims(int W, int H, const int gridx[2], const int gridy[2],
                      int winsize, int step, const int search[2], int *nx, int *ny);
ALDIC_API int aldic_int_search(aldic_ctx *ctx, const int gridx[2], const int gridy[2],
                     int winsize, int step, const int search[2], double *x,
                     double *y, double *u, double *v, double *ccmax,
                     double *qfactors);

/* Multigrid integer search -- funIntegerSearchMg.m:1, the search that
 * IntegerSearch.m:117-120 runs when DICpara.InitFFTSearchMethod is neither 1
 * nor 2 (large displacements): a whole-ROI normxcorr2 for one global shift,
 * then regions halved level by level (x, y or both by their aspect ratio,
 * while wider than winsize), each searched within +-5 px of its parent's
 * shift, and gridfit 'springs' of the last level onto
 * xList = gridx(1):step:gridx(2), yList likewise, with borders from the
 * extreme regions' displacements (funIntegerSearchMg.m:210-244).
 * The node grid is data dependent: *nx, *ny receive numel(xList),
 * numel(yList); x, y, u, v, ccmax (cc.max) receive nx*ny values each
 * (x fastest: the ny x nx arrays of the reference in row-major order) and
 * qfactors (may be NULL) the two normalised q-factor grids, 2*nx*ny values.
 * cap = capacity of each output in values; (W/step+1)*(H/step+1) always
 * suffices; a smaller cap than nx*ny returns ALDIC_E_ARG with *nx, *ny set.
 * info (may be NULL, else 10 values): {levels, last-level regions, regions
 * whose correlation raised (NaN), level-1 u, level-1 v, level-1 peak, host
 * ms of: tables + level 1, levels 2 .. last-1, last level, gridfit}.  The whole ROI must fit
 * an 8192-point transform per side (ROI <= 4096 px). */
ALDIC_API int aldic_int_search_mg(aldic_ctx *ctx, const int gridx[2], const int gridy[2],
                                  int winsize, int step, int *nx, int *ny, int64_t cap, double *x,
                                  double *y, double *u, double *v, double *ccmax, double *qfactors,
                                  double *info);

/* Local IC-GN -- funICGN.m:1 for every node (the loop of LocalICGN.m:64-81,
 * one launch): 6-DOF affine inverse-compositional Gauss-Newton with the
 * ZNSSD residual.  winsize_arr (n subsets, may be NULL) overrides winsize
 * per subset. */
ALDIC_API int aldic_icgn(aldic_ctx *ctx, const double *coords, int64_t n, const double *U0,
               const int32_t *winsize_arr, int winsize, double tol, int precision,
               double *U, double *F, int32_t *iters, double *H21);

/* LocalICGN.m:114-161: bad subsets (status < 0 or > 99, plus iterations
 * above mean + 0.15 std of the good ones) set to NaN and refilled on the
 * M x N node grid (4-neighbour spring inpainting).  U, F modified in place.
 * bad_num receives LocalICGNBadPtNum. */
ALDIC_API int aldic_localicgn_post(aldic_ctx *ctx, int M, int N, const int32_t *iters,
                         double *U, double *F, int *bad_num);

/* ADMM local step -- funICGN_Subpb1.m:1 for every node (Subpb1.m:64-103):
 * translation-only IC-GN with F fixed at FOld and the augmented-Lagrangian
 * penalty mu (P - UOld - vdual), reusing H(5:6,5:6) from H21. */
ALDIC_API int aldic_subpb1(aldic_ctx *ctx, const double *coords, int64_t n,
                 const double *UOld, const double *FOld, const double *vdual,
                 const double *H21, const int32_t *winsize_arr, int winsize,
                 double mu, double tol, int precision, double *U, int32_t *iters);
/* Subpb1.m:162-199: bad -> NaN, then gridfit 'springs' of u and v. */
ALDIC_API int aldic_subpb1_post(aldic_ctx *ctx, int M, int N, const int32_t *iters, double *U,
                      int *bad_num);

/* ADMM global step -- Subpb2.m:1 on the uniform Q4 mesh of MeshSetUp.m
 * (M x N nodes, spacing step, no Dirichlet/Neumann nodes): the right-hand
 * side of the 3x3 Gauss rule of Subpb2.m:100-149 per node, then the direct
 * solve of beta*DN'DN + mu*N'N (the reference's A\b, Subpb2.m:195) by fast
 * diagonalisation -- the operator is a Kronecker sum of 1-D linear-element
 * stiffness and mass matrices (see aldic_fdm_basis). */
ALDIC_API int aldic_subpb2(aldic_ctx *ctx, int M, int N, double step, double beta, double mu,
                 const double *U, const double *F, const double *udual,
                 const double *vdual, double *Uhat);

/* No counterpart in the reference.  Subproblem 2 as aldic_subpb2, for callers
 * that cannot allocate device memory (a host framework that owns every
 * device byte, a real-time loop that must not stall on an allocation, a
 * process with audited or capped allocations).  All arrays are DEVICE
 * pointers (U 2n, F 4n, udual 4n, vdual 2n in; Uhat 2n out, n = M*N); the
 * solver's work vectors live in one fixed static device array of the library
 * (about 12.7 MB, held on every GPU that loads the library until exit), so at
 * most 65536 nodes are accepted -- larger grids return ALDIC_E_ARG.  The
 * first call on a device looks up that array's device address and keeps it
 * for the process; a cudaDeviceReset
 * of that device invalidates it, so do not call this entry point on a device
 * after resetting it.  The array is shared by every call: calls whose GPU
 * work overlaps (other streams or threads) race.  Every call synchronises
 * the stream before it returns (it reads the solver's status back).  The
 * solve is iterative (PCG to relative residual 1e-11), where aldic_subpb2
 * solves directly.  stream: cudaStream_t. */
ALDIC_API int aldic_subpb2_noalloc(int M, int N, double step, double beta, double mu,
                                   const double *U, const double *F, const double *udual,
                                   const double *vdual, double *Uhat, void *stream);

/* The 1-D eigenbasis behind the direct Subproblem 2 solves (host only, no
 * device work; exposed for testing and for callers that want the basis):
 * type ALDIC_FDM_FE -- the linear-element stiffness K and mass M of n nodes
 * at spacing h (the 1-D factors of Subpb2.m's operator), type ALDIC_FDM_FD --
 * G = d'd with d the 1-D difference of funDerivativeOp.m and M = I.  On
 * return K V = M V diag(lam) and V' M V = I; V is n x n row-major (column p
 * is eigenvector p). */
#define ALDIC_FDM_FE 0
#define ALDIC_FDM_FD 1
ALDIC_API int aldic_fdm_basis(int type, int n, double h, double *V, double *lam);

/* Finite-difference Subproblem 2 (main_ALDIC.m:243-278, funDerivativeOp.m):
 * the interior (M-2) x (N-2) nodes solve (beta D'D + mu I) x = beta D'(F -
 * udual) + mu (U - vdual) with D the central differences of
 * funDerivativeOp.m (one-sided at the interior grid's edges); the border
 * nodes keep U.  Direct solve by fast diagonalisation, as aldic_subpb2. */
ALDIC_API int aldic_subpb2_fd(aldic_ctx *ctx, int M, int N, double step, double beta, double mu,
                              const double *U, const double *F, const double *udual,
                              const double *vdual, double *Uhat);
/* F = funDerivativeOp(M, N, step) * U: [du/dx dv/dx du/dy dv/dy] per node. */
ALDIC_API int aldic_fd_strain(aldic_ctx *ctx, int M, int N, double step, const double *U, double *F);

/* ComputeStrain.m (Section 8 of main_ALDIC.m) on the uniform M x N grid:
 * method 0 the solved F, 1 central differences (funDerivativeOp), 2 plane
 * fitting over a (2 rad + 1)^2 window on the interior (PlaneFit2.m; the
 * border keeps the differences), 3 finite-element nodal strains
 * (funGlobal_NodalStrainAvg); strain_type 0 infinitesimal, 1 Eulerian, 2
 * Green-Lagrangian.  F (4n) is read by method 0 only; strain (4n, may be
 * NULL) receives FStrain, finite (4n) FStrainFinite, both full-grid
 * [F11 F21 F12 F22] slots as the reference fills them. */
ALDIC_API int aldic_compute_strain(aldic_ctx *ctx, int M, int N, double step, int method, int rad,
                                   int strain_type, const double *U, const double *F,
                                   double *strain, double *finite);

/* funGlobal_NodalStrainAvg.m:1 on the uniform mesh (2x2 Gauss points,
 * extrapolation to the nodes, average over elements).  Output slots per node
 * are [du/dx du/dy dv/dx dv/dy], the order funGlobal_NodalStrainAvg.m:97,
 * 123-137 writes them (the middle two are swapped against funICGN's F). */
ALDIC_API int aldic_nodal_strain(aldic_ctx *ctx, int M, int N, double step, const double *U,
                       double *F);

/* gridfit.m (regularizer 'springs', smoothness 1, data on the nodes, NaN =
 * no data) for nf fields of M*N values; out may alias in. */
ALDIC_API int aldic_gridfit_springs(aldic_ctx *ctx, int M, int N, int nf, const double *in,
                          double *out);
/* inpaint_nans.m method 4 for nf fields of M*N values, in place. */
ALDIC_API int aldic_inpaint_springs(aldic_ctx *ctx, int M, int N, int nf, double *z);
/* funSmoothDisp.m / funSmoothStrain.m core: gridfit + 3x3 Gaussian nanconv,
 * twice, on nf interleaved fields (stride nf). */
ALDIC_API int aldic_smooth(aldic_ctx *ctx, int M, int N, int nf, double *vals);

/* ---- Quadtree meshes (func_quadtree/*) ----
 * A mesh object: nodes (n x 2 column-major, like DICmesh.coordinatesFEM),
 * elements (ne x 8 column-major int32, 1-based: corners 1-4, hanging nodes
 * on edges 2-3, 3-4, 4-1, 1-2 in slots 5-8, 0 = none, like
 * DICmesh.elementsFEM) and Dirichlet nodes (DICmesh.dirichlet).  Host data;
 * device copies are made on first use. */
typedef struct aldic_qt_mesh aldic_qt_mesh;
/* GenerateQuadtreeMesh.m:17-115 from the uniform mesh of MeshSetUp.m
 * (coords n0 x 2, elems ne0 x 4): refine elements whose box straddles the
 * edge of mask (ImgRefMask, W x H doubles, Img(x,y) at (y-1)*W + x-1) until
 * their smaller side is at most 2*min_size (QrefineR red refinement,
 * 1-irregular), drop elements less than half inside the mask, mark the
 * Dirichlet nodes (refined elements and the ROI border band, two rings
 * wider).  Host computation. */
ALDIC_API int aldic_qt_mesh_generate(int n0, const double *coords, int ne0, const int32_t *elems,
                                     const double *mask, int W, int H, double step,
                                     int min_size, aldic_qt_mesh **out);
/* A mesh from the reference's own DICmesh arrays. */
ALDIC_API int aldic_qt_mesh_create(int n, const double *coords, int ne, const int32_t *elems,
                                   int ndir, const int32_t *dirichlet, aldic_qt_mesh **out);
ALDIC_API int aldic_qt_mesh_info(const aldic_qt_mesh *m, int *n, int *ne, int *ndir);
ALDIC_API int aldic_qt_mesh_get(const aldic_qt_mesh *m, double *coords, int32_t *elems,
                                int32_t *dirichlet);
ALDIC_API int aldic_qt_mesh_destroy(aldic_qt_mesh *m);
/* Subpb2Quadtree.m:1 with GaussPtOrder 2 and alpha 0: the global step on the
 * quadtree mesh (hanging-node shape functions, Dirichlet nodes keep U, nodes
 * in no element get 0).  The reference multiplies udual and vdual by zero
 * (Subpb2Quadtree.m:60-61), so they are not arguments.  U 2n, F 4n -> Uhat
 * 2n; FP64 PCG to relative residual 1e-11 replaces the direct solve. */
ALDIC_API int aldic_qt_subpb2(aldic_ctx *ctx, aldic_qt_mesh *m, double beta, double mu,
                              const double *U, const double *F, double *Uhat);
/* funGlobalNodalStrainQuadtree.m:1 Gauss-point strains (corners only, as the
 * reference zeroes slots 5-8) extrapolated to the element corners and
 * averaged per node (the reference interpolates them with
 * scatteredInterpolant instead); output slots [du/dx du/dy dv/dx dv/dy]. */
ALDIC_API int aldic_qt_nodal_strain(aldic_ctx *ctx, aldic_qt_mesh *m, const double *U, double *F);
/* Refill of flagged nodes (bad[k] != 0) of nf interleaved fields in place:
 * graph-Laplacian interpolation over the mesh edges with a 1e-6 tether to 0
 * (the reference: scatteredInterpolant 'natural', LocalICGN.m:144-161,
 * Subpb1Quadtree.m:194-199). */
ALDIC_API int aldic_qt_fill(aldic_ctx *ctx, aldic_qt_mesh *m, int nf, double *vals,
                            const uint8_t *bad);

/* One quadtree frame, main_ALDIC_Quadtree.m Sections 3-6, driven from C++
 * with every array on the device: the whole-field integer search on the
 * uniform grid of the ROI, NaN inside the mask's hole (IntegerSearch.m:
 * 68-73), Init's inpainting, the quadtree mesh of GenerateQuadtreeMesh.m
 * (generated on the host; kept and reused while the search grid and the
 * mask are unchanged -- the reference regenerates the same mesh every
 * search frame), U0 interpolated onto its nodes, LocalICGN with the flags
 * and refill, the three-value beta sweep of Subpb2Quadtree + nodal strain
 * with the Dirichlet nodes keeping Subproblem 1's strains, then ADMM steps
 * (Subpb1Quadtree flags with the floor 20 and refill, Subpb2Quadtree) until
 * n_admm steps or an update norm below tol2.  The images come from
 * aldic_set_ref (with the mask ImgRefMask) and aldic_set_def.  *mesh
 * receives the frame's mesh, owned by the context (valid until its next
 * quadtree frame); the results stay on the device for aldic_qt_frame_get.
 * Left out as in the reference's non-interactive use: the outlier clicks
 * of funRemoveOutliersQuadtree and the strain smoothing (regularizeNd). */
typedef struct {
  int winsize, step, search;
  int gridx[2], gridy[2];   /* ROI; {0,0} = whole image */
  double tol, mu, tol2;     /* 1e-2, 1e-3, 1e-2 in main_ALDIC_Quadtree.m */
  int n_admm;               /* ADMM steps after step 1 at most (reference: 3) */
  int min_size;             /* DICmesh.elementMinSize (reference: 2) */
  int precision;            /* ALDIC_FP32 / ALDIC_FP64 */
  int subsets;              /* 0: winsize everywhere (Subpb1Quadtree.m:50);
                               1: twice the node's smallest element side, 16..64 */
} aldic_qt_frame_params;
typedef struct {
  int n, ne, ndir;          /* mesh nodes, elements, Dirichlet nodes */
  int bad_icgn;             /* LocalICGNBadPtNum */
  int admm_steps;
  int mesh_reused;          /* 1: the previous frame's mesh was kept */
  double beta;
  double update_y[16], update_y2[16];
  double t_ms[6];           /* host wall time (ms): search + Init, mesh + U0, LocalICGN + refill,
                               Section 5, ADMM, frame */
} aldic_qt_frame_stats;
ALDIC_API int aldic_qt_frame(aldic_ctx *ctx, const aldic_qt_frame_params *p, aldic_qt_mesh **mesh,
                             aldic_qt_frame_stats *stats);
/* The last quadtree frame's arrays (any pointer may be NULL; host or
 * device): U0 (2n, the interpolated start), U_icgn (2n, LocalICGN after the
 * refill), U (2n) and F (4n) of the last Subproblem 2, iters (n,
 * ConvItPerEle of LocalICGN), wins (n, subset sizes). */
ALDIC_API int aldic_qt_frame_get(aldic_ctx *ctx, double *U0, double *U_icgn, double *U, double *F,
                                 int32_t *iters, int32_t *wins);

/* Bad-subset flags on any node set: status < 0 or > 99, or iterations above
 * max(mean + 0.15 std over the good subsets, floor) -- LocalICGN.m:117-131
 * with floor = NaN, Subpb1Quadtree.m:172-181 with floor = 20.  bad: n bytes;
 * nbad: the reference's bad-point count (status 102 not counted). */
ALDIC_API int aldic_icgn_flags(aldic_ctx *ctx, long long n, const int32_t *iters, double floor,
                               uint8_t *bad, int *nbad);

/* ---- BF16 tensor-core GEMM (the learned initial guess's layers; no
 * counterpart in the reference) ----
 * D[M x N] = A[M x K] . B[N x K]^T in FP32 on the tcgen05 tensor cores.
 * Operands are bf16 device arrays read in one of four ways (mode):
 *   0 rows     (r, k) at p[r * ld + k]
 *   1 patches  im2col of an NHWC tensor [*, Hin, Win, C] with
 *              non-overlapping ps x ps patches (row = output position, column =
 *              (di, dj, c)); ps * C must be a multiple of 8
 *   2 rows read transposed   (r, k) at p[k * ld + r]
 *   3 patches read transposed (r, k) = patch element (k, r)
 * Output: rows (ld) or (mode 1) scattered back into the NHWC tensor a patch
 * operand reads; x (+ bias[n]) (ReLU), zeroed where mask <= 0 (bf16, output
 * layout); FP32 or bf16.  splits > 1 splits K, split s writing its partial
 * product at p + s * split_stride.  Device pointers, 16-byte aligned. */
typedef struct {
  const void *p;
  long long ld;
  int mode;
  long long rows, kdim;
  int Hin, Win, C, ps;
  long long bstride;        /* batches > 1: elements between the products' operands */
} aldic_gemm_operand;
typedef struct {
  void *p;
  long long ld;
  int mode;
  int fp32;
  const float *bias;
  int relu;
  const void *mask;
  int Hin, Win, C, ps;
  long long M, N;
  long long split_stride;
  float scale;              /* x = scale * acc (+ bias); 0 is read as 1 */
  long long bstride;        /* batches > 1: elements between the products' outputs */
} aldic_gemm_output;
/* batches > 1 runs that many independent products (strides bstride). */
ALDIC_API int aldic_gemm_bf16(aldic_ctx *ctx, const aldic_gemm_operand *A,
                              const aldic_gemm_operand *B, const aldic_gemm_output *D, int splits,
                              int batches);

/* ---- Learned initial guess (no counterpart in the reference; its
 * data-driven guess is POD-GPR over earlier frames) ----
 * A Siamese patch network on a reference / deformed 64 x 64 patch pair: a
 * shared encoder (8x8 patch embedding to 128 channels with ReLU, then a
 * linear 1x1 layer to 128), the all-pairs correlation of the two patches'
 * 8 x 8 cell features (64 x 64 / sqrt(128)), a 4096 -> 256 dense layer with
 * ReLU (all bf16 on the tcgen05 GEMM, FP32 accumulation) and a 256 -> 8 FP32
 * output: [u/16, v/16, 20 du/dx, 20 dv/dx, 20 du/dy, 20 dv/dy, confidence
 * logit, 0].  Inputs x: B x 64 x 64 x 2 (channel 0 the reference patch, 1 the
 * deformed one), FP32 (host or device) or bf16 (device).  Parameters:
 * 1 075 720 FP32 values, blocks W1 b1 .. W4 b4, Wl row-major [out x in],
 * W1's inputs in the patch order (dy, dx). */
typedef struct aldic_cnn aldic_cnn;
ALDIC_API int aldic_cnn_create(int device, unsigned long long seed, aldic_cnn **out);
ALDIC_API int aldic_cnn_destroy(aldic_cnn *net);
ALDIC_API long long aldic_cnn_num_params(void);
ALDIC_API int aldic_cnn_get_params(aldic_cnn *net, float *params);
ALDIC_API int aldic_cnn_set_params(aldic_cnn *net, const float *params);
/* One training step on B pairs with targets (B x 6, the first six outputs'
 * scaling): forward, loss (squared error + confidence cross-entropy against
 * "translation within 0.5 px"), backward, and an Adam step when lr > 0.
 * Optional outputs: loss, grads (n_params), out (B x 8). */
ALDIC_API int aldic_cnn_train_step(aldic_cnn *net, const void *x, int x_bf16, const float *targets,
                                   int B, float lr, void *stream, double *loss, float *grads,
                                   float *out);
ALDIC_API int aldic_cnn_predict(aldic_cnn *net, const void *x, int x_bf16, int B, void *stream,
                                float *out);
/* 64 x 64 patch pairs around n nodes (coords n x 2 column-major, 1-based)
 * from the context's normalised images, each patch normalised to zero mean
 * and unit deviation; out: n x 64 x 64 x 2, bf16 (bf16 = 1) or FP32 device
 * array. */
ALDIC_API int aldic_cnn_patches(aldic_ctx *ctx, const double *coords, long long n, int bf16,
                                void *out);
/* U0 (2n), F0 (4n, [F11 F21 F12 F22]) and confidence (n) from network
 * outputs (n x 8); any output may be NULL.  Device arrays. */
ALDIC_API int aldic_cnn_to_init(aldic_ctx *ctx, const float *out, long long n, double *U0,
                                double *F0, float *conf);

/* One frame of main_ALDIC.m Sections 3-6 on the images set on the context:
 * the initial guess (integer search + MeshSetUp/Init, or one of the
 * sequence modes below), LocalICGN and its post-processing, beta selection,
 * Subproblem 2, then n_admm ADMM iterations (Subpb1 + post, Subpb2, nodal
 * strain, dual update).  The device part is recorded once as a CUDA graph
 * and replayed on later calls with the same geometry.
 *
 * Initial guess (main_ALDIC.m:60-151, Section 3 of each frame):
 *   ALDIC_INIT_SEARCH  integer search + Init (NewFFTSearch = 1);
 *   ALDIC_INIT_PREV    U of the previous frame on this context
 *                      (U0 = ResultDisp{ImgSeqNum-2}.U, main_ALDIC.m:131);
 *   ALDIC_INIT_ZERO    zeros (reference-image update, main_ALDIC.m:123);
 *   ALDIC_INIT_EXTRAP  2 U(k-1) - U(k-2) from the last two frames, a
 *                      constant-rate predictor standing in for the POD-GPR
 *                      prediction of main_ALDIC.m:133-146;
 *   ALDIC_INIT_GIVEN   the 2n values set by aldic_set_init;
 *   ALDIC_INIT_GATED   the integer search + Init, then every node whose
 *                      confidence set by aldic_set_init_gated reaches its
 *                      threshold starts IC-GN from the given U0 and F0 instead
 *                      (a learned guess with the search as its fallback);
 *   ALDIC_INIT_SEARCH_MG  the multigrid search (aldic_int_search_mg,
 *                      InitFFTSearchMethod other than 1 and 2) + Init: the
 *                      search decides the node grid, which the frame
 *                      reports in aldic_frame_stats.node_grid; the output
 *                      arrays must then hold (W/step+1)*(H/step+1) nodes.
 * The node grid is the whole-field search grid of the same parameters, or
 * node_grid when its M is set (for the frames after a multigrid-search
 * frame, pass the grid that frame reported).  The context keeps the final U
 * of its last two frames on the device; it is valid while the node grid does
 * not change. */
#define ALDIC_INIT_SEARCH 0
#define ALDIC_INIT_PREV 1
#define ALDIC_INIT_ZERO 2
#define ALDIC_INIT_EXTRAP 3
#define ALDIC_INIT_GIVEN 4
#define ALDIC_INIT_SEARCH_MG 5
#define ALDIC_INIT_GATED 6
typedef struct {
  int winsize, step;
  int search[2];
  int gridx[2], gridy[2];   /* ROI; {0,0} = whole image */
  double tol;               /* IC-GN / Subpb1 tolerance (reference: 1e-2) */
  double mu;                /* 1e-3 */
  double beta;              /* <= 0: tune over betaList (main_ALDIC.m:237) */
  int n_admm;               /* ADMM iterations after step 1 (reference: 4) */
  double tol2;              /* ADMM stop threshold (reference 1e-4); <= 0 off */
  int precision;            /* ALDIC_FP32 or ALDIC_FP64 */
  int smooth;               /* 1: funSmoothDisp/funSmoothStrain as main_ALDIC */
  int use_graph;            /* 1: capture/replay the device work as a CUDA graph */
  int init;                 /* ALDIC_INIT_* */
  int subpb2_fd;            /* 1: finite-difference Subproblem 2 (DICpara.Subpb2FDOrFEM = 1) */
  double node_grid[4];      /* {x, y of the first node, M, N}: an explicit node grid
                               (step apart) for the modes that do not search;
                               M = 0: the whole-field search grid */
} aldic_frame_params;

typedef struct {
  int M, N;                 /* node grid */
  int admm_steps;           /* ADMM iterations run */
  int bad_icgn;             /* LocalICGNBadPtNum of step 1 */
  int converged_icgn;       /* subsets with status 1..100 in step 1 */
  double beta;              /* beta used */
  double update_y[16];      /* ||dU Subpb2|| / sqrt(2n) per ADMM iteration */
  double update_y2[16];     /* ||dU Subpb1|| / sqrt(2n) per ADMM iteration */
  double mean_iters_icgn;   /* mean status over converged subsets */
  int kernel_launches;      /* kernels launched by the frame (graph kernel nodes) */
  /* device time of the frame's stages (CUDA events recorded on the context
   * stream inside the frame, ms): 0 deformed-image normalisation, 1 integer
   * search + Init, 2 IC-GN kernel, 3 LocalICGN post-processing, 4 Section 5
   * (beta, Subpb2, nodal strain), 5 ADMM iterations, 6 whole frame */
  double t_stage_ms[8];
  int max_pcg_iters;        /* most PCG iterations taken by one node-grid solve */
  double node_grid[4];      /* the node grid used: {x, y of the first node, M, N} */
  double t_search_mg_ms;    /* host time of the multigrid search (ALDIC_INIT_SEARCH_MG) */
  int gated_init;           /* ALDIC_INIT_GATED: nodes started from the given guess */
} aldic_frame_stats;

/* Launch-shape autotuner of the IC-GN and Subpb1 kernels (no counterpart
 * in the reference, whose funICGN runs one subset per call): the first
 * launch of a geometry that may synchronise times every launch shape (warps
 * per CTA x register cap, each computing bit-identical results) on its own
 * data and keeps the fastest for the process; aldic_frame runs one eager
 * frame before its first capture of a geometry for that.  enable = 0 turns
 * the trials off (and forgets the choices): the default shape is used. */
ALDIC_API int aldic_icgn_autotune(int enable);
/* The shape chosen for (precision, instance, winsize -- -1 for per-subset
 * sizes --, n subsets): warps per CTA, resident CTAs per SM in the launch
 * bounds, and the trial time of each candidate shape (ms[count], count <= 8).
 * instance (the argument named subpb1): 0 LocalICGN -- in an FP32 frame its
 * iteration launch, which follows a separate setup launch --, 1 Subpb1, 2
 * that LocalICGN setup launch.  ALDIC_E_STATE if that geometry has not been
 * tuned. */
ALDIC_API int aldic_icgn_shape(int precision, int subpb1, int winsize, long long n, int *nwarps,
                               int *minb, float *ms, int *count);

ALDIC_API int aldic_frame_dims(aldic_ctx *ctx, const aldic_frame_params *p, int *M, int *N);
/* Initial guess for ALDIC_INIT_GIVEN: U0 interleaved [u1 v1 u2 v2 ...] on the
 * node grid of aldic_frame_dims (n2 = 2*M*N values, host or device). */
ALDIC_API int aldic_set_init(aldic_ctx *ctx, const double *U0, long long n2);
/* No counterpart in the reference (its data-driven guess is POD-GPR,
 * main_ALDIC.m:133-146): an external initial guess for ALDIC_INIT_GATED
 * frames -- U0 (2n), F0 (4n, [F11 F21 F12 F22] per node; NULL = 0, as
 * funICGN.m:39 starts) and a confidence per node (n floats, NULL = all
 * pass); nodes with conf >= conf_min take (U0, F0) as their IC-GN start,
 * the others the integer search's.  Host or device arrays. */
ALDIC_API int aldic_set_init_gated(aldic_ctx *ctx, const double *U0, const double *F0,
                                   const float *conf, double conf_min, long long n);
ALDIC_API int aldic_frame(aldic_ctx *ctx, const aldic_frame_params *p, double *x0, double *y0,
                double *U, double *F, int32_t *iters, aldic_frame_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
