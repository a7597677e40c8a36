/*
 * aldic_oracle.h -- CPU FP64 restatement of the AL-DIC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm load it.  The product library (libaldic_b200.so) never links or calls it.
 *
 * Parity status: the bicubic sampler (orc_ba_interp2_*) is pinned bit-exactly
 * against the reference's own ba_interp2.cpp compiled under oracle/_ref.  The
 * rest follows the reference MATLAB line by line (citations per function) but
 * MATLAB/Octave cannot run here, so those parts are "parity unpinned" against
 * the reference itself; they are pinned only by known-answer tests written from
 * the algorithms' definitions (see tests/test_oracle_*.py).
 *
 * Conventions (same as the reference after ReadImage's transpose):
 *   images are W x H with Img(x,y), x = image column, 1-based; stored with x
 *   fastest (element (x,y) at (y-1)*W + (x-1)), i.e. a C row-major [y][x] array;
 *   node order x-fastest; U interleaved [u1 v1 u2 v2 ...]; F per node
 *   [F11 F21 F12 F22]; H21 stored as n x 21 column-major (entry k of node j at
 *   k*n + j), the packing order of funICGN.m:320.
 */
#ifndef ALDIC_ORACLE_H
#define ALDIC_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- a3: bicubic (Keys a=-1/2) sampling, ba_interp2.cpp:60-182 ---- */
void orc_ba_interp2_f64(const double *F, int64_t M, int64_t N, int64_t P,
                        const double *X, const double *Y, int64_t n, double *out);
void orc_ba_interp2_f32(const float *F, int64_t M, int64_t N, int64_t P,
                        const float *X, const float *Y, int64_t n, float *out);

/* ---- a1: funNormalizeImg.m:22-39.  dtype 0=u8 1=u16 2=f32 3=f64.
 * roi = {gx1, gx2, gy1, gy2} (1-based inclusive; clamped as :25-28).
 * Writes the normalised image and returns mean/std of the ROI. ---- */
int orc_normalize(const void *img, int dtype, int W, int H, const int roi[4],
                  double *out, double *mean, double *stdev);

/* ---- a2: funImgGradient.m:53-78.  Full-size W x H outputs, zero in the
 * 3-pixel border; interior = 7-tap central difference times mask. ---- */
void orc_gradient(const double *f, const double *mask, int W, int H,
                  double *dfdx, double *dfdy);

/* ---- a4/a5: funIntegerSearch.m:3-203 + findpeak.m + compute_qFactor ----
 * Grid trimming as funIntegerSearch.m:14-25; XList/YList as :90-91.
 * orc_search_dims returns nx = numel(XList), ny = numel(YList) and the trimmed
 * first grid coordinates. */
int orc_search_dims(int W, int H, const int gridx[2], const int gridy[2],
                    int winsize, int step, const int search[2],
                    int *nx, int *ny, int *x_first, int *y_first);
/* f_raw, g_raw: raw images (dtype as above) -- the NCC is affine-invariant, so
 * it is evaluated on raw values with the outside-D padding set to mu_g (the
 * value that maps to 0 after normalisation).  Outputs are ny x nx column-major
 * arrays (MATLAB layout of x,y,u,v,cc.max), qfac is n x 2 column-major (may be
 * NULL to skip the q-factors). */
int orc_int_search(const void *f_raw, const void *g_raw, int dtype, int W, int H,
                   double mu_g, const int gridx[2], const int gridy[2],
                   int winsize, int step, const int search[2],
                   double *x, double *y, double *u, double *v, double *ccmax,
                   double *qfac);

/* ---- a6: MeshSetUp.m:23-39 (uniform Q4 mesh) ---- */
void orc_mesh(int M, int N, const double *xlist, const double *ylist,
              double *coords /* n x 2 col-major */, int32_t *elems /* ne x 4 col-major, 1-based */);

/* ---- a7: funICGN.m (per subset) and a8 LocalICGN.m:64-81 batch ----
 * coords n x 2 column-major; U0 2n; winsize per subset (or NULL -> w);
 * g: normalised deformed image; f: normalised reference; dfdx/dfdy full size.
 * iters: 1..100 converged, 101 not converged, 102 masked, -1 error. */
void orc_icgn_batch(const double *f, const double *g, const double *dfdx,
                    const double *dfdy, int W, int H, const double *coords,
                    int64_t n, const double *U0, const int32_t *winsize_arr,
                    int winsize, double tol, double *U, double *F,
                    int32_t *iters, double *H21);

/* ---- a9: funICGN_Subpb1.m (per subset) batch, Subpb1.m:64-103 ---- */
void orc_subpb1_batch(const double *f, const double *g, const double *dfdx,
                      const double *dfdy, int W, int H, const double *coords,
                      int64_t n, const double *UOld, const double *FOld,
                      const double *vdual, const double *H21,
                      const int32_t *winsize_arr, int winsize, double mu,
                      double tol, double *U, int32_t *iters);

/* ---- LocalICGN.m:114-161 post-processing.  bad = iters<0 | iters>99, then
 * the 0.15-sigma iteration flag (:128-131); flagged nodes are refilled by the
 * 4-neighbour spring inpainting of inpaint_nans(.,4) on the M x N node grid
 * (documented stand-in for scatteredInterpolant 'natural').  Returns the
 * LocalICGNBadPtNum of :122.  U (2n) and F (4n) are modified in place. ---- */
int orc_localicgn_post(int M, int N, const int32_t *iters, double *U, double *F);

/* ---- Subpb1.m:162-199: bad -> NaN, then gridfit 'springs' of u and v ---- */
int orc_subpb1_post(int M, int N, const int32_t *iters, double *U);

/* ---- gridfit.m 'springs', smoothness 1, data on the node grid (NaN = no
 * data).  nf fields of length M*N (x fastest); out may alias in. ---- */
int orc_gridfit_springs(int M, int N, int nf, const double *in, double *out);

/* ---- inpaint_nans.m method 4 on an M x N grid (x fastest) ---- */
int orc_inpaint_springs(int M, int N, double *z);

/* ---- a10: Subpb2.m:72-195 on the uniform mesh (no Dirichlet/Neumann) ----
 * Assembles the FE system exactly as the element loop does and solves it by
 * FP64 CG to a relative residual of 1e-13.  Returns CG iterations. */
int orc_subpb2(int M, int N, double step, double beta, double mu,
               const double *U, const double *F, const double *udual,
               const double *vdual, double *Uhat);

/* ---- a11: funGlobal_NodalStrainAvg.m:32-144 on the uniform mesh ---- */
void orc_nodal_strain(int M, int N, double step, const double *U, double *Fout);

/* ---- a14: funSmoothDisp.m / funSmoothStrain.m core (gridfit + nanconv of a
 * 3x3 sigma-0.5 Gaussian, twice) on nf fields interleaved with stride nf ---- */
int orc_smooth_fields(int M, int N, int nf, double *vals);

/* ---- a12: ADMM core of main_ALDIC.m:166-451 for one frame ---- */
typedef struct {
  int winsize, step, search[2];
  int gridx[2], gridy[2];
  double tol;          /* IC-GN / Subpb1 tolerance */
  double mu;           /* 1e-3 */
  double beta;         /* <= 0: tune over betaList (main_ALDIC.m:237,285-301) */
  int n_admm;          /* ADMM iterations after step 1 (reference: 4) */
  double tol2;         /* ADMM stop (main_ALDIC.m:354); <= 0 disables */
  int smooth;          /* 1: funSmoothDisp/funSmoothStrain as main_ALDIC.m */
  const double *init_U; /* NULL: integer search + Init; else U0 (2n) of a later
                           frame of a sequence (main_ALDIC.m:118-147) on the
                           same node grid */
} orc_frame_params;

typedef struct {
  int M, N;
  double *x0, *y0;     /* M*N node coordinates */
  double *U, *F;       /* final USubpb2 (2n) and FSubpb2 (4n) */
  double *U_icgn, *F_icgn; /* step-1 LocalICGN output after post-processing */
  int32_t *iters_icgn; /* n */
  double beta;         /* beta used */
  int admm_steps;      /* ADMM iterations performed */
  double update_y[16], update_y2[16];
  double t_search, t_icgn, t_subpb1, t_subpb2, t_total; /* seconds */
} orc_frame_result;

int orc_frame(const void *f_raw, const void *g_raw, int dtype, int W, int H,
              const orc_frame_params *p, orc_frame_result *r);
void orc_frame_free(orc_frame_result *r);

/* Multigrid search primitives (func/funIntegerSearchMg.m).  orc_ncc_map:
 * normxcorr2(C, D) for C = f(trect[0]:trect[1], trect[2]:trect[3]) and
 * D = g(drect[0]:drect[1], drect[2]:drect[3]) (1-based, inclusive, inside the
 * W x H image), at the 0-based D offsets [ox0, ox1] x [oy0, oy1] of C's first
 * pixel; out is column-major with rows = x offsets.  D is padded with mu_g
 * (zero in normalised units).  Returns 1 for a constant template (normxcorr2
 * raises), -1 for a bad rectangle, else 0.  orc_findpeak: findpeak.m on an
 * nr x nc column-major map -> (row, col, max_f), 1-based.  orc_qfactor:
 * compute_qFactor -> (PCE, 1/entropy). */
int orc_ncc_map(const void *f_raw, const void *g_raw, int dtype, int W, int H, double mu_g,
                const int trect[4], const int drect[4], int ox0, int ox1, int oy0, int oy1,
                double *out);
void orc_findpeak(const double *map, int nr, int nc, double out[3]);
void orc_qfactor(const double *cc, int n, double out[2]);

/* thread count used by OpenMP regions (0 = default) */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
