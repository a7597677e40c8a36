// qt.cuh -- quadtree meshes (func_quadtree/*): the mesh object behind the
// aldic_qt_* entry points, its host-side generation and its device-side
// operators (Subproblem 2 with hanging nodes, nodal strain, refill).
#pragma once
#include <stdint.h>

#include <vector>

#include "aldic_internal.cuh"
#include "kernels.cuh"

// The mesh of GenerateQuadtreeMesh.m: nodes, 8-slot elements (corners 1-4,
// hanging nodes on edges 2-3, 3-4, 4-1, 1-2 in slots 5-8; 1-based, 0 =
// empty) and the Dirichlet nodes of Subpb2Quadtree.m.  Device arrays are
// built on first use on the device of the calling context.
struct aldic_qt_mesh {
  int n = 0, ne = 0;
  std::vector<double> coords;    // n x 2, column-major (x block, y block)
  std::vector<int32_t> elems;    // ne x 8, column-major, 1-based
  std::vector<int32_t> dirichlet;  // sorted, 1-based
  // ---- device side
  int device = -1;
  long long nnz = 0, ninc = 0, nadj = 0;
  aldic::DevBuf d_coords;        // 2n (x block, y block)
  aldic::DevBuf d_elems;         // ne x 8 row-major, 0-based, -1 empty
  aldic::DevBuf d_row, d_col;    // FE operator pattern (node x node)
  aldic::DevBuf d_dpos;          // position of the diagonal in each row
  aldic::DevBuf d_iptr, d_inc, d_ipos;  // node -> (element*8 + slot), scatter map
  aldic::DevBuf d_kind;          // 0 free, 1 Dirichlet, 2 in no element
  aldic::DevBuf d_val, d_diag, d_ke, d_be, d_es;
  aldic::DevBuf d_valM, d_diagM;  // mass part of the operator (the beta sweep's split)
  aldic::DevBuf d_arow, d_acol, d_aval, d_adiag;  // refill graph Laplacian
  aldic::DevBuf slab;            // one allocation; the arrays above are views into it
  void release();
};

namespace aldic {

// GenerateQuadtreeMesh.m:17-115 on the host: refine the uniform mesh where
// element boxes straddle the mask edge (QrefineR red refinement, 1-irregular),
// record hanging nodes, drop elements inside the mask hole, mark the
// Dirichlet nodes.  coords n0 x 2 and elems ne0 x 4 column-major (1-based);
// mask W x H doubles, Img(x, y) at [(y-1) * W + (x-1)].
int qt_generate(int n0, const double *coords, int ne0, const int32_t *elems, const double *mask,
                int W, int H, double step, int min_size, aldic_qt_mesh &out);
int qt_upload(aldic_qt_mesh &m, cudaStream_t st);
// Subpb2Quadtree.m (GaussPtOrder 2, alpha 0): U, F, Uhat device arrays
int qt_subpb2(aldic_qt_mesh &m, GridWork &w, double beta, double mu, const double *U,
              const double *F, double *Uhat, cudaStream_t st);
// funGlobalNodalStrainQuadtree.m Gauss-point strains, averaged to the nodes
int qt_strain(aldic_qt_mesh &m, const double *U, double *F, cudaStream_t st);
// refill of flagged nodes: nf interleaved fields (stride nf) at nodes with
// bad[k] != 0 from the graph Laplacian of the mesh edges
// the beta sweep of Subpb2Quadtree: the three systems (beta[q], mu) in one
// 6-field solve (stiffness and mass parts assembled apart), candidate q in
// solver fields 2q, 2q + 1; qt_store_candidate interleaves candidate q
int qt_subpb2_sweep(aldic_qt_mesh &m, GridWork &w, const double beta[3], double mu,
                    const double *U, const double *F, cudaStream_t st);
int qt_store_candidate(aldic_qt_mesh &m, const GridWork &w, int q, double *Uhat, cudaStream_t st);
int qt_fill(aldic_qt_mesh &m, GridWork &w, int nf, double *vals, const unsigned char *bad,
            cudaStream_t st);
// the same for two interleaved arrays (nf1 + nf2 <= 6 fields) in one solve
int qt_fill2(aldic_qt_mesh &m, GridWork &w, int nf1, double *vals1, int nf2, double *vals2,
             const unsigned char *bad, cudaStream_t st);

constexpr double kQtFillTether = 1e-6;

}  // namespace aldic
