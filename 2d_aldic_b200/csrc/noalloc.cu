// noalloc.cu -- Subproblem 2 for callers that cannot allocate device memory.
//
// Some hosts of this library must not call cudaMalloc at all: code running
// inside another framework's memory pool (which owns every device byte and
// forbids side allocations), real-time loops where an allocation's implicit
// device synchronisation would break the frame budget, and processes whose
// allocations are audited or capped.  aldic_subpb2_noalloc serves them: the
// caller passes device inputs and the device output, and the PCG work
// vectors live in one file-scope static __device__ array of a fixed maximum
// size, loaded with the library and held on every GPU that loads it until
// the process exits.  No cudaMalloc, cudaFree or allocating library call is
// made.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/aldic_b200.h"
#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {
namespace {

// 2 displacement fields x 12 PCG vectors per node, for at most this many nodes
constexpr long long kNoAllocMaxNodes = 65536;  // e.g. a 256 x 256 node grid
constexpr int kNoAllocMaxBlocks = 192;         // cooperative grid: one block per SM
constexpr long long kVecDoubles = 12 * 2 * kNoAllocMaxNodes;
// two buffers of block partials, laid out for up to 12 right-hand sides
constexpr long long kPartDoubles = 2 * 4 * 12 * kNoAllocMaxBlocks;

struct NoAllocScratch {
  double vec[kVecDoubles];
  double part[kPartDoubles];
  unsigned char mask[2 * kNoAllocMaxNodes];
  unsigned int ctl[16];  // barrier count/generation, error flag, iteration count
};

// The scratch (~12.7 MB).  Host code must not use &g_scratch as a device
// address: it is a host-side stand-in; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) NoAllocScratch g_scratch;

std::mutex g_mu;
NoAllocScratch *g_dev_ptr[64] = {};

// Once per device, with that device current.
int scratch_address(int dev, NoAllocScratch **out) {
  if (dev < 0 || dev >= 64) {
    set_error("subpb2_noalloc: device index out of range");
    return E_ARG;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_dev_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("subpb2_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return E_CUDA;
    }
    g_dev_ptr[dev] = (NoAllocScratch *)p;
  }
  *out = g_dev_ptr[dev];
  return OK;
}

}  // namespace
}  // namespace aldic

using namespace aldic;

extern "C" int aldic_subpb2_noalloc(int M, int N, double step, double beta, double mu,
                                    const double *U, const double *F, const double *udual,
                                    const double *vdual, double *Uhat, void *stream) {
  ALDIC_CHECK(U && F && udual && vdual && Uhat && M > 1 && N > 1 && step > 0, E_ARG,
              "subpb2_noalloc: bad arguments");
  const long long n = (long long)M * N;
  ALDIC_CHECK(n <= kNoAllocMaxNodes, E_ARG,
              "subpb2_noalloc: M*N exceeds the fixed scratch of 65536 nodes; use aldic_subpb2");
  int dev = 0;
  ALDIC_CUDA(cudaGetDevice(&dev));
  NoAllocScratch *S = nullptr;
  int rc = scratch_address(dev, &S);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // PCG vectors for two right-hand sides, 2n values each, packed for this n.
  // grid_pcg keeps its second m buffer 12n after the first, so p0 sits at
  // 0, p1 at 12n, five vectors fill the gap and the rest follow.
  double *v = S->vec;
  GridWork w{};
  w.p = v;
  w.x = v + 2 * n;
  w.r = v + 4 * n;
  w.z = v + 6 * n;
  w.q = v + 8 * n;
  w.b = v + 10 * n;
  w.diag = v + 14 * n;
  w.zz = v + 16 * n;
  w.qq = v + 18 * n;
  w.ss = v + 20 * n;
  w.pp = v + 22 * n;
  w.part = S->part;
  w.mask = S->mask;
  w.bar = S->ctl;
  w.err = (int *)(S->ctl + 2);
  w.iters_out = (int *)(S->ctl + 3);
  w.max_blocks = kNoAllocMaxBlocks;
  // the shared array keeps the previous call's contents: zero the control words
  ALDIC_CUDA(cudaMemsetAsync(S->ctl, 0, sizeof(S->ctl), st));
  if ((rc = fe_rhs(w, M, N, step, beta, mu, U, F, udual, vdual, st))) return rc;
  if ((rc = grid_pcg(w, OP_FE, M, N, 2, beta, mu, step, 0, 1e-11, 4000, st))) return rc;
  if ((rc = fe_store(w, M, N, Uhat, st))) return rc;
  int err = 0;
  ALDIC_CUDA(cudaMemcpyAsync(&err, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  ALDIC_CUDA(cudaStreamSynchronize(st));
  if (err == 1) {
    set_error("subpb2_noalloc: barrier wait timed out");
    return E_TIMEOUT;
  }
  if (err == 2) {
    set_error("subpb2_noalloc: PCG did not reach its tolerance");
    return E_TIMEOUT;
  }
  return OK;
}
