// aldic_internal.cuh -- shared definitions of the sm_100a AL-DIC kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace aldic {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
const char *last_error();

#define ALDIC_CUDA(call)                                                                \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      ::aldic::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));           \
      return -3;                                                                        \
    }                                                                                   \
  } while (0)

#define ALDIC_CHECK(cond, code, msg)                                                    \
  do {                                                                                  \
    if (!(cond)) {                                                                      \
      ::aldic::set_error(msg);                                                          \
      return code;                                                                      \
    }                                                                                   \
  } while (0)

// status codes shared with include/aldic_b200.h
enum { OK = 0, E_ARG = -1, E_STATE = -2, E_CUDA = -3, E_TIMEOUT = -4, E_NOMEM = -5 };

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Bounded grid-wide barrier for cooperative launches.  Every block arrives
// once; the last arrival resets the counter and bumps the generation.  A wait
// longer than `limit` polls sets *err and returns, so a kernel whose blocks
// were not co-resident ends with an error status instead of hanging.
struct GridSync {
  unsigned int *count;
  unsigned int *gen;
  int *err;
};

__device__ __forceinline__ bool grid_sync(const GridSync &g, unsigned int nblocks) {
  __syncthreads();
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_fail = 0;
    volatile unsigned int *vgen = g.gen;
    const unsigned int my_gen = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(g.count, 1u);
    if (arrived == nblocks - 1) {
      *g.count = 0;
      __threadfence();
      atomicAdd(g.gen, 1u);
    } else {
      long long spins = 0;
      while (*vgen == my_gen) {
        if (++spins > (1ll << 22)) {  // ~0.5-2 s with the backoff below
          atomicExch(g.err, 1);
          s_fail = 1;
          break;
        }
        if ((spins & 255) == 0 && *((volatile int *)g.err)) {
          s_fail = 1;
          break;
        }
        if (spins > 256) __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return s_fail == 0;
}

// Keys cubic-convolution weights (a = -1/2), FP32 with FMA: the hot-path form.
__device__ __forceinline__ void keys_w(float t, float w[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = 0.5f * (fmaf(2.0f, t2, -t) - t3);
  w[1] = 0.5f * fmaf(3.0f, t3, fmaf(-5.0f, t2, 2.0f));
  w[2] = 0.5f * fmaf(-3.0f, t3, fmaf(4.0f, t2, t));
  w[3] = 0.5f * (t3 - t2);
}
__device__ __forceinline__ void keys_w(double t, double w[4]) {
  const double t2 = t * t, t3 = t2 * t;
  w[0] = 0.5 * (fma(2.0, t2, -t) - t3);
  w[1] = 0.5 * fma(3.0, t3, fma(-5.0, t2, 2.0));
  w[2] = 0.5 * fma(-3.0, t3, fma(4.0, t2, t));
  w[3] = 0.5 * (t3 - t2);
}

// device buffer that grows on demand (contents are not kept on growth)
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    if (cudaMalloc(&p, want) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of " + std::to_string(want) + " bytes failed");
      return E_NOMEM;
    }
    cap = want;
    return OK;
  }
  template <typename T> T *as() const { return (T *)p; }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace aldic
