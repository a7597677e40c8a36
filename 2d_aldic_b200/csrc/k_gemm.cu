// k_gemm.cu -- BF16 GEMM on the 5th-generation tensor cores (tcgen05) for
// the learned initial guess: D[M x N] = A[M x K] . B[N x K]^T (+ bias, ReLU,
// mask), FP32 accumulation in tensor memory.
//
// One CTA (4 warps) owns a 128 x BN tile.  Per 64-wide K step both operand
// tiles are staged in shared memory in the K-major 128-byte-swizzle layout
// (8 rows x 128 B atoms, 16-B chunk c of row r at chunk c ^ (r & 7)); one
// thread issues four tcgen05.mma (K = 16 each) on shared-memory descriptors
// and commits them to an mbarrier, while all threads stage the next K step
// into the other buffer.  The epilogue reads the accumulator with
// tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and applies
// bias / ReLU / a ReLU mask.  Operands are read through small address
// generators so that the same kernel serves the forward pass (rows or
// non-overlapping patch im2col of an NHWC tensor) and both backward
// products (transposed reads), and the result can be scattered back into
// NHWC patches.  Every wait is bounded and reports through an error flag.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "aldic_internal.cuh"
#include "kernels.cuh"

namespace aldic {

namespace {

constexpr int BM = 128, BK = 64, GEMM_THREADS = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// element address of operand (r, k) for the direct modes (ROW, PATCH)
__device__ __forceinline__ const __nv_bfloat16 *src_addr(const GemmSrc &S, long long r, long long k) {
  if (S.mode == GEMM_ROW) return S.p + r * S.ld + k;
  // GEMM_PATCH: im2col row r of an NHWC tensor with ps x ps patches
  const int Ho = S.Hin / S.ps, Wo = S.Win / S.ps;
  const long long hw = (long long)Ho * Wo;
  const long long b = r / hw, rem = r - b * hw;
  const int i = (int)(rem / Wo), j = (int)(rem - (long long)i * Wo);
  const int seg = S.ps * S.C;
  const int di = (int)(k / seg), rest = (int)(k - (long long)di * seg);
  return S.p + (((b * S.Hin + (long long)S.ps * i + di) * S.Win + (long long)S.ps * j) * S.C + rest);
}

// stage rows [r0, r0 + R) x K [k0, k0 + 64) of an operand into the swizzled
// tile at `tile` (zeros outside the operand)
template <int R>
__device__ __forceinline__ void stage(const GemmSrc &S, long long r0, long long k0, unsigned char *tile) {
  const int tid = threadIdx.x;
  if (S.mode == GEMM_ROW || S.mode == GEMM_PATCH) {
    for (int q = tid; q < R * 8; q += GEMM_THREADS) {
      const int r = q >> 3, c = q & 7;
      const long long gr = r0 + r, gk = k0 + 8 * c;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gr < S.rows && gk < S.kdim) v = *reinterpret_cast<const uint4 *>(src_addr(S, gr, gk));
      *reinterpret_cast<uint4 *>(tile + r * 128 + ((c ^ (r & 7)) << 4)) = v;
    }
  } else {
    // transposed operand: element (r, k) is source element (k, r) of a ROW
    // or PATCH source; 8 consecutive r are one 16-B source chunk
    GemmSrc T = S;
    T.mode = S.mode == GEMM_TRANS ? GEMM_ROW : GEMM_PATCH;
    for (int q = tid; q < BK * (R / 8); q += GEMM_THREADS) {
      const int k = q / (R / 8), g = q - k * (R / 8);
      const long long gk = k0 + k, gr = r0 + 8 * g;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (gk < S.kdim && gr < S.rows) v = *reinterpret_cast<const uint4 *>(src_addr(T, gk, gr));
      const __nv_bfloat16 *e = reinterpret_cast<const __nv_bfloat16 *>(&v);
      const int c = k >> 3, off = (k & 7) * 2;
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int r = 8 * g + t;
        *reinterpret_cast<__nv_bfloat16 *>(tile + r * 128 + ((c ^ (r & 7)) << 4) + off) = e[t];
      }
    }
  }
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (sm_100 format:
// start >> 4 in [0,14), LBO 16 B in [16,30), SBO 1024 B (8 rows x 128 B)
// in [32,46), version 1 in [46,48), layout SWIZZLE_128B = 2 in [61,64))
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// kind::f16 instruction descriptor: D F32, A and B BF16, both K-major,
// N >> 3 in [17,23), M >> 4 in [24,29)
template <int BN>
__device__ __forceinline__ uint32_t idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(id), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// bounded wait on an mbarrier phase; false after ~2^26 polls
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < (1u << 26); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// destination element offset of (m, n)
__device__ __forceinline__ long long dst_off(const GemmDst &D, long long m, long long n) {
  if (D.mode == GEMM_ROW) return m * D.ld + n;
  const int Ho = D.Hin / D.ps, Wo = D.Win / D.ps;
  const long long hw = (long long)Ho * Wo;
  const long long b = m / hw, rem = m - b * hw;
  const int i = (int)(rem / Wo), j = (int)(rem - (long long)i * Wo);
  const int seg = D.ps * D.C;
  const int di = (int)(n / seg), rest = (int)(n - (long long)di * seg);
  return ((b * D.Hin + (long long)D.ps * i + di) * D.Win + (long long)D.ps * j) * D.C + rest;
}

template <int BN>
__global__ void __launch_bounds__(GEMM_THREADS) k_gemm(GemmSrc A, GemmSrc B, GemmDst D, int kt_per,
                                                      int batched, int *err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = BM * 128, STAGE = A_BYTES + BN * 128;
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.x * BM, n0 = (long long)blockIdx.y * BN;
  const int kt_total = (int)((A.kdim + BK - 1) / BK);
  if (batched) {  // grid z = product index
    A.p += blockIdx.z * A.bstride;
    B.p += blockIdx.z * B.bstride;
    if (D.fp32) D.p = reinterpret_cast<float *>(D.p) + blockIdx.z * D.bstride;
    else D.p = reinterpret_cast<__nv_bfloat16 *>(D.p) + blockIdx.z * D.bstride;
    if (D.mask) D.mask += blockIdx.z * D.bstride;
  }
  const int kt0 = batched ? 0 : blockIdx.z * kt_per;
  const int kt1 = min(kt0 + kt_per, kt_total);
  const int nk = kt1 > kt0 ? kt1 - kt0 : 0;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    failed = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t id = idesc<BN>();
  uint32_t phase[2] = {0, 0};

  if (nk > 0) {
    stage<BM>(A, m0, (long long)kt0 * BK, smem);
    stage<BN>(B, n0, (long long)kt0 * BK, smem + A_BYTES);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    for (int t = 0; t < nk; ++t) {
      const int buf = t & 1;
      unsigned char *sa = smem + buf * STAGE;
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t da = sdesc(smem_u32(sa)), db = sdesc(smem_u32(sa + A_BYTES));
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)  // +32 B per K = 16 step: +2 in the address field
          mma_bf16(tmem, da + 2 * kk, db + 2 * kk, id, (t > 0 || kk > 0) ? 1u : 0u);
        mma_commit(&bar[buf]);
      }
      if (t + 1 < nk) {
        const int nb = (t + 1) & 1;
        if (t >= 1) {
          if (!bar_wait(&bar[nb], phase[nb])) failed = 1;
          phase[nb] ^= 1;
        }
        unsigned char *sn = smem + nb * STAGE;
        stage<BM>(A, m0, (long long)(kt0 + t + 1) * BK, sn);
        stage<BN>(B, n0, (long long)(kt0 + t + 1) * BK, sn + A_BYTES);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      __syncthreads();
    }
    const int lb = (nk - 1) & 1;
    if (!bar_wait(&bar[lb], phase[lb])) failed = 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  __syncthreads();
  if (D.split_stride && !batched) {  // split-K: each split writes its own partial product
    if (D.fp32) D.p = reinterpret_cast<float *>(D.p) + blockIdx.z * D.split_stride;
    else D.p = reinterpret_cast<__nv_bfloat16 *>(D.p) + blockIdx.z * D.split_stride;
  }
  if (failed) {
    if (tid == 0) atomicExch(err, 3);
  } else {
    // epilogue: row r = 32 * warp + lane of the tile
    const long long m = m0 + 32 * warp + lane;
    const bool base_aligned = ((uintptr_t)D.p & 15) == 0 && ((uintptr_t)D.mask & 15) == 0;
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      if (nk > 0) {
        tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.f;
      }
      if (m >= D.M) continue;
      const long long nf = n0 + c0;
      // 16 contiguous, 16-byte aligned destination elements: vector stores
      if (nf + 16 <= D.N) {
        const long long o0 = dst_off(D, m, nf);
        const int seg = D.ps * D.C;
        const bool contig = D.mode == GEMM_ROW || (nf % seg) + 16 <= seg;
        const bool aligned = (o0 & 7) == 0 && base_aligned;
        if (contig && aligned) {
          float x[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            x[i] = v[i] * D.scale;
            if (D.bias) x[i] += D.bias[nf + i];
            if (D.relu) x[i] = fmaxf(x[i], 0.f);
          }
          if (D.mask) {
            const uint4 *mp = reinterpret_cast<const uint4 *>(D.mask + o0);
            const uint4 q0 = mp[0], q1 = mp[1];
            const __nv_bfloat16 *mb0 = reinterpret_cast<const __nv_bfloat16 *>(&q0);
            const __nv_bfloat16 *mb1 = reinterpret_cast<const __nv_bfloat16 *>(&q1);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              if (!(__bfloat162float(mb0[i]) > 0.f)) x[i] = 0.f;
              if (!(__bfloat162float(mb1[i]) > 0.f)) x[8 + i] = 0.f;
            }
          }
          if (D.fp32) {
            float4 *dp = reinterpret_cast<float4 *>(reinterpret_cast<float *>(D.p) + o0);
#pragma unroll
            for (int i = 0; i < 4; ++i) dp[i] = make_float4(x[4 * i], x[4 * i + 1], x[4 * i + 2], x[4 * i + 3]);
          } else {
            uint32_t pk[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              __nv_bfloat162 h = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
              pk[i] = *reinterpret_cast<uint32_t *>(&h);
            }
            uint4 *dp = reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(D.p) + o0);
            dp[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            dp[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
          }
          continue;
        }
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const long long n = nf + i;
        if (n >= D.N) continue;
        float x = v[i] * D.scale;
        if (D.bias) x += D.bias[n];
        if (D.relu) x = fmaxf(x, 0.f);
        const long long o = dst_off(D, m, n);
        if (D.mask && !(__bfloat162float(D.mask[o]) > 0.f)) x = 0.f;
        if (D.fp32) reinterpret_cast<float *>(D.p)[o] = x;
        else reinterpret_cast<__nv_bfloat16 *>(D.p)[o] = __float2bfloat16_rn(x);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

template <int BN>
int launch_gemm(const GemmSrc &A, const GemmSrc &B, const GemmDst &D, int splits, int batches,
                int *err, cudaStream_t st) {
  const size_t smem = 2 * (size_t)(BM * 128 + BN * 128) + 1024;
  ALDIC_CUDA(cudaFuncSetAttribute(k_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int kt_total = (int)((A.kdim + BK - 1) / BK);
  const int kt_per = (kt_total + splits - 1) / splits;
  dim3 grid((unsigned)((A.rows + BM - 1) / BM), (unsigned)((B.rows + BN - 1) / BN),
            (unsigned)(batches > 1 ? batches : splits));
  k_gemm<BN><<<grid, GEMM_THREADS, smem, st>>>(A, B, D, kt_per < 1 ? 1 : kt_per, batches > 1, err);
  ALDIC_CUDA(cudaGetLastError());
  return OK;
}

bool src_ok(const GemmSrc &S) {
  if (!S.p || S.rows <= 0 || S.kdim <= 0) return false;
  const uintptr_t a = (uintptr_t)S.p;
  if (a % 16) return false;
  if (S.mode == GEMM_ROW || S.mode == GEMM_TRANS) return S.ld % 8 == 0 && S.ld > 0;
  if (S.mode == GEMM_PATCH || S.mode == GEMM_PATCHT)
    return S.ps > 0 && S.C > 0 && (S.ps * S.C) % 8 == 0 && S.Hin % S.ps == 0 && S.Win % S.ps == 0;
  return false;
}

}  // namespace

int gemm_bf16(const GemmSrc &A, const GemmSrc &B, const GemmDst &D, int splits, int *err,
              cudaStream_t st, int batches) {
  ALDIC_CHECK(src_ok(A) && src_ok(B), E_ARG,
              "gemm: operands must be 16-byte aligned with rows of whole 16-byte chunks");
  ALDIC_CHECK(A.kdim == B.kdim, E_ARG, "gemm: A and B disagree on K");
  // transposed operands read 8 rows per chunk: their row count must allow it
  ALDIC_CHECK((A.mode < GEMM_TRANS || A.rows % 8 == 0) && (B.mode < GEMM_TRANS || B.rows % 8 == 0),
              E_ARG, "gemm: transposed operands need a multiple of 8 rows");
  ALDIC_CHECK(A.kdim % 8 == 0, E_ARG, "gemm: K must be a multiple of 8");
  ALDIC_CHECK(D.p && D.M <= A.rows && D.N <= B.rows && splits >= 1 && err, E_ARG, "gemm: bad output");
  ALDIC_CHECK(splits == 1 || D.split_stride > 0, E_ARG, "gemm: split-K needs a partial-product stride");
  ALDIC_CHECK(batches >= 1 && batches <= 65535 && (batches == 1 || splits == 1), E_ARG,
              "gemm: 1..65535 batched products, without split-K");
  ALDIC_CHECK(batches == 1 || (A.bstride % 8 == 0 && B.bstride % 8 == 0), E_ARG,
              "gemm: batch strides must keep 16-byte alignment");
  ALDIC_CHECK(D.mode == GEMM_ROW || (D.ps > 0 && D.C > 0), E_ARG, "gemm: bad output geometry");
  if (B.rows <= 64) return launch_gemm<64>(A, B, D, splits, batches, err, st);
  if (B.rows <= 128) return launch_gemm<128>(A, B, D, splits, batches, err, st);
  return launch_gemm<256>(A, B, D, splits, batches, err, st);
}

}  // namespace aldic
