// Low-precision trailing update of the mixed-precision LU / Cholesky:
//
//     C(row0 + i, col0 + j) += alpha * sum_k L(i, k) * U(j, k)
//
// with L (M x K) and U (N x K) in bf16 or fp16, both K-contiguous, and C the
// fp32 working copy of the matrix (column-major).  One CTA per 128 x 128
// tile of C, 128 threads:
//   thread 0   : TMA loads of the whole K extent of both operands (128-byte
//                swizzle, one mbarrier), then K/16 tcgen05.mma (kind::f16,
//                fp32 accumulate in TMEM), then tcgen05.commit;
//   all warps  : wait for the MMAs, tcgen05.ld their 32 TMEM lanes, scale by
//                alpha and stage the tile in shared memory (reusing the
//                operand buffers), then one TMA reduce-add folds the tile
//                into C in L2 -- the read-modify-write of C never passes
//                through the SM.
// Every wait is bounded: on timeout the kernel records PLA_K_TIMEOUT, waits
// (bounded) for its own copies, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

constexpr int TM = 128, TN = 128, KBOX = 64, THREADS = 128;
constexpr int BOX_BYTES = TM * KBOX * 2;  // 16 KB: 128 rows x 128 bytes
constexpr long kSpin = 20000000;          // bounded polling (~1-2 s)

__device__ __forceinline__ uint32_t su32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (long i = 0; i < kSpin; i++) {
    if (mbar_try(bar, parity)) return true;
    if (i > 32) __nanosleep(40);
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(su32(dst)),
      "l"(map), "r"(su32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap *map, const void *src, int x,
                                                  int y) {
  asm volatile(
      "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group"
      " [%0, {%2, %3}], [%1];" ::"l"(map),
      "r"(su32(src)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart; the start address advances by 32 bytes per 16-wide K step
__device__ __forceinline__ uint64_t sdesc(const void *p) {
  uint64_t a = su32(p);
  uint64_t d = (a & 0x3FFFFull) >> 4;
  d |= (uint64_t)(16 >> 4) << 16;    // leading byte offset (unused for this layout)
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1 << 46;            // descriptor version for tcgen05
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int KB>
__global__ void __launch_bounds__(THREADS, 1)
tc_update_k(const __grid_constant__ CUtensorMap mapL, const __grid_constant__ CUtensorMap mapU,
            const __grid_constant__ CUtensorMap mapC, int row0, int col0, float alpha,
            uint32_t idesc, int lower, int *status) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full, bar_mma;
  __shared__ uint32_t tmem_s;
  __shared__ int s_bad;
  uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *sL = base;
  uint8_t *sU = base + KB * BOX_BYTES;
  float *sC = reinterpret_cast<float *>(base);  // reused once the MMAs are done
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  // SYRK-shaped update: tiles strictly above the diagonal are not needed
  if (lower && m0 + TM - 1 < n0) return;
  if (*(volatile int *)status != PLA_K_OK) return;

  if (warp == 0) tmem_alloc(&tmem_s, TN);
  if (threadIdx.x == 32) {
    mbar_init(&bar_full, 1);
    mbar_init(&bar_mma, 1);
    mbar_fence_init();
    s_bad = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_s;

  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar_full, 2 * KB * BOX_BYTES);
#pragma unroll
    for (int kb = 0; kb < KB; kb++) {
      tma_load_2d(sL + kb * BOX_BYTES, &mapL, &bar_full, kb * KBOX, m0);
      tma_load_2d(sU + kb * BOX_BYTES, &mapU, &bar_full, kb * KBOX, n0);
    }
    if (!mbar_wait(&bar_full, 0)) {
      s_bad = 1;
      atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
      mbar_wait(&bar_full, 0);  // give the copies in flight one more bounded chance
    } else {
      tc_fence_after();
#pragma unroll
      for (int k = 0; k < KB * (KBOX / 16); k++) {
        const int kb = k / (KBOX / 16), kk = k % (KBOX / 16);
        mma_f16(tmem, sdesc(sL + kb * BOX_BYTES + kk * 32), sdesc(sU + kb * BOX_BYTES + kk * 32),
                idesc, k > 0 ? 1u : 0u);
      }
      mma_commit(&bar_mma);
    }
  }
  __syncthreads();
  bool ok = s_bad == 0;
  if (ok && !mbar_wait(&bar_mma, 0)) {
    atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
    ok = false;
  }
  __syncthreads();
  if (ok && s_bad == 0) {
    tc_fence_after();
#pragma unroll
    for (int c0 = 0; c0 < TN; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c0, r);
#pragma unroll
      for (int j = 0; j < 32; j++)
        sC[(c0 + j) * TM + warp * 32 + lane] = alpha * __uint_as_float(r[j]);
    }
    fence_proxy_async();
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && ok && s_bad == 0) {
    tma_reduce_add_2d(&mapC, sC, row0 + m0, col0 + n0);
    bulk_commit();
    bulk_wait_read();
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, TN);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

int encode(CUtensorMap *map, CUtensorMapDataType dt, int esize, const void *ptr, uint64_t inner,
           uint64_t outer, uint64_t ld_elems, uint32_t box_inner, uint32_t box_outer,
           CUtensorMapSwizzle sw) {
  auto fn = encode_fn();
  if (!fn) return (int)cudaErrorNotSupported;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {ld_elems * (uint64_t)esize};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, dt, 2, const_cast<void *>(ptr), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

template <int KB>
int launch(const CUtensorMap &mL, const CUtensorMap &mU, const CUtensorMap &mC, int M, int N,
           int row0, int col0, float alpha, uint32_t idesc, int lower, int *status,
           cudaStream_t s) {
  // operand tiles, reused afterwards as the 128 x 128 fp32 staging tile
  size_t ops = (size_t)2 * KB * BOX_BYTES, stage = (size_t)TM * TN * sizeof(float);
  size_t sm = (ops > stage ? ops : stage) + 1024;
  cudaFuncSetAttribute(tc_update_k<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  dim3 grid((M + TM - 1) / TM, (N + TN - 1) / TN);
  tc_update_k<KB><<<grid, THREADS, sm, s>>>(mL, mU, mC, row0, col0, alpha, idesc, lower, status);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" int pla_k_tc_update(int prec, int M, int N, int K, float alpha, const void *L,
                               long ldl, long l_rows, const void *U, long ldu, long u_rows,
                               float *C, long ldc, long c_rows, long c_cols, int row0, int col0,
                               int lower, int *status, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  if (K % KBOX != 0 || K > 4 * KBOX) return (int)cudaErrorInvalidValue;
  if (ldl % 8 || ldu % 8 || ldc % 4 || (row0 % 4) || ((uintptr_t)C % 16) || ((uintptr_t)L % 16) ||
      ((uintptr_t)U % 16))
    return (int)cudaErrorMisalignedAddress;
  const CUtensorMapDataType abt =
      prec == PLA_K_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  CUtensorMap mL, mU, mC;
  int r;
  if ((r = encode(&mL, abt, 2, L, (uint64_t)K, (uint64_t)l_rows, (uint64_t)ldl, KBOX, TM,
                  CU_TENSOR_MAP_SWIZZLE_128B)))
    return r;
  if ((r = encode(&mU, abt, 2, U, (uint64_t)K, (uint64_t)u_rows, (uint64_t)ldu, KBOX, TN,
                  CU_TENSOR_MAP_SWIZZLE_128B)))
    return r;
  if ((r = encode(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, (uint64_t)c_rows, (uint64_t)c_cols,
                  (uint64_t)ldc, TM, TN, CU_TENSOR_MAP_SWIZZLE_NONE)))
    return r;
  // instruction descriptor: fp32 accumulate, A/B bf16 (1) or fp16 (0), both
  // K-major, N = 128, M = 128
  const uint32_t ab = prec == PLA_K_BF16 ? 1u : 0u;
  const uint32_t idesc = (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)(TN >> 3) << 17) |
                         ((uint32_t)(TM >> 4) << 24);
  switch (K / KBOX) {
    case 1: return launch<1>(mL, mU, mC, M, N, row0, col0, alpha, idesc, lower, status, s);
    case 2: return launch<2>(mL, mU, mC, M, N, row0, col0, alpha, idesc, lower, status, s);
    case 3: return launch<3>(mL, mU, mC, M, N, row0, col0, alpha, idesc, lower, status, s);
    default: return launch<4>(mL, mU, mC, M, N, row0, col0, alpha, idesc, lower, status, s);
  }
}
