// Low-precision trailing update of the mixed-precision LU / Cholesky:
//
//     C(row0 + i, col0 + j) += alpha * sum_k L(i, k) * U(j, k)
//
// with L (M x K) and U (N x K) in bf16 or fp16 (kind::f16), or in fp8 E4M3
// with one power-of-two scale per 128-row tile of each operand (kind::f8f6f4,
// the scales applied in the epilogue), both K-contiguous, and C the fp32
// working copy of the matrix (column-major).  The C traffic (an fp32
// read and write per element) is the bound, so the kernel is built to keep
// HBM busy: one persistent CTA per SM walks 128 x 128 tiles of C with three
// roles that overlap one tile's epilogue with the next tile's loads and MMAs:
//   warp 0 (one thread): TMA loads of 64-wide K chunks of L and U (128-byte
//            swizzle) into a ring of STAGES shared-memory stages (4, or 5 for
//            K > 512, where the chunks of a tile outnumber the stages and
//            the load latency from L2 must be covered);
//   warp 1 (one thread): tcgen05.mma (kind::f16, fp32 accumulate) into one of
//            two TMEM accumulators; tcgen05.commit frees each stage and, after
//            the last chunk, hands the accumulator to the epilogue;
//   warps 2-5: tcgen05.ld 32 columns at a time, scale by alpha, stage them in
//            one of kChunks shared-memory buffers and fold them into C with a
//            TMA reduce-add (the read-modify-write of C happens in L2).
// Every wait is bounded: on timeout the kernel records PLA_K_TIMEOUT, stops
// issuing work, waits (bounded) for its own copies and MMAs, frees its TMEM
// and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

constexpr int TM = 128, TN = 128, KBOX = 64;
constexpr int BOX_BYTES = TM * KBOX * 2;      // 16 KB: 128 rows x 128 bytes
constexpr int STAGE_BYTES = 2 * BOX_BYTES;    // 32 KB
constexpr int CW = 32;                        // epilogue chunk: 32 columns of a tile
constexpr int kChunks = 4;                    // staging buffers for the reduce-adds
constexpr int CHUNK_BYTES = TM * CW * 4;      // 16 KB of fp32
constexpr int THREADS = 192;                  // TMA warp, MMA warp, 4 epilogue warps
// dynamic shared memory with `stages` operand stages (the ring, then the
// reduce-add staging buffers, 1 KB of alignment slack)
constexpr int smem_bytes(int stages) { return stages * STAGE_BYTES + kChunks * CHUNK_BYTES + 1024; }
constexpr long kSpin = 20000000;              // bounded polling (~1-2 s)

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
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}
// barrier 1 among the 128 epilogue threads (warps 2-5)
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }
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
// fp8 operands (E4M3 x E4M3, fp32 accumulate): K = 32 per instruction, so a
// 128-byte row of the swizzled box is again four instructions 32 bytes apart
__device__ __forceinline__ void mma_f8(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
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

// Tile t of the walk: bands of `band` tile rows, each band walked column by
// column.  band = tiles_m is the plain column-major walk; a narrower band
// keeps the L rows of the tiles in flight few enough to stay in L2 while the
// band's columns pass (long K: the split operands of the bf16 x 6 update).
__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int band, int &tm,
                                            int &tn) {
  const int span = band * tiles_n;
  const int b = t / span, w = t - b * span;
  const int rows = min(band, tiles_m - b * band);
  tm = b * band + w % rows;
  tn = w / rows;
}

// F8: E4M3 operands with one power-of-two scale per 128-row tile of L and of
// U (inv_l, inv_u); a K chunk is then 128 elements (still 128 bytes per row)
template <bool F8, int STAGES>
__global__ void __launch_bounds__(THREADS, 1)
tc_update_k(const __grid_constant__ CUtensorMap mapL, const __grid_constant__ CUtensorMap mapU,
            const __grid_constant__ CUtensorMap mapC, int M, int N, int kchunks, int row0,
            int col0, float alpha, uint32_t idesc, int lower, int band, const float *inv_l,
            const float *inv_u, int *status) {
  constexpr int KE = F8 ? 128 : KBOX;  // elements per K chunk
  extern __shared__ uint8_t smem_raw[];
  constexpr int kStages = STAGES;
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2],
      bar_drain;
  __shared__ uint32_t tmem_s;
  __shared__ volatile int s_abort;
  __shared__ int s_skip, s_epi_stop;
  uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *ring = base;                                   // kStages x (L box, U box)
  float *stagec = reinterpret_cast<float *>(base + kStages * STAGE_BYTES);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles_m = (M + TM - 1) / TM, tiles_n = (N + TN - 1) / TN;
  const int ntiles = tiles_m * tiles_n;
  // one thread reads the status so that every thread takes the same branch
  if (threadIdx.x == 0) s_skip = *(volatile int *)status != PLA_K_OK;
  __syncthreads();
  if (s_skip) return;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 128);
    }
    mbar_init(&bar_drain, 1);
    mbar_fence_init();
    s_abort = 0;
  }
  if (warp == 1) tmem_alloc(&tmem_s, 2 * TN);  // two 128-column fp32 accumulators
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_s;
  auto fail = [&]() {
    atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
    s_abort = 1;
  };
  // SYRK-shaped update: tiles strictly above the diagonal are not needed
  auto skip = [&](int tm, int tn) { return lower && tm * TM + TM - 1 < tn * TN; };

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer ----
      int stage = 0;
      uint32_t ph = 0;
      int issued_ph[kStages];
      for (int s = 0; s < kStages; s++) issued_ph[s] = -1;
      for (int t = blockIdx.x; t < ntiles && !s_abort; t += gridDim.x) {
        int tm, tn;
        tile_coords(t, tiles_m, tiles_n, band, tm, tn);
        if (skip(tm, tn)) continue;
        for (int kc = 0; kc < kchunks && !s_abort; kc++) {
          if (!mbar_wait(&empty[stage], ph ^ 1)) {
            fail();
            break;
          }
          uint8_t *sl = ring + stage * STAGE_BYTES;
          mbar_expect_tx(&full[stage], STAGE_BYTES);
          tma_load_2d(sl, &mapL, &full[stage], kc * KE, tm * TM);
          tma_load_2d(sl + BOX_BYTES, &mapU, &full[stage], kc * KE, tn * TN);
          issued_ph[stage] = (int)ph;
          if (++stage == kStages) {
            stage = 0;
            ph ^= 1;
          }
        }
      }
      // every load must have landed before the shared memory is released
      for (int s = 0; s < kStages; s++)
        if (issued_ph[s] >= 0 && !mbar_wait(&full[s], (uint32_t)issued_ph[s])) fail();
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer ----
      int stage = 0, count = 0;
      uint32_t ph = 0;
      bool issued = false;
      for (int t = blockIdx.x; t < ntiles && !s_abort; t += gridDim.x) {
        int tm, tn;
        tile_coords(t, tiles_m, tiles_n, band, tm, tn);
        if (skip(tm, tn)) continue;
        const int ab = count & 1;
        if (!mbar_wait(&acc_empty[ab], ((count >> 1) & 1) ^ 1)) {
          fail();
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(ab * TN);
        bool ok = true;
        for (int kc = 0; kc < kchunks; kc++) {
          if (!mbar_wait(&full[stage], ph)) {
            fail();
            ok = false;
            break;
          }
          tc_fence_after();
          uint8_t *sl = ring + stage * STAGE_BYTES;
#pragma unroll
          for (int kk = 0; kk < 4; kk++) {  // 32-byte K steps through the 128-byte rows
            if constexpr (F8)
              mma_f8(d, sdesc(sl + kk * 32), sdesc(sl + BOX_BYTES + kk * 32), idesc,
                     (kc | kk) ? 1u : 0u);
            else
              mma_f16(d, sdesc(sl + kk * 32), sdesc(sl + BOX_BYTES + kk * 32), idesc,
                      (kc | kk) ? 1u : 0u);
          }
          issued = true;
          mma_commit(&empty[stage]);  // the stage is free once these MMAs have read it
          if (++stage == kStages) {
            stage = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        mma_commit(&acc_full[ab]);
        count++;
      }
      // all MMAs complete before the TMEM is freed
      if (issued) {
        mma_commit(&bar_drain);
        if (!mbar_wait(&bar_drain, 0)) fail();
      }
    }
  } else {  // ---- epilogue: warps 2-5, TMEM lanes 32 * (warp % 4) ----
    // The 128 epilogue threads meet at named barrier 1, so they must leave
    // the tile loop together: the decision to stop is sampled by one thread
    // and read by all from s_epi_stop.
    const int lanes = 32 * (warp & 3);
    const int row = lanes + lane;
    const bool elected = threadIdx.x == 64;
    int count = 0, chunk = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int tm, tn;
        tile_coords(t, tiles_m, tiles_n, band, tm, tn);
      if (skip(tm, tn)) continue;
      const int ab = count & 1;
      if (!mbar_wait(&acc_full[ab], (count >> 1) & 1)) fail();
      epi_sync();
      if (elected) s_epi_stop = s_abort;
      epi_sync();
      if (s_epi_stop) break;
      const float scale = F8 ? alpha * inv_l[tm] * inv_u[tn] : alpha;
      tc_fence_after();
#pragma unroll 1
      for (int c = 0; c < TN / CW; c++) {
        float *sc = stagec + (chunk % kChunks) * (TM * CW);
        if (elected) bulk_wait_read<kChunks - 1>();  // the reduce that used sc has read it
        epi_sync();
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)lanes << 16) + (uint32_t)(ab * TN + c * CW), r);
#pragma unroll
        for (int j = 0; j < CW; j++) sc[j * TM + row] = scale * __uint_as_float(r[j]);
        fence_proxy_async();
        epi_sync();
        if (elected) {
          tma_reduce_add_2d(&mapC, sc, row0 + tm * TM, col0 + tn * TN + c * CW);
          bulk_commit();
        }
        chunk++;
      }
      tc_fence_before();
      mbar_arrive(&acc_empty[ab]);  // this thread's reads of the accumulator are done
      count++;
    }
    if (elected) bulk_wait_all();
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * TN);
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

int g_sms = 0;

template <bool F8, int STAGES>
int launch(const CUtensorMap &mL, const CUtensorMap &mU, const CUtensorMap &mC, int M, int N,
           int kchunks, int row0, int col0, float alpha, uint32_t idesc, int lower, int band,
           const float *inv_l, const float *inv_u, int max_ctas, int *status, cudaStream_t s) {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  constexpr int kSmem = smem_bytes(STAGES);
  cudaFuncSetAttribute(tc_update_k<F8, STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       kSmem);
  const long tiles = (long)((M + TM - 1) / TM) * ((N + TN - 1) / TN);
  const int cap = max_ctas > 0 && max_ctas < g_sms ? max_ctas : g_sms;
  const int grid = (int)(tiles < cap ? tiles : cap);
  const int tiles_m = (M + TM - 1) / TM;
  if (band <= 0 || band > tiles_m) band = tiles_m;
  tc_update_k<F8, STAGES><<<grid, THREADS, kSmem, s>>>(mL, mU, mC, M, N, kchunks, row0, col0,
                                                       alpha, idesc, lower, band, inv_l, inv_u,
                                                       status);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" int pla_k_tc_update_ex(int prec, int M, int N, int K, float alpha, const void *L,
                                  long ldl, long l_rows, const void *U, long ldu, long u_rows,
                                  float *C, long ldc, long c_rows, long c_cols, int row0,
                                  int col0, int lower, int max_ctas, int *status, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  if (K % KBOX != 0) return (int)cudaErrorInvalidValue;
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
                  (uint64_t)ldc, TM, CW, CU_TENSOR_MAP_SWIZZLE_NONE)))
    return r;
  // instruction descriptor: fp32 accumulate, A/B bf16 (1) or fp16 (0), both
  // K-major, N = 128, M = 128
  const uint32_t ab = prec == PLA_K_BF16 ? 1u : 0u;
  const uint32_t idesc = (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)(TN >> 3) << 17) |
                         ((uint32_t)(TM >> 4) << 24);
  // K past 512 (split operands): bands of 32 tile rows, so that the L rows
  // in flight (32 x 128 rows x 2K bytes) stay in L2 across the band's columns
  const int band = K > 512 ? 32 : 0;
  // a fifth stage for the long K: 8 % faster at K = 1536 (16384^2), 2 % slower at K = 256
  if (K > 512)
    return launch<false, 5>(mL, mU, mC, M, N, K / KBOX, row0, col0, alpha, idesc, lower, band,
                            nullptr, nullptr, max_ctas, status, s);
  return launch<false, 4>(mL, mU, mC, M, N, K / KBOX, row0, col0, alpha, idesc, lower, band,
                          nullptr, nullptr, max_ctas, status, s);
}

extern "C" int pla_k_tc_update(int prec, int M, int N, int K, float alpha, const void *L,
                               long ldl, long l_rows, const void *U, long ldu, long u_rows,
                               float *C, long ldc, long c_rows, long c_cols, int row0, int col0,
                               int lower, int *status, cudaStream_t s) {
  return pla_k_tc_update_ex(prec, M, N, K, alpha, L, ldl, l_rows, U, ldu, u_rows, C, ldc, c_rows,
                            c_cols, row0, col0, lower, 0, status, s);
}

// The same update with fp8 E4M3 operands (row-major, K-contiguous, ldl / ldu
// bytes) and per-128-row-tile inverse scales: C += alpha * inv_l[i / 128] *
// inv_u[j / 128] * sum_k L(i, k) U(j, k).
extern "C" int pla_k_tc_update_fp8_ex(int M, int N, int K, float alpha, const void *L,
                                      long ldl, long l_rows, const float *inv_l, const void *U,
                                      long ldu, long u_rows, const float *inv_u, float *C,
                                      long ldc, long c_rows, long c_cols, int row0, int col0,
                                      int lower, int max_ctas, int *status, cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0) return 0;
  if (K % 128 != 0 || !inv_l || !inv_u) return (int)cudaErrorInvalidValue;
  if (ldl % 16 || ldu % 16 || ldc % 4 || (row0 % 4) || ((uintptr_t)C % 16) ||
      ((uintptr_t)L % 16) || ((uintptr_t)U % 16))
    return (int)cudaErrorMisalignedAddress;
  CUtensorMap mL, mU, mC;
  int r;
  if ((r = encode(&mL, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, L, (uint64_t)K, (uint64_t)l_rows,
                  (uint64_t)ldl, 128, TM, CU_TENSOR_MAP_SWIZZLE_128B)))
    return r;
  if ((r = encode(&mU, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, U, (uint64_t)K, (uint64_t)u_rows,
                  (uint64_t)ldu, 128, TN, CU_TENSOR_MAP_SWIZZLE_128B)))
    return r;
  if ((r = encode(&mC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, (uint64_t)c_rows, (uint64_t)c_cols,
                  (uint64_t)ldc, TM, CW, CU_TENSOR_MAP_SWIZZLE_NONE)))
    return r;
  // instruction descriptor, kind::f8f6f4: fp32 accumulate, A and B both E4M3
  // (format 0), both K-major, N = 128, M = 128
  const uint32_t idesc = (1u << 4) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
  return launch<true, 4>(mL, mU, mC, M, N, K / 128, row0, col0, alpha, idesc, lower, 0, inv_l,
                         inv_u, max_ctas, status, s);
}

extern "C" int pla_k_tc_update_fp8(int M, int N, int K, float alpha, const void *L, long ldl,
                                   long l_rows, const float *inv_l, const void *U, long ldu,
                                   long u_rows, const float *inv_u, float *C, long ldc,
                                   long c_rows, long c_cols, int row0, int col0, int lower,
                                   int *status, cudaStream_t s) {
  return pla_k_tc_update_fp8_ex(M, N, K, alpha, L, ldl, l_rows, inv_l, U, ldu, u_rows, inv_u, C,
                                ldc, c_rows, c_cols, row0, col0, lower, 0, status, s);
}
