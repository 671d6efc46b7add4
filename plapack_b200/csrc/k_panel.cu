// Panel LU with partial pivoting: the per-column loop of the reference's
// PLA_LU_right_mv (SOLVERS/LU/PLA_LU_mv.c:52-82) fused into one cooperative
// kernel.  Per column j:
//   PLA_Iamax        -> block argmax + grid-wide pick of (max |a|, first index)
//                       (BLAS1/PLA_Iamax.c:86,108-115)
//   Pivot_rows_mv    -> swap row j with the pivot row over the panel width
//                       (SOLVERS/LU/PLA_Apply_pivots_new.c:245-290)
//   PLA_Local_inv_scal -> a21 *= 1/alpha11 (Local_BLAS/PLA_Local_BLAS1.c:256-263)
//   PLA_Local_ger    -> A22 += a21 * (-a12') (Local_BLAS/PLA_Local_BLAS2.c:632)
//
// Layout: CTA b owns rows [b*R, b*R + R) of the r x w panel.  When they fit,
// the CTA keeps its rows in shared memory for the whole panel; otherwise it
// works in place in global memory (the panel is L2-resident).
//
// Exchange, one round per column: every CTA publishes a record -- its best
// candidate (|value|, row) as two 64-bit words that each carry a generation
// bit, the candidate's whole row, and, from the owner of the diagonal row,
// that row -- and then gathers every CTA's record.  All CTAs pick the same
// winner from the same records, so no barrier precedes the reads.  Records
// alternate between two slots by column parity; the generation bit
// ((j >> 1) & 1) ^ 1 tells the record of column j from that of column j - 2
// in the same slot, and the slots are zeroed before each launch (generation
// 0, which no record of column 0 or 1 has).  A CTA can only overwrite a slot
// after every CTA has published the next column, that is after every CTA has
// finished reading the slot.
//
// Lookahead inside the panel: after the pivot of column j a CTA updates only
// column j + 1 of its rows, publishes the record of column j + 1 (its rows
// carry the rest of the update, computed with the same fma as below, so the
// published values are bitwise those the CTA stores later), and then updates
// its remaining columns while the other CTAs publish.  Every wait is bounded;
// on timeout the kernel records PLA_K_TIMEOUT and exits.
#include <climits>
#include <cstdio>
#include <mutex>

#include "pla_internal.h"
#include "pla_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr long kSpinLimit = 4000000;  // polls before giving up (~1-2 s)
constexpr int kPerLane = 5;           // records per lane of the gathering warp: P <= 160

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// record words: bit 63 the generation, below it |value| (>= 0, so its own
// sign bit is free) or the row index
template <typename T>
__device__ __forceinline__ unsigned long long enc_val(T v, unsigned long long gen) {
  if constexpr (sizeof(T) == 8)
    return (gen << 63) | (unsigned long long)__double_as_longlong(v);
  else
    return (gen << 63) | (unsigned long long)__float_as_uint(v);
}
template <typename T>
__device__ __forceinline__ T dec_val(unsigned long long w) {
  if constexpr (sizeof(T) == 8)
    return __longlong_as_double((long long)(w & ~(1ull << 63)));
  else
    return __uint_as_float((unsigned)(w & 0xffffffffull));
}

// (abs, idx) ordering: larger |value| first, then smaller index
template <typename T>
__device__ __forceinline__ bool better(T av, int ai, T bv, int bi) {
  return av > bv || (av == bv && ai < bi);
}

template <typename T>
__device__ void block_argmax(T &v, int &i, T *sv, int *si) {
  for (int o = 16; o; o >>= 1) {
    T ov = __shfl_down_sync(0xffffffffu, v, o);
    int oi = __shfl_down_sync(0xffffffffu, i, o);
    if (better(ov, oi, v, i)) { v = ov; i = oi; }
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) { sv[w] = v; si[w] = i; }
  __syncthreads();
  if (w == 0) {
    v = l < (kThreads / 32) ? sv[l] : T(-1);
    i = l < (kThreads / 32) ? si[l] : INT_MAX;
    for (int o = 16; o; o >>= 1) {
      T ov = __shfl_down_sync(0xffffffffu, v, o);
      int oi = __shfl_down_sync(0xffffffffu, i, o);
      if (better(ov, oi, v, i)) { v = ov; i = oi; }
    }
    if (l == 0) { sv[0] = v; si[0] = i; }
  }
  __syncthreads();
  v = sv[0];
  i = si[0];
}

// rec: [2 slots][P CTAs][2 words]; cand_row: [2][P][w]; top_row: [2][w]
template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
panel_lu_k(T *A, long lda, int r, int w, int R, int use_smem, int *piv, int *status,
           int *zero_info, int row_base, unsigned long long *rec, T *cand_row, T *top_row) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ T s_v[32];
  __shared__ int s_i[32];
  __shared__ int s_abort, s_p, s_q;

  const int P = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const int row0 = b * R;
  const int row1 = min(row0 + R, r);
  const int nrows = max(row1 - row0, 0);
  T *u = reinterpret_cast<T *>(smem_raw);  // pivot row, w entries
  T *S;
  long lds;
  if (use_smem) {
    S = u + ((w + 1) & ~1);
    lds = R;
    for (long t = tid; t < (long)nrows * w; t += kThreads) {
      int i = (int)(t % nrows), c = (int)(t / nrows);
      S[i + c * lds] = A[(long)(row0 + i) + (long)c * lda];
    }
  } else {
    S = A + row0;
    lds = lda;
  }
  if (tid == 0) s_abort = 0;
  __syncthreads();
#define E(i, c) S[(long)(i) + (long)(c) * lds]

  // Publish the record of column `col`.  With `pend` the rows still owe the
  // rank-1 update of pivot col - 1 in the columns right of col (multiplier
  // E(., col - 1), pivot row u): the published rows include it.
  auto publish = [&](int col, bool pend) {
    const int par = col & 1;
    const unsigned long long gen = (unsigned long long)(((col >> 1) & 1) ^ 1);
    T best = T(-1);
    int bidx = INT_MAX;
    const int lo = max(col - row0, 0);
    for (int li = lo + tid; li < nrows; li += kThreads) {
      T v = fabs(E(li, col));
      if (better(v, row0 + li, best, bidx)) { best = v; bidx = row0 + li; }
    }
    block_argmax(best, bidx, s_v, s_i);
    auto row_val = [&](int li, int c) -> T {
      const T e = E(li, c);
      return (pend && c > col) ? fma(E(li, col - 1), -u[c], e) : e;
    };
    if (bidx != INT_MAX)
      for (int c = tid; c < w; c += kThreads)
        cand_row[((long)par * P + b) * w + c] = row_val(bidx - row0, c);
    if (col >= row0 && col < row1)
      for (int c = tid; c < w; c += kThreads) top_row[(long)par * w + c] = row_val(col - row0, c);
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      unsigned long long *rp = rec + ((long)par * P + b) * 2;
      const bool none = bidx == INT_MAX;  // no candidate: every entry is NaN
      st_relaxed64(rp, enc_val<T>(none ? T(0) : best, gen));
      st_relaxed64(rp + 1, (gen << 63) | (unsigned)(none ? INT_MAX : bidx));
    }
  };

  // Gather the records of column `col` into (s_p = winning row or INT_MAX,
  // s_q = its CTA); false when a wait gave up.  Lane l of warp 0 watches the
  // records of CTAs l, l + 32, ...: each poll loads all of them at once
  // (independent loads, one round trip), and one acquire fence follows once
  // every record carries the column's generation.
  auto gather = [&](int col) -> bool {
    const int par = col & 1;
    const unsigned long long gen = (unsigned long long)(((col >> 1) & 1) ^ 1);
    if (tid < 32) {
      unsigned long long w0[kPerLane], w1[kPerLane];
      bool done[kPerLane];
#pragma unroll
      for (int i = 0; i < kPerLane; i++) {
        done[i] = tid + 32 * i >= P;
        w0[i] = w1[i] = 0;
      }
      bool ok = true;
      for (long spins = 0;; spins++) {
#pragma unroll
        for (int i = 0; i < kPerLane; i++)
          if (!done[i]) {
            const unsigned long long *rp = rec + ((long)par * P + tid + 32 * i) * 2;
            w0[i] = ld_relaxed64(rp);
            w1[i] = ld_relaxed64(rp + 1);
          }
        bool all = true;
#pragma unroll
        for (int i = 0; i < kPerLane; i++)
          if (!done[i]) {
            if ((w0[i] >> 63) == gen && (w1[i] >> 63) == gen) done[i] = true;
            else all = false;
          }
        if (all) break;
        if (spins > kSpinLimit || *(volatile int *)status != PLA_K_OK) {
          ok = false;
          break;
        }
      }
      __threadfence();  // acquire: the rows published before the records are visible
      T bv = T(-1);
      int bi = INT_MAX, bq = 0;
#pragma unroll
      for (int i = 0; i < kPerLane; i++) {
        const int q = tid + 32 * i;
        if (q >= P) continue;
        const T v = dec_val<T>(w0[i]);
        const int ix = (int)(unsigned)(w1[i] & 0xffffffffull);
        if (better(v, ix, bv, bi)) { bv = v; bi = ix; bq = q; }
      }
      const bool all_ok = __all_sync(0xffffffffu, ok);
      for (int o = 16; o; o >>= 1) {
        T ov = __shfl_down_sync(0xffffffffu, bv, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        int oq = __shfl_down_sync(0xffffffffu, bq, o);
        if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; bq = oq; }
      }
      if (tid == 0) {
        if (!all_ok) {
          atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
          s_abort = 1;
        }
        s_p = bi;
        s_q = bq;
      }
    }
    __syncthreads();
    return s_abort == 0;
  };

  publish(0, false);
  for (int j = 0; j < w; j++) {
    if (!gather(j)) return;
    const int par = j & 1;
    // A column of NaNs has no candidate (NaN never compares greater): keep
    // row j as its own pivot, whose contents the owner of row j published.
    const bool none = s_p == INT_MAX;
    const int p = none ? j : s_p, wq = s_q;
    for (int c = tid; c < w; c += kThreads)
      u[c] = none ? __ldcg(&top_row[(long)par * w + c])
                  : __ldcg(&cand_row[((long)par * P + wq) * w + c]);
    __syncthreads();
    // the interchange of rows j and p over the panel width
    if (j >= row0 && j < row1)
      for (int c = tid; c < w; c += kThreads) E(j - row0, c) = u[c];
    if (p != j && p >= row0 && p < row1)
      for (int c = tid; c < w; c += kThreads) E(p - row0, c) = __ldcg(&top_row[(long)par * w + c]);
    if (b == 0 && tid == 0) {
      piv[j] = p - j;
      if (zero_info && u[j] == T(0)) atomicCAS(zero_info, 0, row_base + j + 1);
    }
    __syncthreads();
    // scale by the reciprocal and update the next column first ...
    const T inv = T(1) / u[j];
    const int lo = max(j + 1 - row0, 0);
    for (int li = lo + tid; li < nrows; li += kThreads) {
      const T l = E(li, j) * inv;
      E(li, j) = l;
      if (j + 1 < w) E(li, j + 1) = fma(l, -u[j + 1], E(li, j + 1));
    }
    if (j + 1 < w) {
      __syncthreads();
      publish(j + 1, true);
      // ... then the rest of the rank-1 update while the others publish
      for (int li = lo + tid; li < nrows; li += kThreads) {
        const T l = E(li, j);
        for (int c = j + 2; c < w; c++) E(li, c) = fma(l, -u[c], E(li, c));
      }
      __syncthreads();
    }
  }
  if (use_smem) {
    __syncthreads();
    for (long t = tid; t < (long)nrows * w; t += kThreads) {
      int i = (int)(t % nrows), c = (int)(t / nrows);
      A[(long)(row0 + i) + (long)c * lda] = S[i + c * lds];
    }
  }
#undef E
}

// workspace layout for P CTAs and width w: the record slots (zeroed before
// every launch), the candidate rows and the diagonal rows
struct Layout {
  size_t rec_bytes, off_row, off_top, total;
};
template <typename T>
Layout layout(int P, int w) {
  Layout l;
  l.rec_bytes = ((size_t)2 * P * 2 * sizeof(unsigned long long) + 255) & ~(size_t)255;
  l.off_row = l.rec_bytes;
  l.off_top = l.off_row + (size_t)2 * P * w * sizeof(T);
  l.total = l.off_top + (size_t)2 * w * sizeof(T);
  return l;
}

struct Workspace {
  void *ptr = nullptr;
  size_t bytes = 0;
};
Workspace g_ws;

void *workspace(size_t bytes) {
  if (g_ws.bytes >= bytes) return g_ws.ptr;
  if (g_ws.ptr) cudaFree(g_ws.ptr);
  g_ws.ptr = nullptr;
  g_ws.bytes = 0;
  if (cudaMalloc(&g_ws.ptr, bytes) != cudaSuccess) return nullptr;
  g_ws.bytes = bytes;
  return g_ws.ptr;
}

int g_sms = 0, g_smem_optin = 0;

template <typename T>
int launch(int r, int w, void *A, long lda, int *piv, int *status, int *zero_info, int row_base,
           cudaStream_t s) {
  if (!g_sms) {
    int dev;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&g_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  }
  // rows per CTA: at least 32, at most enough CTAs for one per SM
  int P = (r + 31) / 32;
  if (P > g_sms) P = g_sms;
  if (P > 32 * kPerLane) P = 32 * kPerLane;  // the records one warp gathers
  if (P < 1) P = 1;
  int R = (r + P - 1) / P;
  P = (r + R - 1) / R;
  size_t ubytes = (size_t)((w + 1) & ~1) * sizeof(T);
  size_t sbytes = ubytes + (size_t)R * w * sizeof(T);
  int use_smem = sbytes + 1024 <= (size_t)g_smem_optin - 2048;
  size_t dyn = use_smem ? sbytes : ubytes;
  cudaFuncSetAttribute(panel_lu_k<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_lu_k<T>, kThreads, dyn);
  if (per_sm * g_sms < P) return (int)cudaErrorCooperativeLaunchTooLarge;
  const Layout lay = layout<T>(P, w);
  char *ws = (char *)workspace(lay.total);
  if (!ws) return (int)cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemsetAsync(ws, 0, lay.rec_bytes, s);
  if (e) return (int)e;
  unsigned long long *rec = (unsigned long long *)ws;
  T *cand_row = (T *)(ws + lay.off_row);
  T *top_row = (T *)(ws + lay.off_top);
  T *Ap = (T *)A;
  void *args[] = {&Ap, &lda, &r, &w, &R, &use_smem, &piv, &status, &zero_info, &row_base, &rec,
                  &cand_row, &top_row};
  e = cudaLaunchCooperativeKernel((void *)panel_lu_k<T>, dim3(P), dim3(kThreads), args, dyn, s);
  pla_k_count(1);
  return (int)e;
}

}  // namespace

extern "C" int pla_k_lu_panel(int dt, int r, int w, void *A, long lda, int *piv, int *status,
                              int *zero_info, int row_base, cudaStream_t s) {
  if (r <= 0 || w <= 0) return 0;
  if (w > r) return (int)cudaErrorInvalidValue;
  if (dt == MPI_DOUBLE) return launch<double>(r, w, A, lda, piv, status, zero_info, row_base, s);
  if (dt == MPI_FLOAT) return launch<float>(r, w, A, lda, piv, status, zero_info, row_base, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" void pla_kernels_release(void) {
  if (g_ws.ptr) cudaFree(g_ws.ptr);
  g_ws.ptr = nullptr;
  g_ws.bytes = 0;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the panel factorization.
//
// Some callers cannot let a library call cudaMalloc: programs whose GPU memory
// is owned by another allocator (a framework's caching allocator that has
// reserved the device, for instance), and memory-budgeted or real-time
// services that forbid allocation once they are running.  For them the panel
// kernel's workspace -- the per-CTA pivot records and candidate rows -- lives
// in the fixed device array below instead of memory the library allocates.
// The array holds the workspace of at most kNoAllocCtas CTAs for panels of at
// most kNoAllocWidth columns in double precision (about 335 KB); every GPU
// that loads the library keeps it until the process exits.  Every call shares
// it, so calls whose kernels overlap on the GPU (on different streams, or from
// different host threads) race.
namespace {
constexpr int kNoAllocCtas = 160;
constexpr int kNoAllocWidth = 128;
// the double-precision layout at the limits; a float panel needs less
constexpr size_t kNoAllocRec = ((size_t)2 * kNoAllocCtas * 2 * 8 + 255) & ~(size_t)255;
constexpr size_t kNoAllocBytes = kNoAllocRec +
                                 (size_t)2 * kNoAllocCtas * kNoAllocWidth * sizeof(double) +
                                 (size_t)2 * kNoAllocWidth * sizeof(double);
}  // namespace

static __device__ __align__(256) unsigned char g_panel_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_addr[128] = {};

// The array's device address on the current device, looked up once per
// device (the host-side name of the array is only a stand-in).
int noalloc_scratch(char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= 128) return (int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_panel_scratch);
    if (e != cudaSuccess) return (int)e;
    g_noalloc_addr[dev] = p;
  }
  *out = (char *)g_noalloc_addr[dev];
  return 0;
}

template <typename T>
int launch_noalloc(int r, int w, T *A, long lda, int *piv, int *status, cudaStream_t s) {
  int dev = 0, sms = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int P = (r + 31) / 32;
  if (P > sms) P = sms;
  if (P > kNoAllocCtas) P = kNoAllocCtas;
  if (P > 32 * kPerLane) P = 32 * kPerLane;
  if (P < 1) P = 1;
  int R = (r + P - 1) / P;
  P = (r + R - 1) / R;
  size_t ubytes = (size_t)((w + 1) & ~1) * sizeof(T);
  size_t sbytes = ubytes + (size_t)R * w * sizeof(T);
  int use_smem = sbytes + 1024 <= (size_t)optin - 2048;
  size_t dyn = use_smem ? sbytes : ubytes;
  cudaFuncSetAttribute(panel_lu_k<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_lu_k<T>, kThreads, dyn);
  if (per_sm * sms < P) return (int)cudaErrorCooperativeLaunchTooLarge;
  char *ws = nullptr;
  int rc = noalloc_scratch(&ws);
  if (rc) return rc;
  // the record slots must start at zero (their generation bits); the
  // candidate rows are written before they are read, so the last call's
  // contents are harmless
  const Layout lay = layout<T>(P, w);
  if (lay.total > kNoAllocBytes) return (int)cudaErrorInvalidValue;
  e = cudaMemsetAsync(ws, 0, lay.rec_bytes, s);
  if (e != cudaSuccess) return (int)e;
  unsigned long long *rec = (unsigned long long *)ws;
  T *cand_row = (T *)(ws + lay.off_row);
  T *top_row = (T *)(ws + lay.off_top);
  int *zero_info = nullptr;
  int row_base = 0;
  void *args[] = {&A,        &lda,      &r,   &w,        &R,        &use_smem, &piv,
                  &status,   &zero_info, &row_base, &rec, &cand_row, &top_row};
  e = cudaLaunchCooperativeKernel((void *)panel_lu_k<T>, dim3(P), dim3(kThreads), args, dyn, s);
  pla_k_count(1);
  return (int)e;
}

}  // namespace

// See include/pla_b200.h.  No cudaMalloc, cudaFree or allocating library call
// is made on this path.
extern "C" int PLA_B200_lu_panel_noalloc(MPI_Datatype datatype, int m, int w, void *A, int lda,
                                         int *pivots, int *status, void *stream) {
  if (datatype != MPI_DOUBLE && datatype != MPI_FLOAT)
    return pla::fail("PLA_B200_lu_panel_noalloc: datatype must be MPI_DOUBLE or MPI_FLOAT",
                     __LINE__, __FILE__);
  if (m < 0 || w < 0 || lda < (m > 1 ? m : 1))
    return pla::fail("PLA_B200_lu_panel_noalloc: invalid m, w or lda", __LINE__, __FILE__);
  if (m == 0 || w == 0) return PLA_SUCCESS;
  if (w > m)
    return pla::fail("PLA_B200_lu_panel_noalloc: the panel has more columns than rows",
                     __LINE__, __FILE__);
  if (w > kNoAllocWidth)
    return pla::fail("PLA_B200_lu_panel_noalloc: panel wider than 128 columns, the limit of "
                     "its fixed workspace",
                     __LINE__, __FILE__);
  if (!A || !pivots || !status)
    return pla::fail("PLA_B200_lu_panel_noalloc: null pointer", __LINE__, __FILE__);
  cudaStream_t s = (cudaStream_t)stream;
  int e = datatype == MPI_DOUBLE
              ? launch_noalloc<double>(m, w, (double *)A, lda, pivots, status, s)
              : launch_noalloc<float>(m, w, (float *)A, lda, pivots, status, s);
  if (e) return pla::cuda_fail((cudaError_t)e, __LINE__, __FILE__);
  return PLA_SUCCESS;
}
