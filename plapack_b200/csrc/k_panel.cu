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
// works in place in global memory (the panel is L2-resident).  Each column
// costs one grid barrier: before it, every CTA publishes its best candidate
// (|value|, row, the whole row) and the owner of row j publishes row j, so
// after it every CTA can perform the swap and the update without reading a
// row another CTA may be writing.  Candidate buffers alternate between two
// slots by column parity.  The barrier is a monotonically increasing counter
// with a bounded spin; on timeout the kernel records PLA_K_TIMEOUT and exits.
#include <climits>
#include <cstdio>
#include <mutex>

#include "pla_internal.h"
#include "pla_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr long kSpinLimit = 4000000;  // ~0.5-1 s of polling, then give up

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// returns false when the wait timed out (status already recorded)
__device__ bool grid_barrier(unsigned *bar, unsigned target, int *status, int *s_abort) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    long spins = 0;
    while (ld_acquire(bar) < target) {
      if (++spins > kSpinLimit || *(volatile int *)status != PLA_K_OK) {
        atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
        *s_abort = 1;
        break;
      }
      __nanosleep(20);
    }
    __threadfence();
  }
  __syncthreads();
  return *s_abort == 0;
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

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
panel_lu_k(T *A, long lda, int r, int w, int R, int use_smem, int *piv, int *status,
           int *zero_info, int row_base, unsigned *bar, T *cand_abs, int *cand_idx, T *cand_row,
           T *top_row) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ T s_v[32];
  __shared__ int s_i[32];
  __shared__ int s_abort, s_p;

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

  unsigned phase = 0;
  // publish the candidate for a column `col` into slot `par`
  auto publish = [&](int col, int par) {
    T best = T(-1);
    int bidx = INT_MAX;
    int lo = max(col - row0, 0);
    for (int li = lo + tid; li < nrows; li += kThreads) {
      T v = fabs(E(li, col));
      if (better(v, row0 + li, best, bidx)) { best = v; bidx = row0 + li; }
    }
    block_argmax(best, bidx, s_v, s_i);
    if (tid == 0) {
      cand_abs[par * P + b] = best;
      cand_idx[par * P + b] = bidx;
    }
    if (bidx != INT_MAX)
      for (int c = tid; c < w; c += kThreads) cand_row[((long)par * P + b) * w + c] = E(bidx - row0, c);
    if (col >= row0 && col < row1)
      for (int c = tid; c < w; c += kThreads) top_row[(long)par * w + c] = E(col - row0, c);
  };

  publish(0, 0);
  if (!grid_barrier(bar, ++phase * P, status, &s_abort)) return;

  for (int j = 0; j < w; j++) {
    const int par = j & 1;
    // winner over all CTAs' candidates
    if (tid < 32) {
      T bv = T(-1);
      int bi = INT_MAX, bb = 0;
      for (int q = tid; q < P; q += 32) {
        // other CTAs wrote these: read through L2, never a stale L1 line
        T v = __ldcg(&cand_abs[par * P + q]);
        int ix = __ldcg(&cand_idx[par * P + q]);
        if (better(v, ix, bv, bi)) { bv = v; bi = ix; bb = q; }
      }
      for (int o = 16; o; o >>= 1) {
        T ov = __shfl_down_sync(0xffffffffu, bv, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        int ob = __shfl_down_sync(0xffffffffu, bb, o);
        if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; bb = ob; }
      }
      if (tid == 0) { s_p = bi; s_i[0] = bb; }
    }
    __syncthreads();
    // A column of NaNs has no candidate (NaN never compares greater): keep
    // row j as its own pivot, whose contents the owner of row j published.
    const bool none = s_p == INT_MAX;
    const int p = none ? j : s_p, wb = s_i[0];
    for (int c = tid; c < w; c += kThreads)
      u[c] = none ? __ldcg(&top_row[(long)par * w + c])
                  : __ldcg(&cand_row[((long)par * P + wb) * w + c]);
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
    // scale by the reciprocal, then the rank-1 update of the columns to the right
    const T inv = T(1) / u[j];
    const int lo = max(j + 1 - row0, 0);
    for (int li = lo + tid; li < nrows; li += kThreads) {
      T l = E(li, j) * inv;
      E(li, j) = l;
      for (int c = j + 1; c < w; c++) E(li, c) = fma(l, -u[c], E(li, c));
    }
    if (j + 1 < w) {
      __syncthreads();
      publish(j + 1, par ^ 1);
      if (!grid_barrier(bar, ++phase * P, status, &s_abort)) return;
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
  // workspace: barrier | cand_abs[2P] | cand_idx[2P] | cand_row[2P*w] | top_row[2w]
  size_t off_abs = 256, off_idx = off_abs + 2 * P * sizeof(T);
  size_t off_row = (off_idx + 2 * P * sizeof(int) + 255) & ~(size_t)255;
  size_t off_top = off_row + (size_t)2 * P * w * sizeof(T);
  size_t total = off_top + (size_t)2 * w * sizeof(T);
  char *ws = (char *)workspace(total);
  if (!ws) return (int)cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemsetAsync(ws, 0, 256, s);
  if (e) return (int)e;
  unsigned *bar = (unsigned *)ws;
  T *cand_abs = (T *)(ws + off_abs);
  int *cand_idx = (int *)(ws + off_idx);
  T *cand_row = (T *)(ws + off_row);
  T *top_row = (T *)(ws + off_top);
  T *Ap = (T *)A;
  void *args[] = {&Ap, &lda, &r, &w, &R, &use_smem, &piv, &status, &zero_info, &row_base, &bar,
                  &cand_abs, &cand_idx, &cand_row, &top_row};
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
// kernel's workspace -- the grid-barrier counter and the per-CTA pivot
// candidates -- lives in the fixed device array below instead of memory the
// library allocates.  The array holds the workspace of at most kNoAllocCtas
// CTAs for panels of at most kNoAllocWidth columns in double precision
// (about 334 KB); every GPU that loads the library keeps it until the process
// exits.  Every call shares it, so calls whose kernels overlap on the GPU (on
// different streams, or from different host threads) race.
namespace {
constexpr int kNoAllocCtas = 160;
constexpr int kNoAllocWidth = 128;
constexpr size_t kNoAllocAbs = 256;  // bytes [0, 256): the barrier counter
constexpr size_t kNoAllocIdx = kNoAllocAbs + 2 * kNoAllocCtas * sizeof(double);
constexpr size_t kNoAllocRow =
    (kNoAllocIdx + 2 * kNoAllocCtas * sizeof(int) + 255) & ~(size_t)255;
constexpr size_t kNoAllocTop =
    kNoAllocRow + (size_t)2 * kNoAllocCtas * kNoAllocWidth * sizeof(double);
constexpr size_t kNoAllocBytes = kNoAllocTop + (size_t)2 * kNoAllocWidth * sizeof(double);
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
  // the barrier counter must start at zero; the candidate slots are written
  // before they are read, so the last call's contents are harmless
  e = cudaMemsetAsync(ws, 0, kNoAllocAbs, s);
  if (e != cudaSuccess) return (int)e;
  unsigned *bar = (unsigned *)ws;
  T *cand_abs = (T *)(ws + kNoAllocAbs);
  int *cand_idx = (int *)(ws + kNoAllocIdx);
  T *cand_row = (T *)(ws + kNoAllocRow);
  T *top_row = (T *)(ws + kNoAllocTop);
  int *zero_info = nullptr;
  int row_base = 0;
  void *args[] = {&A,   &lda,        &r,         &w,        &R,         &use_smem,
                  &piv, &status,     &zero_info, &row_base, &bar,       &cand_abs,
                  &cand_idx, &cand_row, &top_row};
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
