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
// Exchange, one round per column, with no grid barrier and no memory fence:
// every CTA publishes a record -- its best candidate (|value|, row) -- the
// candidate's whole row, and, from the owner of the diagonal row, that row.
// Every 32-bit datum travels in a 64-bit word together with the tag of its
// launch and column, so a reader that polls a word until the tag matches has
// the datum, whatever order the writer's stores became visible in.  Warp 0
// of every CTA polls all records in one batch of loads per round and picks
// the winner; then the CTA polls the winner's row and the diagonal row.  All
// CTAs pick the same winner from the same records.  Records alternate
// between two slots by column parity: a CTA can only overwrite a slot after
// every CTA has published the next column, that is after every CTA has
// finished reading the slot.
//
// Lookahead inside the panel: after the pivot of column j a CTA updates only
// column j + 1 of its rows, publishes the record of column j + 1 (its rows
// carry the rest of the update, computed with the same fma as below, so the
// published values are bitwise those the CTA stores later), and then updates
// its remaining columns while the other CTAs publish.  Every wait is bounded;
// on timeout the kernel records PLA_K_TIMEOUT and exits.
#include <cuda.h>

#include <atomic>
#include <climits>
#include <cstdio>
#include <mutex>

#include "pla_internal.h"
#include "pla_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr long kSpinLimit = 4000000;  // polls before giving up (~1-2 s)
constexpr int kPerLane = 5;           // records per lane of the gathering warp: P <= 160
constexpr int kMaxWidth = 256;        // columns per launch: the column is 8 bits of the tag

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Published words: the high 32 bits carry the tag of the column they belong
// to, (launch sequence << 8) | column, the low 32 bits one 32-bit datum (a
// float, half of a double, or a row index).  A 64-bit relaxed load sees a
// whole word, so a reader that finds the expected tag has the datum of this
// launch and column, whatever order the writer's stores became visible in.
__device__ __forceinline__ unsigned long long word(unsigned tag, unsigned bits) {
  return ((unsigned long long)tag << 32) | bits;
}
template <typename T>
__device__ __forceinline__ unsigned half_bits(T v, int h) {
  if constexpr (sizeof(T) == 8) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return h ? (unsigned)(b >> 32) : (unsigned)b;
  } else {
    return __float_as_uint(v);
  }
}
// store element v as sizeof(T) / 4 tagged words at p
template <typename T>
__device__ __forceinline__ void put(unsigned long long *p, T v, unsigned tag) {
#pragma unroll
  for (int h = 0; h < (int)(sizeof(T) / 4); h++) st_relaxed64(p + h, word(tag, half_bits(v, h)));
}

// Pivot candidates compare as unsigned integer keys: key(x) = bits(|x|) + 1,
// and 0 for NaN (and for "no candidate").  For |x| >= 0 the bit pattern
// orders like the value, so (larger key, then smaller row) picks the pivot of
// (larger |x|, then smaller row) -- the first index of the maximum, as
// idamax and BLAS1/PLA_Iamax.c:108-111 -- and a NaN never wins.  Integer
// comparisons keep the reductions below exact total orders: with
// floating-point comparisons a NaN that slipped into a reduction compares
// false both ways and lanes could end with different winners.
template <typename T>
struct KeyOf {
  using K = unsigned;
};
template <>
struct KeyOf<double> {
  using K = unsigned long long;
};
template <typename T>
__device__ __forceinline__ typename KeyOf<T>::K pivot_key(T x) {
  if constexpr (sizeof(T) == 8) {
    const unsigned long long b =
        (unsigned long long)__double_as_longlong(x) & 0x7fffffffffffffffull;
    return b > 0x7ff0000000000000ull ? 0ull : b + 1ull;
  } else {
    const unsigned b = __float_as_uint(x) & 0x7fffffffu;
    return b > 0x7f800000u ? 0u : b + 1u;
  }
}
template <typename K>
__device__ __forceinline__ bool key_better(K a, int ai, K b, int bi) {
  return a > b || (a == b && ai < bi);
}

// CTA argmax with one barrier: every lane of every warp ends with the same
// (key, index); the lanes past the warp count hold the empty candidate.
template <typename K>
__device__ __forceinline__ void block_argmax(K &v, int &i, K *sv, int *si) {
  const int l = threadIdx.x & 31;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const K ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (key_better(ov, oi, v, i)) { v = ov; i = oi; }
  }
  if (l == 0) {
    sv[threadIdx.x >> 5] = v;
    si[threadIdx.x >> 5] = i;
  }
  __syncthreads();
  v = l < kThreads / 32 ? sv[l] : K(0);
  i = l < kThreads / 32 ? si[l] : INT_MAX;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const K ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (key_better(ov, oi, v, i)) { v = ov; i = oi; }
  }
}

// Workspace, in tagged words (NW = sizeof(T) / 4 words per element), two
// slots by column parity:
//   rec  [2][P][NW + 1]  pivot key of each CTA's candidate, then its row index
//   crow [2][P][w][NW]   each candidate's row
//   trow [2][w][NW]      the diagonal row, published by its owner
//
// spin_limit bounds every poll (kSpinLimit in production).  mute_cta >= 0
// makes that CTA skip its stores of published words, so every wait on them
// runs out: the test of the timeout path uses it with a small spin_limit.
template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
panel_lu_k(T *A, long lda, int r, int w, int R, int use_smem, int *piv, int *status,
           int *zero_info, int row_base, unsigned seq, unsigned long long *rec,
           unsigned long long *crow, unsigned long long *trow, long spin_limit, int mute_cta) {
  constexpr int NW = (int)(sizeof(T) / 4), NR = NW + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using K = typename KeyOf<T>::K;
  __shared__ K s_v[32];
  __shared__ int s_i[32];
  __shared__ int s_p, s_q;

  const int P = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
  const bool mute = b == mute_cta;
  const int row0 = b * R;
  const int row1 = min(row0 + R, r);
  const int nrows = max(row1 - row0, 0);
  const int wp = (w + 1) & ~1;
  T *u = reinterpret_cast<T *>(smem_raw);  // the pivot row, w entries
  T *tr = u + wp;                          // the diagonal row as it was before the swap
  T *S;
  long lds;
  if (use_smem) {
    S = tr + wp;
    lds = R;
    for (long t = tid; t < (long)nrows * w; t += kThreads) {
      int i = (int)(t % nrows), c = (int)(t / nrows);
      S[i + c * lds] = A[(long)(row0 + i) + (long)c * lda];
    }
  } else {
    S = A + row0;
    lds = lda;
  }
  __syncthreads();
  const unsigned tag0 = (seq & 0xffffffu) << 8;
#define E(i, c) S[(long)(i) + (long)(c) * lds]

  // Publish the record of column `col`.  With `pend` the rows still owe the
  // rank-1 update of pivot col - 1 in the columns right of col (multiplier
  // E(., col - 1), pivot row u): the published rows include it.
  auto publish = [&](int col, bool pend) {
    const int par = col & 1;
    const unsigned tag = tag0 | (unsigned)col;
    K best = 0;
    int bidx = INT_MAX;
    const int lo = max(col - row0, 0);
    for (int li = lo + tid; li < nrows; li += kThreads) {
      const K v = pivot_key(E(li, col));
      if (v != 0 && key_better(v, row0 + li, best, bidx)) { best = v; bidx = row0 + li; }
    }
    block_argmax(best, bidx, s_v, s_i);
    auto row_val = [&](int li, int c) -> T {
      const T e = E(li, c);
      return (pend && c > col) ? fma(E(li, col - 1), -u[c], e) : e;
    };
    if (bidx != INT_MAX && !mute)
      for (int c = tid; c < w; c += kThreads)
        put<T>(crow + (((long)par * P + b) * w + c) * NW, row_val(bidx - row0, c), tag);
    if (col >= row0 && col < row1 && !mute)
      for (int c = tid; c < w; c += kThreads)
        put<T>(trow + ((long)par * w + c) * NW, row_val(col - row0, c), tag);
    if (tid == 0 && !mute) {
      unsigned long long *rp = rec + ((long)par * P + b) * NR;
      const bool none = bidx == INT_MAX;  // no candidate: every entry is NaN
      const K kv = none ? K(0) : best;
#pragma unroll
      for (int h = 0; h < NW; h++) st_relaxed64(rp + h, word(tag, (unsigned)(kv >> (32 * h))));
      st_relaxed64(rp + NW, word(tag, (unsigned)(none ? INT_MAX : bidx)));
    }
    __syncthreads();  // the rows above are read before the update below writes them
  };

  // Gather column `col`: warp 0 polls every CTA's record (one batch of loads
  // per poll) and picks the winner; then all threads poll the winner's row
  // into u and the diagonal row into tr.  False when a wait gave up.
  auto gather = [&](int col) -> bool {
    const int par = col & 1;
    const unsigned tag = tag0 | (unsigned)col;
    bool ok = true;
    if (tid < 32) {
      unsigned long long wv[kPerLane][NR];
      bool done[kPerLane];
#pragma unroll
      for (int i = 0; i < kPerLane; i++) {
        done[i] = tid + 32 * i >= P;
#pragma unroll
        for (int h = 0; h < NR; h++) wv[i][h] = 0;
      }
      for (long spins = 0;; spins++) {
#pragma unroll
        for (int i = 0; i < kPerLane; i++)
          if (!done[i]) {
            const unsigned long long *rp = rec + ((long)par * P + tid + 32 * i) * NR;
#pragma unroll
            for (int h = 0; h < NR; h++) wv[i][h] = ld_relaxed64(rp + h);
          }
        bool all = true;
#pragma unroll
        for (int i = 0; i < kPerLane; i++)
          if (!done[i]) {
            bool v = true;
#pragma unroll
            for (int h = 0; h < NR; h++) v = v && (unsigned)(wv[i][h] >> 32) == tag;
            if (v) done[i] = true;
            else all = false;
          }
        if (all) break;
        if (spins > spin_limit || *(volatile int *)status != PLA_K_OK) {
          ok = false;
          break;
        }
      }
      K bv = 0;
      int bi = INT_MAX, bq = 0;
#pragma unroll
      for (int i = 0; i < kPerLane; i++) {
        const int q = tid + 32 * i;
        if (q >= P) continue;
        K v = (K)(unsigned)wv[i][0];
        if constexpr (NW == 2) v |= (K)(unsigned)wv[i][1] << 32;
        const int ix = (int)(unsigned)wv[i][NW];
        if (v != 0 && key_better(v, ix, bv, bi)) { bv = v; bi = ix; bq = q; }
      }
      for (int o = 16; o; o >>= 1) {
        K ov = __shfl_down_sync(0xffffffffu, bv, o);
        int oi = __shfl_down_sync(0xffffffffu, bi, o);
        int oq = __shfl_down_sync(0xffffffffu, bq, o);
        if (key_better(ov, oi, bv, bi)) { bv = ov; bi = oi; bq = oq; }
      }
      if (tid == 0) {
        s_p = bi;
        s_q = bq;
      }
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
      return false;
    }
    // A column of NaNs has no candidate (NaN never compares greater): row col
    // stays its own pivot, and u is the diagonal row.
    const bool none = s_p == INT_MAX;
    const int q = s_q, half = w * NW;
    unsigned *ub = reinterpret_cast<unsigned *>(u), *tb = reinterpret_cast<unsigned *>(tr);
    for (int e = tid; e < 2 * half; e += kThreads) {
      const bool top = e >= half || none;
      const int k = e < half ? e : e - half;
      const unsigned long long *src =
          top ? trow + (long)par * half + k : crow + ((long)par * P + q) * half + k;
      unsigned long long v = 0;
      for (long spins = 0;; spins++) {
        v = ld_relaxed64(src);
        if ((unsigned)(v >> 32) == tag) break;
        if (spins > spin_limit || *(volatile int *)status != PLA_K_OK) {
          ok = false;
          break;
        }
      }
      (e < half ? ub : tb)[k] = (unsigned)v;
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
      return false;
    }
    return true;
  };

  publish(0, false);
  for (int j = 0; j < w; j++) {
    if (!gather(j)) return;
    const int p = s_p == INT_MAX ? j : s_p;
    // the interchange of rows j and p over the panel width
    if (j >= row0 && j < row1)
      for (int c = tid; c < w; c += kThreads) E(j - row0, c) = u[c];
    if (p != j && p >= row0 && p < row1)
      for (int c = tid; c < w; c += kThreads) E(p - row0, c) = tr[c];
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

// workspace layout for P CTAs and width w, in tagged words
struct Layout {
  size_t off_crow, off_trow, words;
};
template <typename T>
Layout layout(int P, int w) {
  const size_t nw = sizeof(T) / 4;
  Layout l;
  l.off_crow = (size_t)2 * P * (nw + 1);
  l.off_trow = l.off_crow + (size_t)2 * P * w * nw;
  l.words = l.off_trow + (size_t)2 * w * nw;
  return l;
}

// Launch sequence number for the tags: never 0 in its low 24 bits, so no tag
// matches a zeroed word.  A tag carries only those 24 bits, so once the
// sequence has wrapped a word left by a launch 2^24 launches earlier (with a
// larger grid or width than any launch since) could carry a current tag.  The
// bits above 24 number the epoch: every workspace is cleared before its first
// launch of each epoch (and before its first launch at all), so a word a
// reader accepts was written in the current epoch, that is by this launch.
std::atomic<unsigned> g_seq{0};
unsigned next_seq() {
  unsigned v;
  do v = ++g_seq;
  while ((v & 0xffffffu) == 0);
  return v;
}
constexpr unsigned kNoEpoch = 0xffffffffu;  // a workspace never cleared
inline unsigned epoch_of(unsigned seq) { return seq >> 24; }

struct Workspace {
  void *ptr = nullptr;
  size_t bytes = 0;
  unsigned epoch = kNoEpoch;  // epoch it was last cleared in
};
Workspace g_ws;

void *workspace(size_t bytes) {
  if (g_ws.bytes >= bytes) return g_ws.ptr;
  if (g_ws.ptr) cudaFree(g_ws.ptr);
  g_ws.ptr = nullptr;
  g_ws.bytes = 0;
  g_ws.epoch = kNoEpoch;
  if (cudaMalloc(&g_ws.ptr, bytes) != cudaSuccess) return nullptr;
  g_ws.bytes = bytes;
  return g_ws.ptr;
}

// spin limit and muted CTA of the next launch (test hook; see panel_lu_k)
long g_test_spin_limit = 0;
int g_test_mute_cta = -1;

int g_sms = 0, g_smem_optin = 0;

template <typename T>
int launch(int r, int w, void *A, long lda, int *piv, int *status, int *zero_info, int row_base,
           int max_ctas, cudaStream_t s) {
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
  if (max_ctas > 0 && P > max_ctas) P = max_ctas;
  if (P < 1) P = 1;
  int R = (r + P - 1) / P;
  P = (r + R - 1) / R;
  size_t ubytes = (size_t)2 * ((w + 1) & ~1) * sizeof(T);  // u and tr
  size_t sbytes = ubytes + (size_t)R * w * sizeof(T);
  int use_smem = sbytes + 1024 <= (size_t)g_smem_optin - 2048;
  size_t dyn = use_smem ? sbytes : ubytes;
  cudaFuncSetAttribute(panel_lu_k<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_lu_k<T>, kThreads, dyn);
  if (per_sm * g_sms < P) return (int)cudaErrorCooperativeLaunchTooLarge;
  const Layout lay = layout<T>(P, w);
  unsigned long long *ws =
      (unsigned long long *)workspace(lay.words * sizeof(unsigned long long));
  if (!ws) return (int)cudaErrorMemoryAllocation;
  unsigned long long *rec = ws, *crow = ws + lay.off_crow, *trow = ws + lay.off_trow;
  unsigned seq = next_seq();
  if (g_ws.epoch != epoch_of(seq)) {
    cudaError_t ce = cudaMemsetAsync(g_ws.ptr, 0, g_ws.bytes, s);
    if (ce != cudaSuccess) return (int)ce;
    g_ws.epoch = epoch_of(seq);
  }
  long spin_limit = g_test_spin_limit > 0 ? g_test_spin_limit : kSpinLimit;
  int mute_cta = g_test_mute_cta;
  g_test_spin_limit = 0;
  g_test_mute_cta = -1;
  T *Ap = (T *)A;
  void *args[] = {&Ap,      &lda, &r,   &w,    &R,    &use_smem,   &piv,     &status,
                  &zero_info, &row_base, &seq, &rec, &crow, &trow, &spin_limit, &mute_cta};
  cudaError_t e =
      cudaLaunchCooperativeKernel((void *)panel_lu_k<T>, dim3(P), dim3(kThreads), args, dyn, s);
  pla_k_count(1);
  return (int)e;
}

}  // namespace

extern "C" int pla_k_lu_panel_ex(int dt, int r, int w, void *A, long lda, int *piv, int *status,
                                 int *zero_info, int row_base, int max_ctas, cudaStream_t s) {
  if (r <= 0 || w <= 0) return 0;
  if (w > r || w > kMaxWidth) return (int)cudaErrorInvalidValue;
  if (dt == MPI_DOUBLE)
    return launch<double>(r, w, A, lda, piv, status, zero_info, row_base, max_ctas, s);
  if (dt == MPI_FLOAT)
    return launch<float>(r, w, A, lda, piv, status, zero_info, row_base, max_ctas, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int pla_k_lu_panel(int dt, int r, int w, void *A, long lda, int *piv, int *status,
                              int *zero_info, int row_base, cudaStream_t s) {
  return pla_k_lu_panel_ex(dt, r, w, A, lda, piv, status, zero_info, row_base, 0, s);
}

// Test hooks, not part of the public interface: read or move the launch
// sequence (to make the tag wrap), and give the next panel launch a spin limit
// and a CTA that publishes nothing (to make its waits run out).
extern "C" unsigned pla_k_panel_sequence(void) { return g_seq.load(); }
extern "C" void pla_k_panel_set_sequence(unsigned v) { g_seq.store(v); }
extern "C" void pla_k_panel_test_timeout(long spin_limit, int mute_cta) {
  g_test_spin_limit = spin_limit;
  g_test_mute_cta = mute_cta;
}

namespace {
void release_noalloc();
}

extern "C" void pla_kernels_release(void) {
  if (g_ws.ptr) cudaFree(g_ws.ptr);
  g_ws.ptr = nullptr;
  g_ws.bytes = 0;
  g_ws.epoch = kNoEpoch;
  release_noalloc();
  pla_tslu_release();
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
// most kNoAllocWidth columns in double precision (about 667 KB); every GPU
// that loads the library keeps it until the process exits.  Every call shares
// it, so calls whose kernels overlap on the GPU (on different streams, or from
// different host threads) race.
namespace {
constexpr int kNoAllocCtas = 160;
constexpr int kNoAllocWidth = 128;
// the double-precision layout at the limits, in 8-byte words; a float panel
// needs less
constexpr size_t kNoAllocBytes =
    8 * ((size_t)2 * kNoAllocCtas * 3 + (size_t)2 * kNoAllocCtas * kNoAllocWidth * 2 +
         (size_t)2 * kNoAllocWidth * 2);
}  // namespace

static __device__ __align__(256) unsigned char g_panel_scratch[kNoAllocBytes];

namespace {

// Per device: the array's device address, the context it was looked up in,
// and the sequence epoch the array was last cleared in.
struct NoAllocSlot {
  void *addr = nullptr;
  unsigned long long ctx_id = 0;
  unsigned epoch = kNoEpoch;
};
std::mutex g_noalloc_mu;
NoAllocSlot g_noalloc[128];

void release_noalloc() {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  for (auto &s : g_noalloc) s = NoAllocSlot{};
}

// The array's device address on the current device (the host-side name of
// the array is only a stand-in), looked up on the first call in each context:
// after cudaDeviceReset the device has a new primary context, the module is
// loaded again and the old address is stale, so the cache is keyed by the
// context's unique id.  *clear is set when the array must be zeroed before
// the launch with sequence `seq` (a new context, or a new sequence epoch).
int noalloc_scratch(unsigned seq, char **out, bool *clear) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= 128) return (int)cudaErrorInvalidDevice;
  // driver entry points resolved at run time: the library does not link libcuda
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void *p1 = nullptr, *p2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p1, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &p2, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess)
      return (int)cudaErrorSymbolNotFound;
    get_current = (GetCurrent)p1;
    get_id = (GetId)p2;
  }
  auto context_id = [](unsigned long long *id) -> bool {
    CUcontext ctx = nullptr;
    return get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, id) == CUDA_SUCCESS;
  };
  unsigned long long id = 0;
  const bool known = context_id(&id);  // false before the runtime's first use of the device
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot &s = g_noalloc[dev];
  if (!known || !s.addr || s.ctx_id != id) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_panel_scratch);  // loads the module if needed
    if (e != cudaSuccess) return (int)e;
    if (!context_id(&id)) return (int)cudaErrorDeviceUninitialized;
    s.addr = p;
    s.ctx_id = id;
    s.epoch = kNoEpoch;
  }
  *clear = s.epoch != epoch_of(seq);
  s.epoch = epoch_of(seq);
  *out = (char *)s.addr;
  return 0;
}

template <typename T>
int launch_noalloc(int r, int w, T *A, long lda, int *piv, int *status, int *zero_info,
                   cudaStream_t s) {
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
  size_t ubytes = (size_t)2 * ((w + 1) & ~1) * sizeof(T);  // u and tr
  size_t sbytes = ubytes + (size_t)R * w * sizeof(T);
  int use_smem = sbytes + 1024 <= (size_t)optin - 2048;
  size_t dyn = use_smem ? sbytes : ubytes;
  cudaFuncSetAttribute(panel_lu_k<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, panel_lu_k<T>, kThreads, dyn);
  if (per_sm * sms < P) return (int)cudaErrorCooperativeLaunchTooLarge;
  const Layout lay = layout<T>(P, w);
  if (lay.words * sizeof(unsigned long long) > kNoAllocBytes) return (int)cudaErrorInvalidValue;
  unsigned seq = next_seq();
  char *ws = nullptr;
  bool clear = false;
  int rc = noalloc_scratch(seq, &ws, &clear);
  if (rc) return rc;
  // Every word a call reads carries the call's own tag, so what earlier calls
  // left in the array is never taken for data -- within one sequence epoch.
  // The array is zeroed at the first call of each epoch and of each context.
  if (clear) {
    e = cudaMemsetAsync(ws, 0, kNoAllocBytes, s);
    if (e != cudaSuccess) return (int)e;
  }
  unsigned long long *wsw = (unsigned long long *)ws;
  unsigned long long *rec = wsw, *crow = wsw + lay.off_crow, *trow = wsw + lay.off_trow;
  int row_base = 0;
  long spin_limit = kSpinLimit;
  int mute_cta = -1;
  void *args[] = {&A,      &lda,      &r,    &w,   &R,    &use_smem, &piv,       &status,
                  &zero_info, &row_base, &seq, &rec, &crow, &trow,     &spin_limit, &mute_cta};
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
  // status[1] receives the first exact zero pivot
  int e = datatype == MPI_DOUBLE
              ? launch_noalloc<double>(m, w, (double *)A, lda, pivots, status, status + 1, s)
              : launch_noalloc<float>(m, w, (float *)A, lda, pivots, status, status + 1, s);
  if (e) return pla::cuda_fail((cudaError_t)e, __LINE__, __FILE__);
  return PLA_SUCCESS;
}
