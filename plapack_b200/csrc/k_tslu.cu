// Tournament pivoting for the fp32 sub-panels of the mixed-precision LU
// (communication-avoiding LU, "TSLU": Grigori, Demmel and Xiang, SIAM J.
// Matrix Anal. Appl. 32 (2011)).  The mixed LU's pivots need not be the
// reference's -- it only preconditions an FP64 refinement -- so its panel
// trades PLA_LU_mv's one global pivot search per column (SOLVERS/LU/
// PLA_LU_mv.c:52-82, one grid-wide exchange round per column) for a
// reduction tree over the panel's rows with no exchange inside a column:
//
//   tslu_select_k  every CTA factors its own block of rows (LU with partial
//                  pivoting, in registers, one barrier per column) and keeps
//                  the w rows its pivots chose.  The candidate sets of
//                  kGroup CTAs meet in the last of them to finish (an atomic
//                  counter: no CTA ever waits for another), which factors
//                  their ORIGINAL rows again and keeps w; and so on up to one
//                  set.  The root keeps the rows in the order its pivots chose
//                  them, the LU of those rows (L11 \ U11) and U11's inverse,
//                  the interchanges that bring them to the top as sequential
//                  swaps (the reference's offset encoding, so every later
//                  step of the loop is unchanged), and a copy of the panel's
//                  original top rows.
//   tslu_apply_k   the panel without further pivoting: rows 0..w-1 get
//                  L11 \ U11, every other row i gets (P A)_i inv(U11),
//                  reading a displaced row from the copy.
//
// A CTA factors at most kMaxCand candidate rows per pass (kRows per thread);
// taller blocks run several passes, carrying the w rows kept so far.  No
// kernel here waits on another CTA, so none can hang; the counters a group
// used are reset by the CTA that finished it.  The column loop is not
// unrolled (an unrolled loop overflowed the instruction cache); the rows stay
// in registers, shifted one column left per step so every index is static.
#include <climits>
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

#include "pla_internal.h"
#include "pla_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kW = 32;                  // sub-panel width (columns)
// Candidate rows per thread.  Each tree level costs w column steps, each
// step's time grows with the rows a thread updates: measured at 32768 x 32 on
// 72 CTAs, 2 rows (3 levels) took 92 us, 4 rows (2 levels) 99 us.
constexpr int kRows = 2;
constexpr int kMaxCand = kRows * kThreads;  // candidate rows one pass factors
constexpr int kGroup = kMaxCand / kW;       // candidate sets merged per tree node (16)

// Candidate order: larger |value| first (bits(|x|) + 2; NaN 1; 0 = none), then
// the smaller row.
__device__ __forceinline__ unsigned cand_key(float x) {
  const unsigned b = __float_as_uint(x) & 0x7fffffffu;
  return b > 0x7f800000u ? 1u : b + 2u;
}

struct SelectSmem {
  // each warp's best candidate, by column parity: its order key (candidate
  // key above the complement of its row; 0 = none), candidate slot,
  // reciprocal pivot and values from the current column on
  unsigned long long wkey[2][kWarps];
  int wslot[2][kWarps];
  float winv[2][kWarps];
  __align__(16) float wrow[2][kWarps][kW];
  int ids[kMaxCand];    // candidate rows of the current pass
  int keep[kW];         // rows kept, in pivot order
  int kslot[kW];        // their candidate slots
  float rows[kW * kW];  // root: L11 \ U11 (row-major)
};
// the multipliers of every candidate, column by column (hist[j * kMaxCand + slot])
constexpr size_t kHistBytes = (size_t)kW * kMaxCand * sizeof(float);

// the largest 64-bit order key over the warp (two 32-bit reductions)
__device__ __forceinline__ unsigned long long warp_max_key(unsigned long long x) {
  const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)(x >> 32));
  const unsigned lo = __reduce_max_sync(0xffffffffu, (unsigned)(x >> 32) == hi ? (unsigned)x : 0u);
  return ((unsigned long long)hi << 32) | lo;
}

// Column steps j0 .. j1-1 of select_rows on a window of WIN columns: at step
// j the columns still to be eliminated sit at positions 0 .. w-1-j of v, so
// a window of WIN >= w - j positions carries every value that matters; the
// positions past it are never read again.  The arithmetic on each element is
// that of the full-width step, in the same order.
template <int WIN>
__device__ __forceinline__ void column_steps(int j0, int j1, int w, float (&v)[kRows][kW],
                                             const int (&id)[kRows], bool (&live)[kRows],
                                             SelectSmem &sm, float *hist, bool root) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = j0; j < j1; j++) {
    const int par = j & 1;
    unsigned long long mine = 0;
    int mh = 0;
#pragma unroll
    for (int h = 0; h < kRows; h++) {
      const unsigned long long key =
          live[h] ? ((unsigned long long)cand_key(v[h][0]) << 32) | (0xffffffffu - (unsigned)id[h])
                  : 0ull;
      if (key > mine) { mine = key; mh = h; }
    }
    const unsigned long long best = warp_max_key(mine);
    if (best != 0 && mine == best) {
      float4 *dst = reinterpret_cast<float4 *>(sm.wrow[par][warp]);
#pragma unroll
      for (int h = 0; h < kRows; h++)
        if (h == mh) {
#pragma unroll
          for (int q = 0; q < WIN / 4; q++)
            dst[q] = make_float4(v[h][4 * q], v[h][4 * q + 1], v[h][4 * q + 2], v[h][4 * q + 3]);
          sm.winv[par][warp] = 1.0f / v[h][0];
        }
      sm.wslot[par][warp] = tid + mh * kThreads;
    }
    if (lane == 0) sm.wkey[par][warp] = best;
    __syncthreads();
    // the winner over the warps, the same in every thread
    const unsigned long long e = lane < kWarps ? sm.wkey[par][lane] : 0ull;
    const unsigned long long g = warp_max_key(e);
    const int gw = __ffs(__ballot_sync(0xffffffffu, e == g)) - 1;
    const int gr = (int)(0xffffffffu - (unsigned)g);
    float u[WIN];
    {
      const float4 *src = reinterpret_cast<const float4 *>(sm.wrow[par][gw]);
#pragma unroll
      for (int q = 0; q < WIN / 4; q++) {
        const float4 f = src[q];
        u[4 * q] = f.x;
        u[4 * q + 1] = f.y;
        u[4 * q + 2] = f.z;
        u[4 * q + 3] = f.w;
      }
    }
    const float inv = sm.winv[par][gw];
#pragma unroll
    for (int h = 0; h < kRows; h++)
      if (live[h] && id[h] == gr) live[h] = false;
    if (tid == 0) {
      sm.keep[j] = gr;
      sm.kslot[j] = sm.wslot[par][gw];
    }
    if (root && tid < w - j) sm.rows[j * kW + j + tid] = sm.wrow[par][gw][tid];  // U part
#pragma unroll
    for (int h = 0; h < kRows; h++) {
      const float l = v[h][0] * inv;
      if (live[h]) {
        hist[j * kMaxCand + tid + h * kThreads] = l;
#pragma unroll
        for (int c = 1; c < WIN; c++) v[h][c - 1] = fmaf(-l, u[c], v[h][c]);
        v[h][WIN - 1] = 0.f;
      }
    }
  }
}

// LU with partial pivoting of the candidate rows ids[0..cnt) (entries < 0 are
// empty) of the column-major panel A (w columns), cnt <= kMaxCand.  Keeps
// k = min(candidates, w) rows: sm.keep[j] = the row chosen as pivot j; with
// `root`, sm.rows row j = the kept row j's factored values (row j of
// L11 \ U11).  All threads call it.
//
// Each thread holds kRows candidate rows in registers (slots tid + h kThreads),
// shifted left by one column after every step, so the current column is
// always v[h][0] and every index is static.  The multipliers shifted out go
// to `hist` (needed only for the rows the root keeps).  One barrier per
// column: every warp posts its best candidate (row, reciprocal pivot) before
// it, every thread picks the same winner after it.  Steps 8 q .. 8 q + 7 run
// on a window of 32 - 8 q columns (column_steps), so the multiply-adds follow
// the shrinking trailing part instead of all 32 positions.
__device__ __forceinline__ int select_rows(const float *__restrict__ A, long lda, int w, int cnt,
                                           SelectSmem &sm, float *hist, bool root) {
  const int tid = threadIdx.x;
  float v[kRows][kW];
  int id[kRows];
  bool live[kRows];
#pragma unroll
  for (int h = 0; h < kRows; h++) {
    const int s = tid + h * kThreads;
    id[h] = s < cnt ? sm.ids[s] : -1;
    live[h] = id[h] >= 0;
#pragma unroll
    for (int c = 0; c < kW; c++)
      v[h][c] = (live[h] && c < w) ? A[(long)id[h] + (long)c * lda] : 0.f;
  }
  int nlive = 0;
#pragma unroll
  for (int h = 0; h < kRows; h++) nlive += __syncthreads_count(live[h]);
  const int k = nlive < w ? nlive : w;
  static_assert(kW == 32, "the windows below assume 32-column sub-panels");
  column_steps<32>(0, min(k, 8), w, v, id, live, sm, hist, root);
  column_steps<24>(8, min(k, 16), w, v, id, live, sm, hist, root);
  column_steps<16>(16, min(k, 24), w, v, id, live, sm, hist, root);
  column_steps<8>(24, k, w, v, id, live, sm, hist, root);
  __syncthreads();  // keep[] complete; ids[] and wrow[] free for the caller
  if (root)  // the multipliers of the kept rows: row j's columns left of j
    for (int i = tid; i < k * kW; i += kThreads) {
      const int j = i / kW, c = i % kW;
      if (c < j) sm.rows[i] = hist[c * kMaxCand + sm.kslot[j]];
    }
  __syncthreads();
  return k;
}

// Outputs of the root, in the workspace (all sized for kW):
struct Out {
  int *piv;        // w offsets, the reference's encoding (row j <-> row j + piv[j])
  float *lu11;     // w x kW row-major: L11 \ U11
  float *uinv;     // kW x kW row-major: inv(U11) (upper)
  float *stage;    // w x kW row-major: the panel's original rows 0..w-1
  int *disp;       // [0] = count, then pairs (row i >= w, original top row q)
  int *zero_info;  // optional: 1-based first exact zero pivot + row_base
  int row_base;
};

// The tree: level 0 has P candidate sets (one per CTA), level l + 1 has
// ceil(n_l / kGroup); the sets of level l start at slot sum(n_0 .. n_{l-1}),
// and the group counters of level l at sum(ceil(n_0 / kGroup) ..).
__global__ void __launch_bounds__(kThreads, 1)
tslu_select_k(const float *__restrict__ A, long lda, int r, int w, int R, int *slots,
              unsigned *counters, Out out) {
  __shared__ SelectSmem sm;
  __shared__ int s_last;
  extern __shared__ __align__(16) float hist[];  // kHistBytes
  const int tid = threadIdx.x, P = gridDim.x;
  const int row0 = blockIdx.x * R, row1 = min(row0 + R, r);

  // one loop over every pass of this CTA: its own rows (in passes of at most
  // kMaxCand candidates), then, while it is the last of its group, the
  // group's candidate sets one level up
  int kept = 0, next = row0;
  int nsets = P, level_off = 0, cnt_off = 0, my = blockIdx.x;
  bool leaf = true;
  for (;;) {
    int cnt;
    bool final_pass;
    if (leaf) {
      const int take = min(row1 - next, kMaxCand - kept);
      for (int i = tid; i < kept; i += kThreads) sm.ids[i] = sm.keep[i];
      __syncthreads();
      for (int i = tid; i < take; i += kThreads) sm.ids[kept + i] = next + i;
      __syncthreads();
      next += take;
      cnt = kept + take;
      final_pass = next >= row1;
    } else {
      cnt = min(kGroup, nsets - my * kGroup) * kW;
      for (int i = tid; i < cnt; i += kThreads)
        sm.ids[i] = __ldcg(slots + ((long)level_off + my * kGroup) * kW + i);
      __syncthreads();
      level_off += nsets;
      cnt_off += (nsets + kGroup - 1) / kGroup;
      nsets = (nsets + kGroup - 1) / kGroup;
      final_pass = true;
    }
    const bool root = final_pass && nsets == 1;
    if (leaf && final_pass && !root && cnt <= w) {  // too few rows to choose among: keep all
      for (int i = tid; i < kW; i += kThreads) sm.keep[i] = i < cnt ? sm.ids[i] : -1;
      __syncthreads();
      kept = cnt;
    } else {
      kept = select_rows(A, lda, w, cnt, sm, hist, root);
    }
    if (!final_pass) continue;
    if (root) break;
    // publish this set; the last CTA of the group carries on with the group
    int *slot = slots + ((long)level_off + my) * kW;
    for (int i = tid; i < kW; i += kThreads) slot[i] = i < kept ? sm.keep[i] : -1;
    __threadfence();
    __syncthreads();
    const int group = my / kGroup;
    const int gsize = min(kGroup, nsets - group * kGroup);
    if (tid == 0) {
      const unsigned prev = atomicAdd(counters + cnt_off + group, 1u);
      s_last = prev == (unsigned)gsize - 1;
      if (s_last) counters[cnt_off + group] = 0;  // ready for the next launch
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    my = group;
    leaf = false;
  }

  // root.  The interchanges as sequential swaps: entries are positions
  // 0..w-1 (holding rows 0..w-1) and every kept row below w (holding itself);
  // swap j brings keep[j] from wherever it is to position j.
  __shared__ int e_pos[2 * kW], e_row[2 * kW];
  __shared__ int s_ne;
  if (tid == 0) {
    int ne = w;
    for (int i = 0; i < w; i++) { e_pos[i] = i; e_row[i] = i; }
    for (int j = 0; j < w; j++)
      if (sm.keep[j] >= w) { e_pos[ne] = sm.keep[j]; e_row[ne] = sm.keep[j]; ne++; }
    s_ne = ne;
  }
  __syncthreads();
  if (tid < 32) {
    const int ne = s_ne;
    for (int j = 0; j < w; j++) {
      const int want = sm.keep[j];
      const bool m0 = tid < ne && e_row[tid] == want;
      const bool m1 = tid + 32 < ne && e_row[tid + 32] == want;
      const unsigned b0 = __ballot_sync(0xffffffffu, m0), b1 = __ballot_sync(0xffffffffu, m1);
      const int e = b0 ? __ffs(b0) - 1 : 32 + __ffs(b1) - 1;
      const int p = e_pos[e];
      __syncwarp();
      if (tid == 0) {
        out.piv[j] = p - j;
        e_row[e] = e_row[j];
        e_row[j] = want;
      }
      __syncwarp();
    }
    if (tid == 0) {
      int nd = 0;
      for (int e = w; e < ne; e++)
        if (e_row[e] != e_pos[e]) {
          out.disp[1 + 2 * nd] = e_pos[e];
          out.disp[2 + 2 * nd] = e_row[e];
          nd++;
        }
      out.disp[0] = nd;
    }
  } else if (tid < 64) {
    // inv(U11), one column per lane: U y = e_c by back substitution
    const int c = tid - 32;
    float y[kW];
#pragma unroll
    for (int i = 0; i < kW; i++) y[i] = 0.f;
    if (c < w) {
#pragma unroll
      for (int i = kW - 1; i >= 0; i--) {
        if (i <= c) {
          float acc = i == c ? 1.f : 0.f;
#pragma unroll
          for (int q = i + 1; q < kW; q++)
            if (q <= c) acc = fmaf(-sm.rows[i * kW + q], y[q], acc);
          y[i] = acc * (1.0f / sm.rows[i * kW + i]);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kW; i++) out.uinv[i * kW + c] = y[i];
  }
  for (int i = tid; i < w * kW; i += kThreads) {
    const int j = i / kW, c = i % kW;
    out.lu11[i] = c < w ? sm.rows[i] : 0.f;
    out.stage[i] = c < w ? A[(long)j + (long)c * lda] : 0.f;
  }
  if (tid == 0 && out.zero_info)
    for (int j = 0; j < w; j++)
      if (sm.rows[j * kW + j] == 0.f) {
        atomicCAS(out.zero_info, 0, out.row_base + j + 1);
        break;
      }
}

// Rows 0..w-1 := L11 \ U11; row i >= w := (source row) inv(U11), the source
// being the staged original top row for a displaced row, else row i itself.
// x_c = sum_{k <= c} b_k inv(U11)_kc, accumulated in k order.
__global__ void __launch_bounds__(kThreads)
tslu_apply_k(float *__restrict__ A, long lda, int r, int w, const float *__restrict__ lu11,
             const float *__restrict__ uinv, const float *__restrict__ stage,
             const int *__restrict__ disp) {
  __shared__ __align__(16) float ui[kW * kW];
  __shared__ int dp[2 * kW];
  __shared__ int nd;
  const int tid = threadIdx.x;
  for (int i = tid; i < kW * kW; i += kThreads) ui[i] = uinv[i];
  if (tid == 0) nd = disp[0];
  __syncthreads();
  for (int i = tid; i < 2 * nd; i += kThreads) dp[i] = disp[1 + i];
  __syncthreads();
  for (long i = (long)blockIdx.x * kThreads + tid; i < r; i += (long)gridDim.x * kThreads) {
    if (i < w) {
      for (int c = 0; c < w; c++) A[i + (long)c * lda] = lu11[i * kW + c];
      continue;
    }
    int q = -1;
    for (int d = 0; d < nd; d++)
      if (dp[2 * d] == (int)i) q = dp[2 * d + 1];
    float b[kW], x[kW];
#pragma unroll
    for (int c = 0; c < kW; c++) {
      b[c] = c < w ? (q >= 0 ? stage[q * kW + c] : A[i + (long)c * lda]) : 0.f;
      x[c] = 0.f;
    }
    // x_c += b_k inv(U11)_kc for k = 0, 1, ... and c >= k: row k of inv(U11)
    // read in 16-byte pieces from column 4 floor(k / 4) on
#pragma unroll
    for (int k = 0; k < kW; k++)
#pragma unroll
      for (int q = k / 4; q < kW / 4; q++) {
        const float4 f = reinterpret_cast<const float4 *>(ui + k * kW)[q];
        if (4 * q >= k) x[4 * q] = fmaf(b[k], f.x, x[4 * q]);
        if (4 * q + 1 >= k) x[4 * q + 1] = fmaf(b[k], f.y, x[4 * q + 1]);
        if (4 * q + 2 >= k) x[4 * q + 2] = fmaf(b[k], f.z, x[4 * q + 2]);
        x[4 * q + 3] = fmaf(b[k], f.w, x[4 * q + 3]);
      }
#pragma unroll
    for (int c = 0; c < kW; c++)
      if (c < w) A[i + (long)c * lda] = x[c];
  }
}

// The rest of a sub-panel's step inside the panel, after its interchanges:
// U12 = inv(L11) A12 and A22 -= L21 U12, in one launch.  P is the sub-panel's
// top-left corner (m rows, w <= 32 columns, then ncols more columns of the
// panel to its right).  CTA (x, y) takes rows x kPU + w .. of the kPG columns
// of group y.  It stages the group's A12 and L11 in shared memory (coalesced
// loads), forms the group's U12 there (forward substitution, a column per
// thread, u_j -= L(j, k) u_k for k = 0 .. j-1 in order), then each thread
// updates one row of the group (a_c -= l_k U12(k, c) for k = 0 .. w-1 in
// order, U12 read back by columns in 16-byte pieces).  A12 is only read; the
// last CTA of a group to finish (an atomic counter per group, no CTA waits)
// writes the group's U12 over it.  W32 compiles the common w = 32.
constexpr int kPU = 256;  // threads (rows) of a panel_update_k CTA
constexpr int kPG = 16;   // columns of a panel_update_k group

template <bool W32>
__global__ void __launch_bounds__(kPU)
panel_update_k(int m, int w_, int ncols, float *__restrict__ P, long lda, unsigned *counters) {
  const int w = W32 ? kW : w_;
  __shared__ __align__(16) float ut[kPG][kW];  // the group's U12, by columns
  __shared__ float a12[kPG][kW + 1];
  __shared__ float l11[kW][kW + 1];
  __shared__ int s_last;
  const int tid = threadIdx.x;
  const int c0 = blockIdx.y * kPG, nc = min(kPG, ncols - c0);
  float *A12 = P + (long)(w + c0) * lda;
  for (int e = tid; e < kW * kW; e += kPU) {
    const int j = e % kW, k = e / kW;
    l11[j][k] = k < j && j < w ? P[j + (long)k * lda] : 0.f;
  }
  for (int e = tid; e < kPG * kW; e += kPU) {
    const int j = e % kW, c = e / kW;
    a12[c][j] = j < w && c < nc ? A12[j + (long)c * lda] : 0.f;
  }
  __syncthreads();
  if (tid < kPG) {
    float u[kW];
#pragma unroll
    for (int j = 0; j < kW; j++) u[j] = a12[tid][j];
#pragma unroll
    for (int k = 0; k < kW - 1; k++) {
      asm volatile("" ::: "memory");  // one column step's L11 loads at a time
#pragma unroll
      for (int j = k + 1; j < kW; j++) u[j] = fmaf(-l11[j][k], u[k], u[j]);
    }
#pragma unroll
    for (int q = 0; q < kW / 4; q++)
      *reinterpret_cast<float4 *>(&ut[tid][4 * q]) =
          make_float4(u[4 * q], u[4 * q + 1], u[4 * q + 2], u[4 * q + 3]);
  }
  __syncthreads();
  const long i = (long)blockIdx.x * kPU + tid + w;
  if (i < m) {
    float l[kW], a[kPG];
#pragma unroll
    for (int k = 0; k < kW; k++) l[k] = k < w ? P[i + (long)k * lda] : 0.f;
#pragma unroll
    for (int c = 0; c < kPG; c++) a[c] = c < nc ? A12[i + (long)c * lda] : 0.f;
#pragma unroll
    for (int c = 0; c < kPG; c++) {
#pragma unroll
      for (int q = 0; q < kW / 4; q++) {
        const float4 f = *reinterpret_cast<const float4 *>(&ut[c][4 * q]);
        if (W32 || 4 * q < w) a[c] = fmaf(-l[4 * q], f.x, a[c]);
        if (W32 || 4 * q + 1 < w) a[c] = fmaf(-l[4 * q + 1], f.y, a[c]);
        if (W32 || 4 * q + 2 < w) a[c] = fmaf(-l[4 * q + 2], f.z, a[c]);
        if (W32 || 4 * q + 3 < w) a[c] = fmaf(-l[4 * q + 3], f.w, a[c]);
      }
    }
#pragma unroll
    for (int c = 0; c < kPG; c++)
      if (c < nc) A12[i + (long)c * lda] = a[c];
  }
  // the group's last CTA writes its U12 (every CTA of the group has read A12
  // before it counts)
  __syncthreads();
  if (tid == 0) {
    const unsigned prev = atomicAdd(&counters[blockIdx.y], 1u);
    s_last = prev == gridDim.x - 1;
    if (s_last) counters[blockIdx.y] = 0;  // ready for the next launch
  }
  __syncthreads();
  if (s_last)
    for (int e = tid; e < w * nc; e += kPU) {
      const int k = e % w, c = e / w;
      A12[k + (long)c * lda] = ut[c][k];
    }
}

struct Ws {
  void *ptr = nullptr;
  size_t bytes = 0;
};

// panel_update_k's group counters, one set per (device, stream): launches on
// one stream run in order and leave them at zero; launches on different
// streams may overlap, so they do not share a set.  Freed by pla_tslu_release.
struct PuCounters {
  int dev;
  cudaStream_t stream;
  unsigned *ptr;
};
std::mutex g_pu_mu;
std::vector<PuCounters> g_pu;
Ws g_tws;
int g_tsms = 0;

}  // namespace

// Tournament-pivoted LU of the r x w fp32 panel at A (w <= 32): pivots (the
// reference's offset encoding) to piv, the panel overwritten by its L \ U
// factors under those interchanges.  At most max_ctas CTAs (0: one per SM).
extern "C" int pla_k_lu_panel_tslu(int r, int w, float *A, long lda, int *piv, int *zero_info,
                                   int row_base, int max_ctas, cudaStream_t s) {
  if (r <= 0 || w <= 0) return 0;
  if (w > kW || w > r) return (int)cudaErrorInvalidValue;
  if (!g_tsms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_tsms, cudaDevAttrMultiProcessorCount, dev);
  }
  int P = g_tsms;
  if (max_ctas > 0 && P > max_ctas) P = max_ctas;
  // no more leaves than it takes to give each one pass (kMaxCand rows): every
  // tree level costs w dependent column steps whatever the leaves' heights,
  // and fewer, fuller leaves need fewer levels (r <= 512: the root alone;
  // r <= 16 kMaxCand: one merge)
  const int maxP = (r + kMaxCand - 1) / kMaxCand;
  if (P > maxP) P = maxP;
  if (P < 1) P = 1;
  const int R = (r + P - 1) / P;
  P = (r + R - 1) / R;
  // workspace: the group counters first, at a fixed place (zeroed when the
  // workspace is allocated; every launch leaves them zero), then the root's
  // outputs, then the candidate sets (fewer than 2P of them in all levels)
  constexpr size_t kCounters = 1024;
  const size_t cnt_bytes = kCounters * sizeof(unsigned);
  const size_t out_bytes =
      (size_t)3 * kW * kW * sizeof(float) + (size_t)(2 * kW + 1) * sizeof(int);
  const size_t slot_off = (cnt_bytes + out_bytes + 255) / 256 * 256;
  const size_t need = slot_off + (size_t)2 * P * kW * sizeof(int);
  if (P > (int)kCounters) return (int)cudaErrorInvalidValue;
  if (g_tws.bytes < need) {
    if (g_tws.ptr) cudaFree(g_tws.ptr);
    g_tws.ptr = nullptr;
    g_tws.bytes = 0;
    const size_t want = need < ((size_t)1 << 20) ? ((size_t)1 << 20) : need;
    cudaError_t e = cudaMalloc(&g_tws.ptr, want);
    if (e != cudaSuccess) return (int)e;
    e = cudaMemsetAsync(g_tws.ptr, 0, want, s);
    if (e != cudaSuccess) return (int)e;
    g_tws.bytes = want;
  }
  char *base = (char *)g_tws.ptr;
  unsigned *counters = (unsigned *)base;
  float *lu11 = (float *)(base + cnt_bytes);
  float *uinv = lu11 + kW * kW;
  float *stage = uinv + kW * kW;
  int *disp = (int *)(stage + kW * kW);
  int *slots = (int *)(base + slot_off);
  Out out{piv, lu11, uinv, stage, disp, zero_info, row_base};
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(tslu_select_k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kHistBytes);
    attr = true;
  }
  tslu_select_k<<<P, kThreads, kHistBytes, s>>>(A, lda, r, w, R, slots, counters, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  int Pa = (r + kThreads - 1) / kThreads;
  if (max_ctas > 0 && Pa > 2 * max_ctas) Pa = 2 * max_ctas;
  if (Pa > 2 * g_tsms) Pa = 2 * g_tsms;
  tslu_apply_k<<<Pa, kThreads, 0, s>>>(A, lda, r, w, lu11, uinv, stage, disp);
  pla_k_count(2);
  return (int)cudaGetLastError();
}

// U12 = inv(L11) A12 and A22 -= L21 U12 for the m x w sub-panel at P (w <= 32)
// and the ncols columns right of it (ncols <= PLA_K_PANEL_UPDATE_MAX), one
// launch.  Each stream has its own group counters (launches on one stream run
// in order; launches on different streams may overlap).
extern "C" int pla_k_panel_update(int m, int w, int ncols, float *P, long lda, cudaStream_t s) {
  if (m <= 0 || w <= 0 || ncols <= 0) return 0;
  if (w > kW || w > m || ncols > PLA_K_PANEL_UPDATE_MAX) return (int)cudaErrorInvalidValue;
  constexpr int kGroups = (PLA_K_PANEL_UPDATE_MAX + kPG - 1) / kPG;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  unsigned *counters = nullptr;
  {
    std::lock_guard<std::mutex> g(g_pu_mu);
    for (const PuCounters &pc : g_pu)
      if (pc.dev == dev && pc.stream == s) counters = pc.ptr;
    if (!counters) {
      e = cudaMalloc(&counters, kGroups * sizeof(unsigned));
      if (e != cudaSuccess) return (int)e;
      e = cudaMemsetAsync(counters, 0, kGroups * sizeof(unsigned), s);  // before the first launch
      if (e != cudaSuccess) {
        cudaFree(counters);
        return (int)e;
      }
      g_pu.push_back({dev, s, counters});
    }
  }
  dim3 grid(std::max(1, (m - w + kPU - 1) / kPU), (ncols + kPG - 1) / kPG);
  if (w == kW)
    panel_update_k<true><<<grid, kPU, 0, s>>>(m, w, ncols, P, lda, counters);
  else
    panel_update_k<false><<<grid, kPU, 0, s>>>(m, w, ncols, P, lda, counters);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" void pla_tslu_release(void) {
  if (g_tws.ptr) cudaFree(g_tws.ptr);
  g_tws.ptr = nullptr;
  g_tws.bytes = 0;
  std::lock_guard<std::mutex> g(g_pu_mu);
  for (const PuCounters &pc : g_pu) cudaFree(pc.ptr);
  g_pu.clear();
}
