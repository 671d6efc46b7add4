// Batched factor-and-solve: thousands of independent LU (partial pivoting)
// and Cholesky systems of uneven order in ONE persistent launch.
//
// The host sorts the instances by decreasing order and cuts them into tasks:
//   mode 0 ("warp")   : up to 8 instances with n <= 32, one warp each, the
//                       matrix in shared memory, warp-synchronous;
//   mode 1 ("smem")   : one instance per CTA, matrix and right-hand sides in
//                       shared memory;
//   mode 2, 3 ("global"): one instance per CTA working in place in global
//                       memory: blocked (panels of 16 (mode 2) or 32 (mode 3)
//                       columns in shared memory, the trailing matrix updated
//                       once per panel from register tiles, the solves by
//                       blocks of 32 rows) when the panel fits the launch's
//                       shared memory, else the column algorithm in place.
// CTAs pull tasks from an atomic queue, largest first, so the long instances
// start early and the short ones fill the tail.  Each instance runs the same
// column algorithms as the reference's sequential kernels: LU as PLA_dlu
// (SOLVERS/LU/PLA_seq_lu.c:21-46: first-index argmax, full-row swap,
// reciprocal scaling, rank-1 update), Cholesky right-looking with the
// reciprocal scaling of PLA_dchol (SOLVERS/Cholesky/PLA_Local_chol.c:124-137),
// then the forward and backward substitutions.  Status per instance is a
// LAPACK-style info: LU the first exact zero pivot, Cholesky the failing
// column (1-based), 0 otherwise.
#include <climits>
#include <type_traits>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

constexpr int THREADS = 256;
// shared memory of one warp-mode instance: a 32 x 33 matrix and 4 x 33 RHS
constexpr int kWarpSmem = 32 * 33 + 4 * 33;

template <typename T>
struct Inst {
  int n, nrhs, kind, pad;
  T *A;
  T *B;
  int *piv;
};

struct Task {
  int first, count, mode, pad;
};

// ---------------------------------------------------------------- warp ----
template <typename T>
__device__ void warp_instance(const Inst<T> &in, T *S, int *info) {
  const int lane = threadIdx.x & 31, n = in.n, ld = 33;
  T *Bs = S + 32 * ld;  // up to 4 right-hand sides, ld 33
  for (int c = 0; c < n; c++)
    if (lane < n) S[lane + c * ld] = in.A[lane + (long)c * n];
  for (int r = 0; r < in.nrhs; r++)
    if (lane < n) Bs[lane + r * ld] = in.B[lane + (long)r * n];
  __syncwarp();
  int bad = 0;
  if (in.kind == 0) {
    for (int j = 0; j < n; j++) {
      T v = (lane >= j && lane < n) ? fabs(S[lane + j * ld]) : T(-1);
      int idx = lane >= j && lane < n ? lane : INT_MAX;
      for (int o = 16; o; o >>= 1) {
        T ov = __shfl_down_sync(0xffffffffu, v, o);
        int oi = __shfl_down_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
      }
      const int best = __shfl_sync(0xffffffffu, idx, 0);
      const int p = best == INT_MAX ? j : best;  // all-NaN column: no interchange
      if (lane == 0) in.piv[j] = p - j;
      if (p != j && lane < n) {
        T a = S[j + lane * ld];
        S[j + lane * ld] = S[p + lane * ld];
        S[p + lane * ld] = a;
      }
      __syncwarp();
      const T piv = S[j + j * ld];
      if (piv == T(0) && !bad) bad = j + 1;
      const T inv = T(1) / piv;
      if (lane > j && lane < n) {
        const T l = S[lane + j * ld] * inv;
        S[lane + j * ld] = l;
        for (int c = j + 1; c < n; c++) S[lane + c * ld] = fma(l, -S[j + c * ld], S[lane + c * ld]);
      }
      __syncwarp();
    }
    // P b, then L (unit) and U solves
    for (int r = 0; r < in.nrhs; r++) {
      if (lane == 0)
        for (int j = 0; j < n; j++) {
          int p = j + in.piv[j];
          if (p != j) {
            T a = Bs[j + r * ld];
            Bs[j + r * ld] = Bs[p + r * ld];
            Bs[p + r * ld] = a;
          }
        }
      __syncwarp();
      for (int j = 0; j < n; j++) {
        const T x = Bs[j + r * ld];
        if (lane > j && lane < n) Bs[lane + r * ld] -= S[lane + j * ld] * x;
        __syncwarp();
      }
      for (int j = n - 1; j >= 0; j--) {
        if (lane == 0) Bs[j + r * ld] = Bs[j + r * ld] / S[j + j * ld];
        __syncwarp();
        const T x = Bs[j + r * ld];
        if (lane < j) Bs[lane + r * ld] -= S[lane + j * ld] * x;
        __syncwarp();
      }
    }
  } else {
    for (int j = 0; j < n; j++) {
      const T d = S[j + j * ld];
      if (d <= T(0)) {
        bad = j + 1;
        break;
      }
      const T s = sqrt(d);
      const T inv = T(1) / s;
      __syncwarp();
      if (lane == j) S[j + j * ld] = s;
      if (lane > j && lane < n) S[lane + j * ld] *= inv;
      __syncwarp();
      if (lane > j && lane < n) {
        const T l = S[lane + j * ld];
        for (int c = j + 1; c <= lane; c++) S[lane + c * ld] = fma(-l, S[c + j * ld], S[lane + c * ld]);
      }
      __syncwarp();
    }
    if (!bad)
      for (int r = 0; r < in.nrhs; r++) {
        for (int j = 0; j < n; j++) {
          if (lane == 0) Bs[j + r * ld] = Bs[j + r * ld] / S[j + j * ld];
          __syncwarp();
          const T x = Bs[j + r * ld];
          if (lane > j && lane < n) Bs[lane + r * ld] -= S[lane + j * ld] * x;
          __syncwarp();
        }
        for (int j = n - 1; j >= 0; j--) {
          if (lane == 0) Bs[j + r * ld] = Bs[j + r * ld] / S[j + j * ld];
          __syncwarp();
          const T x = Bs[j + r * ld];
          if (lane < j) Bs[lane + r * ld] -= S[j + lane * ld] * x;  // L' column = L row
          __syncwarp();
        }
      }
  }
  __syncwarp();
  for (int c = 0; c < n; c++)
    if (lane < n && (in.kind == 0 || lane >= c)) in.A[lane + (long)c * n] = S[lane + c * ld];
  if (!(in.kind == 1 && bad))
    for (int r = 0; r < in.nrhs; r++)
      if (lane < n) in.B[lane + (long)r * n] = Bs[lane + r * ld];
  if (lane == 0) *info = bad;
}

// ----------------------------------------------------------------- CTA ----
template <typename T>
__device__ void block_argmax(T &v, int &i, T *sv, int *si) {
  for (int o = 16; o; o >>= 1) {
    T ov = __shfl_down_sync(0xffffffffu, v, o);
    int oi = __shfl_down_sync(0xffffffffu, i, o);
    if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sv[w] = v; si[w] = i; }
  __syncthreads();
  if (w == 0) {
    v = l < THREADS / 32 ? sv[l] : T(-1);
    i = l < THREADS / 32 ? si[l] : INT_MAX;
    for (int o = 16; o; o >>= 1) {
      T ov = __shfl_down_sync(0xffffffffu, v, o);
      int oi = __shfl_down_sync(0xffffffffu, i, o);
      if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
    }
    if (l == 0) { sv[0] = v; si[0] = i; }
  }
  __syncthreads();
  v = sv[0];
  i = si[0];
  __syncthreads();
}

// the instance's matrix at M (ld lm) and right-hand sides at X (ld lx):
// shared memory in mode 1, the instance's own global buffers in mode 2
template <typename T>
__device__ void cta_instance(const Inst<T> &in, T *M, long lm, T *X, long lx, int *info) {
  __shared__ T sv[32];
  __shared__ int si[32];
  __shared__ int s_bad;
  const int n = in.n, tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  if (in.kind == 0) {
    for (int j = 0; j < n; j++) {
      T v = T(-1);
      int idx = INT_MAX;
      for (int i = j + tid; i < n; i += THREADS) {
        T a = fabs(M[i + j * lm]);
        if (a > v) { v = a; idx = i; }
      }
      block_argmax(v, idx, sv, si);
      const int p = idx == INT_MAX ? j : idx;  // all-NaN column: no interchange
      if (tid == 0) in.piv[j] = p - j;
      if (p != j)
        for (int c = tid; c < n; c += THREADS) {
          T a = M[j + c * lm];
          M[j + c * lm] = M[p + c * lm];
          M[p + c * lm] = a;
        }
      __syncthreads();
      const T piv = M[j + j * lm];
      if (tid == 0 && piv == T(0) && !s_bad) s_bad = j + 1;
      const T inv = T(1) / piv;
      for (int i = j + 1 + tid; i < n; i += THREADS) M[i + j * lm] *= inv;
      __syncthreads();
      const int rows = n - j - 1;
      const long tot = (long)rows * rows;
      for (long e = tid; e < tot; e += THREADS) {
        const int i = j + 1 + (int)(e % rows), c = j + 1 + (int)(e / rows);
        M[i + c * lm] = fma(M[i + j * lm], -M[j + c * lm], M[i + c * lm]);
      }
      __syncthreads();
    }
    for (int r = tid; r < in.nrhs; r += THREADS)
      for (int j = 0; j < n; j++) {
        int p = j + in.piv[j];
        if (p != j) {
          T a = X[j + r * lx];
          X[j + r * lx] = X[p + r * lx];
          X[p + r * lx] = a;
        }
      }
    __syncthreads();
    for (int j = 0; j < n; j++) {
      for (long e = tid; e < (long)(n - j - 1) * in.nrhs; e += THREADS) {
        const int i = j + 1 + (int)(e % (n - j - 1)), r = (int)(e / (n - j - 1));
        X[i + r * lx] -= M[i + j * lm] * X[j + r * lx];
      }
      __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {
      if (tid < in.nrhs) X[j + tid * lx] = X[j + tid * lx] / M[j + j * lm];
      __syncthreads();
      for (long e = tid; e < (long)j * in.nrhs; e += THREADS) {
        const int i = (int)(e % j), r = (int)(e / j);
        X[i + r * lx] -= M[i + j * lm] * X[j + r * lx];
      }
      __syncthreads();
    }
  } else {
    for (int j = 0; j < n; j++) {
      const T d = M[j + j * lm];
      if (d <= T(0)) {
        if (tid == 0) s_bad = j + 1;
        break;
      }
      const T s = sqrt(d), inv = T(1) / s;
      __syncthreads();
      if (tid == 0) M[j + j * lm] = s;
      for (int i = j + 1 + tid; i < n; i += THREADS) M[i + j * lm] *= inv;
      __syncthreads();
      const int rows = n - j - 1;
      const long tot = (long)rows * rows;
      for (long e = tid; e < tot; e += THREADS) {
        const int i = j + 1 + (int)(e % rows), c = j + 1 + (int)(e / rows);
        if (i >= c) M[i + c * lm] = fma(-M[i + j * lm], M[c + j * lm], M[i + c * lm]);
      }
      __syncthreads();
    }
    __syncthreads();
    if (!s_bad) {
      for (int j = 0; j < n; j++) {
        if (tid < in.nrhs) X[j + tid * lx] = X[j + tid * lx] / M[j + j * lm];
        __syncthreads();
        for (long e = tid; e < (long)(n - j - 1) * in.nrhs; e += THREADS) {
          const int i = j + 1 + (int)(e % (n - j - 1)), r = (int)(e / (n - j - 1));
          X[i + r * lx] -= M[i + j * lm] * X[j + r * lx];
        }
        __syncthreads();
      }
      for (int j = n - 1; j >= 0; j--) {
        if (tid < in.nrhs) X[j + tid * lx] = X[j + tid * lx] / M[j + j * lm];
        __syncthreads();
        for (long e = tid; e < (long)j * in.nrhs; e += THREADS) {
          const int i = (int)(e % j), r = (int)(e / j);
          X[i + r * lx] -= M[j + i * lm] * X[j + r * lx];
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();
  if (tid == 0) *info = s_bad;
}

// Blocked form of cta_instance for an instance in global memory (modes 2 and
// 3, panels of PW = 16 or 32 columns) whose panel fits the CTA's shared
// memory.  Per panel:
//   - the panel is factored in shared memory with the column algorithm; every
//     thread owns the panel rows i = tid (mod THREADS), so a column costs two
//     barriers (the pivot search, the interchange) and the rank-1 update of a
//     thread's own rows needs none;
//   - the interchanges go to the other columns and U12 = inv(L11) A12 is
//     solved, a column per thread;
//   - the trailing matrix is updated once per panel, in chunks of CW columns,
//     each thread holding a 4 x 8 block of C in registers (L21 read from the
//     panel in shared memory, U12 from a chunk staged there), so an element
//     passes through the SM once per panel.
// Every element receives the same fma operations in the same order as in the
// column algorithm, so the factors, pivots and info are bitwise those of
// cta_instance.  The substitutions then run by blocks of 32 rows: one warp
// solves the block's triangle, every thread applies its columns to the rows
// below (above, going back) -- again each element's operations in the
// column algorithm's order.
constexpr int kCW = 64;  // columns of a trailing-update chunk
// rows x columns of C per thread: 4 x 8 in fp32, 4 x 4 in FP64 (the
// accumulators of two CTAs per SM fit the register file)
constexpr int kRB = 4;
template <typename T>
constexpr int col_block() { return sizeof(T) == 8 ? 4 : 8; }

template <typename T>
__host__ __device__ constexpr long panel_ld(int n) {
  return (n + 3) & ~3;
}

// C(rows, cols) -= L21 U12 (LU) or the lower part of L21 L21' (Cholesky) for
// one chunk: rows [r0, m2) of the trailing block (relative to the panel's row
// jb), columns [cc, cc + cw).  L21(i, k) = P[jb + i + k ldp]; U(k, c) =
// Uc[k kCW + c - cc].  C(i, c) is A[(j0 + jb + i) + (j0 + jb + c) n] for the
// Cholesky, A[(j0 + jb + i) + c n] for the LU (cc there is a global column).
template <typename T>
__device__ void update_chunk(T *A, long n, long c_row0, long c_col_off, const T *P, long ldp,
                             int jb, const T *Uc, int m2, int cc, int cw, bool lower) {
  constexpr int kCB = col_block<T>();
  const int tid = threadIdx.x;
  const int r0 = lower ? (cc / kRB) * kRB : 0;  // rows above the chunk's diagonal hold nothing
  const int nrq = (m2 - r0 + kRB - 1) / kRB, ncb = (cw + kCB - 1) / kCB;
  for (int e = tid; e < nrq * ncb; e += THREADS) {
    const int i0 = r0 + (e % nrq) * kRB, c0 = (e / nrq) * kCB;  // c0 relative to cc
    if (lower && i0 + kRB - 1 < cc + c0) continue;                // strictly above the diagonal
    T acc[kRB][kCB];
#pragma unroll
    for (int r = 0; r < kRB; r++)
#pragma unroll
      for (int q = 0; q < kCB; q++) {
        const int i = i0 + r, c = cc + c0 + q;
        const bool ok = i < m2 && c0 + q < cw && (!lower || i >= c);
        acc[r][q] = ok ? A[c_row0 + i + (long)(c + c_col_off) * n] : T(0);
      }
    const T *lp = P + jb + i0;
    const T *up = Uc + c0;
    for (int k = 0; k < jb; k++) {
      // the thread's kRB rows of L21 column k in 16-byte pieces: jb is the
      // full panel width here (a trailing block exists) and ldp a multiple of
      // 4, so the address is 16-byte aligned, and a warp's loads are one
      // contiguous stretch (element loads kRB apart would conflict on banks)
      T l[kRB], u[kCB];
      constexpr int V = 16 / sizeof(T);
      using Vec = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
#pragma unroll
      for (int r = 0; r < kRB; r += V) {
        const Vec x = *reinterpret_cast<const Vec *>(lp + r + (long)k * ldp);
        const T *xs_ = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int s = 0; s < V; s++) l[r + s] = xs_[s];
      }
#pragma unroll
      for (int q = 0; q < kCB; q += V) {
        const Vec x = *reinterpret_cast<const Vec *>(up + k * kCW + q);
        const T *xs_ = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int s = 0; s < V; s++) u[q + s] = xs_[s];
      }
#pragma unroll
      for (int r = 0; r < kRB; r++)
#pragma unroll
        for (int q = 0; q < kCB; q++) acc[r][q] = fma(-l[r], u[q], acc[r][q]);
    }
#pragma unroll
    for (int r = 0; r < kRB; r++)
#pragma unroll
      for (int q = 0; q < kCB; q++) {
        const int i = i0 + r, c = cc + c0 + q;
        if (i < m2 && c0 + q < cw && (!lower || i >= c))
          A[c_row0 + i + (long)(c + c_col_off) * n] = acc[r][q];
      }
  }
}

// Substitutions with the n x n factor F (global, ld n) for nrhs <= 4 columns
// of X (ld n), by blocks of 32 rows.  lower: x_i -= F(i, j) x_j for j < i
// (unit diagonal unless `divide`, which first divides x_j by F(j, j));
// otherwise backward: x_j /= G(j, j), x_i -= G(i, j) x_j for i < j, with
// G = F (upper, LU) or F' (`trans`, Cholesky).  xs: 32 x 4 shared buffer.
template <typename T>
__device__ void solve_blocked(const T *F, int n, T *X, int nrhs, bool lower, bool divide,
                              bool trans, T *xs) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (n + 31) / 32;
  for (int bb = 0; bb < nblk; bb++) {
    const int blk = lower ? bb : nblk - 1 - bb;
    const int b0 = blk * 32, bw = min(32, n - b0);
    if (warp == 0) {  // the block's triangle, one lane per row
      T x[4];
      const int i = b0 + lane;
#pragma unroll
      for (int r = 0; r < 4; r++) x[r] = (lane < bw && r < nrhs) ? X[i + (long)r * n] : T(0);
      if (lower) {
        for (int j = 0; j < bw; j++) {
          if (divide && lane == j)
#pragma unroll
            for (int r = 0; r < 4; r++) x[r] = x[r] / F[(b0 + j) + (long)(b0 + j) * n];
          const T f = (lane > j && lane < bw) ? F[i + (long)(b0 + j) * n] : T(0);
#pragma unroll
          for (int r = 0; r < 4; r++) {
            const T xj = __shfl_sync(0xffffffffu, x[r], j);
            if (lane > j && lane < bw) x[r] -= f * xj;
          }
        }
      } else {
        for (int j = bw - 1; j >= 0; j--) {
          if (lane == j)
#pragma unroll
            for (int r = 0; r < 4; r++) x[r] = x[r] / F[(b0 + j) + (long)(b0 + j) * n];
          const T g = lane < j ? (trans ? F[(b0 + j) + (long)i * n] : F[i + (long)(b0 + j) * n])
                               : T(0);
#pragma unroll
          for (int r = 0; r < 4; r++) {
            const T xj = __shfl_sync(0xffffffffu, x[r], j);
            if (lane < j) x[r] -= g * xj;
          }
        }
      }
#pragma unroll
      for (int r = 0; r < 4; r++)
        if (lane < bw && r < nrhs) {
          X[i + (long)r * n] = x[r];
          xs[lane + 32 * r] = x[r];
        }
    }
    __syncthreads();
    // the block's columns applied to the rows below (lower) or above it,
    // column by column in the column algorithm's order
    if (lower) {
      for (int i = b0 + bw + tid; i < n; i += THREADS) {
        T x[4];
#pragma unroll
        for (int r = 0; r < 4; r++) x[r] = r < nrhs ? X[i + (long)r * n] : T(0);
        for (int j = 0; j < bw; j++) {
          const T f = F[i + (long)(b0 + j) * n];
#pragma unroll
          for (int r = 0; r < 4; r++) x[r] -= f * xs[j + 32 * r];
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
          if (r < nrhs) X[i + (long)r * n] = x[r];
      }
    } else {
      for (int i = tid; i < b0; i += THREADS) {
        T x[4];
#pragma unroll
        for (int r = 0; r < 4; r++) x[r] = r < nrhs ? X[i + (long)r * n] : T(0);
        for (int j = bw - 1; j >= 0; j--) {
          const T g = trans ? F[(b0 + j) + (long)i * n] : F[i + (long)(b0 + j) * n];
#pragma unroll
          for (int r = 0; r < 4; r++) x[r] -= g * xs[j + 32 * r];
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
          if (r < nrhs) X[i + (long)r * n] = x[r];
      }
    }
    __syncthreads();
  }
}

template <typename T, int PW>
__device__ void cta_blocked(const Inst<T> &in, T *S, int *info) {
  __shared__ T sv[32];
  __shared__ int si[32];
  __shared__ int s_bad, s_piv[PW];
  __shared__ T xs[32 * 4];
  const int n = in.n, tid = threadIdx.x;
  const long ldp = panel_ld<T>(n);
  T *A = in.A;
  T *P = S;              // panel: rows j0 .. n-1 of PW columns, ld ldp
  T *Uc = S + ldp * PW;  // a PW x kCW chunk of U12 (or L21'), row-major
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int j0 = 0; j0 < n; j0 += PW) {
    const int jb = min(PW, n - j0), m = n - j0;
    for (int e = tid; e < m * jb; e += THREADS) {
      const int i = e % m, c = e / m;
      P[i + (long)c * ldp] = A[(j0 + i) + (long)(j0 + c) * n];
    }
    __syncthreads();
    if (in.kind == 0) {
      for (int j = 0; j < jb; j++) {
        T v = T(-1);
        int idx = INT_MAX;
        for (int i = tid; i < m; i += THREADS)
          if (i >= j) {
            const T a = fabs(P[i + (long)j * ldp]);
            if (a > v) { v = a; idx = i; }
          }
        block_argmax(v, idx, sv, si);
        const int p = idx == INT_MAX ? j : idx;  // all-NaN column: no interchange
        if (tid == 0) {
          in.piv[j0 + j] = p - j;
          s_piv[j] = p;
        }
        if (p != j && tid < jb) {
          const T a = P[j + (long)tid * ldp];
          P[j + (long)tid * ldp] = P[p + (long)tid * ldp];
          P[p + (long)tid * ldp] = a;
        }
        __syncthreads();
        const T piv = P[j + (long)j * ldp];
        if (tid == 0 && piv == T(0) && !s_bad) s_bad = j0 + j + 1;
        const T inv = T(1) / piv;
        for (int i = tid; i < m; i += THREADS)
          if (i > j) {
            const T l = P[i + (long)j * ldp] * inv;
            P[i + (long)j * ldp] = l;
            for (int c = j + 1; c < jb; c++)
              P[i + (long)c * ldp] = fma(l, -P[j + (long)c * ldp], P[i + (long)c * ldp]);
          }
        // the next column's search reads only this thread's own rows; its
        // barrier orders these updates before the next interchange
      }
      __syncthreads();
      for (int e = tid; e < m * jb; e += THREADS) {
        const int i = e % m, c = e / m;
        A[(j0 + i) + (long)(j0 + c) * n] = P[i + (long)c * ldp];
      }
      // the panel's interchanges on every other column, in order, a column
      // per thread
      for (int c = tid; c < n; c += THREADS) {
        if (c >= j0 && c < j0 + jb) continue;
        T *col = A + (long)c * n + j0;
        for (int j = 0; j < jb; j++) {
          const int p = s_piv[j];
          if (p != j) {
            const T a = col[j];
            col[j] = col[p];
            col[p] = a;
          }
        }
      }
      __syncthreads();
      if (j0 + jb < n) {
        // U12 := inv(L11) A12, a column per thread (the updates of column i
        // reach row k in the order i = 0, 1, ... as in the column algorithm)
        for (int c = j0 + jb + tid; c < n; c += THREADS) {
          T u[PW];
          T *col = A + (long)c * n + j0;
#pragma unroll
          for (int k = 0; k < PW; k++) u[k] = k < jb ? col[k] : T(0);
#pragma unroll
          for (int i = 0; i < PW; i++)
#pragma unroll
            for (int k = i + 1; k < PW; k++)
              if (k < jb) u[k] = fma(P[k + (long)i * ldp], -u[i], u[k]);
#pragma unroll
          for (int k = 0; k < PW; k++)
            if (k < jb) col[k] = u[k];
        }
        __syncthreads();
        // A22 -= L21 U12 in chunks of kCW columns
        const int m2 = m - jb;
        for (int cc = j0 + jb; cc < n; cc += kCW) {
          const int cw = min(kCW, n - cc);
          for (int e = tid; e < jb * kCW; e += THREADS) {
            const int k = e / kCW, c = e % kCW;
            Uc[e] = c < cw ? A[(j0 + k) + (long)(cc + c) * n] : T(0);
          }
          __syncthreads();
          update_chunk(A, n, (long)(j0 + jb), 0, P, ldp, jb, Uc, m2, cc, cw, false);
          __syncthreads();
        }
      }
    } else {
      bool stop = false;
      for (int j = 0; j < jb; j++) {
        const T d = P[j + (long)j * ldp];
        if (d <= T(0)) {
          if (tid == 0) s_bad = j0 + j + 1;
          stop = true;
          break;
        }
        const T sq = sqrt(d), inv = T(1) / sq;
        __syncthreads();
        if (tid == 0) P[j + (long)j * ldp] = sq;
        for (int i = j + 1 + tid; i < m; i += THREADS) P[i + (long)j * ldp] *= inv;
        __syncthreads();
        const int rows = m - j - 1, cols = jb - j - 1;
        for (int e = tid; e < rows * cols; e += THREADS) {
          const int i = j + 1 + e % rows, c = j + 1 + e / rows;
          if (i >= c)
            P[i + (long)c * ldp] =
                fma(-P[i + (long)j * ldp], P[c + (long)j * ldp], P[i + (long)c * ldp]);
        }
        __syncthreads();
      }
      if (stop) break;
      for (int e = tid; e < m * jb; e += THREADS) {
        const int i = e % m, c = e / m;
        if (i >= c) A[(j0 + i) + (long)(j0 + c) * n] = P[i + (long)c * ldp];
      }
      // A22 -= L21 L21' (lower part), in chunks of kCW columns; the chunk's
      // L21' columns staged row-major
      const int m2 = m - jb;
      for (int cc = 0; cc < m2; cc += kCW) {
        const int cw = min(kCW, m2 - cc);
        __syncthreads();
        for (int e = tid; e < jb * kCW; e += THREADS) {
          const int k = e / kCW, c = e % kCW;
          Uc[e] = c < cw ? P[(jb + cc + c) + (long)k * ldp] : T(0);
        }
        __syncthreads();
        update_chunk(A, n, (long)(j0 + jb), (long)(j0 + jb), P, ldp, jb, Uc, m2, cc, cw, true);
      }
      __syncthreads();
    }
  }
  __syncthreads();
  const int bad = s_bad;
  // the solves, in global memory
  T *X = in.B;
  if (in.kind == 0) {
    for (int r = tid; r < in.nrhs; r += THREADS)
      for (int j = 0; j < n; j++) {
        int p = j + in.piv[j];
        if (p != j) {
          T a = X[j + (long)r * n];
          X[j + (long)r * n] = X[p + (long)r * n];
          X[p + (long)r * n] = a;
        }
      }
    __syncthreads();
    solve_blocked(A, n, X, in.nrhs, true, false, false, xs);
    solve_blocked(A, n, X, in.nrhs, false, true, false, xs);
  } else if (!bad) {
    solve_blocked(A, n, X, in.nrhs, true, true, false, xs);
    solve_blocked(A, n, X, in.nrhs, false, true, true, xs);
  }
  __syncthreads();
  if (tid == 0) *info = bad;
}

// shared memory the blocked form needs for an instance of order n
template <typename T>
__host__ __device__ constexpr size_t blocked_smem(int n, int pw) {
  return ((size_t)panel_ld<T>(n) * pw + (size_t)pw * kCW) * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(THREADS, 2)
batched_k(const Inst<T> *inst, const int *order, const Task *tasks, int ntasks, int *queue,
          int *info, size_t smem_bytes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *S = (T *)smem_raw;
  __shared__ int s_task;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_task = atomicAdd(queue, 1);
    __syncthreads();
    const int t = s_task;
    if (t >= ntasks) return;
    const Task tk = tasks[t];
    if (tk.mode == 0) {
      const int w = threadIdx.x >> 5;
      if (w < tk.count) {
        const int id = order[tk.first + w];
        warp_instance(inst[id], S + (long)w * kWarpSmem, &info[id]);
      }
    } else {
      const int id = order[tk.first];
      const Inst<T> in = inst[id];
      if (tk.mode == 1) {
        const int n = in.n;
        const long lm = n + 1, lx = n + 1;
        T *M = S, *X = S + lm * n;
        for (long e = threadIdx.x; e < (long)n * n; e += THREADS)
          M[(e % n) + (e / n) * lm] = in.A[e];
        for (long e = threadIdx.x; e < (long)n * in.nrhs; e += THREADS)
          X[(e % n) + (e / n) * lx] = in.B[e];
        __syncthreads();
        cta_instance(in, M, lm, X, lx, &info[id]);
        __syncthreads();
        const bool keep_b = !(in.kind == 1 && info[id]);
        for (long e = threadIdx.x; e < (long)n * n; e += THREADS) {
          const int i = (int)(e % n), c = (int)(e / n);
          if (in.kind == 0 || i >= c) in.A[e] = M[i + c * lm];
        }
        if (keep_b)
          for (long e = threadIdx.x; e < (long)n * in.nrhs; e += THREADS)
            in.B[e] = X[(e % n) + (e / n) * lx];
      } else if (tk.mode == 3 && blocked_smem<T>(in.n, 32) <= smem_bytes) {
        cta_blocked<T, 32>(in, S, &info[id]);
      } else if (blocked_smem<T>(in.n, 16) <= smem_bytes) {
        cta_blocked<T, 16>(in, S, &info[id]);
      } else {
        cta_instance(in, in.A, in.n, in.B, in.n, &info[id]);
      }
    }
  }
}

}  // namespace

extern "C" size_t pla_k_batched_smem(int dt, int n_smem_max) {
  const size_t es = dt == MPI_DOUBLE ? 8 : 4;
  size_t warp = (size_t)8 * kWarpSmem * es;
  size_t cta = ((size_t)(n_smem_max + 1) * n_smem_max + (size_t)(n_smem_max + 1) * 4) * es;
  return warp > cta ? warp : cta;
}

// shared memory of the blocked form (panels of pw = 16 or 32 columns) for an
// instance of order n
extern "C" size_t pla_k_batched_blocked_smem(int dt, int n, int pw) {
  return dt == MPI_DOUBLE ? blocked_smem<double>(n, pw) : blocked_smem<float>(n, pw);
}

// inst: device array of {n, nrhs, kind, pad, A, B, piv}; order: instance ids
// by task; tasks: device {first, count, mode}; queue: zeroed int.
extern "C" int pla_k_batched(int dt, const void *inst, const int *order, const void *tasks,
                             int ntasks, int *queue, int *info, int grid, size_t smem,
                             cudaStream_t s) {
  if (ntasks <= 0) return 0;
  if (dt == MPI_DOUBLE) {
    cudaFuncSetAttribute(batched_k<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    batched_k<double><<<grid, THREADS, smem, s>>>((const Inst<double> *)inst, order,
                                                  (const Task *)tasks, ntasks, queue, info, smem);
  } else if (dt == MPI_FLOAT) {
    cudaFuncSetAttribute(batched_k<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    batched_k<float><<<grid, THREADS, smem, s>>>((const Inst<float> *)inst, order,
                                                 (const Task *)tasks, ntasks, queue, info, smem);
  } else {
    return (int)cudaErrorInvalidValue;
  }
  pla_k_count(1);
  return (int)cudaGetLastError();
}
