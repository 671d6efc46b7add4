// Batched factor-and-solve: thousands of independent LU (partial pivoting)
// and Cholesky systems of uneven order in ONE persistent launch.
//
// The host sorts the instances by decreasing order and cuts them into tasks:
//   mode 0 ("warp")   : up to 8 instances with n <= 32, one warp each, the
//                       matrix in shared memory, warp-synchronous;
//   mode 1 ("smem")   : one instance per CTA, matrix and right-hand sides in
//                       shared memory;
//   mode 2 ("global") : one instance per CTA working in place in global memory:
//                       blocked (panels of 16 / 32 columns in shared memory,
//                       the trailing matrix updated once per panel) when the
//                       panel fits the launch's shared memory, else the
//                       column algorithm in place.
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

// Blocked form of cta_instance for an instance in global memory (mode 2) whose
// panel fits the CTA's shared memory: panels of PW columns are factored in
// shared memory with the column algorithm; then the interchanges go to the
// other columns, U12 is solved, and the trailing matrix is updated once per
// panel in chunks of 64 columns (its elements pass through the SM once per
// panel instead of once per column).  Every element receives the same fma
// operations in the same order as in the column algorithm, so the factors,
// pivots and info are bitwise those of cta_instance.
template <typename T>
__device__ void cta_blocked(const Inst<T> &in, T *S, int *info) {
  constexpr int PW = sizeof(T) == 8 ? 16 : 32, CW = 64;
  __shared__ T sv[32];
  __shared__ int si[32];
  __shared__ int s_bad, s_piv[32];
  const int n = in.n, tid = threadIdx.x;
  T *A = in.A;
  T *P = S;              // panel: rows j0 .. n-1 of PW columns, ld n
  T *Uc = S + (long)n * PW;  // a PW x CW chunk of U12 (LU), ld PW
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int j0 = 0; j0 < n; j0 += PW) {
    const int jb = min(PW, n - j0), m = n - j0;
    for (int e = tid; e < m * jb; e += THREADS) {
      const int i = e % m, c = e / m;
      P[i + (long)c * n] = A[(j0 + i) + (long)(j0 + c) * n];
    }
    __syncthreads();
    if (in.kind == 0) {
      for (int j = 0; j < jb; j++) {
        T v = T(-1);
        int idx = INT_MAX;
        for (int i = j + tid; i < m; i += THREADS) {
          const T a = fabs(P[i + (long)j * n]);
          if (a > v) { v = a; idx = i; }
        }
        block_argmax(v, idx, sv, si);
        const int p = idx == INT_MAX ? j : idx;  // all-NaN column: no interchange
        if (tid == 0) {
          in.piv[j0 + j] = p - j;
          s_piv[j] = p;
        }
        if (p != j)
          for (int c = tid; c < jb; c += THREADS) {
            const T a = P[j + (long)c * n];
            P[j + (long)c * n] = P[p + (long)c * n];
            P[p + (long)c * n] = a;
          }
        __syncthreads();
        const T piv = P[j + (long)j * n];
        if (tid == 0 && piv == T(0) && !s_bad) s_bad = j0 + j + 1;
        const T inv = T(1) / piv;
        for (int i = j + 1 + tid; i < m; i += THREADS) P[i + (long)j * n] *= inv;
        __syncthreads();
        const int rows = m - j - 1, cols = jb - j - 1;
        for (int e = tid; e < rows * cols; e += THREADS) {
          const int i = j + 1 + e % rows, c = j + 1 + e / rows;
          P[i + (long)c * n] = fma(P[i + (long)j * n], -P[j + (long)c * n], P[i + (long)c * n]);
        }
        __syncthreads();
      }
      for (int e = tid; e < m * jb; e += THREADS) {
        const int i = e % m, c = e / m;
        A[(j0 + i) + (long)(j0 + c) * n] = P[i + (long)c * n];
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
              if (k < jb) u[k] = fma(P[k + (long)i * n], -u[i], u[k]);
#pragma unroll
          for (int k = 0; k < PW; k++)
            if (k < jb) col[k] = u[k];
        }
        __syncthreads();
        // A22 -= L21 U12 in chunks of CW columns, four columns a thread
        const int m2 = m - jb;
        for (int cc = j0 + jb; cc < n; cc += CW) {
          const int cw = min(CW, n - cc);
          for (int e = tid; e < jb * cw; e += THREADS) {
            const int k = e % jb, c = e / jb;
            Uc[k + c * PW] = A[(j0 + k) + (long)(cc + c) * n];
          }
          __syncthreads();
          const int groups = (cw + 3) / 4;
          for (int e = tid; e < m2 * groups; e += THREADS) {
            const int i = e % m2, c4 = 4 * (e / m2);
            T *row = A + (j0 + jb + i);
            T acc[4];
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] = c4 + q < cw ? row[(long)(cc + c4 + q) * n] : T(0);
            for (int k = 0; k < jb; k++) {
              const T l = P[(jb + i) + (long)k * n];
#pragma unroll
              for (int q = 0; q < 4; q++) acc[q] = fma(l, -Uc[k + (c4 + q) * PW], acc[q]);
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
              if (c4 + q < cw) row[(long)(cc + c4 + q) * n] = acc[q];
          }
          __syncthreads();
        }
      }
    } else {
      bool stop = false;
      for (int j = 0; j < jb; j++) {
        const T d = P[j + (long)j * n];
        if (d <= T(0)) {
          if (tid == 0) s_bad = j0 + j + 1;
          stop = true;
          break;
        }
        const T sq = sqrt(d), inv = T(1) / sq;
        __syncthreads();
        if (tid == 0) P[j + (long)j * n] = sq;
        for (int i = j + 1 + tid; i < m; i += THREADS) P[i + (long)j * n] *= inv;
        __syncthreads();
        const int rows = m - j - 1, cols = jb - j - 1;
        for (int e = tid; e < rows * cols; e += THREADS) {
          const int i = j + 1 + e % rows, c = j + 1 + e / rows;
          if (i >= c)
            P[i + (long)c * n] = fma(-P[i + (long)j * n], P[c + (long)j * n], P[i + (long)c * n]);
        }
        __syncthreads();
      }
      if (stop) break;
      for (int e = tid; e < m * jb; e += THREADS) {
        const int i = e % m, c = e / m;
        if (i >= c) A[(j0 + i) + (long)(j0 + c) * n] = P[i + (long)c * n];
      }
      // A22 -= L21 L21' (lower part), L21 read from the panel, 4 columns a thread
      const int m2 = m - jb;
      for (int cc = 0; cc < m2; cc += CW) {
        const int cw = min(CW, m2 - cc);
        const int groups = (cw + 3) / 4, rows = m2 - cc;  // rows i >= cc of the chunk
        for (int e = tid; e < rows * groups; e += THREADS) {
          const int i = cc + e % rows, c4 = cc + 4 * (e / rows);
          T *row = A + (j0 + jb + i);
          T acc[4];
#pragma unroll
          for (int q = 0; q < 4; q++)
            acc[q] = (c4 + q < cc + cw && i >= c4 + q) ? row[(long)(j0 + jb + c4 + q) * n] : T(0);
          for (int k = 0; k < jb; k++) {
            const T l = P[(jb + i) + (long)k * n];
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] = fma(-l, P[(jb + c4 + q) + (long)k * n], acc[q]);
          }
#pragma unroll
          for (int q = 0; q < 4; q++)
            if (c4 + q < cc + cw && i >= c4 + q) row[(long)(j0 + jb + c4 + q) * n] = acc[q];
        }
      }
      __syncthreads();
    }
  }
  __syncthreads();
  const int bad = s_bad;
  // the solves, in global memory, as in cta_instance
  T *X = in.B;
  const long lx = n;
  if (in.kind == 0) {
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
        X[i + r * lx] -= A[i + (long)j * n] * X[j + r * lx];
      }
      __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {
      if (tid < in.nrhs) X[j + tid * lx] = X[j + tid * lx] / A[j + (long)j * n];
      __syncthreads();
      for (long e = tid; e < (long)j * in.nrhs; e += THREADS) {
        const int i = (int)(e % j), r = (int)(e / j);
        X[i + r * lx] -= A[i + (long)j * n] * X[j + r * lx];
      }
      __syncthreads();
    }
  } else if (!bad) {
    for (int j = 0; j < n; j++) {
      if (tid < in.nrhs) X[j + tid * lx] = X[j + tid * lx] / A[j + (long)j * n];
      __syncthreads();
      for (long e = tid; e < (long)(n - j - 1) * in.nrhs; e += THREADS) {
        const int i = j + 1 + (int)(e % (n - j - 1)), r = (int)(e / (n - j - 1));
        X[i + r * lx] -= A[i + (long)j * n] * X[j + r * lx];
      }
      __syncthreads();
    }
    for (int j = n - 1; j >= 0; j--) {
      if (tid < in.nrhs) X[j + tid * lx] = X[j + tid * lx] / A[j + (long)j * n];
      __syncthreads();
      for (long e = tid; e < (long)j * in.nrhs; e += THREADS) {
        const int i = (int)(e % j), r = (int)(e / j);
        X[i + r * lx] -= A[j + (long)i * n] * X[j + r * lx];
      }
      __syncthreads();
    }
  }
  __syncthreads();
  if (tid == 0) *info = bad;
}

// shared memory the blocked form needs for an instance of order n
template <typename T>
__host__ __device__ constexpr size_t blocked_smem(int n) {
  return ((size_t)n * (sizeof(T) == 8 ? 16 : 32) + (size_t)(sizeof(T) == 8 ? 16 : 32) * 64) *
         sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(THREADS)
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
      } else if (blocked_smem<T>(in.n) <= smem_bytes) {
        cta_blocked(in, S, &info[id]);
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
