// Triangular solves with a diagonal block held in shared memory, the
// unblocked Cholesky of a diagonal block, and the blocked triangular solve
// with right-hand sides built from them and the GEMM.
//
//  trsm_small  : one b x b triangle (b <= 128) against many columns (side L)
//                or rows (side R).  Each CTA loads the triangle once and loops
//                over its share of right-hand-side blocks; substitution runs
//                in shared memory with one barrier per eliminated row.  The
//                operation order is that of the reference BLAS dtrsm
//                (left: divide by the diagonal; right: multiply by its
//                reciprocal), used by PLA_LU (SOLVERS/LU/PLA_LU.c:174-178) and
//                PLA_Chol (SOLVERS/Cholesky/PLA_Chol.c:193-195).
//  potrf_lower : PLA_dchol's left-looking column algorithm
//                (SOLVERS/Cholesky/PLA_Local_chol.c:114-138) on one CTA.
#include "PLA.h"
#include "pla_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxTri = 128;

template <typename T>
__device__ __forceinline__ T opT(const T *Ts, int ldt, bool trans, int i, int j) {
  return trans ? Ts[j + i * ldt] : Ts[i + j * ldt];
}

// side 'L': B(b x ncols) := alpha inv(op(T)) B.  RHS blocks of CB columns.
template <typename T, int CB>
__global__ void __launch_bounds__(kThreads)
trsm_left_k(int b, int ncols, T alpha, const T *Tg, long ldt, T *B, long ldb, bool lower_op,
            bool trans, bool unit, const int *status) {
  extern __shared__ __align__(16) unsigned char sm[];
  if (status && *status != PLA_K_OK) return;
  T *Ts = (T *)sm;            // b x b, ld = b
  T *Xs = Ts + b * b;         // b x CB, ld = b + 1
  const int ldx = b + 1;
  for (int t = threadIdx.x; t < b * b; t += kThreads) {
    int i = t % b, j = t / b;
    Ts[t] = Tg[i + (long)j * ldt];
  }
  const int nblk = (ncols + CB - 1) / CB;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const int c0 = blk * CB, nc = min(CB, ncols - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < b * CB; t += kThreads) {
      int i = t % b, c = t / b;
      Xs[i + c * ldx] = c < nc ? alpha * B[i + (long)(c0 + c) * ldb] : T(0);
    }
    __syncthreads();
    const int c = threadIdx.x % CB, grp = threadIdx.x / CB, ngrp = kThreads / CB;
    if (lower_op) {
      for (int l = 0; l < b; l++) {
        if (!unit) {
          if (grp == 0) Xs[l + c * ldx] = Xs[l + c * ldx] / opT(Ts, b, trans, l, l);
          __syncthreads();
        }
        const T x = Xs[l + c * ldx];
        for (int i = l + 1 + grp; i < b; i += ngrp) Xs[i + c * ldx] -= x * opT(Ts, b, trans, i, l);
        __syncthreads();
      }
    } else {
      for (int l = b - 1; l >= 0; l--) {
        if (!unit) {
          if (grp == 0) Xs[l + c * ldx] = Xs[l + c * ldx] / opT(Ts, b, trans, l, l);
          __syncthreads();
        }
        const T x = Xs[l + c * ldx];
        for (int i = grp; i < l; i += ngrp) Xs[i + c * ldx] -= x * opT(Ts, b, trans, i, l);
        __syncthreads();
      }
    }
    for (int t = threadIdx.x; t < b * CB; t += kThreads) {
      int i = t % b, cc = t / b;
      if (cc < nc) B[i + (long)(c0 + cc) * ldb] = Xs[i + cc * ldx];
    }
  }
}

// side 'R': B(nrows x b) := alpha B inv(op(T)).  RHS blocks of RB rows,
// eliminated column by column: B(:,l) *= 1/opT(l,l), then the columns that
// depend on it are updated (the reference dtrsm's right-side order).
template <typename T, int RB>
__global__ void __launch_bounds__(kThreads)
trsm_right_k(int b, int nrows, T alpha, const T *Tg, long ldt, T *B, long ldb, bool upper_op,
             bool trans, bool unit, const int *status) {
  extern __shared__ __align__(16) unsigned char sm[];
  if (status && *status != PLA_K_OK) return;
  T *Ts = (T *)sm;
  T *Xs = Ts + b * b;  // RB x b, ld = RB + 1
  const int ldx = RB + 1;
  for (int t = threadIdx.x; t < b * b; t += kThreads) {
    int i = t % b, j = t / b;
    Ts[t] = Tg[i + (long)j * ldt];
  }
  const int nblk = (nrows + RB - 1) / RB;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const int r0 = blk * RB, nr = min(RB, nrows - r0);
    __syncthreads();
    for (int t = threadIdx.x; t < RB * b; t += kThreads) {
      int i = t % RB, j = t / RB;
      Xs[i + j * ldx] = i < nr ? alpha * B[(long)(r0 + i) + (long)j * ldb] : T(0);
    }
    __syncthreads();
    const int i = threadIdx.x % RB, grp = threadIdx.x / RB, ngrp = kThreads / RB;
    for (int step = 0; step < b; step++) {
      const int l = upper_op ? step : b - 1 - step;
      if (!unit) {
        if (grp == 0) Xs[i + l * ldx] *= T(1) / opT(Ts, b, trans, l, l);
        __syncthreads();
      }
      const T x = Xs[i + l * ldx];
      if (upper_op) {
        for (int j = l + 1 + grp; j < b; j += ngrp) Xs[i + j * ldx] -= x * opT(Ts, b, trans, l, j);
      } else {
        for (int j = grp; j < l; j += ngrp) Xs[i + j * ldx] -= x * opT(Ts, b, trans, l, j);
      }
      __syncthreads();
    }
    for (int t = threadIdx.x; t < RB * b; t += kThreads) {
      int ii = t % RB, j = t / RB;
      if (ii < nr) B[(long)(r0 + ii) + (long)j * ldb] = Xs[ii + j * ldx];
    }
  }
}

// Cholesky of the b x b lower block (SOLVERS/Cholesky/PLA_Local_chol.c:114-138):
// column k fails when a(k,k) <= 0, then a(k,k) = sqrt and the column below is
// scaled by the reciprocal.  The reference's column k is left-looking,
// a(k:b,k) -= A(k:b,0:k) a(k,0:k)' as one dgemv; here the same products are
// applied right-looking, step k subtracting l(j,k) l(i,k) from every a(i,j)
// with k < j <= i.  Each element receives the same fma in the same order
// (k = 0, 1, ...), so the result is bitwise that of the left-looking loop.
//
// The block lives in registers: thread (tx, ty) of a 16 x 16 grid holds the
// 8 x 8 elements (tx + 16p, ty + 16q), lower triangle only.  Per column one
// barrier: the owners of column k (ty = k mod 16) leave its raw values and
// the diagonal in shared memory (two slots by parity), every thread reads
// the diagonal, takes the square root and the reciprocal, scales the column
// values it needs itself (the same multiply the owners keep), and updates its
// elements; tiles wholly left of or above column k are skipped.  The
// left-looking form serialised each thread on a chain of dependent
// shared-memory loads and took 219 us for b = 128 (FP64).
template <typename T>
__global__ void __launch_bounds__(kThreads)
potrf_lower_k(int b, T *A, long lda, int *status, int *info, int base) {
  static_assert(kThreads == 256 && kMaxTri == 128, "a 16 x 16 grid of 8 x 8 register tiles");
  __shared__ T col[2][kMaxTri];  // column k before scaling (rows >= k), by parity of k
  if (*status != PLA_K_OK) return;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T a[8][8];
#pragma unroll
  for (int p = 0; p < 8; p++)
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = tx + 16 * p, j = ty + 16 * q;
      a[p][q] = (i < b && i >= j) ? A[i + (long)j * lda] : T(0);
    }
  if (ty == 0) {
#pragma unroll
    for (int p = 0; p < 8; p++)
      if (tx + 16 * p < b) col[0][tx + 16 * p] = a[p][0];
  }
  __syncthreads();
  int fail = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) {  // columns 16q .. 16q + 15
    for (int kk = 0; kk < 16; kk++) {
      const int k = 16 * q + kk;
      if (k >= b) break;
      const int par = k & 1;
      const T d = col[par][k];  // the same value in every thread: the test is uniform
      if (d <= T(0)) {
        fail = k + 1;
        break;
      }
      const T dk = sqrt(d);
      const T inv = T(1) / dk;
      T li[8], lj[8];
#pragma unroll
      for (int p = 0; p < 8; p++) {
        li[p] = lj[p] = T(0);
        if (16 * p + 15 <= k) continue;
        const int i = tx + 16 * p, j = ty + 16 * p;
        if (i > k && i < b) li[p] = col[par][i] * inv;
        if (j > k && j < b) lj[p] = col[par][j] * inv;
      }
      if (ty == kk) {  // the owners keep column k of L
#pragma unroll
        for (int p = 0; p < 8; p++) {
          const int i = tx + 16 * p;
          if (i == k) a[p][q] = dk;
          else if (i > k) a[p][q] = li[p];
        }
      }
      // Tiles wholly at or left of column k are skipped (a test uniform over
      // the block); only the tile holding column k tests j > k, and only the
      // diagonal tiles i >= j.  Rows at or past b are never written back, so
      // they take part without a test.
#pragma unroll
      for (int p = 0; p < 8; p++) {
        if (16 * p + 15 <= k) continue;
#pragma unroll
        for (int qq = 0; qq <= p; qq++) {
          if (16 * qq + 15 <= k) continue;
          bool ok = qq < p || tx >= ty;
          if (16 * qq <= k) ok = ok && ty + 16 * qq > k;
          if (ok) a[p][qq] = fma(-lj[qq], li[p], a[p][qq]);
        }
      }
      // column k + 1 before scaling, and its diagonal, for the next step
      if (k + 1 < b) {
        if (kk < 15) {
          if (ty == kk + 1) {
#pragma unroll
            for (int p = 0; p < 8; p++)
              if (tx + 16 * p > k && tx + 16 * p < b) col[par ^ 1][tx + 16 * p] = a[p][q];
          }
        } else if (q + 1 < 8) {
          if (ty == 0) {
#pragma unroll
            for (int p = 0; p < 8; p++)
              if (tx + 16 * p > k && tx + 16 * p < b) col[par ^ 1][tx + 16 * p] = a[p][q + 1];
          }
        }
      }
      __syncthreads();
    }
    if (fail) break;
  }
  if (fail) {
    if (threadIdx.x == 0) {
      *info = base + fail;
      *status = PLA_K_NOT_SPD;
    }
    return;  // the reference leaves A11 unwritten on failure (PLA_Chol.c:181-185)
  }
#pragma unroll
  for (int p = 0; p < 8; p++)
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = tx + 16 * p, j = ty + 16 * q;
      if (i < b && i >= j) A[i + (long)j * lda] = a[p][q];
    }
}

int g_sms = 0;
int sms() {
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  return g_sms;
}

template <typename T>
int trsm_small_t(char side, char uplo, char trans, char diag, int b, int other, double alpha,
                 const void *Tm, long ldt, void *B, long ldb, const int *status, cudaStream_t s) {
  if (b <= 0 || other <= 0) return 0;
  if (b > kMaxTri) return (int)cudaErrorInvalidValue;
  const bool tr = trans != 'N', unit = diag == 'U';
  if (side == 'L') {
    constexpr int CB = 32;
    const bool lower_op = (uplo == 'L') != tr;
    size_t sm = ((size_t)b * b + (size_t)(b + 1) * CB) * sizeof(T);
    cudaFuncSetAttribute(trsm_left_k<T, CB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int nblk = (other + CB - 1) / CB;
    int grid = nblk < sms() ? nblk : sms();
    trsm_left_k<T, CB><<<grid, kThreads, sm, s>>>(b, other, (T)alpha, (const T *)Tm, ldt, (T *)B,
                                                  ldb, lower_op, tr, unit, status);
  } else {
    constexpr int RB = 64;
    const bool upper_op = (uplo == 'U') != tr;
    size_t sm = ((size_t)b * b + (size_t)(RB + 1) * b) * sizeof(T);
    cudaFuncSetAttribute(trsm_right_k<T, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int nblk = (other + RB - 1) / RB;
    int grid = nblk < sms() ? nblk : sms();
    trsm_right_k<T, RB><<<grid, kThreads, sm, s>>>(b, other, (T)alpha, (const T *)Tm, ldt, (T *)B,
                                                   ldb, upper_op, tr, unit, status);
  }
  pla_k_count(1);
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" int pla_k_trsm_small(int dt, char side, char uplo, char trans, char diag, int b,
                                int other, double alpha, const void *T, long ldt, void *B,
                                long ldb, const int *status, cudaStream_t s) {
  if (dt == MPI_DOUBLE)
    return trsm_small_t<double>(side, uplo, trans, diag, b, other, alpha, T, ldt, B, ldb, status, s);
  if (dt == MPI_FLOAT)
    return trsm_small_t<float>(side, uplo, trans, diag, b, other, alpha, T, ldt, B, ldb, status, s);
  return (int)cudaErrorInvalidValue;
}

extern "C" int pla_k_potrf_lower(int dt, int b, void *A, long lda, int *status, int *info,
                                 int base, cudaStream_t s) {
  if (b <= 0) return 0;
  if (b > kMaxTri) return (int)cudaErrorInvalidValue;
  if (dt == MPI_DOUBLE) {
    potrf_lower_k<double><<<1, kThreads, 0, s>>>(b, (double *)A, lda, status, info, base);
  } else if (dt == MPI_FLOAT) {
    potrf_lower_k<float><<<1, kThreads, 0, s>>>(b, (float *)A, lda, status, info, base);
  } else {
    return (int)cudaErrorInvalidValue;
  }
  pla_k_count(1);
  return (int)cudaGetLastError();
}

// Blocked solve op(A) X = B (A n x n triangular, B n x nrhs): diagonal blocks
// of 128 by substitution, the rest of the rows updated by GEMV (one
// right-hand side) or GEMM, in the order op(A)'s triangle dictates.
extern "C" int pla_k_trsv_blocked(int dt, char uplo, char trans, char diag, int n, int nrhs,
                                  const void *A, long lda, void *B, long ldb, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return 0;
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  const bool tr = trans != 'N';
  const bool forward = (uplo == 'L') != tr;  // op(A) lower -> top to bottom
  const int nb = kMaxTri;
  auto a_at = [&](long i, long j) { return (const char *)A + (i + j * lda) * es; };
  auto b_at = [&](long i) { return (char *)B + i * es; };
  const int nblk = (n + nb - 1) / nb;
  for (int q = 0; q < nblk; q++) {
    const int blk = forward ? q : nblk - 1 - q;
    const int k0 = blk * nb, kb = n - k0 < nb ? n - k0 : nb;
    int r = pla_k_trsm_small(dt, 'L', uplo, trans, diag, kb, nrhs, 1.0, a_at(k0, k0), lda,
                             b_at(k0), ldb, nullptr, s);
    if (r) return r;
    // remaining rows: B_rest -= op(A)(rest, blk) X_blk
    int r0, rn;
    if (forward) { r0 = k0 + kb; rn = n - r0; }
    else { r0 = 0; rn = k0; }
    if (rn <= 0) continue;
    // op(A)(rest, blk): for no-transpose it is A(rest, blk); for transpose it
    // is A(blk, rest)'
    const void *Ablk = tr ? a_at(k0, r0) : a_at(r0, k0);
    if (nrhs == 1) {
      r = pla_k_gemv(dt, tr ? PLA_TRANSPOSE : PLA_NO_TRANSPOSE, tr ? kb : rn, tr ? rn : kb, -1.0,
                     Ablk, lda, b_at(k0), 1.0, b_at(r0), s);
    } else {
      r = pla_k_gemm(dt, tr ? PLA_TRANSPOSE : PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, rn, nrhs, kb,
                     -1.0, Ablk, lda, b_at(k0), ldb, 1.0, b_at(r0), ldb, 0, nullptr, s);
    }
    if (r) return r;
  }
  return 0;
}
