/*
 * CPU oracle for the dense direct-solve path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms, used by tests/, by
 * __graft_entry__.smoke() and by the CPU-baseline leg of bench.py as the
 * checker.  The product never links or calls this file.
 *
 * Pinned against the upstream PLAPACK compiled from its own sources
 * (oracle/_ref, see the Makefile): tests/test_oracle.py checks that both give
 * identical pivot vectors and factors within rounding on the committed golden
 * inputs, and tests/golden/ holds the reference's outputs.
 *
 * Storage is column-major with an explicit leading dimension; pivots use the
 * reference encoding: piv[i] = offset (>= 0) from row i to the row swapped
 * into position i (SOLVERS/LU/PLA_seq_lu.c:35, zero_or_one = 0).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

/* uniform [-1,1) fill exactly as TEST/create_problem.c:31,49-51 on rank 0:
 * srand48(0 * 1793) once, then drand48()*2-1 in column-major order */
void oracle_fill_drand48(long seed, long count, double *out) {
  long i;
  srand48(seed);
  for (i = 0; i < count; i++) out[i] = drand48() * 2.0 - 1.0;
}

#define DEFINE_ORACLE(T, P)                                                    \
  /* BLAS idamax: first index of the largest |x_i| (0-based here) */           \
  static int P##_iamax(int n, const T *x) {                                    \
    int i, best = 0;                                                           \
    T m;                                                                       \
    if (n <= 0) return 0;                                                      \
    m = (T)fabs(x[0]);                                                         \
    for (i = 1; i < n; i++)                                                    \
      if ((T)fabs(x[i]) > m) { m = (T)fabs(x[i]); best = i; }                  \
    return best;                                                               \
  }                                                                            \
                                                                               \
  /* Unblocked right-looking LU with partial pivoting, full-width row swaps,   \
   * reciprocal scaling and a rank-1 update per column:                        \
   * SOLVERS/LU/PLA_seq_lu.c:21-46 (PLA_dlu / PLA_slu). */                     \
  void oracle_##P##lu_unblocked(int m, int n, T *A, int lda, int *piv) {       \
    int j, i, c, k = m < n ? m : n;                                            \
    for (j = 0; j < k; j++) {                                                  \
      int p = j + P##_iamax(m - j, &A[IDX(j, j, lda)]);                        \
      T inv;                                                                   \
      piv[j] = p - j;                                                          \
      if (p != j)                                                              \
        for (c = 0; c < n; c++) {                                              \
          T t = A[IDX(j, c, lda)];                                             \
          A[IDX(j, c, lda)] = A[IDX(p, c, lda)];                               \
          A[IDX(p, c, lda)] = t;                                               \
        }                                                                      \
      inv = (T)1.0 / A[IDX(j, j, lda)];                                        \
      for (i = j + 1; i < m; i++) A[IDX(i, j, lda)] = inv * A[IDX(i, j, lda)]; \
      for (c = j + 1; c < n; c++) {                                            \
        T y = A[IDX(j, c, lda)];                                               \
        if (y != 0) {                                                          \
          T t = (T)-1.0 * y;                                                   \
          for (i = j + 1; i < m; i++)                                          \
            A[IDX(i, c, lda)] += A[IDX(i, j, lda)] * t;                        \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }                                                                            \
                                                                               \
  /* Row interchanges in sequence, as PLA_Apply_pivots_to_rows does           \
   * (SOLVERS/LU/PLA_Apply_pivots_new.c:104-164): for i = 0..npiv-1 swap row   \
   * i with row i + piv[i], over columns [c0, c1). */                          \
  void oracle_##P##apply_pivots(int npiv, const int *piv, T *B, int ldb,       \
                                int c0, int c1) {                              \
    int i, c;                                                                  \
    for (i = 0; i < npiv; i++) {                                               \
      int p = i + piv[i];                                                      \
      if (p == i) continue;                                                    \
      for (c = c0; c < c1; c++) {                                              \
        T t = B[IDX(i, c, ldb)];                                               \
        B[IDX(i, c, ldb)] = B[IDX(p, c, ldb)];                                 \
        B[IDX(p, c, ldb)] = t;                                                 \
      }                                                                        \
    }                                                                          \
  }                                                                            \
                                                                               \
  /* Blocked right-looking LU, SOLVERS/LU/PLA_LU.c:103-192 on a 1x1 template:  \
   *  - panel A(k:m, k:k+b) factored unblocked, row swaps inside the panel     \
   *    only (PLA_LU_mv.c:52-82: Iamax, Pivot_rows_mv, inv_scal, ger)          \
   *  - the panel's pivots applied to the remaining columns of A_B (the        \
   *    already-factored L columns and the trailing columns, :152)             \
   *  - A12 <- inv(L11) A12 (unit lower, :174-178)                             \
   *  - A22 <- A22 - A21 A12 (:185-186).                                      \
   * With left == 0 the pivots skip the already-factored L columns: the       \
   * LINPACK-style variant, SOLVERS/LINPACK/PLA_LU_linpack.c:145 (pivots      \
   * applied to A_BR only). */                                                 \
  static void P##lu_blocked_ex(int m, int n, int nb, T *A, int lda, int *piv,   \
                               int left) {                                      \
    int k, kmax = m < n ? m : n;                                               \
    for (k = 0; k < kmax; k += nb) {                                           \
      int b = kmax - k < nb ? kmax - k : nb;                                   \
      int r = m - k, i, j, l, c;                                               \
      T *Ak = &A[IDX(k, k, lda)];                                              \
      /* panel: r x b, pivots relative to row k */                             \
      for (j = 0; j < b; j++) {                                                \
        int p = j + P##_iamax(r - j, &Ak[IDX(j, j, lda)]);                     \
        T inv;                                                                 \
        piv[k + j] = p - j;                                                    \
        if (p != j)                                                            \
          for (c = 0; c < b; c++) {                                            \
            T t = Ak[IDX(j, c, lda)];                                          \
            Ak[IDX(j, c, lda)] = Ak[IDX(p, c, lda)];                           \
            Ak[IDX(p, c, lda)] = t;                                            \
          }                                                                    \
        inv = (T)1.0 / Ak[IDX(j, j, lda)];                                     \
        for (i = j + 1; i < r; i++)                                            \
          Ak[IDX(i, j, lda)] = inv * Ak[IDX(i, j, lda)];                       \
        for (c = j + 1; c < b; c++) {                                          \
          T y = Ak[IDX(j, c, lda)];                                            \
          if (y != 0) {                                                        \
            T t = (T)-1.0 * y;                                                 \
            for (i = j + 1; i < r; i++)                                        \
              Ak[IDX(i, c, lda)] += Ak[IDX(i, j, lda)] * t;                    \
          }                                                                    \
        }                                                                      \
      }                                                                        \
      /* pivots to the columns left and right of the panel */                  \
      if (left)                                                                \
        oracle_##P##apply_pivots(b, &piv[k], &A[IDX(k, 0, lda)], lda, 0, k);   \
      oracle_##P##apply_pivots(b, &piv[k], &A[IDX(k, 0, lda)], lda, k + b, n); \
      /* A12 <- inv(L11) A12, column by column */                              \
      for (c = k + b; c < n; c++)                                              \
        for (l = 0; l < b; l++) {                                              \
          T x = A[IDX(k + l, c, lda)];                                         \
          if (x != 0)                                                          \
            for (i = l + 1; i < b; i++)                                        \
              A[IDX(k + i, c, lda)] -= x * A[IDX(k + i, k + l, lda)];          \
        }                                                                      \
      /* A22 <- A22 - A21 A12 */                                               \
      for (c = k + b; c < n; c++)                                              \
        for (l = 0; l < b; l++) {                                              \
          T t = (T)-1.0 * A[IDX(k + l, c, lda)];                               \
          for (i = k + b; i < m; i++)                                          \
            A[IDX(i, c, lda)] += t * A[IDX(i, k + l, lda)];                    \
        }                                                                      \
    }                                                                          \
  }                                                                            \
  void oracle_##P##lu_blocked(int m, int n, int nb, T *A, int lda, int *piv) { \
    P##lu_blocked_ex(m, n, nb, A, lda, piv, 1);                                \
  }                                                                            \
  void oracle_##P##lu_linpack(int m, int n, int nb, T *A, int lda, int *piv) { \
    P##lu_blocked_ex(m, n, nb, A, lda, piv, 0);                                \
  }                                                                            \
                                                                               \
  /* Unblocked lower Cholesky, left-looking column form of PLA_dchol           \
   * (SOLVERS/Cholesky/PLA_Local_chol.c:103-143): gemv update of column k,     \
   * fail with k+1 when a(k,k) <= 0, sqrt, scale below by the reciprocal. */   \
  int oracle_##P##chol_unblocked(int n, T *A, int lda) {                       \
    int k, i, l;                                                               \
    for (k = 0; k < n; k++) {                                                  \
      T inv;                                                                   \
      for (l = 0; l < k; l++) {                                                \
        T t = (T)-1.0 * A[IDX(k, l, lda)];                                     \
        for (i = k; i < n; i++) A[IDX(i, k, lda)] += t * A[IDX(i, l, lda)];    \
      }                                                                        \
      if (A[IDX(k, k, lda)] <= 0) return k + 1;                                \
      A[IDX(k, k, lda)] = (T)sqrt(A[IDX(k, k, lda)]);                          \
      inv = (T)1.0 / A[IDX(k, k, lda)];                                        \
      for (i = k + 1; i < n; i++) A[IDX(i, k, lda)] = inv * A[IDX(i, k, lda)]; \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  /* Blocked right-looking lower Cholesky, SOLVERS/Cholesky/PLA_Chol.c:159-224:\
   * unblocked factor of A11, A21 <- A21 inv(L11'), A22 <- A22 - A21 A21'     \
   * (lower triangle only).  Returns k + the local failing index. */          \
  int oracle_##P##chol_blocked(int n, int nb, T *A, int lda) {                 \
    int k;                                                                     \
    for (k = 0; k < n; k += nb) {                                              \
      int b = n - k < nb ? n - k : nb, i, j, l;                                \
      int info = oracle_##P##chol_unblocked(b, &A[IDX(k, k, lda)], lda);       \
      if (info) return k + info;                                               \
      /* dtrsm(R, L, T, N): columns in order, reciprocal of the diagonal */    \
      for (l = 0; l < b; l++) {                                                \
        T inv = (T)1.0 / A[IDX(k + l, k + l, lda)];                            \
        for (i = k + b; i < n; i++) A[IDX(i, k + l, lda)] *= inv;              \
        for (j = l + 1; j < b; j++) {                                          \
          T t = A[IDX(k + j, k + l, lda)];                                     \
          if (t != 0)                                                          \
            for (i = k + b; i < n; i++)                                        \
              A[IDX(i, k + j, lda)] -= t * A[IDX(i, k + l, lda)];              \
        }                                                                      \
      }                                                                        \
      /* lower A22 -= A21 A21' */                                              \
      for (j = k + b; j < n; j++)                                              \
        for (l = 0; l < b; l++) {                                              \
          T t = (T)-1.0 * A[IDX(j, k + l, lda)];                               \
          for (i = j; i < n; i++)                                              \
            A[IDX(i, j, lda)] += t * A[IDX(i, k + l, lda)];                    \
        }                                                                      \
    }                                                                          \
    return 0;                                                                  \
  }                                                                            \
                                                                               \
  /* op(A) x = b in place; uplo 'L'/'U', trans 'N'/'T', diag 'U'/'N'.         \
   * The lower no-transpose case is the dot (left-looking) form of            \
   * BLAS2/PLA_Trsv_ln.c:54-79 (b1 -= A10 x0, then solve the diagonal). */    \
  void oracle_##P##trsv(char uplo, char trans, char diag, int n, const T *A,   \
                        int lda, T *x) {                                       \
    int i, j;                                                                  \
    const int unit = (diag == 'U');                                            \
    const int lower = (uplo == 'L'), notrans = (trans == 'N');                 \
    if (lower == notrans) {                                                    \
      /* forward: L x = b or U' x = b */                                       \
      for (i = 0; i < n; i++) {                                                \
        T s = x[i];                                                            \
        for (j = 0; j < i; j++)                                                \
          s -= (lower ? A[IDX(i, j, lda)] : A[IDX(j, i, lda)]) * x[j];         \
        x[i] = unit ? s : s / A[IDX(i, i, lda)];                               \
      }                                                                        \
    } else {                                                                   \
      for (i = n - 1; i >= 0; i--) {                                           \
        T s = x[i];                                                            \
        for (j = i + 1; j < n; j++)                                            \
          s -= (lower ? A[IDX(j, i, lda)] : A[IDX(i, j, lda)]) * x[j];         \
        x[i] = unit ? s : s / A[IDX(i, i, lda)];                               \
      }                                                                        \
    }                                                                          \
  }                                                                            \
                                                                               \
  /* C := alpha op(A) op(B) + beta C, plain triple loop */                     \
  void oracle_##P##gemm(char ta, char tb, int m, int n, int k, T alpha,        \
                        const T *A, int lda, const T *B, int ldb, T beta,      \
                        T *C, int ldc) {                                       \
    int i, j, l;                                                               \
    for (j = 0; j < n; j++)                                                    \
      for (i = 0; i < m; i++) {                                                \
        T s = 0;                                                               \
        for (l = 0; l < k; l++) {                                              \
          T a = (ta == 'N') ? A[IDX(i, l, lda)] : A[IDX(l, i, lda)];           \
          T b = (tb == 'N') ? B[IDX(l, j, ldb)] : B[IDX(j, l, ldb)];           \
          s += a * b;                                                          \
        }                                                                      \
        C[IDX(i, j, ldc)] =                                                    \
            (beta == 0) ? alpha * s : alpha * s + beta * C[IDX(i, j, ldc)];    \
      }                                                                        \
  }                                                                            \
                                                                               \
  /* B := alpha inv(op(A)) B (side 'L') or alpha B inv(op(A)) (side 'R'),     \
   * solved column by column / row by row with oracle_trsv. */                \
  void oracle_##P##trsm(char side, char uplo, char trans, char diag, int m,    \
                        int n, T alpha, const T *A, int lda, T *B, int ldb) {  \
    int i, j;                                                                  \
    if (side == 'L') {                                                         \
      for (j = 0; j < n; j++) {                                                \
        for (i = 0; i < m; i++) B[IDX(i, j, ldb)] *= alpha;                    \
        oracle_##P##trsv(uplo, trans, diag, m, A, lda, &B[IDX(0, j, ldb)]);    \
      }                                                                        \
    } else {                                                                   \
      /* X op(A) = alpha B  <=>  op(A)' X' = alpha B' */                      \
      T *row = (T *)malloc(sizeof(T) * (size_t)(n > 0 ? n : 1));               \
      char t2 = (trans == 'N') ? 'T' : 'N';                                    \
      for (i = 0; i < m; i++) {                                                \
        for (j = 0; j < n; j++) row[j] = alpha * B[IDX(i, j, ldb)];            \
        oracle_##P##trsv(uplo, t2, diag, n, A, lda, row);                      \
        for (j = 0; j < n; j++) B[IDX(i, j, ldb)] = row[j];                    \
      }                                                                        \
      free(row);                                                               \
    }                                                                          \
  }

DEFINE_ORACLE(double, d)
DEFINE_ORACLE(float, s)

/* ---------------------------------------------------------------------------
 * Model of the library's OWN tournament-pivoted fp32 panel (the mixed LU's
 * sub-panels, plapack_b200/csrc/k_tslu.cu).  It has no counterpart in the
 * reference -- whose panel is partial pivoting -- and is here only so the GPU
 * test can check that kernel bit for bit: the same tree (leaf row blocks of R
 * rows, passes of at most 512 candidate rows carrying the rows kept, sets of
 * 16 merged per node), the same candidate order (|x| as bits + 2, NaN 1,
 * then the smaller row), the same arithmetic (l = x * (1/u), fmaf(-l, u, x);
 * inv(U11) by back substitution per column, the rows below as (row) inv(U11)
 * accumulated with fmaf) in the same order.
 * r x w panel (w <= 32), column-major A (lda), P = min(max_ctas, ceil(r / 512))
 * leaf blocks of R = ceil(r / P) rows.  Pivots in the
 * reference's offset encoding; A overwritten by L \ U under them.
 * ------------------------------------------------------------------------- */
#define TS_W 32
#define TS_CAND 512
#define TS_GROUP 16

static unsigned long long ts_key(float x, int row) {
  unsigned b;
  unsigned k;
  memcpy(&b, &x, 4);
  b &= 0x7fffffffu;
  k = b > 0x7f800000u ? 1u : b + 2u;
  return ((unsigned long long)k << 32) | (0xffffffffu - (unsigned)row);
}

/* partial-pivoting LU of the candidate rows ids (entries < 0 empty); keeps
 * min(live, w) rows in keep[] in pivot order, their factored rows in rows[] */
static int ts_select(const float *A, int lda, int w, const int *ids, int cnt, int *keep,
                     float *rows) {
  static float v[TS_CAND][TS_W];
  int live[TS_CAND], i, j, c, nlive = 0, k;
  for (i = 0; i < cnt; i++) {
    live[i] = ids[i] >= 0;
    nlive += live[i];
    for (c = 0; c < TS_W; c++) v[i][c] = (live[i] && c < w) ? A[IDX(ids[i], c, lda)] : 0.f;
  }
  k = nlive < w ? nlive : w;
  for (j = 0; j < k; j++) {
    unsigned long long best = 0;
    int bi = -1;
    float u[TS_W], inv;
    for (i = 0; i < cnt; i++)
      if (live[i]) {
        unsigned long long kk = ts_key(v[i][j], ids[i]);
        if (kk > best) { best = kk; bi = i; }
      }
    for (c = 0; c < TS_W; c++) u[c] = v[bi][c];
    live[bi] = 0;
    keep[j] = ids[bi];
    if (rows)
      for (c = 0; c < w; c++) rows[j * TS_W + c] = v[bi][c];
    inv = 1.0f / u[j];
    for (i = 0; i < cnt; i++)
      if (live[i]) {
        float l = v[i][j] * inv;
        v[i][j] = l;
        for (c = j + 1; c < TS_W; c++) v[i][c] = fmaf(-l, u[c], v[i][c]);
      }
  }
  return k;
}

void oracle_slu_tournament(int r, int w, int max_ctas, float *A, int lda, int *piv) {
  int P = max_ctas, R, b, nsets, level_off = 0, i, j, c;
  int maxP = (r + TS_CAND - 1) / TS_CAND;
  int *slots, ids[TS_CAND], keep[TS_W], kept, root_done = 0;
  static float rows[TS_W * TS_W], stage[TS_W * TS_W], uinv[TS_W * TS_W];
  int e_pos[2 * TS_W], e_row[2 * TS_W], ne;
  if (P > maxP) P = maxP;
  if (P < 1) P = 1;
  R = (r + P - 1) / P;
  P = (r + R - 1) / R;
  slots = (int *)malloc(sizeof(int) * 2 * (size_t)P * TS_W);
  /* leaves */
  for (b = 0; b < P; b++) {
    int row0 = b * R, row1 = row0 + R < r ? row0 + R : r, next = row0;
    kept = 0;
    for (;;) {
      int take = row1 - next < TS_CAND - kept ? row1 - next : TS_CAND - kept, cnt, last;
      for (i = 0; i < kept; i++) ids[i] = keep[i];
      for (i = 0; i < take; i++) ids[kept + i] = next + i;
      next += take;
      last = next >= row1;
      cnt = kept + take;
      if (last && P > 1 && cnt <= w) {
        for (i = 0; i < TS_W; i++) keep[i] = i < cnt ? ids[i] : -1;
        kept = cnt;
      } else {
        kept = ts_select(A, lda, w, ids, cnt, keep, (last && P == 1) ? rows : NULL);
      }
      if (last) break;
    }
    for (i = 0; i < TS_W; i++) slots[(size_t)b * TS_W + i] = i < kept ? keep[i] : -1;
  }
  root_done = P == 1;
  nsets = P;
  while (!root_done) {
    int ngroups = (nsets + TS_GROUP - 1) / TS_GROUP, g;
    for (g = 0; g < ngroups; g++) {
      int gsize = nsets - g * TS_GROUP < TS_GROUP ? nsets - g * TS_GROUP : TS_GROUP;
      int cnt = gsize * TS_W;
      for (i = 0; i < cnt; i++) ids[i] = slots[(size_t)(level_off + g * TS_GROUP) * TS_W + i];
      kept = ts_select(A, lda, w, ids, cnt, keep, ngroups == 1 ? rows : NULL);
      for (i = 0; i < TS_W; i++)
        slots[(size_t)(level_off + nsets + g) * TS_W + i] = i < kept ? keep[i] : -1;
    }
    level_off += nsets;
    nsets = ngroups;
    root_done = nsets == 1;
  }
  /* the interchanges as sequential swaps */
  ne = w;
  for (i = 0; i < w; i++) { e_pos[i] = i; e_row[i] = i; }
  for (j = 0; j < w; j++)
    if (keep[j] >= w) { e_pos[ne] = keep[j]; e_row[ne] = keep[j]; ne++; }
  for (j = 0; j < w; j++) {
    int e = 0;
    while (e_row[e] != keep[j]) e++;
    piv[j] = e_pos[e] - j;
    e_row[e] = e_row[j];
    e_row[j] = keep[j];
  }
  for (j = 0; j < w; j++)
    for (c = 0; c < w; c++) stage[j * TS_W + c] = A[IDX(j, c, lda)];
  /* inv(U11), column by column: U y = e_c by back substitution */
  for (c = 0; c < TS_W; c++) {
    float y[TS_W];
    int q;
    for (i = 0; i < TS_W; i++) y[i] = 0.f;
    if (c < w)
      for (i = c; i >= 0; i--) {
        float acc = i == c ? 1.f : 0.f;
        for (q = i + 1; q <= c; q++) acc = fmaf(-rows[i * TS_W + q], y[q], acc);
        y[i] = acc * (1.0f / rows[i * TS_W + i]);
      }
    for (i = 0; i < TS_W; i++) uinv[i * TS_W + c] = y[i];
  }
  /* the panel without further pivoting: row i >= w := (source row) inv(U11) */
  for (i = w; i < r; i++) {
    float b2[TS_W], x[TS_W];
    int q = -1, e, k2;
    for (e = w; e < ne; e++)
      if (e_pos[e] == i && e_row[e] != e_pos[e]) q = e_row[e];
    for (c = 0; c < TS_W; c++) {
      b2[c] = c < w ? (q >= 0 ? stage[q * TS_W + c] : A[IDX(i, c, lda)]) : 0.f;
      x[c] = 0.f;
    }
    for (k2 = 0; k2 < TS_W; k2++)
      for (c = k2; c < TS_W; c++) x[c] = fmaf(b2[k2], uinv[k2 * TS_W + c], x[c]);
    for (c = 0; c < w; c++) A[IDX(i, c, lda)] = x[c];
  }
  for (i = 0; i < w; i++)
    for (c = 0; c < w; c++) A[IDX(i, c, lda)] = rows[i * TS_W + c];
  free(slots);
}
