/*
 * Host BLAS for the CPU oracle (test infrastructure only).
 *
 * The upstream PLAPACK build links `-lblas` (Make.include:41), and its
 * Dockerfile installs Ubuntu 16.04's `libblas-dev`, i.e. the netlib reference
 * BLAS (LAPACK 3.6.0 era).  That library is not part of the reference tree, so
 * this file restates the published reference-BLAS algorithms for the real
 * routines PLAPACK's hot path calls, following the netlib loop orders so that
 * rounding matches a plain reference BLAS (no FMA contraction: build with
 * -ffp-contract=off).  Complex routines are not on the path and abort.
 *
 * Fortran calling convention: every argument by reference, trailing '_'.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

static int lsame(const char *a, char b) {
  char c = *a;
  if (c >= 'a' && c <= 'z') c = (char)(c - 'a' + 'A');
  return c == b;
}

/* start offset for a strided vector of length n with increment inc */
#define VSTART(n, inc) ((inc) > 0 ? 0 : (long)(1 - (n)) * (inc))

#define DEFINE_REAL_BLAS(T, P)                                                 \
  /* index of the first element of max |x| (1-based; 0 when n < 1) */          \
  int i##P##amax_(const int *n, const T *x, const int *incx) {                 \
    int i, best = 1;                                                           \
    T m;                                                                       \
    long ix;                                                                   \
    if (*n < 1 || *incx <= 0) return 0;                                        \
    if (*n == 1) return 1;                                                     \
    m = (T)fabs(x[0]);                                                         \
    ix = *incx;                                                                \
    for (i = 2; i <= *n; i++, ix += *incx) {                                   \
      T v = (T)fabs(x[ix]);                                                    \
      if (v > m) { best = i; m = v; }                                          \
    }                                                                          \
    return best;                                                               \
  }                                                                            \
  T P##asum_(const int *n, const T *x, const int *incx) {                      \
    int i;                                                                     \
    T s = 0;                                                                   \
    long ix = 0;                                                               \
    if (*n < 1 || *incx <= 0) return 0;                                        \
    for (i = 0; i < *n; i++, ix += *incx) s += (T)fabs(x[ix]);                 \
    return s;                                                                  \
  }                                                                            \
  void P##axpy_(const int *n, const T *a, const T *x, const int *incx, T *y,   \
                const int *incy) {                                             \
    int i;                                                                     \
    long ix = VSTART(*n, *incx), iy = VSTART(*n, *incy);                       \
    if (*n < 1 || *a == 0) return;                                             \
    for (i = 0; i < *n; i++, ix += *incx, iy += *incy) y[iy] += *a * x[ix];    \
  }                                                                            \
  void P##copy_(const int *n, const T *x, const int *incx, T *y,               \
                const int *incy) {                                             \
    int i;                                                                     \
    long ix = VSTART(*n, *incx), iy = VSTART(*n, *incy);                       \
    for (i = 0; i < *n; i++, ix += *incx, iy += *incy) y[iy] = x[ix];          \
  }                                                                            \
  T P##dot_(const int *n, const T *x, const int *incx, const T *y,             \
            const int *incy) {                                                 \
    int i;                                                                     \
    T s = 0;                                                                   \
    long ix = VSTART(*n, *incx), iy = VSTART(*n, *incy);                       \
    for (i = 0; i < *n; i++, ix += *incx, iy += *incy) s += x[ix] * y[iy];     \
    return s;                                                                  \
  }                                                                            \
  /* scaled sum of squares, so that no intermediate overflows */               \
  T P##nrm2_(const int *n, const T *x, const int *incx) {                      \
    int i;                                                                     \
    T scale = 0, ssq = 1;                                                      \
    long ix = 0;                                                               \
    if (*n < 1 || *incx < 1) return 0;                                         \
    if (*n == 1) return (T)fabs(x[0]);                                         \
    for (i = 0; i < *n; i++, ix += *incx) {                                    \
      if (x[ix] != 0) {                                                        \
        T ax = (T)fabs(x[ix]);                                                 \
        if (scale < ax) {                                                      \
          ssq = 1 + ssq * (scale / ax) * (scale / ax);                         \
          scale = ax;                                                          \
        } else {                                                               \
          ssq += (ax / scale) * (ax / scale);                                  \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    return scale * (T)sqrt(ssq);                                               \
  }                                                                            \
  void P##scal_(const int *n, const T *a, T *x, const int *incx) {             \
    int i;                                                                     \
    long ix = 0;                                                               \
    if (*n < 1 || *incx <= 0) return;                                          \
    for (i = 0; i < *n; i++, ix += *incx) x[ix] = *a * x[ix];                  \
  }                                                                            \
  void P##swap_(const int *n, T *x, const int *incx, T *y, const int *incy) {  \
    int i;                                                                     \
    long ix = VSTART(*n, *incx), iy = VSTART(*n, *incy);                       \
    for (i = 0; i < *n; i++, ix += *incx, iy += *incy) {                       \
      T t = x[ix];                                                             \
      x[ix] = y[iy];                                                           \
      y[iy] = t;                                                               \
    }                                                                          \
  }                                                                            \
  /* y := alpha*op(A)*x + beta*y */                                            \
  void P##gemv_(const char *tr, const int *m, const int *n, const T *alpha,    \
                const T *A, const int *lda, const T *x, const int *incx,       \
                const T *beta, T *y, const int *incy) {                        \
    int i, j, leny, lenx;                                                      \
    long ix, iy, kx, ky;                                                       \
    const long ld = *lda;                                                      \
    if (*m == 0 || *n == 0 || (*alpha == 0 && *beta == 1)) return;             \
    if (lsame(tr, 'N')) { lenx = *n; leny = *m; }                              \
    else { lenx = *m; leny = *n; }                                             \
    kx = VSTART(lenx, *incx);                                                  \
    ky = VSTART(leny, *incy);                                                  \
    if (*beta != 1) {                                                          \
      for (i = 0, iy = ky; i < leny; i++, iy += *incy)                         \
        y[iy] = (*beta == 0) ? (T)0 : *beta * y[iy];                           \
    }                                                                          \
    if (*alpha == 0) return;                                                   \
    if (lsame(tr, 'N')) {                                                      \
      for (j = 0, ix = kx; j < *n; j++, ix += *incx) {                         \
        T temp = *alpha * x[ix];                                               \
        for (i = 0, iy = ky; i < *m; i++, iy += *incy)                         \
          y[iy] += temp * A[i + j * ld];                                       \
      }                                                                        \
    } else {                                                                   \
      for (j = 0, iy = ky; j < *n; j++, iy += *incy) {                         \
        T temp = 0;                                                            \
        for (i = 0, ix = kx; i < *m; i++, ix += *incx)                         \
          temp += A[i + j * ld] * x[ix];                                       \
        y[iy] += *alpha * temp;                                                \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* A := alpha*x*y' + A */                                                    \
  void P##ger_(const int *m, const int *n, const T *alpha, const T *x,         \
               const int *incx, const T *y, const int *incy, T *A,             \
               const int *lda) {                                               \
    int i, j;                                                                  \
    long ix, jy = VSTART(*n, *incy), kx = VSTART(*m, *incx);                   \
    const long ld = *lda;                                                      \
    if (*m == 0 || *n == 0 || *alpha == 0) return;                             \
    for (j = 0; j < *n; j++, jy += *incy) {                                    \
      if (y[jy] != 0) {                                                        \
        T temp = *alpha * y[jy];                                               \
        for (i = 0, ix = kx; i < *m; i++, ix += *incx)                         \
          A[i + j * ld] += x[ix] * temp;                                       \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* solve op(A)*x = b in place, A triangular */                               \
  void P##trsv_(const char *uplo, const char *tr, const char *diag,            \
                const int *n, const T *A, const int *lda, T *x,                \
                const int *incx) {                                             \
    int i, j;                                                                  \
    const int nounit = lsame(diag, 'N');                                       \
    const long ld = *lda, inc = *incx;                                         \
    const long kx = VSTART(*n, *incx);                                         \
    if (*n == 0) return;                                                       \
    if (lsame(tr, 'N')) {                                                      \
      if (lsame(uplo, 'U')) {                                                  \
        for (j = *n - 1; j >= 0; j--) {                                        \
          if (x[kx + j * inc] != 0) {                                          \
            T temp;                                                            \
            if (nounit) x[kx + j * inc] /= A[j + j * ld];                      \
            temp = x[kx + j * inc];                                            \
            for (i = j - 1; i >= 0; i--)                                       \
              x[kx + i * inc] -= temp * A[i + j * ld];                         \
          }                                                                    \
        }                                                                      \
      } else {                                                                 \
        for (j = 0; j < *n; j++) {                                             \
          if (x[kx + j * inc] != 0) {                                          \
            T temp;                                                            \
            if (nounit) x[kx + j * inc] /= A[j + j * ld];                      \
            temp = x[kx + j * inc];                                            \
            for (i = j + 1; i < *n; i++)                                       \
              x[kx + i * inc] -= temp * A[i + j * ld];                         \
          }                                                                    \
        }                                                                      \
      }                                                                        \
    } else {                                                                   \
      if (lsame(uplo, 'U')) {                                                  \
        for (j = 0; j < *n; j++) {                                             \
          T temp = x[kx + j * inc];                                            \
          for (i = 0; i < j; i++) temp -= A[i + j * ld] * x[kx + i * inc];     \
          if (nounit) temp /= A[j + j * ld];                                   \
          x[kx + j * inc] = temp;                                              \
        }                                                                      \
      } else {                                                                 \
        for (j = *n - 1; j >= 0; j--) {                                        \
          T temp = x[kx + j * inc];                                            \
          for (i = *n - 1; i > j; i--) temp -= A[i + j * ld] * x[kx + i * inc];\
          if (nounit) temp /= A[j + j * ld];                                   \
          x[kx + j * inc] = temp;                                              \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* x := op(A)*x, A triangular */                                             \
  void P##trmv_(const char *uplo, const char *tr, const char *diag,            \
                const int *n, const T *A, const int *lda, T *x,                \
                const int *incx) {                                             \
    int i, j;                                                                  \
    const int nounit = lsame(diag, 'N');                                       \
    const long ld = *lda, inc = *incx;                                         \
    const long kx = VSTART(*n, *incx);                                         \
    if (*n == 0) return;                                                       \
    if (lsame(tr, 'N')) {                                                      \
      if (lsame(uplo, 'U')) {                                                  \
        for (j = 0; j < *n; j++) {                                             \
          T temp = x[kx + j * inc];                                            \
          for (i = 0; i < j; i++) x[kx + i * inc] += temp * A[i + j * ld];     \
          if (nounit) x[kx + j * inc] *= A[j + j * ld];                        \
        }                                                                      \
      } else {                                                                 \
        for (j = *n - 1; j >= 0; j--) {                                        \
          T temp = x[kx + j * inc];                                            \
          for (i = *n - 1; i > j; i--) x[kx + i * inc] += temp * A[i + j * ld];\
          if (nounit) x[kx + j * inc] *= A[j + j * ld];                        \
        }                                                                      \
      }                                                                        \
    } else {                                                                   \
      if (lsame(uplo, 'U')) {                                                  \
        for (j = *n - 1; j >= 0; j--) {                                        \
          T temp = x[kx + j * inc];                                            \
          if (nounit) temp *= A[j + j * ld];                                   \
          for (i = j - 1; i >= 0; i--) temp += A[i + j * ld] * x[kx + i * inc];\
          x[kx + j * inc] = temp;                                              \
        }                                                                      \
      } else {                                                                 \
        for (j = 0; j < *n; j++) {                                             \
          T temp = x[kx + j * inc];                                            \
          if (nounit) temp *= A[j + j * ld];                                   \
          for (i = j + 1; i < *n; i++) temp += A[i + j * ld] * x[kx + i * inc];\
          x[kx + j * inc] = temp;                                              \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* y := alpha*A*x + beta*y, A symmetric (one triangle referenced) */         \
  void P##symv_(const char *uplo, const int *n, const T *alpha, const T *A,    \
                const int *lda, const T *x, const int *incx, const T *beta,    \
                T *y, const int *incy) {                                       \
    int i, j;                                                                  \
    const long ld = *lda;                                                      \
    const long kx = VSTART(*n, *incx), ky = VSTART(*n, *incy);                 \
    const long ix = *incx, iy = *incy;                                         \
    if (*n == 0 || (*alpha == 0 && *beta == 1)) return;                        \
    if (*beta != 1)                                                            \
      for (i = 0; i < *n; i++)                                                 \
        y[ky + i * iy] = (*beta == 0) ? (T)0 : *beta * y[ky + i * iy];         \
    if (*alpha == 0) return;                                                   \
    if (lsame(uplo, 'U')) {                                                    \
      for (j = 0; j < *n; j++) {                                               \
        T t1 = *alpha * x[kx + j * ix], t2 = 0;                                \
        for (i = 0; i < j; i++) {                                              \
          y[ky + i * iy] += t1 * A[i + j * ld];                                \
          t2 += A[i + j * ld] * x[kx + i * ix];                                \
        }                                                                      \
        y[ky + j * iy] += t1 * A[j + j * ld] + *alpha * t2;                    \
      }                                                                        \
    } else {                                                                   \
      for (j = 0; j < *n; j++) {                                               \
        T t1 = *alpha * x[kx + j * ix], t2 = 0;                                \
        y[ky + j * iy] += t1 * A[j + j * ld];                                  \
        for (i = j + 1; i < *n; i++) {                                         \
          y[ky + i * iy] += t1 * A[i + j * ld];                                \
          t2 += A[i + j * ld] * x[kx + i * ix];                                \
        }                                                                      \
        y[ky + j * iy] += *alpha * t2;                                         \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* A := alpha*x*y' + alpha*y*x' + A, one triangle */                         \
  void P##syr2_(const char *uplo, const int *n, const T *alpha, const T *x,    \
                const int *incx, const T *y, const int *incy, T *A,            \
                const int *lda) {                                              \
    int i, j;                                                                  \
    const long ld = *lda;                                                      \
    const long kx = VSTART(*n, *incx), ky = VSTART(*n, *incy);                 \
    const long ix = *incx, iy = *incy;                                         \
    if (*n == 0 || *alpha == 0) return;                                        \
    for (j = 0; j < *n; j++) {                                                 \
      if (x[kx + j * ix] != 0 || y[ky + j * iy] != 0) {                        \
        T t1 = *alpha * y[ky + j * iy], t2 = *alpha * x[kx + j * ix];          \
        int lo = lsame(uplo, 'U') ? 0 : j;                                     \
        int hi = lsame(uplo, 'U') ? j + 1 : *n;                                \
        for (i = lo; i < hi; i++)                                              \
          A[i + j * ld] += x[kx + i * ix] * t1 + y[ky + i * iy] * t2;          \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* C := alpha*op(A)*op(B) + beta*C */                                        \
  void P##gemm_(const char *ta, const char *tb, const int *m, const int *n,    \
                const int *k, const T *alpha, const T *A, const int *lda,      \
                const T *B, const int *ldb, const T *beta, T *C,               \
                const int *ldc) {                                              \
    int i, j, l;                                                               \
    const int nota = lsame(ta, 'N'), notb = lsame(tb, 'N');                    \
    const long la = *lda, lb = *ldb, lc = *ldc;                                \
    if (*m == 0 || *n == 0 ||                                                  \
        ((*alpha == 0 || *k == 0) && *beta == 1))                              \
      return;                                                                  \
    if (*alpha == 0) {                                                         \
      for (j = 0; j < *n; j++)                                                 \
        for (i = 0; i < *m; i++)                                               \
          C[i + j * lc] = (*beta == 0) ? (T)0 : *beta * C[i + j * lc];         \
      return;                                                                  \
    }                                                                          \
    if (notb) {                                                                \
      if (nota) {                                                              \
        for (j = 0; j < *n; j++) {                                             \
          if (*beta == 0) for (i = 0; i < *m; i++) C[i + j * lc] = 0;          \
          else if (*beta != 1)                                                 \
            for (i = 0; i < *m; i++) C[i + j * lc] *= *beta;                   \
          for (l = 0; l < *k; l++) {                                           \
            T temp = *alpha * B[l + j * lb];                                   \
            for (i = 0; i < *m; i++) C[i + j * lc] += temp * A[i + l * la];    \
          }                                                                    \
        }                                                                      \
      } else {                                                                 \
        for (j = 0; j < *n; j++)                                               \
          for (i = 0; i < *m; i++) {                                           \
            T temp = 0;                                                        \
            for (l = 0; l < *k; l++) temp += A[l + i * la] * B[l + j * lb];    \
            C[i + j * lc] = (*beta == 0) ? *alpha * temp                       \
                                         : *alpha * temp + *beta * C[i + j * lc];\
          }                                                                    \
      }                                                                        \
    } else {                                                                   \
      if (nota) {                                                              \
        for (j = 0; j < *n; j++) {                                             \
          if (*beta == 0) for (i = 0; i < *m; i++) C[i + j * lc] = 0;          \
          else if (*beta != 1)                                                 \
            for (i = 0; i < *m; i++) C[i + j * lc] *= *beta;                   \
          for (l = 0; l < *k; l++) {                                           \
            T temp = *alpha * B[j + l * lb];                                   \
            for (i = 0; i < *m; i++) C[i + j * lc] += temp * A[i + l * la];    \
          }                                                                    \
        }                                                                      \
      } else {                                                                 \
        for (j = 0; j < *n; j++)                                               \
          for (i = 0; i < *m; i++) {                                           \
            T temp = 0;                                                        \
            for (l = 0; l < *k; l++) temp += A[l + i * la] * B[j + l * lb];    \
            C[i + j * lc] = (*beta == 0) ? *alpha * temp                       \
                                         : *alpha * temp + *beta * C[i + j * lc];\
          }                                                                    \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* C := alpha*A*A' + beta*C (tr N) or alpha*A'*A + beta*C (tr T) */          \
  void P##syrk_(const char *uplo, const char *tr, const int *n, const int *k,  \
                const T *alpha, const T *A, const int *lda, const T *beta,     \
                T *C, const int *ldc) {                                        \
    int i, j, l;                                                               \
    const int upper = lsame(uplo, 'U');                                        \
    const long la = *lda, lc = *ldc;                                           \
    if (*n == 0 || ((*alpha == 0 || *k == 0) && *beta == 1)) return;           \
    for (j = 0; j < *n; j++) {                                                 \
      int lo = upper ? 0 : j, hi = upper ? j + 1 : *n;                         \
      if (lsame(tr, 'N')) {                                                    \
        if (*beta == 0) for (i = lo; i < hi; i++) C[i + j * lc] = 0;           \
        else if (*beta != 1)                                                   \
          for (i = lo; i < hi; i++) C[i + j * lc] *= *beta;                    \
        if (*alpha == 0) continue;                                             \
        for (l = 0; l < *k; l++) {                                             \
          if (A[j + l * la] != 0) {                                            \
            T temp = *alpha * A[j + l * la];                                   \
            for (i = lo; i < hi; i++) C[i + j * lc] += temp * A[i + l * la];   \
          }                                                                    \
        }                                                                      \
      } else {                                                                 \
        for (i = lo; i < hi; i++) {                                            \
          T temp = 0;                                                          \
          for (l = 0; l < *k; l++) temp += A[l + i * la] * A[l + j * la];      \
          C[i + j * lc] = (*beta == 0) ? *alpha * temp                         \
                                       : *alpha * temp + *beta * C[i + j * lc];\
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  /* C := alpha*A*B + beta*C (side L) or alpha*B*A + beta*C, A symmetric */    \
  void P##symm_(const char *side, const char *uplo, const int *m,              \
                const int *n, const T *alpha, const T *A, const int *lda,      \
                const T *B, const int *ldb, const T *beta, T *C,               \
                const int *ldc) {                                              \
    int i, j, l;                                                               \
    const int left = lsame(side, 'L'), upper = lsame(uplo, 'U');               \
    const long la = *lda, lb = *ldb, lc = *ldc;                                \
    const int na = left ? *m : *n;                                             \
    if (*m == 0 || *n == 0) return;                                            \
    for (j = 0; j < *n; j++)                                                   \
      for (i = 0; i < *m; i++) {                                               \
        T temp = 0;                                                            \
        for (l = 0; l < na; l++) {                                             \
          int r = left ? i : l, c = left ? l : j;                              \
          T a;                                                                 \
          if ((upper && r <= c) || (!upper && r >= c)) a = A[r + c * la];      \
          else a = A[c + r * la];                                              \
          temp += left ? a * B[l + j * lb] : B[i + l * lb] * a;                \
        }                                                                      \
        C[i + j * lc] = (*beta == 0) ? *alpha * temp                           \
                                     : *alpha * temp + *beta * C[i + j * lc];  \
      }                                                                        \
  }                                                                            \
  /* B := alpha*op(A)*B (side L) or alpha*B*op(A), A triangular */             \
  void P##trmm_(const char *side, const char *uplo, const char *ta,            \
                const char *diag, const int *m, const int *n, const T *alpha,  \
                const T *A, const int *lda, T *B, const int *ldb) {            \
    int i, j, l;                                                               \
    const int left = lsame(side, 'L'), upper = lsame(uplo, 'U');               \
    const int tr = !lsame(ta, 'N'), nounit = lsame(diag, 'N');                 \
    const long la = *lda, lb = *ldb;                                           \
    const int na = left ? *m : *n;                                             \
    T *col;                                                                    \
    if (*m == 0 || *n == 0) return;                                            \
    col = (T *)malloc(sizeof(T) * (size_t)(left ? *m : *n));                   \
    if (left) {                                                                \
      for (j = 0; j < *n; j++) {                                               \
        for (i = 0; i < *m; i++) {                                             \
          T temp = 0;                                                          \
          for (l = 0; l < na; l++) {                                           \
            int r = tr ? l : i, c = tr ? i : l;                                \
            T a;                                                               \
            if (r == c) a = nounit ? A[r + c * la] : (T)1;                     \
            else if ((upper && r < c) || (!upper && r > c)) a = A[r + c * la]; \
            else a = 0;                                                        \
            temp += a * B[l + j * lb];                                         \
          }                                                                    \
          col[i] = *alpha * temp;                                              \
        }                                                                      \
        for (i = 0; i < *m; i++) B[i + j * lb] = col[i];                       \
      }                                                                        \
    } else {                                                                   \
      for (i = 0; i < *m; i++) {                                               \
        for (j = 0; j < *n; j++) {                                             \
          T temp = 0;                                                          \
          for (l = 0; l < na; l++) {                                           \
            int r = tr ? j : l, c = tr ? l : j;                                \
            T a;                                                               \
            if (r == c) a = nounit ? A[r + c * la] : (T)1;                     \
            else if ((upper && r < c) || (!upper && r > c)) a = A[r + c * la]; \
            else a = 0;                                                        \
            temp += B[i + l * lb] * a;                                         \
          }                                                                    \
          col[j] = *alpha * temp;                                              \
        }                                                                      \
        for (j = 0; j < *n; j++) B[i + j * lb] = col[j];                       \
      }                                                                        \
    }                                                                          \
    free(col);                                                                 \
  }                                                                            \
  /* solve op(A)*X = alpha*B (side L) or X*op(A) = alpha*B, X overwrites B */  \
  void P##trsm_(const char *side, const char *uplo, const char *ta,            \
                const char *diag, const int *m, const int *n, const T *alpha,  \
                const T *A, const int *lda, T *B, const int *ldb) {            \
    int i, j, k;                                                               \
    const int left = lsame(side, 'L'), upper = lsame(uplo, 'U');               \
    const int nounit = lsame(diag, 'N');                                       \
    const long la = *lda, lb = *ldb;                                           \
    if (*m == 0 || *n == 0) return;                                            \
    if (*alpha == 0) {                                                         \
      for (j = 0; j < *n; j++)                                                 \
        for (i = 0; i < *m; i++) B[i + j * lb] = 0;                            \
      return;                                                                  \
    }                                                                          \
    if (left) {                                                                \
      if (lsame(ta, 'N')) {                                                    \
        /* B := alpha*inv(A)*B, column by column, axpy form */                 \
        for (j = 0; j < *n; j++) {                                             \
          if (*alpha != 1)                                                     \
            for (i = 0; i < *m; i++) B[i + j * lb] *= *alpha;                  \
          if (upper) {                                                         \
            for (k = *m - 1; k >= 0; k--)                                      \
              if (B[k + j * lb] != 0) {                                        \
                if (nounit) B[k + j * lb] /= A[k + k * la];                    \
                for (i = 0; i < k; i++)                                        \
                  B[i + j * lb] -= B[k + j * lb] * A[i + k * la];              \
              }                                                                \
          } else {                                                             \
            for (k = 0; k < *m; k++)                                           \
              if (B[k + j * lb] != 0) {                                        \
                if (nounit) B[k + j * lb] /= A[k + k * la];                    \
                for (i = k + 1; i < *m; i++)                                   \
                  B[i + j * lb] -= B[k + j * lb] * A[i + k * la];              \
              }                                                                \
          }                                                                    \
        }                                                                      \
      } else {                                                                 \
        /* B := alpha*inv(A')*B, dot form */                                   \
        for (j = 0; j < *n; j++) {                                             \
          if (upper) {                                                         \
            for (i = 0; i < *m; i++) {                                         \
              T temp = *alpha * B[i + j * lb];                                 \
              for (k = 0; k < i; k++) temp -= A[k + i * la] * B[k + j * lb];   \
              if (nounit) temp /= A[i + i * la];                               \
              B[i + j * lb] = temp;                                            \
            }                                                                  \
          } else {                                                             \
            for (i = *m - 1; i >= 0; i--) {                                    \
              T temp = *alpha * B[i + j * lb];                                 \
              for (k = i + 1; k < *m; k++) temp -= A[k + i * la] * B[k + j * lb];\
              if (nounit) temp /= A[i + i * la];                               \
              B[i + j * lb] = temp;                                            \
            }                                                                  \
          }                                                                    \
        }                                                                      \
      }                                                                        \
    } else {                                                                   \
      if (lsame(ta, 'N')) {                                                    \
        /* B := alpha*B*inv(A) */                                              \
        if (upper) {                                                           \
          for (j = 0; j < *n; j++) {                                           \
            if (*alpha != 1)                                                   \
              for (i = 0; i < *m; i++) B[i + j * lb] *= *alpha;                \
            for (k = 0; k < j; k++)                                            \
              if (A[k + j * la] != 0)                                          \
                for (i = 0; i < *m; i++)                                       \
                  B[i + j * lb] -= A[k + j * la] * B[i + k * lb];              \
            if (nounit) {                                                      \
              T temp = 1 / A[j + j * la];                                      \
              for (i = 0; i < *m; i++) B[i + j * lb] *= temp;                  \
            }                                                                  \
          }                                                                    \
        } else {                                                               \
          for (j = *n - 1; j >= 0; j--) {                                      \
            if (*alpha != 1)                                                   \
              for (i = 0; i < *m; i++) B[i + j * lb] *= *alpha;                \
            for (k = j + 1; k < *n; k++)                                       \
              if (A[k + j * la] != 0)                                          \
                for (i = 0; i < *m; i++)                                       \
                  B[i + j * lb] -= A[k + j * la] * B[i + k * lb];              \
            if (nounit) {                                                      \
              T temp = 1 / A[j + j * la];                                      \
              for (i = 0; i < *m; i++) B[i + j * lb] *= temp;                  \
            }                                                                  \
          }                                                                    \
        }                                                                      \
      } else {                                                                 \
        /* B := alpha*B*inv(A') */                                             \
        if (upper) {                                                           \
          for (k = *n - 1; k >= 0; k--) {                                      \
            if (nounit) {                                                      \
              T temp = 1 / A[k + k * la];                                      \
              for (i = 0; i < *m; i++) B[i + k * lb] *= temp;                  \
            }                                                                  \
            for (j = 0; j < k; j++)                                            \
              if (A[j + k * la] != 0) {                                        \
                T temp = A[j + k * la];                                        \
                for (i = 0; i < *m; i++) B[i + j * lb] -= temp * B[i + k * lb];\
              }                                                                \
            if (*alpha != 1)                                                   \
              for (i = 0; i < *m; i++) B[i + k * lb] *= *alpha;                \
          }                                                                    \
        } else {                                                               \
          for (k = 0; k < *n; k++) {                                           \
            if (nounit) {                                                      \
              T temp = 1 / A[k + k * la];                                      \
              for (i = 0; i < *m; i++) B[i + k * lb] *= temp;                  \
            }                                                                  \
            for (j = k + 1; j < *n; j++)                                       \
              if (A[j + k * la] != 0) {                                        \
                T temp = A[j + k * la];                                        \
                for (i = 0; i < *m; i++) B[i + j * lb] -= temp * B[i + k * lb];\
              }                                                                \
            if (*alpha != 1)                                                   \
              for (i = 0; i < *m; i++) B[i + k * lb] *= *alpha;                \
          }                                                                    \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  }

DEFINE_REAL_BLAS(double, d)
DEFINE_REAL_BLAS(float, s)

/* complex BLAS is not on the real dense-solve path; reaching one of these
 * is a harness error. */
static void not_on_path(const char *name) {
  fprintf(stderr, "oracle BLAS: %s is not provided (not on the real path)\n",
          name);
  abort();
}
#define STUB(name) \
  void name(void) { not_on_path(#name); }
STUB(caxpy_) STUB(ccopy_) STUB(cgemm_) STUB(cgemv_) STUB(cgeru_) STUB(chemv_)
STUB(cher_) STUB(cherk_) STUB(cscal_) STUB(cswap_) STUB(csymm_) STUB(csyrk_)
STUB(ctrmv_) STUB(ctrsm_) STUB(ctrsv_) STUB(dzasum_) STUB(dznrm2_)
STUB(icamax_) STUB(izamax_) STUB(scasum_) STUB(scnrm2_) STUB(zaxpy_)
STUB(zcopy_) STUB(zgemm_) STUB(zgemv_) STUB(zgeru_) STUB(zhemv_) STUB(zher_)
STUB(zherk_) STUB(zscal_) STUB(zswap_) STUB(zsymm_) STUB(zsyrk_) STUB(ztrmv_)
STUB(ztrsm_) STUB(ztrsv_)
