/*
 * Flat C entry points that drive the upstream PLAPACK (compiled from the
 * reference sources with the single-rank MPI stand-in and the restated
 * netlib BLAS) on a 1x1 template.  Test infrastructure only: the parity tests
 * and the CPU-baseline leg of the benchmark call these through ctypes.
 *
 * Each entry mirrors a reference test driver:
 *   ref_lu            TEST/test_lu.c:118-139 (PLA_Matrix_create, PLA_Mvector of
 *                     MPI_INT pivots, fill through the local buffer as
 *                     TEST/create_problem.c:38-51 does, PLA_LU)
 *   ref_lu_linpack    the same with PLA_LU_linpack (SOLVERS/LINPACK/driver.c's
 *                     augmented-matrix solve factors with the blocked LU)
 *   ref_chol          TEST/test_chol.c:113-135 (PLA_Chol(PLA_LOWER_TRIANGULAR))
 *   ref_general_solve SOLVERS/LU/PLA_General.c:67-119
 *   ref_pos_def_solve SOLVERS/Cholesky/PLA_Pos_def.c:44-99
 *   ref_trsv / ref_trsm / ref_gemm / ref_apply_pivots  the BLAS entry points.
 * Matrices cross this boundary column-major with an explicit leading
 * dimension; datatype 0 = float, 1 = double (test_lu.c's itype codes).
 */
#include "PLA.h"

#include <string.h>

int PLA_LU(PLA_Obj, PLA_Obj);
int PLA_LU_linpack(PLA_Obj, PLA_Obj);
int PLA_Chol(int, PLA_Obj);
int PLA_General_solve(PLA_Obj, PLA_Obj, PLA_Obj);
int PLA_Pos_def_solve(PLA_Obj, PLA_Obj);
int PLA_Trsv(int, int, int, PLA_Obj, PLA_Obj);
int PLA_Trsm(int, int, int, int, PLA_Obj, PLA_Obj, PLA_Obj);
int PLA_Gemm(int, int, PLA_Obj, PLA_Obj, PLA_Obj, PLA_Obj, PLA_Obj);
int PLA_Apply_pivots_to_rows(PLA_Obj, PLA_Obj);
int pla_Environ_set_nb_alg(int, int);
int PLA_Set_error_checking(int, int, int, int);
int PLA_Comm_1D_to_2D(MPI_Comm, int, int, MPI_Comm *);
int PLA_Init(MPI_Comm);
int PLA_Finalize(void);
int PLA_Temp_create(int, int, PLA_Template *);
int PLA_Temp_free(PLA_Template *);

static PLA_Template templ = NULL;
static int ready = 0;

static MPI_Datatype dt(int code) { return code == 0 ? MPI_FLOAT : MPI_DOUBLE; }
static size_t esz(int code) { return code == 0 ? sizeof(float) : sizeof(double); }

int ref_init(int nb_distr, int nb_alg, int error_checking) {
  MPI_Comm comm = MPI_COMM_NULL;
  if (ready) return 0;
  MPI_Init(NULL, NULL);
  pla_Environ_set_nb_alg(PLA_OP_ALL_ALG, nb_alg);
  PLA_Set_error_checking(error_checking, error_checking, 0, FALSE);
  PLA_Comm_1D_to_2D(MPI_COMM_WORLD, 1, 1, &comm);
  PLA_Init(comm);
  PLA_Temp_create(nb_distr, 0, &templ);
  ready = 1;
  return 0;
}

int ref_set_nb_alg(int nb_alg) { return pla_Environ_set_nb_alg(PLA_OP_ALL_ALG, nb_alg); }

int ref_finalize(void) {
  if (!ready) return 0;
  PLA_Temp_free(&templ);
  PLA_Finalize();
  MPI_Finalize();
  ready = 0;
  return 0;
}

/* host column-major (ld) <-> object local buffer (its own ldim) */
static void put(PLA_Obj A, int m, int n, const void *src, int ld, int code) {
  char *buf;
  int ldim, j;
  size_t e = esz(code);
  PLA_Obj_local_buffer(A, (void **)&buf);
  PLA_Obj_local_ldim(A, &ldim);
  for (j = 0; j < n; j++)
    memcpy(buf + (size_t)j * ldim * e, (const char *)src + (size_t)j * ld * e,
           (size_t)m * e);
}
static void get(PLA_Obj A, int m, int n, void *dst, int ld, int code) {
  char *buf;
  int ldim, j;
  size_t e = esz(code);
  PLA_Obj_local_buffer(A, (void **)&buf);
  PLA_Obj_local_ldim(A, &ldim);
  for (j = 0; j < n; j++)
    memcpy((char *)dst + (size_t)j * ld * e, buf + (size_t)j * ldim * e,
           (size_t)m * e);
}

/* PLA_LU (linpack == 0) or PLA_LU_linpack (SOLVERS/LINPACK/PLA_LU_linpack.c:13)
 * on an m x n matrix; pivots (length min(m,n)) are PLAPACK's offsets */
static int lu_either(int linpack, int m, int n, int code, void *A, int lda, int *piv,
                     double *seconds) {
  PLA_Obj a = NULL, p = NULL;
  int r, k = m < n ? m : n, *pb;
  double t;
  PLA_Matrix_create(dt(code), m, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  PLA_Mvector_create(MPI_INT, k, 1, templ, PLA_ALIGN_FIRST, &p);
  put(a, m, n, A, lda, code);
  t = MPI_Wtime();
  r = linpack ? PLA_LU_linpack(a, p) : PLA_LU(a, p);
  t = MPI_Wtime() - t;
  if (seconds) *seconds = t;
  get(a, m, n, A, lda, code);
  PLA_Obj_local_buffer(p, (void **)&pb);
  memcpy(piv, pb, (size_t)k * sizeof(int));
  PLA_Obj_free(&a);
  PLA_Obj_free(&p);
  return r;
}
int ref_lu(int m, int n, int code, void *A, int lda, int *piv, double *seconds) {
  return lu_either(0, m, n, code, A, lda, piv, seconds);
}
int ref_lu_linpack(int m, int n, int code, void *A, int lda, int *piv, double *seconds) {
  return lu_either(1, m, n, code, A, lda, piv, seconds);
}

int ref_chol(int n, int code, void *A, int lda, double *seconds) {
  PLA_Obj a = NULL;
  int r;
  double t;
  PLA_Matrix_create(dt(code), n, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  put(a, n, n, A, lda, code);
  t = MPI_Wtime();
  r = PLA_Chol(PLA_LOWER_TRIANGULAR, a);
  t = MPI_Wtime() - t;
  if (seconds) *seconds = t;
  get(a, n, n, A, lda, code);
  PLA_Obj_free(&a);
  return r;
}

/* right-hand sides: one column -> PLA_Mvector (the Trsv path), several ->
 * PLA_Matrix (the Trsm path), as PLA_General_solve branches on */
static PLA_Obj rhs_create(int n, int nrhs, int code) {
  PLA_Obj b = NULL;
  if (nrhs == 1)
    PLA_Mvector_create(dt(code), n, 1, templ, PLA_ALIGN_FIRST, &b);
  else
    PLA_Matrix_create(dt(code), n, nrhs, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &b);
  return b;
}

int ref_general_solve(int n, int nrhs, int code, void *A, int lda, void *B,
                      int ldb, int *piv, double *seconds) {
  PLA_Obj a = NULL, p = NULL, b = NULL;
  int r, *pb;
  double t;
  PLA_Matrix_create(dt(code), n, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  PLA_Mvector_create(MPI_INT, n, 1, templ, PLA_ALIGN_FIRST, &p);
  b = rhs_create(n, nrhs, code);
  put(a, n, n, A, lda, code);
  put(b, n, nrhs, B, ldb, code);
  t = MPI_Wtime();
  r = PLA_General_solve(a, p, b);
  t = MPI_Wtime() - t;
  if (seconds) *seconds = t;
  get(a, n, n, A, lda, code);
  get(b, n, nrhs, B, ldb, code);
  PLA_Obj_local_buffer(p, (void **)&pb);
  if (piv) memcpy(piv, pb, (size_t)n * sizeof(int));
  PLA_Obj_free(&a);
  PLA_Obj_free(&p);
  PLA_Obj_free(&b);
  return r;
}

int ref_pos_def_solve(int n, int nrhs, int code, void *A, int lda, void *B,
                      int ldb, double *seconds) {
  PLA_Obj a = NULL, b = NULL;
  int r;
  double t;
  PLA_Matrix_create(dt(code), n, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  b = rhs_create(n, nrhs, code);
  put(a, n, n, A, lda, code);
  put(b, n, nrhs, B, ldb, code);
  t = MPI_Wtime();
  r = PLA_Pos_def_solve(a, b);
  t = MPI_Wtime() - t;
  if (seconds) *seconds = t;
  get(a, n, n, A, lda, code);
  get(b, n, nrhs, B, ldb, code);
  PLA_Obj_free(&a);
  PLA_Obj_free(&b);
  return r;
}

int ref_trsv(int uplo, int trans, int diag, int n, int code, void *A, int lda,
             void *x) {
  PLA_Obj a = NULL, v = NULL;
  int r;
  PLA_Matrix_create(dt(code), n, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  PLA_Mvector_create(dt(code), n, 1, templ, PLA_ALIGN_FIRST, &v);
  put(a, n, n, A, lda, code);
  put(v, n, 1, x, n, code);
  r = PLA_Trsv(uplo, trans, diag, a, v);
  get(v, n, 1, x, n, code);
  PLA_Obj_free(&a);
  PLA_Obj_free(&v);
  return r;
}

static PLA_Obj scalar(int code, double value) {
  PLA_Obj s = NULL;
  void *buf;
  PLA_Mscalar_create(dt(code), PLA_ALL_ROWS, PLA_ALL_COLS, 1, 1, templ, &s);
  PLA_Obj_local_buffer(s, &buf);
  if (code == 0) *(float *)buf = (float)value; else *(double *)buf = value;
  return s;
}

int ref_trsm(int side, int uplo, int trans, int diag, int m, int n,
             double alpha, int code, void *A, int lda, void *B, int ldb) {
  PLA_Obj a = NULL, b = NULL, al;
  int r, na = (side == PLA_SIDE_LEFT) ? m : n;
  PLA_Matrix_create(dt(code), na, na, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  PLA_Matrix_create(dt(code), m, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &b);
  al = scalar(code, alpha);
  put(a, na, na, A, lda, code);
  put(b, m, n, B, ldb, code);
  r = PLA_Trsm(side, uplo, trans, diag, al, a, b);
  get(b, m, n, B, ldb, code);
  PLA_Obj_free(&a);
  PLA_Obj_free(&b);
  PLA_Obj_free(&al);
  return r;
}

int ref_gemm(int transa, int transb, int m, int n, int k, double alpha,
             int code, void *A, int lda, void *B, int ldb, double beta,
             void *C, int ldc) {
  PLA_Obj a = NULL, b = NULL, c = NULL, al, be;
  int r;
  int am = (transa == PLA_NO_TRANSPOSE) ? m : k, an = (transa == PLA_NO_TRANSPOSE) ? k : m;
  int bm = (transb == PLA_NO_TRANSPOSE) ? k : n, bn = (transb == PLA_NO_TRANSPOSE) ? n : k;
  PLA_Matrix_create(dt(code), am, an, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &a);
  PLA_Matrix_create(dt(code), bm, bn, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &b);
  PLA_Matrix_create(dt(code), m, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &c);
  al = scalar(code, alpha);
  be = scalar(code, beta);
  put(a, am, an, A, lda, code);
  put(b, bm, bn, B, ldb, code);
  put(c, m, n, C, ldc, code);
  r = PLA_Gemm(transa, transb, al, a, b, be, c);
  get(c, m, n, C, ldc, code);
  PLA_Obj_free(&a);
  PLA_Obj_free(&b);
  PLA_Obj_free(&c);
  PLA_Obj_free(&al);
  PLA_Obj_free(&be);
  return r;
}

/* PLA_Apply_pivots_to_rows(B, ipiv) with ipiv an MVECTOR of MPI_INT */
int ref_apply_pivots(int n, int nrhs, int code, void *B, int ldb,
                     const int *piv, int npiv) {
  PLA_Obj b = NULL, p = NULL;
  int r, *pb;
  PLA_Matrix_create(dt(code), n, nrhs, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &b);
  PLA_Mvector_create(MPI_INT, npiv, 1, templ, PLA_ALIGN_FIRST, &p);
  put(b, n, nrhs, B, ldb, code);
  PLA_Obj_local_buffer(p, (void **)&pb);
  memcpy(pb, piv, (size_t)npiv * sizeof(int));
  r = PLA_Apply_pivots_to_rows(b, p);
  get(b, n, nrhs, B, ldb, code);
  PLA_Obj_free(&b);
  PLA_Obj_free(&p);
  return r;
}
