// Thin C ABI between the host library and the CUDA kernels (sm_100a).
// Every matrix is column-major with an explicit leading dimension (elements);
// every launch goes on the given stream and returns 0 on success, else a
// cudaError_t value.  `dt` is MPI_DOUBLE or MPI_FLOAT unless noted.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status word: kernels report failures here instead of trapping ---- */
#define PLA_K_OK 0
#define PLA_K_TIMEOUT 1        /* a bounded wait gave up (grid barrier)   */
#define PLA_K_NOT_SPD 2        /* Cholesky met a non-positive pivot       */

void pla_kernels_release(void);
/* number of kernels the library has launched (all streams, since load) */
void pla_k_count(int n);
long pla_k_launches(void);

int pla_k_fill(int dt, int m, int n, void *A, long lda, double value, cudaStream_t s);
/* Y := alpha * X + beta * Y (beta == 0 ignores Y's contents) */
int pla_k_axpby(int dt, int m, int n, double alpha, const void *X, long ldx, double beta,
                void *Y, long ldy, cudaStream_t s);
/* Y := X or X' (m x n result) */
int pla_k_copy(int dt, int trans, int m, int n, const void *X, long ldx, void *Y, long ldy,
               cudaStream_t s);
/* convert between precisions: dst(m x n, dt_dst) := src(m x n, dt_src).
 * dt codes: MPI_DOUBLE, MPI_FLOAT, PLA_K_BF16, PLA_K_FP16 */
#define PLA_K_BF16 1001
#define PLA_K_FP16 1002
int pla_k_convert(int dt_src, const void *src, long lds, int dt_dst, void *dst, long ldd, int m,
                  int n, cudaStream_t s);

/* ---- panel LU: factor the r x w panel at A in place with partial pivoting.
 * piv[j] = offset from row j to the pivot row (reference encoding).
 * zero_info (optional): set to the 1-based first exact zero pivot + row_base. */
/* the same with at most max_ctas CTAs (0: one per SM), leaving the other SMs
 * to kernels that run beside it */
int pla_k_lu_panel_ex(int dt, int r, int w, void *A, long lda, int *piv, int *status,
                      int *zero_info, int row_base, int max_ctas, cudaStream_t s);
int pla_k_lu_panel(int dt, int r, int w, void *A, long lda, int *piv, int *status,
                   int *zero_info, int row_base, cudaStream_t s);

/* ---- tournament-pivoted LU of an r x w fp32 panel, w <= 32 (k_tslu.cu): the
 * pivots (offset encoding) to piv, the panel overwritten by L \ U under them;
 * zero_info as above.  One launch sequence at a time (its workspace and
 * counters are shared). */
int pla_k_lu_panel_tslu(int r, int w, float *A, long lda, int *piv, int *zero_info,
                        int row_base, int max_ctas, cudaStream_t s);
void pla_tslu_release(void);
/* U12 = inv(L11) A12 and A22 -= L21 U12 for the m x w fp32 sub-panel at P (w <= 32,
 * unit-lower L11 at its top) and the ncols columns right of it, one launch */
#define PLA_K_PANEL_UPDATE_MAX 480
int pla_k_panel_update(int m, int w, int ncols, float *P, long lda, cudaStream_t s);
/* the mixed / FP64 LU's blocked r x b panel factorization (32-column
 * sub-panels, pivoting PLA_B200_PIVOT_*) on stream s (0: the library stream) */
int pla_k_panel_lu_blocked(int dt, int r, int b, void *P, long lda, int *piv, int *zero_info,
                           int max_ctas, int pivoting, cudaStream_t s);

/* ---- row interchanges: for i in [0, npiv): swap rows i and i + piv[i] of the
 * block whose row 0 is A (rows relative to A), in columns [c0, c1) and
 * [c2, c3). */
int pla_k_laswp(int dt, void *A, long lda, int npiv, const int *piv, int c0, int c1, int c2,
                int c3, cudaStream_t s);
// adds the number of non-trivial interchanges (piv[i] != 0) of piv[0..npiv) to *ctr
int pla_k_count_interchanges(int npiv, const int *piv, unsigned long long *ctr,
                              cudaStream_t s);
/* apply a host pivot vector to m x n B in sequence (device pivots) */
int pla_k_laswp_rows(int dt, void *B, long ldb, int ncols, int npiv, const int *piv,
                     cudaStream_t s);

/* ---- GEMM: C := alpha op(A) op(B) + beta C; uplo_c = 0 full, 'L' lower only,
 * 'U' upper only (SYRK-shaped updates). */
/* rows of C one CTA of pla_k_gemm covers: a GEMM whose C is also its B is
 * safe only when m is at most this (every column tile then has one CTA) */
int pla_k_gemm_tile_rows(int dt);
int pla_k_gemm(int dt, int transa, int transb, int m, int n, int k, double alpha,
               const void *A, long lda, const void *B, long ldb, double beta, void *C,
               long ldc, int uplo_c, const int *status, cudaStream_t s);

/* ---- small triangular solves (the triangle is b x b with b <= 128):
 * side 'L': B := alpha inv(op(T)) B  (B is b x ncols)
 * side 'R': B := alpha B inv(op(T))  (B is nrows x b)
 * uplo 'L'/'U', trans 'N'/'T', diag 'U'/'N'. */
int pla_k_trsm_small(int dt, char side, char uplo, char trans, char diag, int b, int other,
                     double alpha, const void *T, long ldt, void *B, long ldb,
                     const int *status, cudaStream_t s);

/* ---- unblocked lower Cholesky of the b x b block at A (b <= 128); on a
 * non-positive pivot sets *status = PLA_K_NOT_SPD and *info = base + k + 1. */
int pla_k_potrf_lower(int dt, int b, void *A, long lda, int *status, int *info, int base,
                      cudaStream_t s);

/* ---- level-1/2 helpers ---- */
int pla_k_scal(int dt, int m, int n, double alpha, void *X, long ldx, cudaStream_t s);
/* out[0] (device, FP64) := the two-norm of x[0], x[inc], ..., x[(n-1) inc],
 * scaled by max |x_i| as dnrm2; deterministic */
int pla_k_nrm2(int dt, long n, const void *x, long inc, double *out, cudaStream_t s);
/* A(i, i) += v for i < n */
int pla_k_shift_diag(int dt, int n, void *A, long lda, double v, cudaStream_t s);
int pla_k_inv_scal(int dt, int m, int n, double alpha, void *X, long ldx, cudaStream_t s);
int pla_k_swap(int dt, int m, int n, void *X, long ldx, void *Y, long ldy, cudaStream_t s);
int pla_k_ger(int dt, int m, int n, double alpha, const void *x, long incx, const void *y,
              long incy, void *A, long lda, cudaStream_t s);
/* y := alpha op(A) x + beta y ; x, y with unit stride */
int pla_k_gemv(int dt, int trans, int m, int n, double alpha, const void *A, long lda,
               const void *x, double beta, void *y, cudaStream_t s);
/* first index of max |x| (0-based) and the signed value there */
int pla_k_iamax(int dt, int n, const void *x, long incx, int *index_out, void *value_out,
                cudaStream_t s);

/* ---- triangular solve with one or more right-hand sides (n x nrhs, ldb),
 * blocked: diagonal blocks by substitution, off-diagonal by GEMM/GEMV. */
int pla_k_trsv_blocked(int dt, char uplo, char trans, char diag, int n, int nrhs,
                       const void *A, long lda, void *B, long ldb, cudaStream_t s);

/* ---- norms and refinement helpers (FP64 unless noted) ---- */
/* row sums of |A| (m x n): rs[i] = sum_j |A(i,j)| */
int pla_k_row_abs_sums(int dt, int m, int n, const void *A, long lda, double *rs,
                       cudaStream_t s);
/* out[j] = max_i |X(i,j)| for each column j */
int pla_k_col_abs_max(int dt, int m, int n, const void *X, long ldx, double *out,
                      cudaStream_t s);

/* ---- mixed precision ---- */
/* C(row0 + i, col0 + j) += alpha * sum_k L(i,k) U(j,k) on the tensor cores:
 * L (M x K, l_rows allocated) and U (N x K, u_rows allocated) in bf16/fp16
 * with K contiguous (leading dimensions ldl, ldu in elements, multiples of 8);
 * C fp32 column-major with ldc (multiple of 4), c_rows x c_cols allocated.
 * K must be a multiple of 64 and at most 256.  lower != 0 skips the tiles
 * strictly above the diagonal (SYRK-shaped updates). */
int pla_k_tc_update(int prec, int M, int N, int K, float alpha, const void *L, long ldl,
                    long l_rows, const void *U, long ldu, long u_rows, float *C, long ldc,
                    long c_rows, long c_cols, int row0, int col0, int lower, int *status,
                    cudaStream_t s);
/* the tensor-core updates on at most max_ctas persistent CTAs (0: one per SM) */
int pla_k_tc_update_ex(int prec, int M, int N, int K, float alpha, const void *L, long ldl,
                       long l_rows, const void *U, long ldu, long u_rows, float *C, long ldc,
                       long c_rows, long c_cols, int row0, int col0, int lower, int max_ctas,
                       int *status, cudaStream_t s);
int pla_k_tc_update_fp8_ex(int M, int N, int K, float alpha, const void *L, long ldl,
                           long l_rows, const float *inv_l, const void *U, long ldu, long u_rows,
                           const float *inv_u, float *C, long ldc, long c_rows, long c_cols,
                           int row0, int col0, int lower, int max_ctas, int *status,
                           cudaStream_t s);
/* pla_k_tc_update with fp8 E4M3 operands (ldl / ldu in bytes, K % 128 == 0)
 * and per-128-row-tile inverse scales of L (inv_l) and of U (inv_u) */
int pla_k_tc_update_fp8(int M, int N, int K, float alpha, const void *L, long ldl, long l_rows,
                        const float *inv_l, const void *U, long ldu, long u_rows,
                        const float *inv_u, float *C, long ldc, long c_rows, long c_cols,
                        int row0, int col0, int lower, int *status, cudaStream_t s);
/* dst (bf16/fp16, row-major, ldd) := src (fp32, m x kdim column-major, lds) */
int pla_k_pack_rows(int prec, int m, int kdim, const float *src, long lds, void *dst, long ldd,
                    cudaStream_t s);
/* dst (fp8 E4M3, row-major, ldd bytes) := x(i, k) * 2^e(i / 128) for i < m,
 * k < kdim, x(i, k) = src[i * si + k * sk] (fp32); e(b) the largest power with
 * max |x| of rows [128 b, 128 b + 128) * 2^e <= 448; inv[b] := 2^-e(b). */
int pla_k_pack_fp8(int m, int kdim, const float *src, long si, long sk, void *dst, long ldd,
                   float *inv, cudaStream_t s);
/* bf16 split of an fp32 matrix for fp32-like products on the tensor cores:
 * x(i, k) = src[i si + k sk] (i < m, k < kdim) = hi + lo, hi = bf16(x),
 * lo = bf16(x - hi); row i of dst (ld ldd >= 3 kdim, K-contiguous) gets three
 * kdim-wide segments, segment s holding lo if bit s of pattern is set, else
 * hi.  With zero != 0 the source is cleared after it is read. */
int pla_k_pack_split(int m, int kdim, float *src, long si, long sk, void *dst, long ldd,
                     int pattern, int zero, cudaStream_t s);
/* nseg K-wide segments per row, segment s holding part (code >> 2 s) & 3 of
 * the three-way split x = p0 + p1 + p2 (p0 = bf16(x), p1 = bf16(x - p0), p2 =
 * bf16(x - p0 - p1)); nseg <= 8 */
int pla_k_pack_split_ex(int m, int kdim, float *src, long si, long sk, void *dst, long ldd,
                        int nseg, unsigned code, int zero, cudaStream_t s);
/* out[0] = max |A(i, i)|, out[1] = min |A(i, i)| over i < n (fp32, device); NaN in both
 * when a diagonal entry is NaN */
int pla_k_diag_range(int n, const float *A, long lda, float *out, cudaStream_t s);
/* D (ldd) := inv(L) for a unit-lower-triangular fp32 L (n x n, n a multiple
 * of 32 up to 256; only L's strictly lower part is read), one launch of
 * n / 16 CTAs; work is not used (kept for the interface) */
int pla_k_trtri_unit_lower(int n, const float *L, long ldl, float *D, long ldd, float *work,
                           cudaStream_t s);
/* d := diag(A)^-1/2 (1 where A(i, i) <= 0); dst (fp32, ldd) := D A D */
int pla_k_sym_scale(int n, const double *A, long lda, double *d, float *dst, long ldd,
                    cudaStream_t s);
/* X(i, r) *= d(i) for r < nrhs (FP64) */
int pla_k_diag_mul(int n, int nrhs, const double *d, double *X, long ldx, cudaStream_t s);
/* R := B - A X in FP64 (A n x ncols, X ncols x nrhs, nrhs <= 16); with
 * abs_rows, R(:,0) := row sums of |A|.  work: pla_k_residual_work() bytes. */
/* single-launch fp32 triangular solve with one right-hand side: the inverses
 * of the 128 x 128 diagonal blocks of op(A) go to Dinv (ldd >= n rounded up to
 * 128, 128 columns) once per factor; then x := inv(op(A)) b (x may alias b). */
int pla_k_trsv_inv_blocks(int dt, char uplo, char trans, char diag, int n, const void *A,
                          long lda, void *Dinv, long ldd, cudaStream_t s);
int pla_k_trsv_ticket(int dt, char uplo, char trans, int n, const void *A, long lda,
                      const void *Dinv, long ldd, const void *b, void *x, int *status,
                      cudaStream_t s);
/* the same for up to 16 fp32 right-hand sides (n x nrhs, ldb / ldx) in one
 * launch: A read once for all of them; B and X may be the same array */
int pla_k_trsv_ticket_multi(char uplo, char trans, int n, int nrhs, const float *A, long lda,
                            const float *Dinv, long ldd, const float *B, long ldb, float *X,
                            long ldx, int *status, cudaStream_t s);
/* FP64 right-hand sides and arithmetic on an fp32 triangle: the FP64 inverses of
 * its 128 x 128 diagonal blocks, then X := inv(op(A)) B for nrhs <= 16 */
int pla_k_trsv_inv_blocks_f64(char uplo, char trans, char diag, int n, const float *A, long lda,
                              double *Dinv, long ldd, cudaStream_t s);
int pla_k_trsv_ticket_multi_f64(char uplo, char trans, int n, int nrhs, const float *A, long lda,
                                const double *Dinv, long ldd, const double *B, long ldb,
                                double *X, long ldx, int *status, cudaStream_t s);
/* single-column fp32 solve with link blocks G_i = op(A)(i, p) inv(D_p) (p the
 * block solved just before i; ldd x 128 floats, the layout of Dinv): the chain
 * between blocks skips the inverse-block product */
int pla_k_trsv_link_blocks(char uplo, char trans, int n, const float *A, long lda,
                           const float *Dinv, long ldd, float *G, cudaStream_t s);
int pla_k_trsv_ticket_link(char uplo, char trans, int n, const float *A, long lda,
                           const float *Dinv, long ldd, const float *G, const float *b, float *x,
                           int *status, cudaStream_t s);
void pla_trsv_release(void);
/* out (dt_out = MPI_FLOAT or MPI_DOUBLE, n x nrhs, ldo) := rows perm[0..n) of
 * the FP64 in (ldi): a composed row permutation and a conversion in one pass */
int pla_k_gather_rows(int dt_out, int n, int nrhs, const int *perm, const double *in, long ldi,
                      void *out, long ldo, cudaStream_t s);
/* batched Krylov-basis operations for up to 16 columns, column s's basis at
 * V + s ldv (ld n); bit s of `active` selects the columns:
 *   dots:   out[s ldo + c] = V_s(:, a0 + c) . V_s(:, b), c < nc
 *   update: V_s(:, b) -= V_s(:, 0:nc) h_s, h_s = h + s ldh (device)
 *   scale:  V_s(:, b) *= scale[s] (host array) */
int pla_k_basis_dots(int n, int nrhs, const double *V, long ldv, int a0, int nc, int b,
                     unsigned active, double *out, int ldo, cudaStream_t s);
int pla_k_basis_update(int n, int nrhs, double *V, long ldv, int nc, int b, const double *h,
                       int ldh, unsigned active, cudaStream_t s);
int pla_k_basis_scale(int n, int nrhs, double *V, long ldv, int b, const double *scale,
                      unsigned active, cudaStream_t s);
size_t pla_k_residual_work(int n, int ncols, int nrhs);
int pla_k_residual(int n, int ncols, int nrhs, const double *A, long lda, const double *X,
                   long ldx, const double *B, long ldb, double *R, long ldr, int abs_rows,
                   double *work, cudaStream_t s);

#ifdef __cplusplus
}
#endif
