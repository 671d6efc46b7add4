// Solvers and parallel/local BLAS of the dense direct-solve path on a 1x1
// template: the view loops of SOLVERS/LU, SOLVERS/Cholesky, BLAS2/PLA_Trsv*,
// BLAS3/PLA_Trsm*, BLAS3/PLA_Gemm* and Local_BLAS/ become sequences of
// device kernels on the library stream.  Every redistribution the reference
// performs with PLA_Copy (panels to multivectors, transposed projections) is
// a view into the same device buffer here, so no copy is made.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pla_internal.h"
#include "pla_kernels.h"

using namespace pla;

namespace {

constexpr int kTri = 128;  // largest diagonal block solved in shared memory

struct Status {
  int status;     // PLA_K_* of the kernels
  int info;       // Cholesky: failing global column (1-based)
  int zero_info;  // LU: first exact zero pivot (1-based)
};

Status *device_status() {
  return (Status *)scratch(0, sizeof(Status));
}

int finish(const char *what) {
  cudaError_t e = cudaStreamSynchronize(stream());
  if (e != cudaSuccess) return cuda_fail(e, __LINE__, what);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, __LINE__, what);
  return PLA_SUCCESS;
}

#define K(call)                                                    \
  do {                                                             \
    int r_ = (call);                                               \
    if (r_) return cuda_fail((cudaError_t)r_, __LINE__, __FILE__); \
  } while (0)

bool numeric(PLA_Obj o) { return is_double(o) || is_float(o); }

char uplo_c(int uplo) { return uplo == PLA_LOWER_TRIANGULAR ? 'L' : 'U'; }
char trans_c(int t) { return t == PLA_NO_TRANSPOSE ? 'N' : 'T'; }
char diag_c(int d) { return d == PLA_UNIT_DIAG ? 'U' : 'N'; }
int gemm_t(int t) { return t == PLA_NO_TRANSPOSE ? PLA_NO_TRANSPOSE : PLA_TRANSPOSE; }

// Left-side solve with one diagonal block of order kb <= 128 against `other`
// columns.  For many columns the block is inverted once (substitution against
// the identity) and applied as a GEMM, B := alpha inv(op(T)) B.  The GEMM runs
// in place when kb rows fit one CTA tile of the GEMM (every column tile of B
// is then read and written by one CTA only); otherwise B is first copied.
int trsm_left_block(int dt, char uplo, char trans, char diag, int kb, int other, double alpha,
                    const char *T, long ldt, char *B, long ldb, const int *status) {
  if (other < 1024)
    return pla_k_trsm_small(dt, 'L', uplo, trans, diag, kb, other, alpha, T, ldt, B, ldb, status,
                            stream());
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  char *inv = (char *)scratch(3, (size_t)kTri * kTri * es);
  if (!inv) return (int)cudaErrorMemoryAllocation;
  int r = pla_k_fill(dt, kb, kb, inv, kb, 0.0, stream());
  if (!r) r = pla_k_fill(dt, 1, kb, inv, kb + 1, 1.0, stream());  // the diagonal
  if (!r) r = pla_k_trsm_small(dt, 'L', uplo, trans, diag, kb, kb, 1.0, T, ldt, inv, kb, status,
                               stream());
  const char *src = B;
  long lds = ldb;
  if (!r && kb > pla_k_gemm_tile_rows(dt)) {
    char *copy = (char *)scratch(17, (size_t)kb * other * es);
    if (!copy) return (int)cudaErrorMemoryAllocation;
    r = pla_k_copy(dt, PLA_NO_TRANSPOSE, kb, other, B, ldb, copy, kb, stream());
    src = copy;
    lds = kb;
  }
  if (!r) r = pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, kb, other, kb, alpha, inv, kb, src,
                         lds, 0.0, B, ldb, 0, status, stream());
  return r;
}

// op(T) X = alpha B (side L) or X op(T) = alpha B (side R) for a triangle of
// any size: diagonal blocks of <= 128 (inverse-diagonal + GEMM on the left),
// the coupling blocks by GEMM, ordered like BLAS3/PLA_Trsm_left_lower.c:33-78.
int trsm_blocked(int dt, char side, char uplo, char trans, char diag, int nt, int other,
                 double alpha, const char *T, long ldt, char *B, long ldb, const int *status) {
  if (nt <= 0 || other <= 0) return 0;
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  const bool tr = trans != 'N';
  auto t_at = [&](long i, long j) { return T + (i + j * ldt) * es; };
  if (nt <= kTri && side == 'L')
    return trsm_left_block(dt, uplo, trans, diag, nt, other, alpha, T, ldt, B, ldb, status);
  if (nt <= kTri)
    return pla_k_trsm_small(dt, side, uplo, trans, diag, nt, other, alpha, T, ldt, B, ldb,
                            status, stream());
  const int nblk = (nt + kTri - 1) / kTri;
  if (side == 'L') {
    // op(T) lower: forward over row blocks; upper: backward
    const bool forward = (uplo == 'L') != tr;
    auto b_at = [&](long i) { return B + i * es; };
    for (int q = 0; q < nblk; q++) {
      const int blk = forward ? q : nblk - 1 - q;
      const int k0 = blk * kTri, kb = std::min(kTri, nt - k0);
      // alpha scales the first block here and every other row in the first
      // GEMM below (its beta), so later steps use 1
      const double a = q == 0 ? alpha : 1.0;
      int r = trsm_left_block(dt, uplo, trans, diag, kb, other, a, t_at(k0, k0), ldt, b_at(k0),
                              ldb, status);
      if (r) return r;
      int r0 = forward ? k0 + kb : 0, rn = forward ? nt - r0 : k0;
      if (rn <= 0) continue;
      const char *Ablk = tr ? t_at(k0, r0) : t_at(r0, k0);
      // B_rest := a_rest * B_rest - op(T)(rest, blk) X_blk, where the rest
      // rows still carry their original scale on the first step
      r = pla_k_gemm(dt, tr ? PLA_TRANSPOSE : PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, rn, other, kb,
                     -1.0, Ablk, ldt, b_at(k0), ldb, q == 0 ? alpha : 1.0, b_at(r0), ldb, 0,
                     status, stream());
      if (r) return r;
    }
    return 0;
  }
  // side R: X op(T) = alpha B; op(T) upper: forward over column blocks
  const bool forward = (uplo == 'U') != tr;
  auto b_col = [&](long j) { return B + j * ldb * es; };
  for (int q = 0; q < nblk; q++) {
    const int blk = forward ? q : nblk - 1 - q;
    const int k0 = blk * kTri, kb = std::min(kTri, nt - k0);
    int r = pla_k_trsm_small(dt, 'R', uplo, trans, diag, kb, other, q == 0 ? alpha : 1.0,
                             t_at(k0, k0), ldt, b_col(k0), ldb, status, stream());
    if (r) return r;
    int c0 = forward ? k0 + kb : 0, cn = forward ? nt - c0 : k0;
    if (cn <= 0) continue;
    // B(:, rest) := a B(:, rest) - X_blk op(T)(blk, rest)
    const char *Tblk = tr ? t_at(c0, k0) : t_at(k0, c0);
    r = pla_k_gemm(dt, PLA_NO_TRANSPOSE, tr ? PLA_TRANSPOSE : PLA_NO_TRANSPOSE, other, cn, kb,
                   -1.0, b_col(k0), ldb, Tblk, ldt, q == 0 ? alpha : 1.0, b_col(c0), ldb, 0,
                   status, stream());
    if (r) return r;
  }
  return 0;
}

}  // namespace

namespace pla {
// The r x b panel at `P` (row k of the matrix) with partial pivoting.  The
// column loop of PLA_LU_right_mv (SOLVERS/LU/PLA_LU_mv.c:52-82) runs in the
// cooperative kernel on sub-panels of kSub columns, whose rows stay in shared
// memory; after each sub-panel its pivots are applied to the panel's other
// columns and the columns to its right get the unit-lower solve and the
// rank-kSub update (for fp32 both in one launch, pla_k_panel_update).  Pivot
// choices are those of the column-by-column loop; only the rounding order of
// the panel's trailing columns differs.  (Tournament
// pivoting of the sub-panels with their interchanges and U12 solve done in
// the tournament kernels themselves, two launches fewer per sub-panel, was
// measured slower inside the solve: 233 against 225 ms at n = 32768, that
// work then sitting on the root CTA of the critical path.)
int panel_lu(int dt, int r, int b, char *P, long lda, int *piv, int *status, int *zero_info,
             int row_base, int max_ctas, int pivoting) {
  constexpr int kSub = 32;
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  auto at = [&](long i, long j) { return P + (i + j * lda) * es; };
  // one sub-panel of width sb at (s, s): partial pivoting (the reference's
  // column loop, one exchange round per column), or -- fp32 only, for the
  // mixed LU whose pivots need not be the reference's -- tournament pivoting
  auto factor = [&](int s, int sb) -> int {
    if (pivoting == PLA_B200_PIVOT_TOURNAMENT && dt == MPI_FLOAT)
      return pla_k_lu_panel_tslu(r - s, sb, (float *)at(s, s), lda, piv + s, zero_info,
                                 row_base + s, max_ctas, stream());
    return pla_k_lu_panel_ex(dt, r - s, sb, at(s, s), lda, piv + s, status, zero_info,
                             row_base + s, max_ctas, stream());
  };
  if (b <= kSub) return factor(0, b);
  for (int s = 0; s < b; s += kSub) {
    const int sb = std::min(kSub, b - s), rest = b - s - sb;
    int e = factor(s, sb);
    if (e) return e;
    e = pla_k_laswp(dt, at(s, 0), lda, sb, piv + s, 0, s, s + sb, b, stream());
    if (e) return e;
    if (rest <= 0) continue;
    if (dt == MPI_FLOAT && rest <= PLA_K_PANEL_UPDATE_MAX) {  // U12 solve and update, one launch
      e = pla_k_panel_update(r - s, sb, rest, (float *)at(s, s), lda, stream());
      if (e) return e;
      continue;
    }
    e = pla_k_trsm_small(dt, 'L', 'L', 'N', 'U', sb, rest, 1.0, at(s, s), lda, at(s, s + sb), lda,
                         status, stream());
    if (e) return e;
    if (r - s - sb > 0) {
      e = pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, r - s - sb, rest, sb, -1.0,
                     at(s + sb, s), lda, at(s, s + sb), lda, 1.0, at(s + sb, s + sb), lda, 0,
                     status, stream());
      if (e) return e;
    }
  }
  return 0;
}
}  // namespace pla

// The blocked panel factorization alone (panel_lu: the r x b panel at P,
// pivots to piv, first exact zero pivot to zero_info), queued on stream s
// (0: the library stream), for timing and tests.
extern "C" int pla_k_panel_lu_blocked(int dt, int r, int b, void *P, long lda, int *piv,
                                      int *zero_info, int max_ctas, int pivoting,
                                      cudaStream_t s) {
  if (dt != MPI_FLOAT && dt != MPI_DOUBLE) return (int)cudaErrorInvalidValue;
  OnStream on(s);
  int *st = (int *)scratch(0, 4 * sizeof(int));
  if (!st) return (int)cudaErrorMemoryAllocation;
  cudaMemsetAsync(st, 0, 4 * sizeof(int), stream());
  return panel_lu(dt, r, b, (char *)P, lda, piv, st, zero_info, 0, max_ctas, pivoting);
}

namespace {

// Blocked right-looking LU (SOLVERS/LU/PLA_LU.c:103-192) on device memory,
// with a lookahead of one panel.  After the TRSM of step k the columns of
// panel k+1 are updated first; panel k+1 is then factored on the
// high-priority lookahead stream, on at most lookahead_ctas(dt) CTAs, while the
// rest of the trailing update of step k runs on the library stream.  The two
// touch disjoint columns, and step k+1 starts (row interchanges across the
// full width) only after both.  Every operation and its operands are those
// of the loop without lookahead, so the pivots and factors are the same.
// With left_swaps false (PLA_LU_linpack_right, SOLVERS/LINPACK/
// PLA_LU_linpack.c:108-112) each step's interchanges skip the columns left of
// its panel: the L of earlier steps keeps its rows where they were, as in
// LINPACK's dgefa.
int lu_device(int dt, int m, int n, char *A, long lda, int *piv, int nb, Status *st,
              bool left_swaps = true) {
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  auto at = [&](long i, long j) { return A + (i + j * lda) * es; };
  const int kmax = std::min(m, n);
  PLA_Phase_times &ph = state().phases;
  const bool la = kmax >= 4 * nb;  // worth a second stream
  cudaStream_t s0 = stream(), s1 = la ? lookahead_stream() : s0;
  cudaEvent_t ev_next = la ? lookahead_event(0) : nullptr, ev_panel = la ? lookahead_event(1) : nullptr;
  auto update = [&](int k, int b, int c0, int nc) -> int {
    PhaseTimer t(&ph.update_ms);
    int r = pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, m - k - b, nc, b, -1.0,
                       at(k + b, k), lda, at(k, c0), lda, 1.0, at(k + b, c0), lda, 0, &st->status,
                       stream());
    if (t.on) ph.update_launches++;
    return r;
  };
  int ready = -1;  // step whose panel the lookahead stream has factored
  for (int k = 0; k < kmax; k += nb) {
    const int b = std::min(nb, kmax - k), r = m - k;
    if (ready == k) {
      PLA_CUDA(cudaStreamWaitEvent(s0, ev_panel, 0));
    } else {
      PhaseTimer t(&ph.panel_ms);
      K(panel_lu(dt, r, b, at(k, k), lda, piv + k, &st->status, &st->zero_info, k, 0,
                   PLA_B200_PIVOT_PARTIAL));
    }
    {
      PhaseTimer t(&ph.swap_ms);
      K(pla_k_laswp(dt, at(k, 0), lda, b, piv + k, 0, left_swaps ? k : 0, k + b, n, stream()));
    }
    if (k + b >= n) continue;
    {
      PhaseTimer t(&ph.trsm_ms);
      K(trsm_blocked(dt, 'L', 'L', 'N', 'U', b, n - k - b, 1.0, at(k, k), lda, at(k, k + b), lda,
                     &st->status));
    }
    if (m - k - b <= 0) continue;
    const int k2 = k + b, b2 = std::min(nb, kmax - k2);
    if (la && b2 > 0) {
      K(update(k, b, k2, b2));  // the next panel's columns first
      PLA_CUDA(cudaEventRecord(ev_next, s0));
      PLA_CUDA(cudaStreamWaitEvent(s1, ev_next, 0));
      {
        OnStream on(s1);
        PhaseTimer t(&ph.panel_ms);
        K(panel_lu(dt, m - k2, b2, at(k2, k2), lda, piv + k2, &st->status, &st->zero_info, k2,
                   lookahead_ctas(dt), PLA_B200_PIVOT_PARTIAL));
      }
      PLA_CUDA(cudaEventRecord(ev_panel, s1));
      ready = k2;
      if (n - k2 - b2 > 0) K(update(k, b, k2 + b2, n - k2 - b2));
    } else {
      K(update(k, b, k2, n - k2));
    }
  }
  return 0;  // every lookahead panel was awaited at its own step
}

// A21 := A21 inv(L11)' for the rest x b block column below a b x b diagonal
// block (b <= 128).  For tall blocks L11 is inverted once (substitution
// against the identity) and applied as a GEMM from a copy of A21.
int trsm_right_lower_t(int dt, int b, int rest, const char *L11, long lda, char *A21,
                       const int *status) {
  if (rest < 1024)
    return pla_k_trsm_small(dt, 'R', 'L', 'T', 'N', b, rest, 1.0, L11, lda, A21, lda, status,
                            stream());
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  char *inv = (char *)scratch(20, (size_t)kTri * kTri * es);
  char *copy = (char *)scratch(21, (size_t)rest * b * es);
  if (!inv || !copy) return (int)cudaErrorMemoryAllocation;
  int r = pla_k_fill(dt, b, b, inv, b, 0.0, stream());
  if (!r) r = pla_k_fill(dt, 1, b, inv, b + 1, 1.0, stream());  // the diagonal
  if (!r) r = pla_k_trsm_small(dt, 'L', 'L', 'N', 'N', b, b, 1.0, L11, lda, inv, b, status,
                               stream());
  if (!r) r = pla_k_copy(dt, PLA_NO_TRANSPOSE, rest, b, A21, lda, copy, rest, stream());
  if (!r) r = pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_TRANSPOSE, rest, b, b, 1.0, copy, rest, inv, b,
                         0.0, A21, lda, 0, status, stream());
  return r;
}

// Blocked right-looking lower Cholesky (SOLVERS/Cholesky/PLA_Chol.c:159-224),
// with the lookahead of the LU loop: after step k the block column k+1 is
// updated first, its diagonal factorization and solve run on the lookahead
// stream, and the rest of the SYRK update of step k runs beside them.
int chol_device(int dt, int n, char *A, long lda, int nb, Status *st) {
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  auto at = [&](long i, long j) { return A + (i + j * lda) * es; };
  nb = std::min(nb, 4 * kTri);  // a block column of up to 512, factored in steps of <= 128
  PLA_Phase_times &ph = state().phases;
  const bool la = n >= 4 * nb;
  cudaStream_t s0 = stream(), s1 = la ? lookahead_stream() : s0;
  cudaEvent_t ev_next = la ? lookahead_event(0) : nullptr, ev_panel = la ? lookahead_event(1) : nullptr;
  // block column [k, k + b): inner steps of at most 128 columns (diagonal
  // block, the solve below it, the update of the block column's remaining
  // columns), so the trailing SYRK of the outer loop has K = b
  auto panel = [&](int k, int b) -> int {
    for (int kk = k; kk < k + b; kk += kTri) {
      const int bb = std::min(kTri, k + b - kk), rest = n - kk - bb;
      {
        PhaseTimer t(&ph.panel_ms);
        K(pla_k_potrf_lower(dt, bb, at(kk, kk), lda, &st->status, &st->info, kk, stream()));
      }
      if (rest <= 0) break;
      {
        PhaseTimer t(&ph.trsm_ms);
        K(trsm_right_lower_t(dt, bb, rest, at(kk, kk), lda, at(kk + bb, kk), &st->status));
      }
      const int inner = k + b - kk - bb;  // columns of the block column still to update
      if (inner > 0) {
        PhaseTimer t(&ph.panel_ms);
        K(pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_TRANSPOSE, rest, inner, bb, -1.0, at(kk + bb, kk),
                     lda, at(kk + bb, kk), lda, 1.0, at(kk + bb, kk + bb), lda, 'L', &st->status,
                     stream()));
      }
    }
    return 0;
  };
  // columns [c0, c0 + nc) of the trailing matrix (rows c0 .. n-1, lower part)
  auto syrk = [&](int k, int b, int c0, int nc) -> int {
    PhaseTimer t(&ph.update_ms);
    int r = pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_TRANSPOSE, n - c0, nc, b, -1.0, at(c0, k), lda,
                       at(c0, k), lda, 1.0, at(c0, c0), lda, 'L', &st->status, stream());
    if (t.on) ph.update_launches++;
    return r;
  };
  int ready = -1;
  for (int k = 0; k < n; k += nb) {
    const int b = std::min(nb, n - k), rest = n - k - b, k2 = k + b;
    if (ready == k) PLA_CUDA(cudaStreamWaitEvent(s0, ev_panel, 0));
    else K(panel(k, b));
    if (rest <= 0) continue;
    const int b2 = std::min(nb, rest);
    if (la) {
      K(syrk(k, b, k2, b2));  // block column k+1 first
      PLA_CUDA(cudaEventRecord(ev_next, s0));
      PLA_CUDA(cudaStreamWaitEvent(s1, ev_next, 0));
      {
        OnStream on(s1);
        K(panel(k2, b2));
      }
      PLA_CUDA(cudaEventRecord(ev_panel, s1));
      ready = k2;
      if (rest - b2 > 0) K(syrk(k, b, k2 + b2, rest - b2));
    } else {
      K(syrk(k, b, k2, rest));
    }
  }
  return 0;
}


// vector increment of a 1-row or 1-column view
long vinc(PLA_Obj v) { return (v->length == 1 && v->width > 1) ? ld(v) : 1; }
int vlen(PLA_Obj v) { return (v->length == 1) ? v->width : v->length; }

}  // namespace

namespace pla {
// the factorization loops without the final status read-back (callers that
// queue many factorizations and synchronize once)
int lu_async(int dt, int m, int n, char *A, long lda, int *piv, int nb) {
  Status *st = device_status();
  if (!st) PLA_FAIL("cannot allocate the status word");
  PLA_CUDA(cudaMemsetAsync(st, 0, sizeof(Status), stream()));
  return lu_device(dt, m, n, A, lda, piv, nb, st);
}
int chol_async(int dt, int n, char *A, long lda, int nb) {
  Status *st = device_status();
  if (!st) PLA_FAIL("cannot allocate the status word");
  PLA_CUDA(cudaMemsetAsync(st, 0, sizeof(Status), stream()));
  return chol_device(dt, n, A, lda, nb, st);
}
int lu_on_device(int dt, int m, int n, char *A, long lda, int *piv, int nb, int *zero_info_host,
                 bool left_swaps) {
  Status *st = device_status();
  if (!st) PLA_FAIL("cannot allocate the status word");
  PLA_CUDA(cudaMemsetAsync(st, 0, sizeof(Status), stream()));
  int r = lu_device(dt, m, n, A, lda, piv, nb, st, left_swaps);
  if (r) return r;
  count_interchanges(std::min(m, n), piv);
  Status h{};
  PLA_CUDA(cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, stream()));
  r = finish("lu");
  if (r) return r;
  if (h.status == PLA_K_TIMEOUT) PLA_FAIL("panel factorization: grid barrier timed out");
  if (zero_info_host) *zero_info_host = h.zero_info;
  return PLA_SUCCESS;
}
int trsm_device(int dt, char side, char uplo, char trans, char diag, int nt, int other,
                double alpha, const char *T, long ldt, char *B, long ldb) {
  return trsm_blocked(dt, side, uplo, trans, diag, nt, other, alpha, T, ldt, B, ldb, nullptr);
}
int chol_on_device(int dt, int n, char *A, long lda, int nb, int *info_host) {
  Status *st = device_status();
  if (!st) PLA_FAIL("cannot allocate the status word");
  PLA_CUDA(cudaMemsetAsync(st, 0, sizeof(Status), stream()));
  int r = chol_device(dt, n, A, lda, nb, st);
  if (r) return r;
  Status h{};
  PLA_CUDA(cudaMemcpyAsync(&h, st, sizeof h, cudaMemcpyDeviceToHost, stream()));
  r = finish("chol");
  if (r) return r;
  *info_host = h.status == PLA_K_NOT_SPD ? h.info : 0;
  return PLA_SUCCESS;
}
}  // namespace pla

extern "C" {

// ------------------------------------------------------------------- LU ----
static int lu_entry(PLA_Obj A, PLA_Obj pivots, int nb, bool left_swaps, int *info) {
  State &s = state();
  if (s.check_parameters) {
    int value = PLA_SUCCESS;
    // SOLVERS/LU/PLA_LU_enter_exit.c:17-103
    if (!valid(A) || A->objtype != PLA_MATRIX) { warn("Invalid object A"); value--; }
    else if (!numeric(A)) { warn("datatype not yet supported"); value--; }
    if (!valid(pivots) || pivots->objtype != PLA_MVECTOR) {
      return fail("Invalid objtype for pivots: pivots must be a multivector of size n x 1",
                  __LINE__, __FILE__);
    }
    if (pivots->base->datatype != MPI_INT) { warn("pivots must be of type MPI_INT"); value--; }
    if (valid(A) && pivots->length != std::min(A->length, A->width)) {
      warn("length of pivots must match min( length of A, width of A )");
      value--;
    }
    if (value != PLA_SUCCESS) return value;
  }
  if (!valid(A) || !numeric(A)) PLA_FAIL("PLA_LU needs a float or double matrix");
  if (nb <= 0) PLA_Environ_nb_alg(PLA_OP_PAN_PAN, A->templ, &nb);
  int zi = 0;
  int r = lu_on_device(A->base->datatype, A->length, A->width, at(A, 0, 0), ld(A),
                       (int *)at(pivots, 0, 0), nb, &zi, left_swaps);
  if (r) return r;
  if (info) *info = zi;
  return PLA_SUCCESS;  // the reference never reports singularity (PLA_LU.c:29)
}

int PLA_LU_info(PLA_Obj A, PLA_Obj pivots, int *info) {
  return lu_entry(A, pivots, 0, true, info);
}

int PLA_LU(PLA_Obj A, PLA_Obj pivots) { return lu_entry(A, pivots, 0, true, nullptr); }

// SOLVERS/LU/PLA_LU.c:37: the blocked LU with the caller's block size
int PLA_LU_right(int nb_alg, PLA_Obj A, PLA_Obj pivots) {
  if (nb_alg <= 0) PLA_FAIL("PLA_LU_right: nb_alg must be positive");
  return lu_entry(A, pivots, nb_alg, true, nullptr);
}

// SOLVERS/LU/PLA_LU_mv.c:13-102: factor the panel A_mv in place with partial
// pivoting; pivots_msc receives the pivots and A_11_msc a copy of the factored
// top block (row j is copied when it becomes the pivot row, :274, and rows
// above the current column never change afterwards, so the copy is the final
// top min(m, n) x n block).  The pivots are those of the column loop.
int PLA_LU_right_mv(PLA_Obj A_mv, PLA_Obj A_11_msc, PLA_Obj pivots_msc) {
  if (!valid(A_mv) || !valid(A_11_msc) || !valid(pivots_msc)) PLA_FAIL("invalid object");
  if (!numeric(A_mv)) PLA_FAIL("datatype not yet supported");
  if (A_11_msc->base->datatype != A_mv->base->datatype) PLA_FAIL("datatype mismatch");
  if (pivots_msc->base->datatype != MPI_INT) PLA_FAIL("pivots must be of type MPI_INT");
  const int m = A_mv->length, n = A_mv->width, k = std::min(m, n);
  if (A_11_msc->length < k || A_11_msc->width < n) PLA_FAIL("A_11_msc smaller than the panel's top block");
  if (vlen(pivots_msc) < k || vinc(pivots_msc) != 1) PLA_FAIL("pivots_msc must be a column of min(m, n) entries");
  if (k == 0) return PLA_SUCCESS;
  int *dpiv = (int *)scratch(29, (size_t)k * sizeof(int));
  if (!dpiv) PLA_FAIL("cannot allocate scratch");
  int r = lu_on_device(A_mv->base->datatype, m, n, at(A_mv, 0, 0), ld(A_mv), dpiv, kTri, nullptr,
                       true);
  if (r) return r;
  const int es = A_mv->base->esize;
  PLA_CUDA(cudaMemcpy2DAsync(at(A_11_msc, 0, 0), (size_t)ld(A_11_msc) * es, at(A_mv, 0, 0),
                             (size_t)ld(A_mv) * es, (size_t)k * es, n, cudaMemcpyDefault, stream()));
  PLA_CUDA(cudaMemcpyAsync(at(pivots_msc, 0, 0), dpiv, (size_t)k * sizeof(int), cudaMemcpyDefault,
                           stream()));
  return finish("lu_right_mv");
}

// SOLVERS/LINPACK/PLA_LU_linpack.c:13-28 and :30-208: the blocked LU whose
// interchanges leave the columns left of each panel alone
int PLA_LU_linpack(PLA_Obj A, PLA_Obj pivots) { return lu_entry(A, pivots, 0, false, nullptr); }

int PLA_LU_linpack_right(int nb_alg, PLA_Obj A, PLA_Obj pivots) {
  if (nb_alg <= 0) PLA_FAIL("PLA_LU_linpack_right: nb_alg must be positive");
  return lu_entry(A, pivots, nb_alg, false, nullptr);
}

// SOLVERS/LU/PLA_Apply_pivots_new.c:13-179: the interchanges in sequence
int PLA_Apply_pivots_to_rows(PLA_Obj A, PLA_Obj ipiv) {
  if (!valid(A) || !valid(ipiv)) PLA_FAIL("invalid object");
  if (ipiv->base->datatype != MPI_INT) PLA_FAIL("pivots must be of type MPI_INT");
  if (!numeric(A)) PLA_FAIL("datatype not yet supported");
  int npiv = vlen(ipiv);
  if (npiv > A->length) PLA_FAIL("more pivots than rows");
  if (vinc(ipiv) != 1) PLA_FAIL("pivots must be a column");
  {
    // a pivot vector from the caller must name rows of A (the kernel trusts it)
    std::vector<int> h(npiv);
    PLA_CUDA(d2h(h.data(), at(ipiv, 0, 0), npiv * sizeof(int)));
    for (int i = 0; i < npiv; i++)
      if (h[i] < 0 || i + h[i] >= A->length) PLA_FAIL("pivot entry outside the rows of A");
  }
  K(pla_k_laswp_rows(A->base->datatype, at(A, 0, 0), ld(A), A->width, npiv,
                     (const int *)at(ipiv, 0, 0), stream()));
  return finish("apply pivots");
}

// columns j = n-1 .. 0: swap column j with column j + piv[j] (:309-451)
int PLA_Apply_pivots_to_columns_in_reverse(PLA_Obj A, PLA_Obj ipiv) {
  if (!valid(A) || !valid(ipiv)) PLA_FAIL("invalid object");
  if (ipiv->objtype != PLA_MVECTOR) PLA_FAIL("not yet implemented");
  int npiv = std::min(vlen(ipiv), A->width);
  std::vector<int> h(npiv);
  PLA_CUDA(d2h(h.data(), at(ipiv, 0, 0), npiv * sizeof(int)));
  for (int j = npiv - 1; j >= 0; j--) {
    int p = j + h[j];
    if (p == j) continue;
    if (p >= A->width) PLA_FAIL("pivot out of range");
    K(pla_k_swap(A->base->datatype, A->length, 1, at(A, 0, j), ld(A), at(A, 0, p), ld(A),
                 stream()));
  }
  return finish("apply pivots to columns");
}

// -------------------------------------------------------------- Cholesky ----
int PLA_Chol(int uplo, PLA_Obj A) {
  State &s = state();
  if (s.check_parameters) {
    // SOLVERS/Cholesky/PLA_Chol_enter_exit.c:17-60
    if (uplo != PLA_LOWER_TRIANGULAR && uplo != PLA_UPPER_TRIANGULAR) warn("Invalid parameter uplo");
    if (uplo != PLA_LOWER_TRIANGULAR) PLA_FAIL("Only lower triangular factorization supported");
    if (!valid(A) || A->objtype != PLA_MATRIX) { warn("Invalid objtype for A"); return -1; }
    if (A->length != A->width) { warn("A must be square"); return -1; }
  }
  if (!valid(A) || !numeric(A)) PLA_FAIL("PLA_Chol needs a float or double matrix");
  if (uplo != PLA_LOWER_TRIANGULAR) PLA_FAIL("Only lower triangular factorization supported");
  int nb;
  PLA_Environ_nb_alg(PLA_OP_PAN_PAN, A->templ, &nb);
  int info = 0;
  int r = chol_on_device(A->base->datatype, A->length, at(A, 0, 0), ld(A), nb, &info);
  if (r) return r;
  return info;  // global 1-based failing column, as PLA_Chol.c:181-185 computes
}

int PLA_Local_chol(int uplo, PLA_Obj A) {
  if (uplo != PLA_LOWER_TRIANGULAR) PLA_FAIL("Only lower triangular factorization supported");
  if (!valid(A) || !numeric(A)) PLA_FAIL("invalid object");
  int info = 0;
  int r = chol_on_device(A->base->datatype, A->length, at(A, 0, 0), ld(A), kTri, &info);
  return r ? r : info;
}

// --------------------------------------------------------------- solves ----
}  // extern "C"

namespace pla {
// x := inv(op(T)) x for nrhs columns of x: one or two columns of order >= 1024
// go through the single-launch solve (inverse diagonal blocks first, then one
// launch per column); other shapes through the blocked solve.  Queued on the
// library stream; a bounded wait that gives up is reported by finish_solve.
int tri_solve(int dt, char uplo, char trans, char diag, int n, int nrhs, const char *T, long ldt,
              char *X, long ldx) {
  if (n <= 0 || nrhs <= 0) return 0;
  if (n < 1024 || nrhs > 2)
    return pla_k_trsv_blocked(dt, uplo, trans, diag, n, nrhs, T, ldt, X, ldx, stream());
  const int es = dt == MPI_DOUBLE ? 8 : 4, tb = dt == MPI_DOUBLE ? 64 : 128;
  const long ldd = ((long)n + tb - 1) / tb * tb;
  char *dinv = (char *)scratch(22, (size_t)ldd * tb * es);
  int *status = (int *)scratch(23, 64);
  if (!dinv || !status) return (int)cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), stream());
  if (e) return (int)e;
  int r = pla_k_trsv_inv_blocks(dt, uplo, trans, diag, n, T, ldt, dinv, ldd, stream());
  for (int c = 0; c < nrhs && !r; c++) {
    char *col = X + (long)c * ldx * es;
    r = pla_k_trsv_ticket(dt, uplo, trans, n, T, ldt, dinv, ldd, col, col, status, stream());
  }
  return r;
}
// after tri_solve: wait, and report a solve whose bounded wait gave up
int finish_solve(const char *what) {
  int r = finish(what);
  if (r) return r;
  int *status = (int *)scratch(23, 64);
  int h = 0;
  if (status) PLA_CUDA(d2h(&h, status, sizeof h));
  if (h == PLA_K_TIMEOUT) PLA_FAIL("triangular solve: a bounded wait timed out");
  return PLA_SUCCESS;
}
}  // namespace pla

extern "C" {

int PLA_Trsv(int uplo, int trans, int diag, PLA_Obj A, PLA_Obj x) {
  if (!valid(A) || !valid(x)) PLA_FAIL("invalid object");
  if (!numeric(A) || A->base->datatype != x->base->datatype) PLA_FAIL("datatype mismatch");
  if (A->length != A->width || vlen(x) != A->length) PLA_FAIL("nonconformal objects");
  if (vinc(x) != 1) PLA_FAIL("x must be a column vector");
  PhaseTimer t(&state().phases.solve_ms);
  K(tri_solve(A->base->datatype, uplo_c(uplo), trans_c(trans), diag_c(diag), A->length, 1,
              at(A, 0, 0), ld(A), at(x, 0, 0), ld(x)));
  return finish_solve("trsv");
}

int PLA_Local_trsv(int uplo, int trans, int diag, PLA_Obj A, PLA_Obj x) {
  return PLA_Trsv(uplo, trans, diag, A, x);
}

int PLA_Trsm(int side, int uplo, int trans, int diag, PLA_Obj alpha, PLA_Obj A, PLA_Obj B) {
  if (!valid(A) || !valid(B) || !valid(alpha)) PLA_FAIL("invalid object");
  if (!numeric(A) || A->base->datatype != B->base->datatype) PLA_FAIL("datatype mismatch");
  const int nt = side == PLA_SIDE_LEFT ? B->length : B->width;
  const int other = side == PLA_SIDE_LEFT ? B->width : B->length;
  if (A->length != nt || A->width != nt) PLA_FAIL("nonconformal objects");
  PhaseTimer t(&state().phases.solve_ms);
  K(trsm_blocked(A->base->datatype, side == PLA_SIDE_LEFT ? 'L' : 'R', uplo_c(uplo),
                 trans_c(trans), diag_c(diag), nt, other, scalar_value(alpha), at(A, 0, 0), ld(A),
                 at(B, 0, 0), ld(B), nullptr));
  return finish("trsm");
}

int PLA_Local_trsm(int side, int uplo, int trans, int diag, PLA_Obj alpha, PLA_Obj A,
                   PLA_Obj B) {
  return PLA_Trsm(side, uplo, trans, diag, alpha, A, B);
}

static int gemm_objs(int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B, PLA_Obj beta,
                     PLA_Obj C, int uplo_c) {
  if (!valid(A) || !valid(B) || !valid(C) || !valid(alpha) || !valid(beta))
    PLA_FAIL("invalid object");
  if (!numeric(C) || A->base->datatype != C->base->datatype ||
      B->base->datatype != C->base->datatype)
    PLA_FAIL("datatype mismatch");
  const bool ta = transa != PLA_NO_TRANSPOSE, tb = transb != PLA_NO_TRANSPOSE;
  const int m = C->length, n = C->width;
  const int k = ta ? A->length : A->width;
  if ((ta ? A->width : A->length) != m || (tb ? B->length : B->width) != n ||
      (tb ? B->width : B->length) != k)
    PLA_FAIL("nonconformal objects");
  PhaseTimer t(&state().phases.update_ms);
  K(pla_k_gemm(C->base->datatype, gemm_t(transa), gemm_t(transb), m, n, k, scalar_value(alpha),
               at(A, 0, 0), ld(A), at(B, 0, 0), ld(B), scalar_value(beta), at(C, 0, 0), ld(C),
               uplo_c, nullptr, stream()));
  return finish("gemm");
}

// BLAS3/PLA_Gemm_x.c:13: the GEMM with the caller's choice of stationary
// operand (PLA_VERSION_A / _B / _C); on a 1x1 template nothing moves, so
// every version is the same device product
int PLA_Gemm(int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B, PLA_Obj beta,
             PLA_Obj C);
int PLA_Gemm_x(int version, int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B,
               PLA_Obj beta, PLA_Obj C) {
  if (version != PLA_VERSION_A && version != PLA_VERSION_B && version != PLA_VERSION_C)
    PLA_FAIL("PLA_Gemm_x: unknown version");
  return PLA_Gemm(transa, transb, alpha, A, B, beta, C);
}

int PLA_Gemm(int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B, PLA_Obj beta,
             PLA_Obj C) {
  return gemm_objs(transa, transb, alpha, A, B, beta, C, 0);
}

int PLA_Local_gemm(int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B, PLA_Obj beta,
                   PLA_Obj C) {
  return gemm_objs(transa, transb, alpha, A, B, beta, C, 0);
}

// C := beta C + alpha X X_trans restricted to one triangle; X_trans holds X'
// (BLAS3/PLA_Syrk_perform_local_part.c:13-78)
int PLA_Syrk_perform_local_part(int uplo, PLA_Obj alpha, PLA_Obj X, PLA_Obj X_trans,
                                PLA_Obj beta, PLA_Obj A) {
  return gemm_objs(PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, alpha, X, X_trans, beta, A, uplo_c(uplo));
}

// C := beta C + alpha op(A) op(A)' on one triangle (Local_BLAS/PLA_Local_syrk.c)
int PLA_Local_syrk(int uplo, int trans, PLA_Obj alpha, PLA_Obj A, PLA_Obj beta, PLA_Obj C) {
  int t2 = trans == PLA_NO_TRANSPOSE ? PLA_TRANSPOSE : PLA_NO_TRANSPOSE;
  return gemm_objs(trans, t2, alpha, A, A, beta, C, uplo_c(uplo));
}

int PLA_General_solve(PLA_Obj A, PLA_Obj ipiv, PLA_Obj B) {
  // SOLVERS/LU/PLA_General.c:67-119
  int error = PLA_LU(A, ipiv);
  if (error != PLA_SUCCESS) return error;
  if (!valid(B)) PLA_FAIL("invalid object B");
  if (B->width > 0) {
    int r = PLA_Apply_pivots_to_rows(B, ipiv);
    if (r) return r;
    const int dt = A->base->datatype, n = A->length;
    PhaseTimer t(&state().phases.solve_ms);
    // Trsv for one or two right-hand sides (single launch), Trsm for more
    K(tri_solve(dt, 'L', 'N', 'U', n, B->width, at(A, 0, 0), ld(A), at(B, 0, 0), ld(B)));
    K(tri_solve(dt, 'U', 'N', 'N', n, B->width, at(A, 0, 0), ld(A), at(B, 0, 0), ld(B)));
    r = finish_solve("general solve");
    if (r) return r;
  }
  return PLA_SUCCESS;
}

int PLA_Pos_def_solve(PLA_Obj A, PLA_Obj B) {
  // SOLVERS/Cholesky/PLA_Pos_def.c:44-99: warn on failure, solve regardless
  int value = PLA_Chol(PLA_LOWER_TRIANGULAR, A);
  if (value < 0) return value;
  if (value != PLA_SUCCESS) warn("irregular return from PLA_Chol");
  if (!valid(B)) PLA_FAIL("invalid object B");
  const int dt = A->base->datatype, n = A->length;
  PhaseTimer t(&state().phases.solve_ms);
  K(tri_solve(dt, 'L', 'N', 'N', n, B->width, at(A, 0, 0), ld(A), at(B, 0, 0), ld(B)));
  K(tri_solve(dt, 'L', 'T', 'N', n, B->width, at(A, 0, 0), ld(A), at(B, 0, 0), ld(B)));
  int r = finish_solve("pos def solve");
  return r ? r : value;
}

// --------------------------------------------------------- level 1 / 2 -----
int PLA_Gemv(int trans, PLA_Obj alpha, PLA_Obj A, PLA_Obj x, PLA_Obj beta, PLA_Obj y) {
  if (!valid(A) || !valid(x) || !valid(y)) PLA_FAIL("invalid object");
  if (vinc(x) != 1 || vinc(y) != 1) PLA_FAIL("x and y must be column vectors");
  K(pla_k_gemv(A->base->datatype, gemm_t(trans), A->length, A->width, scalar_value(alpha),
               at(A, 0, 0), ld(A), at(x, 0, 0), scalar_value(beta), at(y, 0, 0), stream()));
  return finish("gemv");
}

int PLA_Local_gemv(int trans, PLA_Obj alpha, PLA_Obj A, PLA_Obj x, PLA_Obj beta, PLA_Obj y) {
  return PLA_Gemv(trans, alpha, A, x, beta, y);
}

int PLA_Iamax(PLA_Obj x, PLA_Obj k, PLA_Obj xmax) {
  // BLAS1/PLA_Iamax.c:37-124: value and global index of the first max |x_i|
  if (!valid(x) || !valid(k) || !valid(xmax)) PLA_FAIL("invalid object");
  if (x->base->datatype != xmax->base->datatype) PLA_FAIL("datatype mismatch");
  int *di = (int *)scratch(1, 64);
  char *dv = (char *)di + 16;
  K(pla_k_iamax(x->base->datatype, vlen(x), at(x, 0, 0), vinc(x), di, dv, stream()));
  int hi;
  double hv[1];
  PLA_CUDA(cudaMemcpyAsync(&hi, di, sizeof hi, cudaMemcpyDeviceToHost, stream()));
  PLA_CUDA(cudaMemcpyAsync(hv, dv, x->base->esize, cudaMemcpyDeviceToHost, stream()));
  int r = finish("iamax");
  if (r) return r;
  if (vlen(x) == 0) hi = 0;
  PLA_Obj_set(k, MPI_INT, &hi);
  if (is_double(x)) PLA_Obj_set(xmax, MPI_DOUBLE, hv);
  else PLA_Obj_set(xmax, MPI_FLOAT, hv);
  return PLA_SUCCESS;
}

int PLA_Local_iamax(PLA_Obj x, int *index, void *value) {
  if (!valid(x)) PLA_FAIL("invalid object");
  int *di = (int *)scratch(1, 64);
  char *dv = (char *)di + 16;
  K(pla_k_iamax(x->base->datatype, vlen(x), at(x, 0, 0), vinc(x), di, dv, stream()));
  PLA_CUDA(cudaMemcpyAsync(index, di, sizeof(int), cudaMemcpyDeviceToHost, stream()));
  PLA_CUDA(cudaMemcpyAsync(value, dv, x->base->esize, cudaMemcpyDeviceToHost, stream()));
  return finish("local iamax");
}

int PLA_Local_scal(PLA_Obj alpha, PLA_Obj x) {
  if (!valid(alpha) || !valid(x)) PLA_FAIL("invalid object");
  K(pla_k_scal(x->base->datatype, x->length, x->width, scalar_value(alpha), at(x, 0, 0), ld(x),
               stream()));
  return finish("scal");
}

int PLA_Local_inv_scal(PLA_Obj alpha, PLA_Obj x) {
  if (!valid(alpha) || !valid(x)) PLA_FAIL("invalid object");
  K(pla_k_inv_scal(x->base->datatype, x->length, x->width, scalar_value(alpha), at(x, 0, 0),
                   ld(x), stream()));
  return finish("inv_scal");
}

int PLA_Local_swap(PLA_Obj x, PLA_Obj y) {
  if (!valid(x) || !valid(y)) PLA_FAIL("invalid object");
  if (x->length != y->length || x->width != y->width) PLA_FAIL("nonconformal objects");
  K(pla_k_swap(x->base->datatype, x->length, x->width, at(x, 0, 0), ld(x), at(y, 0, 0), ld(y),
               stream()));
  return finish("swap");
}

int PLA_Local_ger(PLA_Obj alpha, PLA_Obj x, PLA_Obj y, PLA_Obj A) {
  if (!valid(alpha) || !valid(x) || !valid(y) || !valid(A)) PLA_FAIL("invalid object");
  if (vlen(x) != A->length || vlen(y) != A->width) PLA_FAIL("nonconformal objects");
  K(pla_k_ger(A->base->datatype, A->length, A->width, scalar_value(alpha), at(x, 0, 0), vinc(x),
              at(y, 0, 0), vinc(y), at(A, 0, 0), ld(A), stream()));
  return finish("ger");
}

// y := alpha x + y (Local_BLAS/PLA_Local_BLAS1.c daxpy on the local parts;
// BLAS1/PLA_Axpy.c:13 redistributes x first, which a 1x1 template never
// needs).  x may also be the transpose-shaped view of y's data (a row vector
// against a column vector).
static int axpy_objs(PLA_Obj alpha, PLA_Obj x, PLA_Obj y, const char *what) {
  if (!valid(alpha) || !valid(x) || !valid(y)) PLA_FAIL("invalid object");
  if (x->base->datatype != y->base->datatype) PLA_FAIL("datatype mismatch");
  if (!numeric(y)) PLA_FAIL("datatype not yet supported");
  const int dt = y->base->datatype;
  const double a = scalar_value(alpha);
  if (x->length == y->length && x->width == y->width) {
    K(pla_k_axpby(dt, y->length, y->width, a, at(x, 0, 0), ld(x), 1.0, at(y, 0, 0), ld(y),
                  stream()));
  } else if (x->length == y->width && x->width == y->length) {
    char *t = (char *)scratch(28, (size_t)y->length * y->width * y->base->esize);
    if (!t) PLA_FAIL("cannot allocate scratch");
    K(pla_k_copy(dt, PLA_TRANSPOSE, y->length, y->width, at(x, 0, 0), ld(x), t, y->length,
                 stream()));
    K(pla_k_axpby(dt, y->length, y->width, a, t, y->length, 1.0, at(y, 0, 0), ld(y), stream()));
  } else {
    PLA_FAIL("nonconformal objects");
  }
  return finish(what);
}
int PLA_Axpy(PLA_Obj alpha, PLA_Obj x, PLA_Obj y) { return axpy_objs(alpha, x, y, "axpy"); }
int PLA_Local_axpy(PLA_Obj alpha, PLA_Obj x, PLA_Obj y) {
  return axpy_objs(alpha, x, y, "local axpy");
}

// alpha := || x ||_2 (BLAS1/PLA_Nrm2.c:13-66, Local_BLAS/PLA_Local_BLAS1.c:
// 394-441): a one-row x is read along its row, anything else down its first
// column, as the reference's local call does
int PLA_Local_nrm2(PLA_Obj x, PLA_Obj alpha) {
  if (!valid(x) || !valid(alpha)) PLA_FAIL("invalid object");
  if (!numeric(x)) PLA_FAIL("datatype not yet supported");
  double v = 0.0;
  if (x->length * x->width != 0) {
    const bool row = x->length == 1;
    const long n = row ? x->width : x->length, inc = row ? ld(x) : 1;
    double *d = (double *)scratch(1, 64);
    K(pla_k_nrm2(x->base->datatype, n, at(x, 0, 0), inc, d, stream()));
    PLA_CUDA(cudaMemcpyAsync(&v, d, sizeof v, cudaMemcpyDeviceToHost, stream()));
    const int r = finish("nrm2");
    if (r) return r;
  }
  if (x->base->datatype == MPI_FLOAT) {
    float f = (float)v;
    return PLA_Obj_set(alpha, MPI_FLOAT, &f);
  }
  return PLA_Obj_set(alpha, MPI_DOUBLE, &v);
}
int PLA_Nrm2(PLA_Obj x, PLA_Obj alpha) { return PLA_Local_nrm2(x, alpha); }

// add *value (of type datatype) to every diagonal element of obj
// (UTIL/PLA_Shift.c:15-91)
int PLA_Shift(PLA_Obj obj, MPI_Datatype datatype, void *value) {
  if (!valid(obj) || !value) PLA_FAIL("invalid object");
  if (!numeric(obj)) PLA_FAIL("PLA_Shift: Datatype not yet implemented");
  double v;
  if (datatype == MPI_DOUBLE) v = *(const double *)value;
  else if (datatype == MPI_FLOAT) v = *(const float *)value;
  else PLA_FAIL("Datatype not yet implemented");
  K(pla_k_shift_diag(obj->base->datatype, std::min(obj->length, obj->width), at(obj, 0, 0),
                     ld(obj), v, stream()));
  return finish("shift");
}

// ----------------------------------------------------------------- copies ---
static int copy_objs(PLA_Obj from, PLA_Obj to) {
  if (!valid_any(from) || !valid_any(to)) PLA_FAIL("invalid object");
  if (from->base->ooc || to->base->ooc) return ooc_copy(from, to);
  if (from->base->datatype != to->base->datatype) PLA_FAIL("datatype mismatch");
  const int dt = from->base->datatype;
  const int es = from->base->esize;
  bool same = from->length == to->length && from->width == to->width;
  bool transposed = from->length == to->width && from->width == to->length;
  // a row projection stores the rows of the matrix it is conformal to as its
  // columns, so a copy between it and a matrix transposes (COPY/PLA_Copy.c)
  bool proj_from = from->objtype == PLA_PMVECTOR && from->proj_onto == PLA_PROJ_ONTO_ROW;
  bool proj_to = to->objtype == PLA_PMVECTOR && to->proj_onto == PLA_PROJ_ONTO_ROW;
  bool trans = proj_from != proj_to;
  if (trans ? !transposed : !same) PLA_FAIL("objects do not conform");
  if (from->length == 0 || from->width == 0) return PLA_SUCCESS;
  if (from->base->on_host || to->base->on_host) {
    cudaMemcpyKind kind = cudaMemcpyDefault;
    if (trans) PLA_FAIL("transposed copy involving a host multiscalar");
    PLA_CUDA(cudaMemcpy2DAsync(at(to, 0, 0), ld(to) * es, at(from, 0, 0), ld(from) * es,
                               (size_t)from->length * es, from->width, kind, stream()));
    return finish("copy");
  }
  if (dt == MPI_INT && trans) PLA_FAIL("transposed integer copy");
  K(pla_k_copy(dt == MPI_INT ? MPI_FLOAT : dt, trans ? PLA_TRANSPOSE : PLA_NO_TRANSPOSE,
               to->length, to->width, at(from, 0, 0), ld(from), at(to, 0, 0), ld(to), stream()));
  return finish("copy");
}

int PLA_Copy(PLA_Obj from, PLA_Obj to) { return copy_objs(from, to); }
int PLA_Local_copy(PLA_Obj from, PLA_Obj to) { return copy_objs(from, to); }

// -------------------------------------------------- application interface ---
int PLA_API_begin(void) {
  if (state().api_active) PLA_FAIL("PLA_API_begin called twice");
  state().api_active = 1;
  return PLA_SUCCESS;
}
int PLA_API_end(void) {
  state().api_active = 0;
  return finish("api end");
}
int PLA_Obj_API_open(PLA_Obj obj) { return valid(obj) ? PLA_SUCCESS : fail("invalid object", __LINE__, __FILE__); }
int PLA_Obj_API_close(PLA_Obj obj) {
  if (!valid(obj)) PLA_FAIL("invalid object");
  return finish("api close");
}
int PLA_Obj_API_sync(PLA_Obj obj) { return PLA_Obj_API_close(obj); }

// obj(i0:i0+m, j0:j0+n) += alpha * host(m x n, ldim): staged through the
// library's device scratch in column chunks (API/PLA_API.c:390-590)
static int axpy_to_global(int m, int n, void *alpha, const void *host, long ldh, long inch,
                          PLA_Obj obj, int i0, int j0) {
  if (!valid(obj)) PLA_FAIL("invalid object");
  if (m == 0 || n == 0) return PLA_SUCCESS;
  if (i0 < 0 || j0 < 0 || i0 + m > obj->length || j0 + n > obj->width)
    PLA_FAIL("API axpy outside the object");
  const int dt = obj->base->datatype, es = obj->base->esize;
  double a = dt == MPI_DOUBLE ? *(double *)alpha : dt == MPI_FLOAT ? *(float *)alpha : *(int *)alpha;
  if (inch != 1) PLA_FAIL("only unit-stride local vectors are supported");
  const size_t chunk_bytes = (size_t)256 << 20;
  int cols = (int)std::max<size_t>(1, chunk_bytes / ((size_t)m * es));
  cols = std::min(cols, n);
  char *stage = (char *)scratch(2, (size_t)m * cols * es);
  if (!stage) PLA_FAIL("cannot allocate the staging buffer");
  for (int j = 0; j < n; j += cols) {
    int c = std::min(cols, n - j);
    PLA_CUDA(cudaMemcpy2DAsync(stage, (size_t)m * es, (const char *)host + (size_t)j * ldh * es,
                               (size_t)ldh * es, (size_t)m * es, c, cudaMemcpyHostToDevice,
                               stream()));
    K(pla_k_axpby(dt, m, c, a, stage, m, 1.0, at(obj, i0, j0 + j), ld(obj), stream()));
  }
  return finish("api axpy to global");
}

// host(m x n) += alpha * obj(i0.., j0..)
static int axpy_from_global(int m, int n, void *alpha, PLA_Obj obj, int i0, int j0, void *host,
                            long ldh) {
  if (!valid(obj)) PLA_FAIL("invalid object");
  if (m == 0 || n == 0) return PLA_SUCCESS;
  if (i0 < 0 || j0 < 0 || i0 + m > obj->length || j0 + n > obj->width)
    PLA_FAIL("API axpy outside the object");
  const int dt = obj->base->datatype, es = obj->base->esize;
  std::vector<char> tmp((size_t)m * n * es);
  PLA_CUDA(cudaMemcpy2DAsync(tmp.data(), (size_t)m * es, at(obj, i0, j0), ld(obj) * es,
                             (size_t)m * es, n, cudaMemcpyDefault, stream()));
  int r = finish("api axpy from global");
  if (r) return r;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++) {
      size_t src = (size_t)i + (size_t)j * m, dst = (size_t)i + (size_t)j * ldh;
      if (dt == MPI_DOUBLE) ((double *)host)[dst] += *(double *)alpha * ((double *)tmp.data())[src];
      else if (dt == MPI_FLOAT) ((float *)host)[dst] += *(float *)alpha * ((float *)tmp.data())[src];
      else if (dt == MPI_INT) ((int *)host)[dst] += *(int *)alpha * ((int *)tmp.data())[src];
    }
  return PLA_SUCCESS;
}

int PLA_API_axpy_matrix_to_global(int m, int n, void *alpha, void *local, int ldim, PLA_Obj obj,
                                  int disp_row, int disp_col) {
  return axpy_to_global(m, n, alpha, local, ldim, 1, obj, disp_row, disp_col);
}
int PLA_API_axpy_global_to_matrix(int m, int n, void *alpha, PLA_Obj obj, int disp_row,
                                  int disp_col, void *local, int ldim) {
  return axpy_from_global(m, n, alpha, obj, disp_row, disp_col, local, ldim);
}
int PLA_API_axpy_vector_to_global(int size, void *alpha, void *local, int stride, PLA_Obj obj,
                                  int disp) {
  if (!valid(obj)) PLA_FAIL("invalid object");
  return axpy_to_global(size, 1, alpha, local, size, stride, obj, disp, 0);
}
int PLA_API_axpy_global_to_vector(int size, void *alpha, PLA_Obj obj, int disp, void *local,
                                  int stride) {
  if (stride != 1) PLA_FAIL("only unit-stride local vectors are supported");
  return axpy_from_global(size, 1, alpha, obj, disp, 0, local, size);
}

}  // extern "C"
