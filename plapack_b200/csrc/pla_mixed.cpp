// Mixed-precision direct solves with FP64 iterative refinement.
//
// Factorization: an fp32 working copy of A is factored with the same blocked
// right-looking loops as PLA_LU / PLA_Chol (fp32 panel, pivots, triangular
// solves); only the trailing update -- the O(n^3) part -- runs in bf16 or
// fp16 on the tensor cores with fp32 accumulation (k_tc_update.cu).  A itself
// is never modified.
//
// Refinement, both in FP64 with the fp32 factors as the preconditioner M:
//   LU-IR    : x <- x + M^{-1} (b - A x)
//   GMRES-IR : x <- x + d, d from restarted GMRES on M^{-1} A d = M^{-1} r with
//              classical Gram-Schmidt applied twice (CGS2)
// until  ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol  for every
// right-hand side.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include <cuda_bf16.h>

#include "pla_internal.h"
#include "pla_kernels.h"

using namespace pla;

namespace pla {
int lu_on_device(int dt, int m, int n, char *A, long lda, int *piv, int nb, int *zero_info_host,
                 bool left_swaps = true);
int tri_solve(int dt, char uplo, char trans, char diag, int n, int nrhs, const char *T, long ldt,
              char *X, long ldx);
int chol_on_device(int dt, int n, char *A, long lda, int nb, int *info_host);
int trsm_device(int dt, char side, char uplo, char trans, char diag, int nt, int other,
                double alpha, const char *T, long ldt, char *B, long ldb);
int panel_lu(int dt, int r, int b, char *P, long lda, int *piv, int *status, int *zero_info,
             int row_base, int max_ctas, int pivoting);
}

namespace {

// a call that already returns a library code (PLA_SUCCESS or PLA_ERROR with
// its message recorded)
#define PK(call)        \
  do {                  \
    int r_ = (call);    \
    if (r_) return r_;  \
  } while (0)

#define K(call)                                                    \
  do {                                                             \
    int r_ = (call);                                               \
    if (r_) return cuda_fail((cudaError_t)r_, __LINE__, __FILE__); \
  } while (0)

enum Slots { kSlotA32 = 4, kSlotL = 5, kSlotU = 6, kSlotPiv = 7, kSlotVec = 8, kSlotWork = 9,
             kSlotV = 10, kSlotSt = 11, kSlotA64 = 16, kSlotScales = 18, kSlotDiag = 19,
             kSlotLbig = 24, kSlotDinvSteps = 25, kSlotSclSteps = 26, kSlotTmp = 27,
             kSlotSplitL = 31, kSlotSplitU = 32, kSlotUr = 33, kSlotSplitUr = 34 };

long round_up(long v, long m) { return (v + m - 1) / m * m; }

struct Factor {
  int n = 0, ld = 0, prec = 0, kind = 0;  // kind 0 = LU, 1 = Cholesky
  int pivoting = PLA_B200_PIVOT_PARTIAL;   // of the fp32 LU panels
  float *a = nullptr;     // fp32 factors (BF16, FP16, FP32, BF16X6)
  double *a64 = nullptr;  // FP64 factors (FP64)
  double *dsc = nullptr;  // d = diag(A)^-1/2 when the factors are those of D A D
  int *piv = nullptr;
  int *perm = nullptr;    // LU: row i of P v is v[perm[i]] (the pivots composed)
  int *status = nullptr;  // [status, info, zero_info]
  // inverses of the 128 x 128 diagonal blocks of the two triangular factors,
  // and their link blocks (op(T)(i, p) inv(D_p), p the block solved before i)
  float *dinv1 = nullptr, *dinv2 = nullptr;
  float *link1 = nullptr, *link2 = nullptr;
  // BF16X6: the same inverses in FP64, the solves with the fp32 factors then
  // carried out in FP64 (fp32-level factors serve up to kappa near 2^24 times
  // the refinement's reach, and an fp32 solve would round that away)
  double *dinv1d = nullptr, *dinv2d = nullptr;
  long ldd = 0;
};

constexpr int kSlotDinv = 13;
constexpr int kSlotDinv64 = 12;
constexpr int kSlotLink = 28;
constexpr int kSlotPerm = 30;

// The row interchanges of an LU composed into one permutation, once per
// factorization: the refinement applies P to every preconditioned vector, and
// a gather is one parallel pass where the interchanges in sequence are n
// dependent swaps per column.
int prepare_perm(Factor &F) {
  F.perm = nullptr;
  if (F.kind != 0) return PLA_SUCCESS;
  const int n = F.n;
  std::vector<int> piv(n), perm(n);
  PLA_CUDA(d2h(piv.data(), F.piv, (size_t)n * sizeof(int)));
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int i = 0; i < n; i++) {
    const int p = i + piv[i];
    if (p < 0 || p >= n) PLA_FAIL("pivot outside the matrix");
    std::swap(perm[i], perm[p]);
  }
  int *d = (int *)scratch(kSlotPerm, (size_t)n * sizeof(int));
  if (!d) PLA_FAIL("cannot allocate the permutation");
  PLA_CUDA(cudaMemcpyAsync(d, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice,
                           stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));  // perm is a host temporary
  F.perm = d;
  return PLA_SUCCESS;
}

// the per-factor data of the single-launch triangular solves
int prepare_solves(Factor &F) {
  F.ldd = round_up(F.n, 128);
  if (F.prec == PLA_B200_PREC_BF16X6) {
    double *d = (double *)scratch(kSlotDinv64, (size_t)2 * F.ldd * 128 * sizeof(double));
    if (!d) PLA_FAIL("cannot allocate the inverse diagonal blocks");
    F.dinv1d = d;
    F.dinv2d = d + F.ldd * 128;
    const char u2 = F.kind == 0 ? 'U' : 'L', t2 = F.kind == 0 ? 'N' : 'T';
    K(pla_k_trsv_inv_blocks_f64('L', 'N', F.kind == 0 ? 'U' : 'N', F.n, F.a, F.ld, F.dinv1d,
                                F.ldd, stream()));
    K(pla_k_trsv_inv_blocks_f64(u2, t2, 'N', F.n, F.a, F.ld, F.dinv2d, F.ldd, stream()));
    return PLA_SUCCESS;
  }
  float *d = (float *)scratch(kSlotDinv, (size_t)2 * F.ldd * 128 * sizeof(float));
  float *g = (float *)scratch(kSlotLink, (size_t)2 * F.ldd * 128 * sizeof(float));
  if (!d || !g) PLA_FAIL("cannot allocate the inverse diagonal blocks");
  F.dinv1 = d;
  F.dinv2 = d + F.ldd * 128;
  F.link1 = g;
  F.link2 = g + F.ldd * 128;
  const char u1 = 'L', t1 = 'N', d1 = F.kind == 0 ? 'U' : 'N';
  const char u2 = F.kind == 0 ? 'U' : 'L', t2 = F.kind == 0 ? 'N' : 'T';
  K(pla_k_trsv_inv_blocks(MPI_FLOAT, u1, t1, d1, F.n, F.a, F.ld, F.dinv1, F.ldd, stream()));
  K(pla_k_trsv_inv_blocks(MPI_FLOAT, u2, t2, 'N', F.n, F.a, F.ld, F.dinv2, F.ldd, stream()));
  K(pla_k_trsv_link_blocks(u1, t1, F.n, F.a, F.ld, F.dinv1, F.ldd, F.link1, stream()));
  K(pla_k_trsv_link_blocks(u2, t2, F.n, F.a, F.ld, F.dinv2, F.ldd, F.link2, stream()));
  return PLA_SUCCESS;
}

struct EventTimer {
  cudaEvent_t a, b;
  EventTimer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, stream());
  }
  double stop() {
    cudaEventRecord(b, stream());
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~EventTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// U12 := inv(L11) A12 on the tensor cores.  The solve with the unit-lower
// diagonal block is on the factorization's critical path (the next panel
// waits for it); in fp32 on the SIMT pipe it took about 0.25 ms a step at
// n = 32768.  Here inv(L11) is formed once per panel (beside the trailing
// update, on the panel's stream) and both operands are split into bf16
// hi + lo, so that one K = 3b product sums hi*hi + hi*lo + lo*hi in fp32:
// about 16 significant bits, against the 11 of the fp16 operands the trailing
// update rounds U12 to anyway.  The product accumulates into A12 itself,
// which the split-pack clears behind its read.  With bf16 x 6 factors both
// operands are split three ways and the K = 6b product keeps fp32 accuracy.
//
// Segment codes of pla_k_pack_split_ex (two bits per K-wide segment, the part
// of x = p0 + p1 + p2 it holds): the A operand and the B operand of a product
// that sums p0 p1 + p1 p0 + p0 p0 (three segments) or p0 p2 + p1 p1 + p2 p0 +
// p0 p1 + p1 p0 + p0 p0 (six).  The small part products come first: the
// tensor core's fp32 accumulation truncates each addition relative to the
// running sum, so the terms 2^-8 and 2^-16 below the leading ones are summed
// before the leading ones make that sum large.
constexpr unsigned kSplitA3 = 0x4, kSplitB3 = 0x1;      // [0 1 0] x [1 0 0]
constexpr unsigned kSplitA6 = 0x124, kSplitB6 = 0x46;   // [0 1 2 0 1 0] x [2 1 0 1 0 0]

struct SplitU12 {
  int nseg = 3;                                   // 3: bf16 x 3, 6: bf16 x 6
  float *dinv[2] = {nullptr, nullptr};           // inv(L11), b x b column-major
  __nv_bfloat16 *lsplit[2] = {nullptr, nullptr};  // A-operand split of inv(L11), b x nseg b
  __nv_bfloat16 *usplit = nullptr;                // B-operand split of A12', rest x nseg b
};

// inv(L11) of a unit-lower b x b block: pla_k_trtri_unit_lower (independent
// block columns, one launch) when b is a multiple of 32 up to 256, else the
// blocked triangular solve on I.  The inverse sits on the panel chain of the
// factorization; the blocked solve took about 0.16 ms a step at b = 256.
int unit_lower_inverse(const float *L11, long ld, int b, float *D) {
  if (b >= 32 && b <= 256 && b % 32 == 0) {
    K(pla_k_trtri_unit_lower(b, L11, ld, D, b, nullptr, stream()));
    return PLA_SUCCESS;
  }
  K(pla_k_fill(MPI_FLOAT, b, b, D, b, 0.0, stream()));
  K(pla_k_fill(MPI_FLOAT, 1, b, D, b + 1, 1.0, stream()));
  K(trsm_device(MPI_FLOAT, 'L', 'L', 'N', 'U', b, b, 1.0, (const char *)L11, ld, (char *)D, b));
  return PLA_SUCCESS;
}

int split_alloc(SplitU12 &S, int n, int nb, int nseg) {
  S.nseg = nseg;
  const size_t d = (size_t)nb * nb * sizeof(float), l = (size_t)nb * nseg * nb * 2;
  char *p = (char *)scratch(kSlotSplitL, 2 * (d + l) + 1024);
  S.usplit = (__nv_bfloat16 *)scratch(kSlotSplitU, (size_t)n * nseg * nb * 2 + 1024);
  if (!p || !S.usplit) PLA_FAIL("cannot allocate the split operands of the U12 solve");
  for (int q = 0; q < 2; q++) {
    S.dinv[q] = (float *)(p + q * (d + l));
    S.lsplit[q] = (__nv_bfloat16 *)(p + q * (d + l) + d);
  }
  return PLA_SUCCESS;
}

// after the panel at (k, k) (on the current stream): inv(L11) and its split
int split_prepare(SplitU12 &S, int q, const float *L11, long ld, int b) {
  float *D = S.dinv[q];
  PK(unit_lower_inverse(L11, ld, b, D));
  // row i of inv(L11): element (i, k) at D[i + k b]
  K(pla_k_pack_split_ex(b, b, D, 1, b, S.lsplit[q], (long)S.nseg * b, S.nseg,
                        S.nseg == 6 ? kSplitA6 : kSplitA3, 0, stream()));
  return PLA_SUCCESS;
}

// U12 (b x cols at A12, ld) := inv(L11) A12 with the split of step parity q
int split_solve(SplitU12 &S, int q, float *C, long ld, long c_rows, long c_cols, int row0,
                int col0, int b, int cols, int *status) {
  float *A12 = C + row0 + (long)col0 * ld;
  // row j of A12' is column j of A12: element (j, k) at A12[k + j ld]
  const long kk = (long)S.nseg * b;
  K(pla_k_pack_split_ex(cols, b, A12, ld, 1, S.usplit, kk, S.nseg,
                        S.nseg == 6 ? kSplitB6 : kSplitB3, 1, stream()));
  K(pla_k_tc_update_ex(PLA_K_BF16, b, cols, (int)kk, 1.0f, S.lsplit[q], kk, b, S.usplit, kk,
                       cols, C, ld, c_rows, c_cols, row0, col0, 0, 0, status, stream()));
  return PLA_SUCCESS;
}

// fp32 factorization with low-precision trailing updates
int factor_mixed(Factor &F, const double *A, long lda, int nb) {
  const int n = F.n;
  const long ld = F.ld;
  auto at = [&](long i, long j) { return F.a + i + j * ld; };
  if (F.dsc)  // the unit-diagonal D A D of the fp8 Cholesky
    K(pla_k_sym_scale(n, A, lda, F.dsc, F.a, ld, stream()));
  else
    K(pla_k_convert(MPI_DOUBLE, A, lda, MPI_FLOAT, F.a, ld, n, n, stream()));
  const bool lowp = F.prec != PLA_B200_PREC_FP32;
  const bool f8 = F.prec == PLA_B200_PREC_FP8;
  // bf16 x 6: each operand of the update split three ways into bf16, six
  // K-wide segments per packed row, one K = 6b product of fp32 accuracy;
  // bf16 x 3: split two ways, three segments, K = 3b
  const bool x6 = F.prec == PLA_B200_PREC_BF16X6, x3 = F.prec == PLA_B200_PREC_BF16X3;
  const int nseg = x6 ? 6 : x3 ? 3 : 1;
  const int kprec =
      F.prec == PLA_B200_PREC_BF16 || x6 || x3 ? PLA_K_BF16 : PLA_K_FP16;
  const int kmult = f8 ? 128 : 64;  // K granularity of the tensor-core update
  const long ku = (long)nseg * nb;  // elements per packed operand row
  void *Lp = nullptr, *Up = nullptr;
  float *inv_l = nullptr, *inv_u = nullptr;
  if (lowp) {
    Lp = scratch(kSlotL, (size_t)n * ku * 2 + 256);
    Up = scratch(kSlotU, (size_t)n * ku * 2 + 256);
    if (!Lp || !Up) PLA_FAIL("cannot allocate the low-precision panels");
    if (f8) {  // one scale per 128 rows of L and of U'
      const size_t tiles = (size_t)(n + 127) / 128 + 1;
      inv_l = (float *)scratch(kSlotScales, 2 * tiles * sizeof(float) + 256);
      if (!inv_l) PLA_FAIL("cannot allocate the fp8 tile scales");
      inv_u = inv_l + tiles;
    }
  }
  int *st = F.status;
  PLA_Phase_times &ph = state().phases;
  // LU lookahead, as in the FP64 loop: panel k+1 on the lookahead stream
  // beside the rest of update k, which then keeps lookahead_ctas(MPI_FLOAT) SMs free
  const bool la = F.kind == 0 && n >= 4 * nb;
  cudaStream_t s0 = stream(), s1 = la ? lookahead_stream() : s0;
  cudaEvent_t ev_next = la ? lookahead_event(0) : nullptr, ev_panel = la ? lookahead_event(1) : nullptr;
  int sms = 0;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int side_ctas = std::max(1, sms - lookahead_ctas(MPI_FLOAT));
  const int esz = f8 ? 1 : 2;  // bytes per packed element
  // the LU's U12 solves on the tensor cores (low-precision factors only: an
  // fp32 factorization keeps the fp32 solve)
  const bool split = F.kind == 0 && lowp && nb % 64 == 0 && nb <= 256;
  SplitU12 S;
  if (split) PK(split_alloc(S, n, nb, x6 ? 6 : 3));  // bf16 x 3 below fp32-level factors
  int ready = -1;
  for (int k = 0; k < n; k += nb) {
    const int b = std::min(nb, n - k), rest = n - k - b, k2 = k + b;
    if (F.kind == 0) {
      if (ready == k) {
        PLA_CUDA(cudaStreamWaitEvent(s0, ev_panel, 0));
      } else {
        PhaseTimer t(&ph.panel_ms);
        K(panel_lu(MPI_FLOAT, n - k, b, (char *)at(k, k), ld, F.piv + k, &st[0], &st[2], k, 0,
                   F.pivoting));
      }
      {
        PhaseTimer t(&ph.swap_ms);
        K(pla_k_laswp(MPI_FLOAT, at(k, 0), ld, b, F.piv + k, 0, k, k + b, n, stream()));
      }
      if (rest <= 0) continue;
      PhaseTimer t(&ph.trsm_ms);
      if (split) {
        const int q = (k / nb) & 1;
        if (ready != k) PK(split_prepare(S, q, at(k, k), ld, b));
        PK(split_solve(S, q, F.a, ld, ld, n, k, k + b, b, rest, &st[0]));
      } else {
        K(trsm_device(MPI_FLOAT, 'L', 'L', 'N', 'U', b, rest, 1.0, (const char *)at(k, k), ld,
                      (char *)at(k, k + b), ld));
      }
    } else {
      {
        PhaseTimer t(&ph.panel_ms);
        K(pla_k_potrf_lower(MPI_FLOAT, b, at(k, k), ld, &st[0], &st[1], k, stream()));
      }
      if (rest <= 0) continue;
      PhaseTimer t(&ph.trsm_ms);
      K(pla_k_trsm_small(MPI_FLOAT, 'R', 'L', 'T', 'N', b, rest, 1.0, at(k, k), ld, at(k + b, k),
                         ld, &st[0], stream()));
    }
    if (lowp && b % kmult == 0) {
      // L (rest x b, column-major) and U' (U is b x rest: element (j, kk) at
      // kk + j ld) packed row-major, in fp8 with their tile scales or in
      // bf16 / fp16
      const char *Uop = (const char *)Lp;
      const float *su = inv_l;
      {
        PhaseTimer t(&ph.convert_ms);
        if (f8) {
          K(pla_k_pack_fp8(rest, b, at(k + b, k), 1, ld, Lp, nb, inv_l, stream()));
          if (F.kind == 0) {
            K(pla_k_pack_fp8(rest, b, at(k, k + b), ld, 1, Up, nb, inv_u, stream()));
            Uop = (const char *)Up;
            su = inv_u;
          }
        } else if (x6 || x3) {
          // A operand: L; B operand: U' (LU) or L again (Cholesky)
          const unsigned ca = x6 ? kSplitA6 : kSplitA3, cb = x6 ? kSplitB6 : kSplitB3;
          K(pla_k_pack_split_ex(rest, b, at(k + b, k), 1, ld, Lp, ku, nseg, ca, 0, stream()));
          if (F.kind == 0)
            K(pla_k_pack_split_ex(rest, b, at(k, k + b), ld, 1, Up, ku, nseg, cb, 0, stream()));
          else
            K(pla_k_pack_split_ex(rest, b, at(k + b, k), 1, ld, Up, ku, nseg, cb, 0, stream()));
          Uop = (const char *)Up;
        } else {
          K(pla_k_pack_rows(kprec, rest, b, at(k + b, k), ld, Lp, nb, stream()));
          if (F.kind == 0) {
            K(pla_k_convert(MPI_FLOAT, at(k, k + b), ld, kprec, Up, nb, b, rest, stream()));
            Uop = (const char *)Up;
          }
        }
      }
      // C(:, c0 : c0 + nc) of the trailing matrix, on at most `cap` CTAs
      auto upd = [&](int c0, int nc, int cap) -> int {
        const long off = (long)(c0 - k2);  // rows of U' skipped (multiple of 128)
        PhaseTimer t(&ph.update_ms);
        int r = f8 ? pla_k_tc_update_fp8_ex(rest, nc, b, -1.0f, Lp, nb, n, inv_l,
                                            Uop + off * nb * esz, nb, n - off, su + off / 128,
                                            F.a, ld, ld, n, k2, c0, F.kind == 1, cap, &st[0],
                                            stream())
                   : pla_k_tc_update_ex(kprec, rest, nc, nseg * b, -1.0f, Lp, ku, n,
                                        Uop + off * ku * esz, ku, n - off, F.a, ld, ld, n, k2, c0,
                                        F.kind == 1, cap, &st[0], stream());
        if (t.on) ph.update_launches++;
        return r;
      };
      const int b2 = std::min(nb, rest);
      // The next panel's columns must end on a 128-column tile boundary: the
      // update walks whole 128 x 128 tiles, so a partial last tile would also
      // fold its product into the columns the second launch updates (and
      // fp8's U' scales are per 128 rows).  nb = 192 with the split that
      // allows measured slower anyway (factorization 167 against 154 ms).
      if (la && b2 % 128 == 0 && rest > b2) {
        K(upd(k2, b2, 0));  // the next panel's columns first
        PLA_CUDA(cudaEventRecord(ev_next, s0));
        PLA_CUDA(cudaStreamWaitEvent(s1, ev_next, 0));
        {
          OnStream on(s1);
          PhaseTimer t(&ph.panel_ms);
          K(panel_lu(MPI_FLOAT, n - k2, b2, (char *)at(k2, k2), ld, F.piv + k2, &st[0], &st[2],
                     k2, lookahead_ctas(MPI_FLOAT), F.pivoting));
          // the next step's inv(L11) and its split, beside the update
          if (split && b2 == nb && n - k2 - b2 > 0)
            PK(split_prepare(S, (k2 / nb) & 1, at(k2, k2), ld, b2));
        }
        PLA_CUDA(cudaEventRecord(ev_panel, s1));
        ready = k2;
        K(upd(k2 + b2, rest - b2, side_ctas));
      } else {
        K(upd(k2, rest, 0));
      }
    } else if (F.kind == 0) {
      K(pla_k_gemm(MPI_FLOAT, PLA_NO_TRANSPOSE, PLA_NO_TRANSPOSE, rest, rest, b, -1.0, at(k + b, k),
                   ld, at(k, k + b), ld, 1.0, at(k + b, k + b), ld, 0, &st[0], stream()));
    } else {
      K(pla_k_gemm(MPI_FLOAT, PLA_NO_TRANSPOSE, PLA_TRANSPOSE, rest, rest, b, -1.0, at(k + b, k),
                   ld, at(k + b, k), ld, 1.0, at(k + b, k + b), ld, 'L', &st[0], stream()));
    }
  }
  if (F.kind == 0) count_interchanges(n, F.piv);
  return PLA_SUCCESS;
}

// FP64 factors: the plain blocked PLA_LU / PLA_Chol loops on a copy of A.
// Returns PLA_SUCCESS; the LU's first exact zero pivot or the failing
// Cholesky column goes to *info.
int factor_fp64(Factor &F, const double *A, long lda, int *info) {
  const int n = F.n;
  F.a64 = (double *)scratch(kSlotA64, (size_t)F.ld * n * sizeof(double));
  if (!F.a64) PLA_FAIL("cannot allocate the FP64 factors");
  K(pla_k_copy(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, n, A, lda, F.a64, F.ld, stream()));
  // the block size the FP64 loops run fastest at (512-wide DMMA updates at
  // large n); the low-precision nb does not carry over
  const int nb = n >= 8192 ? 512 : 128;
  if (F.kind == 0) return lu_on_device(MPI_DOUBLE, n, n, (char *)F.a64, F.ld, F.piv, nb, info);
  return chol_on_device(MPI_DOUBLE, n, (char *)F.a64, F.ld, nb, info);
}

// out (fp64, n x nrhs, ldo) := M^{-1} v (fp64, ldv) with the factors
int precond(const Factor &F, const double *v, long ldv, double *out, long ldo, int nrhs,
            float *t32) {
  const int n = F.n;
  if (F.dinv1d) {  // bf16 x 6 factors: P, then both solves in FP64 through `out`
    if (F.kind == 0 && F.perm)
      K(pla_k_gather_rows(MPI_DOUBLE, n, nrhs, F.perm, v, ldv, out, ldo, stream()));
    else
      K(pla_k_copy(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, nrhs, v, ldv, out, ldo, stream()));
    if (F.kind == 0 && !F.perm) K(pla_k_laswp_rows(MPI_DOUBLE, out, ldo, nrhs, n, F.piv, stream()));
    const char u2 = F.kind == 0 ? 'U' : 'L', t2 = F.kind == 0 ? 'N' : 'T';
    K(pla_k_trsv_ticket_multi_f64('L', 'N', n, nrhs, F.a, F.ld, F.dinv1d, F.ldd, out, ldo, out,
                                  ldo, F.status, stream()));
    K(pla_k_trsv_ticket_multi_f64(u2, t2, n, nrhs, F.a, F.ld, F.dinv2d, F.ldd, out, ldo, out, ldo,
                                  F.status, stream()));
    return PLA_SUCCESS;
  }
  if (F.prec == PLA_B200_PREC_FP64) {
    if (F.kind == 0 && F.perm)
      K(pla_k_gather_rows(MPI_DOUBLE, n, nrhs, F.perm, v, ldv, out, ldo, stream()));
    else
      K(pla_k_copy(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, nrhs, v, ldv, out, ldo, stream()));
    if (F.kind == 0) {
      if (!F.perm) K(pla_k_laswp_rows(MPI_DOUBLE, out, ldo, nrhs, n, F.piv, stream()));
      const char *f = (const char *)F.a64;
      K(tri_solve(MPI_DOUBLE, 'L', 'N', 'U', n, nrhs, f, F.ld, (char *)out, ldo));
      K(tri_solve(MPI_DOUBLE, 'U', 'N', 'N', n, nrhs, f, F.ld, (char *)out, ldo));
    } else {
      const char *f = (const char *)F.a64;
      K(tri_solve(MPI_DOUBLE, 'L', 'N', 'N', n, nrhs, f, F.ld, (char *)out, ldo));
      K(tri_solve(MPI_DOUBLE, 'L', 'T', 'N', n, nrhs, f, F.ld, (char *)out, ldo));
    }
    return PLA_SUCCESS;
  }
  if (F.dsc) {  // M^{-1} = D (L L')^{-1} D: scale in FP64 through `out`
    K(pla_k_copy(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, nrhs, v, ldv, out, ldo, stream()));
    K(pla_k_diag_mul(n, nrhs, F.dsc, out, ldo, stream()));
    K(pla_k_convert(MPI_DOUBLE, out, ldo, MPI_FLOAT, t32, n, n, nrhs, stream()));
  } else if (F.kind == 0 && F.perm) {
    K(pla_k_gather_rows(MPI_FLOAT, n, nrhs, F.perm, v, ldv, t32, n, stream()));
  } else {
    K(pla_k_convert(MPI_DOUBLE, v, ldv, MPI_FLOAT, t32, n, n, nrhs, stream()));
  }
  if (F.kind == 0 && !F.perm) K(pla_k_laswp_rows(MPI_FLOAT, t32, n, nrhs, n, F.piv, stream()));
  const char u1 = 'L', t1 = 'N', d1 = F.kind == 0 ? 'U' : 'N';
  const char u2 = F.kind == 0 ? 'U' : 'L', t2 = F.kind == 0 ? 'N' : 'T', d2 = 'N';
  if (nrhs <= 2 && F.dinv1) {
    // the single-column solves with link blocks: the successor of a block
    // starts from its y, before the inverse-block product
    for (int j = 0; j < nrhs; j++) {
      float *col = t32 + (long)j * n;
      K(pla_k_trsv_ticket_link(u1, t1, n, F.a, F.ld, F.dinv1, F.ldd, F.link1, col, col,
                               F.status, stream()));
      K(pla_k_trsv_ticket_link(u2, t2, n, F.a, F.ld, F.dinv2, F.ldd, F.link2, col, col,
                               F.status, stream()));
    }
  } else if (nrhs <= 16 && F.dinv1) {
    // all the columns in one launch per triangle: the factors are read once
    K(pla_k_trsv_ticket_multi(u1, t1, n, nrhs, F.a, F.ld, F.dinv1, F.ldd, t32, n, t32, n,
                              F.status, stream()));
    K(pla_k_trsv_ticket_multi(u2, t2, n, nrhs, F.a, F.ld, F.dinv2, F.ldd, t32, n, t32, n,
                              F.status, stream()));
  } else {
    K(pla_k_trsv_blocked(MPI_FLOAT, u1, t1, d1, n, nrhs, F.a, F.ld, t32, n, stream()));
    K(pla_k_trsv_blocked(MPI_FLOAT, u2, t2, d2, n, nrhs, F.a, F.ld, t32, n, stream()));
  }
  K(pla_k_convert(MPI_FLOAT, t32, n, MPI_DOUBLE, out, ldo, n, nrhs, stream()));
  if (F.dsc) K(pla_k_diag_mul(n, nrhs, F.dsc, out, ldo, stream()));
  return PLA_SUCCESS;
}

double host_max(const double *dev, int count) {
  std::vector<double> h(count);
  cudaMemcpyAsync(h.data(), dev, count * sizeof(double), cudaMemcpyDeviceToHost, stream());
  cudaStreamSynchronize(stream());
  double m = 0;
  for (double v : h) m = std::max(m, v);
  return m;
}

struct Norms {
  double a_inf = 0;
  std::vector<double> b_inf;
};

// per-column backward error of x given r = b - A x
int backward_errors(int n, int nrhs, const double *R, long ldr, const double *X, long ldx,
                    const Norms &nm, double *tmp, std::vector<double> &eta) {
  K(pla_k_col_abs_max(MPI_DOUBLE, n, nrhs, R, ldr, tmp, stream()));
  K(pla_k_col_abs_max(MPI_DOUBLE, n, nrhs, X, ldx, tmp + nrhs, stream()));
  std::vector<double> h(2 * nrhs);
  PLA_CUDA(cudaMemcpyAsync(h.data(), tmp, 2 * nrhs * sizeof(double), cudaMemcpyDeviceToHost,
                           stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));
  eta.resize(nrhs);
  for (int j = 0; j < nrhs; j++) {
    double den = nm.a_inf * h[nrhs + j] + nm.b_inf[j];
    eta[j] = den > 0 ? h[j] / den : h[j];
  }
  return PLA_SUCCESS;
}

double dot(int n, const double *x, const double *y, double *tmp) {
  pla_k_gemv(MPI_DOUBLE, PLA_TRANSPOSE, n, 1, 1.0, x, n, y, 0.0, tmp, stream());
  double h = 0;
  cudaMemcpyAsync(&h, tmp, sizeof h, cudaMemcpyDeviceToHost, stream());
  cudaStreamSynchronize(stream());
  return h;
}

// GMRES iterations after which a cycle that has not reduced its residual
// tenfold is cut short (see gmres)
constexpr int kSlowCycle = 16;

// one restarted-GMRES correction: d ~= A^{-1} r (d, r fp64 columns)
int gmres(const Factor &F, const double *A, long lda, const double *r, double *d, int restart,
          double tau, double *V, double *w, double *tmp, float *t32, double *work, int *iters) {
  const int n = F.n, m = restart;
  // z = M^{-1} r, beta = ||z||
  int rc = precond(F, r, n, V, n, 1, t32);
  if (rc) return rc;
  double beta = std::sqrt(dot(n, V, V, tmp));
  K(pla_k_fill(MPI_DOUBLE, n, 1, d, n, 0.0, stream()));
  if (!(beta > 0)) return PLA_SUCCESS;
  K(pla_k_scal(MPI_DOUBLE, n, 1, 1.0 / beta, V, n, stream()));
  std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0);
  g[0] = beta;
  int j = 0;
  for (; j < m; j++) {
    double *vj = V + (long)j * n, *vn = V + (long)(j + 1) * n;
    // w = M^{-1} (A v_j)
    K(pla_k_residual(n, n, 1, A, lda, vj, n, nullptr, n, w, n, 0, work, stream()));
    rc = precond(F, w, n, vn, n, 1, t32);
    if (rc) return rc;
    // CGS2 against v_0 .. v_j
    std::vector<double> h(j + 1, 0.0);
    for (int pass = 0; pass < 2; pass++) {
      K(pla_k_gemv(MPI_DOUBLE, PLA_TRANSPOSE, n, j + 1, 1.0, V, n, vn, 0.0, tmp, stream()));
      std::vector<double> hp(j + 1);
      PLA_CUDA(cudaMemcpyAsync(hp.data(), tmp, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                               stream()));
      PLA_CUDA(cudaStreamSynchronize(stream()));
      // tmp still holds the coefficients on the device
      K(pla_k_gemv(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, j + 1, -1.0, V, n, tmp, 1.0, vn, stream()));
      for (int i = 0; i <= j; i++) h[i] += hp[i];
    }
    double hn = std::sqrt(dot(n, vn, vn, tmp));
    for (int i = 0; i <= j; i++) H[i + (size_t)j * (m + 1)] = h[i];
    H[j + 1 + (size_t)j * (m + 1)] = hn;
    if (hn > 0) K(pla_k_scal(MPI_DOUBLE, n, 1, 1.0 / hn, vn, n, stream()));
    // Givens rotations on column j
    for (int i = 0; i < j; i++) {
      double a = H[i + (size_t)j * (m + 1)], b = H[i + 1 + (size_t)j * (m + 1)];
      H[i + (size_t)j * (m + 1)] = cs[i] * a + sn[i] * b;
      H[i + 1 + (size_t)j * (m + 1)] = -sn[i] * a + cs[i] * b;
    }
    double a = H[j + (size_t)j * (m + 1)], b = H[j + 1 + (size_t)j * (m + 1)];
    double rr = std::hypot(a, b);
    cs[j] = rr > 0 ? a / rr : 1.0;
    sn[j] = rr > 0 ? b / rr : 0.0;
    H[j + (size_t)j * (m + 1)] = rr;
    H[j + 1 + (size_t)j * (m + 1)] = 0.0;
    g[j + 1] = -sn[j] * g[j];
    g[j] = cs[j] * g[j];
    if (std::fabs(g[j + 1]) <= tau * beta || hn == 0) {
      j++;
      break;
    }
    // kSlowCycle iterations without a tenfold reduction of the preconditioned
    // residual: these factors are too far from A for the cycle to converge
    // (kappa times their precision is large).  Stop here, keep the partial
    // correction, and let the caller's stagnation test escalate instead of
    // running out the restart.
    if (j + 1 >= kSlowCycle && std::fabs(g[j + 1]) > 0.1 * beta) {
      j++;
      break;
    }
  }
  // y = H(0:j,0:j) \ g(0:j); d = V y
  std::vector<double> y(j, 0.0);
  for (int i = j - 1; i >= 0; i--) {
    double s = g[i];
    for (int c = i + 1; c < j; c++) s -= H[i + (size_t)c * (m + 1)] * y[c];
    y[i] = s / H[i + (size_t)i * (m + 1)];
  }
  if (j > 0) {
    PLA_CUDA(cudaMemcpyAsync(tmp, y.data(), j * sizeof(double), cudaMemcpyHostToDevice, stream()));
    K(pla_k_gemv(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, j, 1.0, V, n, tmp, 0.0, d, stream()));
  }
  *iters += j;
  return PLA_SUCCESS;
}

// Restarted-GMRES corrections for nrhs columns at once, D(:, s) ~= A^{-1}
// R(:, s).  The columns run in lockstep: one residual launch forms A v_j for
// all of them and one preconditioner application solves with the factors for
// all of them, so A (8.6 GB at n = 32768) and the factors are read once per
// iteration rather than once per column.  The orthogonalisation (CGS2, its
// coefficients read back in one copy per pass), the Givens rotations and the
// convergence test are per column; a column that has converged takes no
// further part.  V holds column s's basis at V + s (restart + 1) n, W is n x
// nrhs, tmp at least (restart + 1) nrhs doubles.
int gmres_block(const Factor &F, const double *A, long lda, const double *R, double *D, int nrhs,
                int restart, double tau, double *V, double *W, double *tmp, float *t32,
                double *work, int *iters) {
  const int n = F.n, m = restart;
  const long ldv = (long)n * (m + 1);
  auto vcol = [&](int s, int j) { return V + (long)s * ldv + (long)j * n; };
  const unsigned all = nrhs >= 32 ? ~0u : (1u << nrhs) - 1u;
  int rc = precond(F, R, n, V, ldv, nrhs, t32);  // z_s = M^{-1} r_s into v_0 of every column
  if (rc) return rc;
  K(pla_k_fill(MPI_DOUBLE, n, nrhs, D, n, 0.0, stream()));
  std::vector<double> beta(nrhs), sc(nrhs);
  K(pla_k_basis_dots(n, nrhs, V, ldv, 0, 1, 0, all, tmp, 1, stream()));
  PLA_CUDA(cudaMemcpyAsync(beta.data(), tmp, nrhs * sizeof(double), cudaMemcpyDeviceToHost,
                           stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));
  const size_t hm = (size_t)(m + 1) * m;
  std::vector<double> H(hm * nrhs, 0.0), cs((size_t)m * nrhs), sn((size_t)m * nrhs),
      g((size_t)(m + 1) * nrhs, 0.0);
  std::vector<int> jend(nrhs, 0);
  unsigned active = 0;
  for (int s = 0; s < nrhs; s++) {
    beta[s] = std::sqrt(beta[s]);
    g[(size_t)s * (m + 1)] = beta[s];
    if (beta[s] > 0) active |= 1u << s;
    sc[s] = beta[s] > 0 ? 1.0 / beta[s] : 1.0;
  }
  K(pla_k_basis_scale(n, nrhs, V, ldv, 0, sc.data(), active, stream()));
  std::vector<double> hp((size_t)(m + 1) * nrhs), hsum((size_t)(m + 1) * nrhs), hn(nrhs);
  for (int j = 0; j < m && active; j++) {
    // W = A [v_j of every column]; v_{j+1} = M^{-1} W
    K(pla_k_residual(n, n, nrhs, A, lda, vcol(0, j), ldv, nullptr, n, W, n, 0, work, stream()));
    rc = precond(F, W, n, vcol(0, j + 1), ldv, nrhs, t32);
    if (rc) return rc;
    // CGS2 against v_0 .. v_j: one launch for the coefficients of every
    // active column, one read-back, one launch for the updates
    std::fill(hsum.begin(), hsum.end(), 0.0);
    for (int pass = 0; pass < 2; pass++) {
      K(pla_k_basis_dots(n, nrhs, V, ldv, 0, j + 1, j + 1, active, tmp, m + 1, stream()));
      PLA_CUDA(cudaMemcpyAsync(hp.data(), tmp, hp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                               stream()));
      PLA_CUDA(cudaStreamSynchronize(stream()));
      // tmp still holds the coefficients on the device
      K(pla_k_basis_update(n, nrhs, V, ldv, j + 1, j + 1, tmp, m + 1, active, stream()));
      for (int s = 0; s < nrhs; s++)
        if ((active >> s) & 1u)
          for (int i = 0; i <= j; i++) hsum[(size_t)s * (m + 1) + i] += hp[(size_t)s * (m + 1) + i];
    }
    K(pla_k_basis_dots(n, nrhs, V, ldv, j + 1, 1, j + 1, active, tmp, 1, stream()));
    PLA_CUDA(cudaMemcpyAsync(hn.data(), tmp, nrhs * sizeof(double), cudaMemcpyDeviceToHost,
                             stream()));
    PLA_CUDA(cudaStreamSynchronize(stream()));
    unsigned next = active;
    for (int s = 0; s < nrhs; s++) {
      sc[s] = 1.0;
      if (!((active >> s) & 1u)) continue;
      const double h1 = std::sqrt(hn[s]);
      double *Hs = H.data() + hm * s, *gs = g.data() + (size_t)s * (m + 1);
      double *css = cs.data() + (size_t)s * m, *sns = sn.data() + (size_t)s * m;
      for (int i = 0; i <= j; i++) Hs[i + (size_t)j * (m + 1)] = hsum[(size_t)s * (m + 1) + i];
      Hs[j + 1 + (size_t)j * (m + 1)] = h1;
      if (h1 > 0) sc[s] = 1.0 / h1;
      for (int i = 0; i < j; i++) {
        const double a = Hs[i + (size_t)j * (m + 1)], b = Hs[i + 1 + (size_t)j * (m + 1)];
        Hs[i + (size_t)j * (m + 1)] = css[i] * a + sns[i] * b;
        Hs[i + 1 + (size_t)j * (m + 1)] = -sns[i] * a + css[i] * b;
      }
      const double a = Hs[j + (size_t)j * (m + 1)], b = Hs[j + 1 + (size_t)j * (m + 1)];
      const double rr = std::hypot(a, b);
      css[j] = rr > 0 ? a / rr : 1.0;
      sns[j] = rr > 0 ? b / rr : 0.0;
      Hs[j + (size_t)j * (m + 1)] = rr;
      Hs[j + 1 + (size_t)j * (m + 1)] = 0.0;
      gs[j + 1] = -sns[j] * gs[j];
      gs[j] = css[j] * gs[j];
      jend[s] = j + 1;
      if (std::fabs(gs[j + 1]) <= tau * beta[s] || h1 == 0) next &= ~(1u << s);
      // a column as slow as the single-column cycle's cut-off stops too
      if (j + 1 >= kSlowCycle && std::fabs(gs[j + 1]) > 0.1 * beta[s]) next &= ~(1u << s);
    }
    K(pla_k_basis_scale(n, nrhs, V, ldv, j + 1, sc.data(), active, stream()));
    active = next;
  }
  // y_s = H_s \ g_s; D(:, s) = V_s y_s
  std::vector<double> y((size_t)(m + 1) * nrhs, 0.0);
  for (int s = 0; s < nrhs; s++) {
    const int js = jend[s];
    if (js == 0) continue;
    const double *Hs = H.data() + hm * s, *gs = g.data() + (size_t)s * (m + 1);
    double *ys = y.data() + (size_t)s * (m + 1);
    for (int i = js - 1; i >= 0; i--) {
      double t = gs[i];
      for (int c = i + 1; c < js; c++) t -= Hs[i + (size_t)c * (m + 1)] * ys[c];
      ys[i] = t / Hs[i + (size_t)i * (m + 1)];
    }
    *iters += js;
  }
  PLA_CUDA(cudaMemcpyAsync(tmp, y.data(), y.size() * sizeof(double), cudaMemcpyHostToDevice,
                           stream()));
  for (int s = 0; s < nrhs; s++)
    if (jend[s] > 0)
      K(pla_k_gemv(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, jend[s], 1.0, vcol(s, 0), n,
                   tmp + (size_t)s * (m + 1), 0.0, D + (long)s * n, stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));  // y must stay alive until copied
  return PLA_SUCCESS;
}

// LU of a matrix that is still arriving from host memory (bf16 / fp16 / fp8
// trailing updates).  The copy stream brings A in groups of columns into the
// FP64 device object and converts each group into the fp32 working copy; an
// event marks each group.  Every step keeps its packed L panel, the inverse
// of its unit lower diagonal block and its pivots, so a group that becomes
// available after some steps replays exactly what those steps would have done
// to it: the row interchanges, U rows as inverse(L_kk) times the block, and
// the tensor-core update.  Every element therefore receives the same
// operations in the same order whatever the arrival times, and the factors
// do not depend on them.  The host polls the arrival events as it queues the
// steps, and stays at most two steps ahead of the device.
int factor_mixed_streamed(Factor &F, const double *Ah, long ldh, double *Ad, long lda, int nb) {
  const int n = F.n;
  const long ld = F.ld;
  auto at = [&](long i, long j) { return F.a + i + j * ld; };
  const bool f8 = F.prec == PLA_B200_PREC_FP8;
  const int kprec = F.prec == PLA_B200_PREC_BF16 ? PLA_K_BF16 : PLA_K_FP16;
  const int esz = f8 ? 1 : 2;
  const int nsteps = (n + nb - 1) / nb;
  // Groups of about n / 8 columns; the first is split into 4 nb, 4 nb and
  // the rest, so the first steps start after a few milliseconds of copying
  // rather than after an eighth of the whole copy.  Boundaries are multiples
  // of nb.
  const int gcols = std::max(nb, (n / 8 + nb - 1) / nb * nb);
  std::vector<int> gb{0};
  if (gcols >= 16 * nb) {
    gb.push_back(4 * nb);
    gb.push_back(8 * nb);
  }
  for (int c = gcols; c < n; c += gcols) gb.push_back(c);
  gb.push_back(n);
  const int ngroups = (int)gb.size() - 1;
  const int tiles = (n + 127) / 128 + 1;
  // per-step storage
  std::vector<size_t> loff(nsteps);
  size_t lbytes = 0;
  for (int k = 0; k < nsteps; k++) {
    const long rest = std::max(0, n - (k + 1) * nb);
    loff[k] = lbytes;
    lbytes += (size_t)round_up(rest * nb * esz, 256);
  }
  char *Lbig = (char *)scratch(kSlotLbig, lbytes + 256);
  float *dinv = (float *)scratch(kSlotDinvSteps, (size_t)nsteps * nb * nb * sizeof(float));
  float *scl = (float *)scratch(kSlotSclSteps, ((size_t)nsteps + 2) * tiles * sizeof(float));
  void *Ub = scratch(kSlotU, (size_t)n * nb * 2 + 256);
  void *Ub_r = scratch(kSlotUr, (size_t)n * nb * 2 + 256);  // the replay stream's U'
  __nv_bfloat16 *usplit_r =
      (__nv_bfloat16 *)scratch(kSlotSplitUr, (size_t)n * 3 * nb * 2 + 256);
  // per step: the split of inv(L11) for the tensor-core U12 solves (replays
  // of late column groups use old steps' splits)
  __nv_bfloat16 *lsplit =
      (__nv_bfloat16 *)scratch(kSlotSplitL, (size_t)nsteps * nb * 3 * nb * 2 + 256);
  __nv_bfloat16 *usplit = (__nv_bfloat16 *)scratch(kSlotSplitU, (size_t)n * 3 * nb * 2 + 256);
  if (!Lbig || !dinv || !scl || !Ub || !lsplit || !usplit || !Ub_r || !usplit_r)
    PLA_FAIL("cannot allocate the streamed-solve buffers");
  float *inv_u = scl + (size_t)nsteps * tiles;  // the U' scales of the launch in flight
  float *inv_u_r = inv_u + tiles;               // ... of the replay stream's
  int *st = F.status;
  PLA_Phase_times &ph = state().phases;
  cudaStream_t s0 = stream(), s1 = lookahead_stream(), sc = copy_stream();
  int sms = 0;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int side_ctas = std::max(1, sms - lookahead_ctas(MPI_FLOAT));
  std::vector<cudaEvent_t> arr(ngroups), thr(4), rep(ngroups + 1);
  for (auto &e : arr) PLA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : thr) PLA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto &e : rep) PLA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  struct Events {  // destroyed on every return path
    std::vector<cudaEvent_t> *a, *b, *c;
    ~Events() {
      for (auto e : *a) cudaEventDestroy(e);
      for (auto e : *b) cudaEventDestroy(e);
      for (auto e : *c) cudaEventDestroy(e);
    }
  } guard{&arr, &thr, &rep};
  cudaEvent_t ev_post0 = rep[ngroups];  // step 0's panel and its packed L, on s0
  cudaStream_t sr = replay_stream();
  cudaEvent_t ev_next = lookahead_event(0), ev_panel = lookahead_event(1);

  // 1. the copies and conversions, group by group, on the copy stream
  for (int g = 0; g < ngroups; g++) {
    const long c0 = gb[g], nc = gb[g + 1] - gb[g];
    PLA_CUDA(cudaMemcpy2DAsync(Ad + c0 * lda, lda * sizeof(double), Ah + c0 * ldh,
                               ldh * sizeof(double), (size_t)n * sizeof(double), nc,
                               cudaMemcpyHostToDevice, sc));
    K(pla_k_convert(MPI_DOUBLE, Ad + c0 * lda, lda, MPI_FLOAT, at(0, c0), ld, n, (int)nc, sc));
    PLA_CUDA(cudaEventRecord(arr[g], sc));
  }
  int known = 0;  // groups [0, known) take part (the library stream waited for them)
  auto poll = [&](int need) -> int {
    while (known < ngroups) {
      bool take = known < need;
      if (!take) {
        cudaError_t q = cudaEventQuery(arr[known]);
        cudaGetLastError();  // a "not ready" answer is not an error
        take = q == cudaSuccess;
      }
      if (!take) break;
      PLA_CUDA(cudaStreamWaitEvent(s0, arr[known], 0));
      known++;
    }
    return 0;
  };
  // after panel s (on the current stream): the inverse of its unit lower
  // diagonal block and its packed L
  auto post_panel = [&](int s) -> int {
    const int k0 = s * nb, b = std::min(nb, n - k0), rest = n - k0 - b;
    float *D = dinv + (size_t)s * nb * nb;
    PK(unit_lower_inverse(at(k0, k0), ld, b, D));
    if (rest <= 0) return 0;
    K(pla_k_pack_split(b, b, D, 1, b, lsplit + (size_t)s * nb * 3 * nb, 3L * b, 0b100, 0,
                       stream()));
    PhaseTimer t(&ph.convert_ms);
    if (f8)
      K(pla_k_pack_fp8(rest, b, at(k0 + b, k0), 1, ld, Lbig + loff[s], nb,
                       scl + (size_t)s * tiles, stream()));
    else
      K(pla_k_pack_rows(kprec, rest, b, at(k0 + b, k0), ld, Lbig + loff[s], nb, stream()));
    return 0;
  };
  // step s on columns [c0, c1): interchanges, U rows, packed U' (into ub,
  // with the split operand us and the fp8 scales iu of the stream it runs on)
  auto prep = [&](int s, int c0, int c1, void *ub, __nv_bfloat16 *us, float *iu) -> int {
    const int k0 = s * nb, b = std::min(nb, n - k0), nc = c1 - c0;
    if (nc <= 0) return 0;
    {
      PhaseTimer t(&ph.swap_ms);
      K(pla_k_laswp(MPI_FLOAT, at(k0, 0), ld, b, F.piv + k0, 0, 0, c0, c1, stream()));
    }
    {
      // U rows := inv(L11) block on the tensor cores, bf16 hi/lo split (see
      // split_solve): the block is split and cleared, then accumulated into
      PhaseTimer t(&ph.trsm_ms);
      K(pla_k_pack_split(nc, b, at(k0, c0), ld, 1, us, 3L * b, 0b010, 1, stream()));
      K(pla_k_tc_update_ex(PLA_K_BF16, b, nc, 3 * b, 1.0f, lsplit + (size_t)s * nb * 3 * nb,
                           3L * b, b, us, 3L * b, nc, F.a, ld, ld, n, k0, c0, 0, 0, &st[0],
                           stream()));
    }
    if (n - k0 - b <= 0) return 0;
    PhaseTimer t(&ph.convert_ms);
    if (f8) K(pla_k_pack_fp8(nc, b, at(k0, c0), ld, 1, ub, nb, iu, stream()));
    else K(pla_k_convert(MPI_FLOAT, at(k0, c0), ld, kprec, ub, nb, b, nc, stream()));
    return 0;
  };
  // step s's update of columns [c0, c1), whose U' (in ub, fp8 scales iu) was
  // packed from column p0
  auto upd = [&](int s, int c0, int c1, int p0, int cap, void *ub, float *iu) -> int {
    const int k0 = s * nb, b = std::min(nb, n - k0), rest = n - k0 - b, nc = c1 - c0;
    if (nc <= 0 || rest <= 0) return 0;
    const long off = c0 - p0;  // columns of U' skipped (a multiple of 128)
    PhaseTimer t(&ph.update_ms);
    K(f8 ? pla_k_tc_update_fp8_ex(rest, nc, b, -1.0f, Lbig + loff[s], nb, rest,
                                  scl + (size_t)s * tiles, (char *)ub + off * nb * esz, nb, nc,
                                  iu + off / 128, F.a, ld, ld, n, k0 + b, c0, 0, cap, &st[0],
                                  stream())
         : pla_k_tc_update_ex(kprec, rest, nc, b, -1.0f, Lbig + loff[s], nb, rest,
                              (char *)ub + off * nb * esz, nb, nc, F.a, ld, ld, n, k0 + b, c0, 0,
                              cap, &st[0], stream()));
    if (t.on) ph.update_launches++;
    return 0;
  };
  // Group g's catch-up on the replay stream: the steps [applied[g], upto) it
  // missed, once it has arrived and those steps' panels are packed.  It runs
  // beside the panel chain and the main update (they work on other
  // columns), from the group's arrival on, so that when the chain reaches the
  // group only the steps since the last call remain.  Every column receives
  // the operations of the in-HBM factorization, in its order.
  std::vector<int> applied(ngroups, 0);  // steps already applied to each group
  std::vector<char> started(ngroups, 0);
  auto replay = [&](int g, int upto) -> int {
    OnStream on(sr);
    if (!started[g]) {
      PLA_CUDA(cudaStreamWaitEvent(sr, arr[g], 0));
      PLA_CUDA(cudaStreamWaitEvent(sr, ev_post0, 0));
      started[g] = 1;
    }
    if (applied[g] < upto) {
      // the panels of steps < upto (upto - 1 <= the chain's step) and their L
      if (upto > 1) PLA_CUDA(cudaStreamWaitEvent(sr, ev_panel, 0));
      for (int s2 = applied[g]; s2 < upto; s2++) {
        const int c0 = std::max(gb[g], (s2 + 1) * nb);
        PK(prep(s2, c0, gb[g + 1], Ub_r, usplit_r, inv_u_r));
        PK(upd(s2, c0, gb[g + 1], c0, side_ctas, Ub_r, inv_u_r));
      }
      applied[g] = upto;
    }
    PLA_CUDA(cudaEventRecord(rep[g], sr));
    return 0;
  };

  // 2. the steps
  PK(poll(1));
  {
    PhaseTimer t(&ph.panel_ms);
    K(panel_lu(MPI_FLOAT, n, std::min(nb, n), (char *)at(0, 0), ld, F.piv, &st[0], &st[2], 0, 0,
               F.pivoting));
  }
  PK(post_panel(0));
  PLA_CUDA(cudaEventRecord(ev_post0, s0));
  int arrived = known;  // groups [known, arrived) have arrived and catch up on sr
  for (int k = 0; k < nsteps; k++) {
    const int k0 = k * nb, b = std::min(nb, n - k0), rest = n - k0 - b;
    if (k > 0) PLA_CUDA(cudaStreamWaitEvent(s0, ev_panel, 0));
    if (k >= 2) PLA_CUDA(cudaEventSynchronize(thr[(k - 2) % 4]));
    // groups through the one holding block k+1 must take part now
    const int upto = (int)std::min<long>(n, (long)(k + 2) * nb);
    int need = 0;
    while (gb[need] < upto) need++;
    // the groups that have arrived catch up (through step k - 1) on sr; the
    // needed ones then join the main update, which takes them from step k on
    while (arrived < ngroups) {
      cudaError_t q = cudaEventQuery(arr[arrived]);
      cudaGetLastError();  // a "not ready" answer is not an error
      if (q != cudaSuccess) break;
      arrived++;
    }
    for (int g = known; g < std::max(arrived, need); g++) PK(replay(g, k));
    for (; known < need; known++) PLA_CUDA(cudaStreamWaitEvent(s0, rep[known], 0));
    arrived = std::max(arrived, known);
    const int kc = gb[known];  // columns that take part
    if (rest > 0) {
      PK(prep(k, k0 + b, kc, Ub, usplit, inv_u));
      const int b2 = std::min(nb, rest);
      if (k + 1 < nsteps) {
        PK(upd(k, k0 + b, k0 + b + b2, k0 + b, 0, Ub, inv_u));  // the next panel's columns first
        PLA_CUDA(cudaEventRecord(ev_next, s0));
        PLA_CUDA(cudaStreamWaitEvent(s1, ev_next, 0));
        {
          OnStream on(s1);
          {
            PhaseTimer t(&ph.panel_ms);
            K(panel_lu(MPI_FLOAT, n - k0 - b, b2, (char *)at(k0 + b, k0 + b), ld, F.piv + k0 + b,
                       &st[0], &st[2], k0 + b, lookahead_ctas(MPI_FLOAT), F.pivoting));
          }
          PK(post_panel(k + 1));
        }
        PLA_CUDA(cudaEventRecord(ev_panel, s1));
        PK(upd(k, k0 + b + b2, kc, k0 + b, side_ctas, Ub, inv_u));
      }
    }
    for (int g = 0; g < known; g++) applied[g] = k + 1;
    PLA_CUDA(cudaEventRecord(thr[k % 4], s0));
  }
  // every group has joined (the last step needs them all); the refinement
  // reads all of A
  for (; known < ngroups; known++) {
    PK(replay(known, nsteps));
    PLA_CUDA(cudaStreamWaitEvent(s0, rep[known], 0));
  }
  // 3. the interchanges of every step on the columns to its left
  for (int k = 1; k < nsteps; k++) {
    const int k0 = k * nb, b = std::min(nb, n - k0);
    PhaseTimer t(&ph.swap_ms);
    K(pla_k_laswp(MPI_FLOAT, at(k0, 0), ld, b, F.piv + k0, 0, k0, 0, 0, stream()));
  }
  count_interchanges(n, F.piv);
  PLA_CUDA(cudaStreamSynchronize(s0));
  return PLA_SUCCESS;
}

// the next precision up when the refinement stagnates (0: none left).  BF16
// and FP16 go to bf16 x 6 factors (fp32 accuracy from the tensor cores at
// about six times the bf16 tensor work), then to FP64.  Plain fp32 factors
// (the SIMT update) are slower than either: at n = 32768 the fp32 LU took
// 1.1 s against 0.8 s for the FP64 LU on the DMMA pipe; they stay available
// on request and go to FP64.
int escalated(int prec) {
  switch (prec) {
    case PLA_B200_PREC_FP8: return PLA_B200_PREC_BF16;
    case PLA_B200_PREC_BF16:
    case PLA_B200_PREC_FP16:
    case PLA_B200_PREC_BF16X3: return PLA_B200_PREC_BF16X6;
    case PLA_B200_PREC_BF16X6:
    case PLA_B200_PREC_FP32: return PLA_B200_PREC_FP64;
    default: return 0;
  }
}

// unit roundoff of the trailing update's operands at each precision
double unit_roundoff(int prec) {
  switch (prec) {
    case PLA_B200_PREC_FP8: return std::ldexp(1.0, -4);
    case PLA_B200_PREC_BF16: return std::ldexp(1.0, -8);
    case PLA_B200_PREC_FP16: return std::ldexp(1.0, -11);
    case PLA_B200_PREC_BF16X3: return std::ldexp(1.0, -16);
    case PLA_B200_PREC_BF16X6:
    case PLA_B200_PREC_FP32: return std::ldexp(1.0, -24);
    default: return std::ldexp(1.0, -53);
  }
}

// Early escalation: factors whose diagonal range (max / min |u_ii|, a lower
// bound on their condition number; squared for a Cholesky factor) times the
// precision's unit roundoff exceeds this have been refactored one precision
// up at once.  Measured on the n = 32768 C3 family: fp16 at kappa = 1e6 is
// about 500 (17 GMRES iterations), at kappa = 1e10 about 5e6 (no convergence
// within a restart cycle).
constexpr double kEarlyEscalate = 1e4;

// Ah: when not null, A's values are in host memory (column-major, ldh) and are
// copied into the device object A during the call
int solve_mixed(int kind, PLA_Obj A, PLA_Obj B, const PLA_Mixed_params *pin,
                PLA_Mixed_report *rep, const double *Ah = nullptr, long ldh = 0) {
  if (!valid(A) || !valid(B)) PLA_FAIL("invalid object");
  if (!is_double(A) || !is_double(B)) PLA_FAIL("the mixed-precision solvers take FP64 objects");
  if (A->length != A->width || B->length != A->length) PLA_FAIL("nonconformal objects");
  PLA_Mixed_params p;
  PLA_Mixed_params_default(&p);
  if (pin) p = *pin;
  if (p.max_iterations <= 0) p.max_iterations = 50;
  if (p.gmres_restart <= 0) p.gmres_restart = 30;
  if (p.precision < PLA_B200_PREC_BF16 || p.precision > PLA_B200_PREC_BF16X3)
    PLA_FAIL("unknown precision");
  if (p.panel_pivoting != PLA_B200_PIVOT_PARTIAL && p.panel_pivoting != PLA_B200_PIVOT_TOURNAMENT)
    PLA_FAIL("unknown panel pivoting");
  const int n = A->length, nrhs = B->width;
  if (n == 0 || nrhs == 0) {
    if (rep) *rep = PLA_Mixed_report{1, 0, 0, 0, 0.0, 0.0, 0.0, p.precision, 0};
    return PLA_SUCCESS;
  }
  if (nrhs > 16) PLA_FAIL("at most 16 right-hand sides per mixed-precision solve");
  int nb0 = p.nb;
  if (nb0 <= 0) PLA_Environ_nb_alg(PLA_OP_PAN_PAN, A->templ, &nb0);
  const double tol = p.tol > 0 ? p.tol : n * std::ldexp(1.0, -53);
  const double *Ad = (const double *)at(A, 0, 0);
  const long lda = ld(A);
  double *Bd = (double *)at(B, 0, 0);
  const long ldb = ld(B);

  const long ldf = round_up(n, 32);
  int *piv = (int *)scratch(kSlotPiv, (size_t)n * sizeof(int) + 64);
  int *status = (int *)scratch(kSlotSt, 64);
  const size_t vec = (size_t)n * 16;
  double *X = (double *)scratch(kSlotVec, (5 * vec + 64) * sizeof(double));
  if (!piv || !status || !X) PLA_FAIL("cannot allocate the mixed-precision workspace");
  double *R = X + vec, *Dv = R + vec, *Bsave = Dv + vec, *tmp = Bsave + vec;
  float *t32b = (float *)scratch(kSlotWork + 3, vec * sizeof(float) + 256);
  double *work = (double *)scratch(kSlotWork, std::max(pla_k_residual_work(n, n, nrhs),
                                                       (size_t)n * sizeof(double)) + 256);
  double *V = nullptr, *w = nullptr;
  if (p.refinement == PLA_B200_IR_GMRES) {
    // one basis per right-hand side (they run in lockstep), then W
    V = (double *)scratch(kSlotV, (size_t)n * ((size_t)(p.gmres_restart + 1) * nrhs + nrhs) *
                                      sizeof(double));
    w = V + (size_t)n * (p.gmres_restart + 1) * nrhs;
  }
  if (!t32b || !work || (p.refinement == PLA_B200_IR_GMRES && !V))
    PLA_FAIL("cannot allocate the refinement workspace");

  if (Ah && ldh < n) PLA_FAIL("leading dimension of the host matrix below n");
  const bool lowp0 = p.precision == PLA_B200_PREC_BF16 || p.precision == PLA_B200_PREC_FP16 ||
                     p.precision == PLA_B200_PREC_FP8;
  // the first factorization overlaps the copy of A when it is an LU with
  // tensor-core updates; otherwise A is copied first
  bool stream_first = Ah && kind == 0 && lowp0 && n >= 4096;
  if (Ah && !stream_first)
    PLA_CUDA(cudaMemcpy2DAsync((void *)Ad, lda * sizeof(double), Ah, ldh * sizeof(double),
                               (size_t)n * sizeof(double), n, cudaMemcpyHostToDevice, stream()));
  // a copy of b (B receives x at the end); the norms of A and b once A is there
  K(pla_k_copy(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, nrhs, Bd, ldb, Bsave, n, stream()));
  Norms nm;
  bool have_norms = false;
  auto norms = [&]() -> int {
    if (have_norms) return 0;
    K(pla_k_residual(n, n, 1, Ad, lda, nullptr, n, nullptr, n, tmp, n, 1, work, stream()));
    nm.a_inf = host_max(tmp, n);
    K(pla_k_col_abs_max(MPI_DOUBLE, n, nrhs, Bsave, n, tmp, stream()));
    nm.b_inf.resize(nrhs);
    PLA_CUDA(d2h(nm.b_inf.data(), tmp, nrhs * sizeof(double)));
    have_norms = true;
    return 0;
  };

  PLA_Mixed_report r{};
  r.backward_error = std::numeric_limits<double>::infinity();
  bool have_x = false;
  double refine_ms = 0;
  for (int prec = p.precision; prec;) {
    Factor F;
    F.n = n;
    F.ld = (int)ldf;
    F.prec = prec;
    F.kind = kind;
    F.pivoting = p.panel_pivoting;
    F.piv = piv;
    F.status = status;
    PLA_CUDA(cudaMemsetAsync(status, 0, 64, stream()));
    // ---- factorization ----
    int info = 0;
    {
      EventTimer t;
      if (prec == PLA_B200_PREC_FP64) {
        int rc = factor_fp64(F, Ad, lda, &info);
        if (rc) return rc;
      } else {
        F.a = (float *)scratch(kSlotA32, (size_t)ldf * n * sizeof(float));
        if (!F.a) PLA_FAIL("cannot allocate the fp32 working copy");
        int nb = nb0;
        if (prec == PLA_B200_PREC_FP8) {
          nb = std::min(std::max(128, nb / 128 * 128), kind == 0 ? 256 : 128);
        } else if (prec != PLA_B200_PREC_FP32) {
          nb = std::max(64, nb / 64 * 64);
          nb = std::min(nb, kind == 0 ? 256 : 128);
        } else if (kind == 1) {
          nb = std::min(nb, 128);
        }
        if (prec == PLA_B200_PREC_FP8 && kind == 1) {
          F.dsc = (double *)scratch(kSlotDiag, (size_t)n * sizeof(double) + 256);
          if (!F.dsc) PLA_FAIL("cannot allocate the diagonal scaling");
        }
        int rc = stream_first ? factor_mixed_streamed(F, Ah, ldh, (double *)Ad, lda, nb)
                              : factor_mixed(F, Ad, lda, nb);
        stream_first = false;
        if (rc) return rc;
        int hst[3];
        PLA_CUDA(d2h(hst, status, sizeof hst));  // after the factorization's kernels
        if (hst[0] == PLA_K_TIMEOUT) PLA_FAIL("factorization: a bounded wait timed out");
        info = kind == 0 ? hst[2] : (hst[0] == PLA_K_NOT_SPD ? hst[1] : 0);
      }
      r.factor_ms += t.stop();
    }
    r.factorizations++;
    r.precision_used = prec;
    r.info = info;
    if (kind == 1 && info) {  // not positive definite at this precision
      if (!p.escalate || !escalated(prec)) break;
      prec = escalated(prec);
      continue;
    }
    if (prec != PLA_B200_PREC_FP64 && p.escalate && escalated(prec)) {
      // the factors' diagonal range says whether to refine them at all; one
      // level up at a time, since low-precision factors of an
      // ill-conditioned matrix can show a range far beyond its condition
      float dr[2];
      K(pla_k_diag_range(n, F.a, F.ld, (float *)tmp, stream()));
      PLA_CUDA(d2h(dr, tmp, sizeof dr));
      double ratio = (double)dr[0] / (double)dr[1];
      if (kind == 1) ratio *= ratio;
      if (!(ratio * unit_roundoff(prec) <= kEarlyEscalate)) {
        prec = escalated(prec);
        continue;
      }
    }

    // ---- refinement ----
    K(norms());
    EventTimer t;
    if (prec != PLA_B200_PREC_FP64) {
      int rc0 = prepare_solves(F);
      if (rc0) return rc0;
    }
    PK(prepare_perm(F));
    if (!have_x) {  // start from x = M^{-1} b
      int rc = precond(F, Bsave, n, X, n, nrhs, t32b);
      if (rc) return rc;
      have_x = true;
    }
    std::vector<double> eta;
    double prev = std::numeric_limits<double>::infinity();
    // A GMRES-IR step that fails to halve the backward error has run a full
    // restart cycle without converging: at that rate the remaining steps cost
    // more than refactoring one precision up, so one such step escalates.
    // Classic LU-IR steps are cheap (one residual and one solve) and get two.
    const int slow_limit = p.refinement == PLA_B200_IR_GMRES ? 1 : 2;
    int slow = 0, it = 0;
    bool stalled = false;
    for (;; it++) {
      K(pla_k_residual(n, n, nrhs, Ad, lda, X, n, Bsave, n, R, n, 0, work, stream()));
      int rc = backward_errors(n, nrhs, R, n, X, n, nm, tmp, eta);
      if (rc) return rc;
      double worst = 0;
      bool finite = true;
      for (double e : eta) {
        if (!(e == e) || std::isinf(e)) finite = false;
        worst = std::max(worst, e);
      }
      r.backward_error = finite ? worst : std::numeric_limits<double>::quiet_NaN();
      if (finite && worst <= tol) break;
      if (!finite) {  // a zero or tiny pivot at this precision: restart the iterate
        have_x = false;
        stalled = true;
        break;
      }
      slow = worst > 0.5 * prev ? slow + 1 : 0;
      prev = worst;
      if (it >= p.max_iterations || (p.escalate && slow >= slow_limit)) {
        stalled = true;
        break;
      }
      if (p.refinement == PLA_B200_IR_GMRES && nrhs == 1) {
        rc = gmres(F, Ad, lda, R, Dv, p.gmres_restart, 1e-8, V, w, tmp, t32b, work,
                   &r.inner_iterations);
        if (rc) return rc;
      } else if (p.refinement == PLA_B200_IR_GMRES) {
        rc = gmres_block(F, Ad, lda, R, Dv, nrhs, p.gmres_restart, 1e-8, V, w, tmp, t32b, work,
                         &r.inner_iterations);
        if (rc) return rc;
      } else {
        rc = precond(F, R, n, Dv, n, nrhs, t32b);
        if (rc) return rc;
      }
      K(pla_k_axpby(MPI_DOUBLE, n, nrhs, 1.0, Dv, n, 1.0, X, n, stream()));
    }
    r.iterations += it;
    refine_ms += t.stop();
    if (!stalled || !p.escalate || !escalated(prec)) break;
    prec = escalated(prec);
  }
  r.converged = r.backward_error <= tol;
  r.refine_ms = refine_ms;
  if (have_x) K(pla_k_copy(MPI_DOUBLE, PLA_NO_TRANSPOSE, n, nrhs, X, n, Bd, ldb, stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));
  if (rep) *rep = r;
  if (kind == 1 && r.info && !r.converged) return r.info;  // not positive definite
  return PLA_SUCCESS;
}

}  // namespace

extern "C" {

void PLA_Mixed_params_default(PLA_Mixed_params *p) {
  if (!p) return;
  p->precision = PLA_B200_PREC_FP16;
  p->refinement = PLA_B200_IR_GMRES;
  p->max_iterations = 50;
  p->gmres_restart = 30;
  p->nb = 0;
  p->escalate = 1;
  p->tol = 0.0;
  p->panel_pivoting = PLA_B200_PIVOT_TOURNAMENT;
}

int PLA_General_solve_mixed(PLA_Obj A, PLA_Obj B, const PLA_Mixed_params *params,
                            PLA_Mixed_report *report) {
  return solve_mixed(0, A, B, params, report);
}

int PLA_Pos_def_solve_mixed(PLA_Obj A, PLA_Obj B, const PLA_Mixed_params *params,
                            PLA_Mixed_report *report) {
  return solve_mixed(1, A, B, params, report);
}

int PLA_General_solve_mixed_host(PLA_Obj A, const void *A_host, int ldh, PLA_Obj B,
                                 const PLA_Mixed_params *params, PLA_Mixed_report *report) {
  if (!A_host) PLA_FAIL("null host matrix");
  return solve_mixed(0, A, B, params, report, (const double *)A_host, ldh);
}

}  // extern "C"
