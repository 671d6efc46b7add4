// GEMM for the trailing updates: C := alpha op(A) op(B) + beta C, optionally
// restricted to the lower or upper triangle of C (the SYRK-shaped update of
// SOLVERS/Cholesky/PLA_Chol.c:207-210).
//
// FP64: tensor-core DMMA (mma.sync m16n8k8 .f64; tcgen05 has no f64 kind).
//   CTA tile 64 x 64, k-step 16, 4 warps as 2 (M) x 2 (N) with a 32 x 32
//   warp tile; three cp.async stages; three CTAs per SM, so that the start of
//   one tile (the reads of C and the first stage) and the stores at its end
//   overlap the other CTAs' main loops.  The stages are stored permuted
//   (rows g and g+8, k and k+4 side by side) so that each thread's fragment
//   pairs are single 16-byte loads, and padded so those loads are
//   bank-conflict free: A stage [16][64+4], B stage [64][16+8].
//   Each thread copies a fixed pattern of 8 + 8 elements per stage: its
//   shared-memory addresses are one register plus compile-time offsets and
//   its global addresses one pointer plus multiples of a fixed stride, and the
//   bounds are tested only in tiles that cross an edge of the matrices.  With
//   the index arithmetic of a per-element copy loop the kernel issued 2.4x the
//   instructions for the same MMAs and reached 29.7 TF/s at M = N = 16384,
//   K = 512; with this copy, 33.5 TF/s (cuBLAS DGEMM on the same GPU: 34.6).
// FP32: SIMT FFMA with 128 x 64 tiles, 8 warps and three stages.
#include <cstdint>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

// tile shapes: BM x BN per CTA, BK per stage, THREADS threads
template <int BM_, int BN_, int STAGES_, int THREADS_>
struct Tile {
  static constexpr int BM = BM_, BN = BN_, BK = 16, STAGES = STAGES_, THREADS = THREADS_;
  static constexpr int LDA_S = BM + 4;  // elements per k-row of the A stage
  static constexpr int LDB_S = BK + 8;  // per n-row of the B stage (16-byte loads conflict free)
  static constexpr int STAGE = BK * LDA_S + BN * LDB_S;
};
using DT = Tile<64, 64, 3, 128>;   // FP64 tensor-core kernel
using ST = Tile<128, 64, 3, 256>;  // FP32 SIMT kernel

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int src_size = valid ? 4 : 0;  // 0 = fill the destination with zeros
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem),
               "r"(src_size));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Positions inside an FP64 stage: rows g and g + 8 of every 16-row group are
// stored next to each other, and so are k and k + 4 of every 8-wide k group,
// so that each pair of f64 fragment elements the m16n8k8 MMA wants from one
// thread is one 16-byte load.
__device__ __forceinline__ int pos_m(int row) {
  return (row & ~15) | ((row & 7) << 1) | ((row >> 3) & 1);
}
__device__ __forceinline__ int pos_k(int kk) {
  return (kk & ~7) | ((kk & 3) << 1) | ((kk >> 2) & 1);
}

// The FP32 kernel's copy of one k-slab of op(A) (BM x BK) and op(B) (BK x BN)
// into shared memory, one 4-byte cp.async per element.
template <typename TL, bool TA, bool TB>
__device__ __forceinline__ void load_stage(float *As, float *Bs, const float *A, long lda,
                                           const float *B, long ldb, int m, int n, int k, int m0,
                                           int n0, int k0, int tid) {
  constexpr int BM = TL::BM, BN = TL::BN, BK = TL::BK, THREADS = TL::THREADS;
  constexpr int LDA_S = TL::LDA_S, LDB_S = TL::LDB_S;
  // A: element (row, kk) of op(A) -> As[kk * LDA_S + row]
#pragma unroll
  for (int it = 0; it < (BM * BK) / THREADS; it++) {
    int e = tid + it * THREADS;
    int row, kk;
    if (!TA) { row = e % BM; kk = e / BM; }   // A is m x k, rows contiguous
    else     { kk = e % BK; row = e / BK; }   // A is k x m, k contiguous
    int gi = m0 + row, gk = k0 + kk;
    bool ok = gi < m && gk < k;
    const float *src = ok ? (TA ? A + gk + (long)gi * lda : A + gi + (long)gk * lda) : A;
    cp_async4(As + kk * LDA_S + row, src, ok);
  }
  // B: element (kk, col) of op(B) -> Bs[col * LDB_S + kk]
#pragma unroll
  for (int it = 0; it < (BK * BN) / THREADS; it++) {
    int e = tid + it * THREADS;
    int col, kk;
    if (!TB) { kk = e % BK; col = e / BK; }   // B is k x n, k contiguous
    else     { col = e % BN; kk = e / BN; }   // B is n x k, n contiguous
    int gj = n0 + col, gk = k0 + kk;
    bool ok = gj < n && gk < k;
    const float *src = ok ? (TB ? B + gj + (long)gk * ldb : B + gk + (long)gj * ldb) : B;
    cp_async4(Bs + col * LDB_S + kk, src, ok);
  }
}

// The FP64 kernel's copy of one stage.  Thread tid copies 8 elements of
// op(A) and 8 of op(B).  Along the contiguous dimension of each operand the
// thread's index is fixed; along the other it is a base plus it * step, it =
// 0..7, so that the shared-memory position of element it is the thread's base
// plus a compile-time offset (positions permuted as pos_m / pos_k):
//   A, not transposed (m x k, rows contiguous): row tid % 64, k tid / 64 + 2 it
//   A, transposed (k x m): k tid % 16, row tid / 16 + 8 it
//   B, not transposed (k x n, k contiguous): k tid % 16, col tid / 16 + 8 it
//   B, transposed (n x k): col tid % 64, k tid / 64 + 2 it
struct DLoad {
  unsigned s;        // shared address of element 0 in stage 0
  const double *g;   // global address of element 0 for k0 = 0
  long gstep;        // elements between consecutive elements it
  long kstep;        // elements per unit of k0
  unsigned inmask;   // bit it: row (A) or column (B) of element it inside the matrix
  int k_first, k_inc;  // k index of element it = k0 + k_first + it * k_inc
};
template <bool TA>
__device__ __forceinline__ constexpr int a_soff(int it) {
  return TA ? 16 * (it >> 1) + (it & 1) : 2 * it * DT::LDA_S;
}
template <bool TB>
__device__ __forceinline__ constexpr int b_soff(int it) {
  return TB ? 8 * (it >> 2) + 4 * (it & 1) + ((it >> 1) & 1) : 8 * it * DT::LDB_S;
}
template <bool TA>
__device__ __forceinline__ DLoad a_load(unsigned sbase, const double *A, long lda, int m, int m0,
                                       int tid) {
  DLoad d;
  if (!TA) {
    const int r = tid & 63, kk = tid >> 6;
    d.s = sbase + 8u * (kk * DT::LDA_S + pos_m(r));
    d.g = A + (m0 + r) + (long)kk * lda;
    d.gstep = 2 * lda;
    d.kstep = lda;
    d.inmask = m0 + r < m ? 0xffu : 0u;
    d.k_first = kk;
    d.k_inc = 2;
  } else {
    const int kk = tid & 15, r0 = tid >> 4;
    d.s = sbase + 8u * (kk * DT::LDA_S + 2 * r0);
    d.g = A + kk + (long)(m0 + r0) * lda;
    d.gstep = 8 * lda;
    d.kstep = 1;
    d.inmask = 0;
#pragma unroll
    for (int it = 0; it < 8; it++) d.inmask |= (m0 + r0 + 8 * it < m ? 1u : 0u) << it;
    d.k_first = kk;
    d.k_inc = 0;
  }
  return d;
}
template <bool TB>
__device__ __forceinline__ DLoad b_load(unsigned sbase, const double *B, long ldb, int n, int n0,
                                       int tid) {
  DLoad d;
  if (!TB) {
    const int kk = tid & 15, c0 = tid >> 4;
    d.s = sbase + 8u * (c0 * DT::LDB_S + pos_k(kk));
    d.g = B + kk + (long)(n0 + c0) * ldb;
    d.gstep = 8 * ldb;
    d.kstep = 1;
    d.inmask = 0;
#pragma unroll
    for (int it = 0; it < 8; it++) d.inmask |= (n0 + c0 + 8 * it < n ? 1u : 0u) << it;
    d.k_first = kk;
    d.k_inc = 0;
  } else {
    const int c = tid & 63, kk0 = tid >> 6;
    d.s = sbase + 8u * (c * DT::LDB_S + 2 * kk0);
    d.g = B + (n0 + c) + (long)kk0 * ldb;
    d.gstep = 2 * ldb;
    d.kstep = ldb;
    d.inmask = n0 + c < n ? 0xffu : 0u;
    d.k_first = kk0;
    d.k_inc = 2;
  }
  return d;
}
// copy the 8 elements of one operand for the stage at k0 into slot offset so
template <bool T, bool ISB, bool EDGE>
__device__ __forceinline__ void d_copy(const DLoad &d, unsigned so, int k0, int k) {
  const double *p = d.g + (long)k0 * d.kstep;
#pragma unroll
  for (int it = 0; it < 8; it++) {
    const unsigned sa = d.s + so + 8u * (ISB ? b_soff<T>(it) : a_soff<T>(it));
    if (!EDGE) {
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(p + it * d.gstep));
    } else {
      const bool ok = ((d.inmask >> it) & 1u) && k0 + d.k_first + it * d.k_inc < k;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa),
                   "l"(ok ? p + it * d.gstep : d.g), "r"(ok ? 8 : 0));
    }
  }
}

__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4],
                                            const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ bool keep(int uplo, int i, int j) {
  return uplo == 0 || (uplo == 'L' ? i >= j : i <= j);
}

// FP64 tensor-core GEMM.  FOLD (alpha = +-1, every trailing update): the
// accumulators start as alpha * beta * C and the result is alpha * acc, so the
// reads of C are issued before the main loop, under the pipeline fill, and the
// epilogue only stores.  Without FOLD the epilogue reads C.
template <bool TA, bool TB, bool FOLD>
__global__ void __launch_bounds__(DT::THREADS, 3)
dgemm_k(int m, int n, int k, double alpha, const double *__restrict__ A, long lda,
        const double *__restrict__ B, long ldb, double beta, double *C, long ldc, int uplo,
        const int *status) {
  constexpr int BM = DT::BM, BN = DT::BN, BK = DT::BK, STAGES = DT::STAGES;
  constexpr int LDA_S = DT::LDA_S, LDB_S = DT::LDB_S;
  extern __shared__ __align__(16) double smem[];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (uplo == 'L' && m0 + BM - 1 < n0) return;  // tile strictly above the diagonal
  if (uplo == 'U' && n0 + BN - 1 < m0) return;  // tile strictly below the diagonal
  if (status && *status != PLA_K_OK) return;
  double *As = smem;                          // [STAGES][BK][LDA_S]
  double *Bs = smem + STAGES * BK * LDA_S;    // [STAGES][BN][LDB_S]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;  // 2 x 2 warps
  const int g = lane >> 2, t = lane & 3;

  const double ab = FOLD && beta != 0.0 ? alpha * beta : 0.0;
  double acc[2][4][4];
  {
    const int ri = m0 + wm + g, cj = n0 + wn + 2 * t;
    const double *cb = C + ri + (long)cj * ldc;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int i = 0; i < 2; i++) {
          const int di = i * 16 + (q >> 1) * 8, dj = j * 8 + (q & 1);
          acc[i][j][q] = ab != 0.0 && ri + di < m && cj + dj < n ? ab * cb[di + (long)dj * ldc]
                                                                  : 0.0;
        }
  }

  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem);
  const DLoad la = a_load<TA>(sbase, A, lda, m, m0, tid);
  const DLoad lb = b_load<TB>(sbase + 8u * STAGES * BK * LDA_S, B, ldb, n, n0, tid);
  const bool interior = m0 + BM <= m && n0 + BN <= n;
  auto load = [&](int slot, int k0) {
    const unsigned soa = 8u * slot * BK * LDA_S, sob = 8u * slot * BN * LDB_S;
    if (interior && k0 + BK <= k) {
      d_copy<TA, false, false>(la, soa, k0, k);
      d_copy<TB, true, false>(lb, sob, k0, k);
    } else {
      d_copy<TA, false, true>(la, soa, k0, k);
      d_copy<TB, true, true>(lb, sob, k0, k);
    }
  };

  const int nk = (k + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < nk) load(s, s * BK);
    cp_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    {  // prefetch stage kt + STAGES - 1 into the slot freed by stage kt - 1
      int ks = kt + STAGES - 1;
      if (ks < nk) load(ks % STAGES, ks * BK);
      cp_commit();
    }
    const double *as = As + (kt % STAGES) * BK * LDA_S;
    const double *bs = Bs + (kt % STAGES) * BN * LDB_S;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double af[2][4], bf[4][2];
      // (a0, a1) = rows g, g+8 at k = kk+t; (a2, a3) the same rows at kk+t+4;
      // (b0, b1) = k = kk+t, kk+t+4 of column g: one 16-byte load each
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int r = wm + i * 16 + 2 * g;
        const double2 lo = *reinterpret_cast<const double2 *>(&as[(kk + t) * LDA_S + r]);
        const double2 hi = *reinterpret_cast<const double2 *>(&as[(kk + t + 4) * LDA_S + r]);
        af[i][0] = lo.x;
        af[i][1] = lo.y;
        af[i][2] = hi.x;
        af[i][3] = hi.y;
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = wn + j * 8 + g;
        const double2 bb = *reinterpret_cast<const double2 *>(&bs[c * LDB_S + kk + 2 * t]);
        bf[j][0] = bb.x;
        bf[j][1] = bb.y;
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dmma_16x8x8(acc[i][j], af[i], bf[j]);
    }
  }
  cp_wait<0>();

  // epilogue: C = alpha * acc + beta * C, fragment (g, 2t), (g, 2t+1), (g+8, ...)
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int gi = m0 + wm + i * 16 + g + (q >> 1) * 8;
        const int gj = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (gi < m && gj < n && keep(uplo, gi, gj)) {
          double *cp = C + gi + (long)gj * ldc;
          double v = alpha * acc[i][j][q];
          *cp = FOLD || beta == 0.0 ? v : fma(beta, *cp, v);
        }
      }
}

// FP32 SIMT GEMM with the same staging; each thread computes an 8 x 4 block
template <bool TA, bool TB, bool FOLD>
__global__ void __launch_bounds__(ST::THREADS, 2)
sgemm_k(int m, int n, int k, float alpha, const float *__restrict__ A, long lda,
        const float *__restrict__ B, long ldb, float beta, float *C, long ldc, int uplo,
        const int *status) {
  constexpr int BM = ST::BM, BN = ST::BN, BK = ST::BK, STAGES = ST::STAGES;
  constexpr int LDA_S = ST::LDA_S, LDB_S = ST::LDB_S;
  extern __shared__ __align__(16) float fsm[];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (uplo == 'L' && m0 + BM - 1 < n0) return;
  if (uplo == 'U' && n0 + BN - 1 < m0) return;
  if (status && *status != PLA_K_OK) return;
  float *As = fsm;
  float *Bs = fsm + STAGES * BK * LDA_S;
  const int tid = threadIdx.x;
  const int tm = (tid & 15) * 8, tn = (tid >> 4) * 4;  // 16 x 16 threads
  float acc[8][4];
  const float ab = FOLD && beta != 0.f ? alpha * beta : 0.f;  // as in dgemm_k
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int gi = m0 + tm + i, gj = n0 + tn + j;
      acc[i][j] = ab != 0.f && gi < m && gj < n ? ab * C[gi + (long)gj * ldc] : 0.f;
    }
  const int nk = (k + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < nk)
      load_stage<ST, TA, TB>(As + s * BK * LDA_S, Bs + s * BN * LDB_S, A, lda, B, ldb, m, n,
                                k, m0, n0, s * BK, tid);
    cp_commit();
  }
  for (int kt = 0; kt < nk; kt++) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    int ks = kt + STAGES - 1;
    if (ks < nk) {
      int slot = ks % STAGES;
      load_stage<ST, TA, TB>(As + slot * BK * LDA_S, Bs + slot * BN * LDB_S, A, lda, B, ldb,
                                m, n, k, m0, n0, ks * BK, tid);
    }
    cp_commit();
    const float *as = As + (kt % STAGES) * BK * LDA_S;
    const float *bs = Bs + (kt % STAGES) * BN * LDB_S;
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      float a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = as[kk * LDA_S + tm + i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = bs[(tn + j) * LDB_S + kk];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
  }
  cp_wait<0>();
#pragma unroll
  for (int j = 0; j < 4; j++)
#pragma unroll
    for (int i = 0; i < 8; i++) {
      int gi = m0 + tm + i, gj = n0 + tn + j;
      if (gi < m && gj < n && keep(uplo, gi, gj)) {
        float *cp = C + gi + (long)gj * ldc;
        float v = alpha * acc[i][j];
        *cp = FOLD || beta == 0.f ? v : fmaf(beta, *cp, v);
      }
    }
}

template <typename K>
void set_smem(K kern, size_t bytes) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

extern "C" int pla_k_gemm_tile_rows(int dt) { return dt == MPI_DOUBLE ? DT::BM : ST::BM; }

extern "C" int pla_k_gemm(int dt, int transa, int transb, int m, int n, int k, double alpha,
                          const void *A, long lda, const void *B, long ldb, double beta, void *C,
                          long ldc, int uplo_c, const int *status, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  if (k <= 0 || alpha == 0.0) {
    if (beta == 1.0) return 0;
    // C := beta C on the requested triangle: an empty main loop
    k = 0;
    alpha = 0.0;
  }
  const bool ta = transa != PLA_NO_TRANSPOSE, tb = transb != PLA_NO_TRANSPOSE;
  const bool fold = alpha == 1.0 || alpha == -1.0;
  if (dt == MPI_DOUBLE) {
    dim3 grid((m + DT::BM - 1) / DT::BM, (n + DT::BN - 1) / DT::BN);
    const unsigned THREADS = DT::THREADS;
    size_t sm = (size_t)DT::STAGES * DT::STAGE * sizeof(double);
    const double *a = (const double *)A, *b = (const double *)B;
    double *c = (double *)C;
#define L(TA_, TB_)                                                                          \
  do {                                                                                       \
    if (fold) {                                                                              \
      set_smem(dgemm_k<TA_, TB_, true>, sm);                                                 \
      dgemm_k<TA_, TB_, true><<<grid, THREADS, sm, s>>>(m, n, k, alpha, a, lda, b, ldb, beta, \
                                                        c, ldc, uplo_c, status);             \
    } else {                                                                                 \
      set_smem(dgemm_k<TA_, TB_, false>, sm);                                                \
      dgemm_k<TA_, TB_, false><<<grid, THREADS, sm, s>>>(m, n, k, alpha, a, lda, b, ldb,      \
                                                         beta, c, ldc, uplo_c, status);      \
    }                                                                                        \
  } while (0)
    if (!ta && !tb) L(false, false);
    else if (!ta && tb) L(false, true);
    else if (ta && !tb) L(true, false);
    else L(true, true);
#undef L
  } else if (dt == MPI_FLOAT) {
    dim3 grid((m + ST::BM - 1) / ST::BM, (n + ST::BN - 1) / ST::BN);
    const unsigned THREADS = ST::THREADS;
    size_t sm = (size_t)ST::STAGES * ST::STAGE * sizeof(float);
    const float *a = (const float *)A, *b = (const float *)B;
    float *c = (float *)C;
#define L(TA_, TB_)                                                                          \
  do {                                                                                       \
    if (fold) {                                                                              \
      set_smem(sgemm_k<TA_, TB_, true>, sm);                                                 \
      sgemm_k<TA_, TB_, true><<<grid, THREADS, sm, s>>>(m, n, k, (float)alpha, a, lda, b,     \
                                                        ldb, (float)beta, c, ldc, uplo_c,    \
                                                        status);                             \
    } else {                                                                                 \
      set_smem(sgemm_k<TA_, TB_, false>, sm);                                                \
      sgemm_k<TA_, TB_, false><<<grid, THREADS, sm, s>>>(m, n, k, (float)alpha, a, lda, b,    \
                                                         ldb, (float)beta, c, ldc, uplo_c,   \
                                                         status);                            \
    }                                                                                        \
  } while (0)
    if (!ta && !tb) L(false, false);
    else if (!ta && tb) L(false, true);
    else if (ta && !tb) L(true, false);
    else L(true, true);
#undef L
  } else {
    return (int)cudaErrorInvalidValue;
  }
  pla_k_count(1);
  return (int)cudaGetLastError();
}
