// Kernels of the mixed-precision solvers:
//   pack_rows   : fp32 column-major panel -> bf16/fp16 row-major (K-contiguous)
//                 operand of the tensor-core trailing update, through a
//                 32 x 32 shared tile so reads and writes stay coalesced;
//   pack_fp8    : the same operand in fp8 E4M3 with a power-of-two scale per
//                 128 rows;
//   sym_scale   : d = diag(A)^-1/2 and the fp32 copy of D A D (the unit-diagonal
//                 matrix the fp8 Cholesky factors);
//   residual    : R = B - A X (or row sums of |A|) in FP64, split over column
//                 slices so every SM streams A at full bandwidth; partial sums
//                 land in a [slices][n] workspace and a second pass adds them
//                 in a fixed order (deterministic).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include <cstdint>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

template <typename D>
__device__ inline D from_f32(float v);
template <>
__device__ inline __nv_bfloat16 from_f32<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <>
__device__ inline __half from_f32<__half>(float v) { return __float2half_rn(v); }

// dst[i * ldd + k] = src[i + k * lds] for i < m, k < kdim
template <typename D>
__global__ void pack_rows_k(int m, int kdim, const float *src, long lds, D *dst, long ldd) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int i = i0 + threadIdx.x, k = k0 + r;
    tile[r][threadIdx.x] = (i < m && k < kdim) ? src[i + (long)k * lds] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int i = i0 + r, k = k0 + threadIdx.x;
    if (i < m && k < kdim) dst[(long)i * ldd + k] = from_f32<D>(tile[threadIdx.x][r]);
  }
}

// fp8 E4M3 operand with one power-of-two scale per block of 128 rows.  For
// block b the scale is 2^e, e the largest integer with max|x| * 2^e <= 448
// (the largest finite E4M3 value), so the block uses the top of the E4M3
// range without overflow; dst[i * ldd + k] = e4m3(x(i, k) * 2^e) and
// inv[b] = 2^-e.  Source element (i, k) is src[i * si + k * sk].  Powers of
// two scale exactly, so the only rounding is the conversion itself.
__global__ void __launch_bounds__(256)
pack_fp8_k(int m, int kdim, const float *__restrict__ src, long si, long sk,
           uint8_t *__restrict__ dst, long ldd, float *__restrict__ inv) {
  __shared__ float red[8];
  __shared__ float s_scale;
  const int b = blockIdx.x, i0 = b * 128;
  const int rows = min(128, m - i0);
  const int total = rows * kdim;
  float amax = 0.f;
  for (int e = threadIdx.x; e < total; e += 256) {
    const int i = e % rows, k = e / rows;
    amax = fmaxf(amax, fabsf(src[(long)(i0 + i) * si + (long)k * sk]));
  }
  for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = red[0];
    for (int w = 1; w < 8; w++) a = fmaxf(a, red[w]);
    float sc = 1.f;
    if (a > 0.f && isfinite(a)) {
      int E;
      const float f = frexpf(a, &E);  // a = f * 2^E, f in [0.5, 1); 448 = 0.875 * 2^9
      sc = ldexpf(1.f, f <= 0.875f ? 9 - E : 8 - E);
    }
    s_scale = sc;
    inv[b] = 1.f / sc;
  }
  __syncthreads();
  const float sc = s_scale;
  for (int e = threadIdx.x; e < total; e += 256) {
    const int k = e % kdim, i = e / kdim;
    const float x = src[(long)(i0 + i) * si + (long)k * sk] * sc;
    dst[(long)(i0 + i) * ldd + k] = (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
  }
}

// Diagonal scaling of an SPD matrix for the fp8 Cholesky: d(i) = 1 / sqrt(A(i, i))
// (1 where A(i, i) <= 0: the factorization then reports the failure itself)
__global__ void diag_rsqrt_k(int n, const double *__restrict__ A, long lda, double *__restrict__ d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = A[i + (long)i * lda];
  d[i] = a > 0.0 ? 1.0 / sqrt(a) : 1.0;
}
// dst(i, j) = fp32(d(i) * A(i, j) * d(j)), column j = blockIdx.y
__global__ void scale_convert_k(int n, const double *__restrict__ A, long lda,
                                const double *__restrict__ d, float *__restrict__ dst, long ldd) {
  const int j = blockIdx.y;
  const double dj = d[j];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i + (long)j * ldd] = (float)(d[i] * A[i + (long)j * lda] * dj);
}
// X(i, r) *= d(i)
__global__ void diag_mul_k(int n, int nrhs, const double *__restrict__ d, double *X, long ldx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double di = d[i];
  for (int r = 0; r < nrhs; r++) X[i + (long)r * ldx] *= di;
}

// out(i, r) := (To) in(perm[i], r): a row permutation (the composed row
// interchanges of an LU) and a conversion in one pass
template <typename Ti, typename To>
__global__ void gather_rows_k(int n, int nrhs, const int *__restrict__ perm,
                              const Ti *__restrict__ in, long ldi, To *__restrict__ out,
                              long ldo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long src = perm[i];
  for (int r = 0; r < nrhs; r++) out[i + (long)r * ldo] = (To)in[src + (long)r * ldi];
}

// Batched helpers of the lockstep GMRES: column s's Krylov basis is
// V + s * ldv (n x (m + 1), ld n); `active` has bit s set for the columns
// still iterating.
// out[s * ldo + c] := V_s(:, a0 + c) . V_s(:, b) for c < nc: one block per
// (c, s), a fixed reduction order
__global__ void __launch_bounds__(256)
basis_dots_k(int n, const double *__restrict__ V, long ldv, int a0, int nc, int b,
             unsigned active, double *__restrict__ out, int ldo) {
  const int c = blockIdx.x, s = blockIdx.y;
  if (!((active >> s) & 1u) || c >= nc) return;
  const double *x = V + (long)s * ldv + (long)(a0 + c) * n, *y = V + (long)s * ldv + (long)b * n;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) acc = fma(x[i], y[i], acc);
  __shared__ double red[8];
  for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
    for (int o = 4; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) out[s * ldo + c] = acc;
  }
}

// V_s(:, b) -= V_s(:, 0:nc) h_s for the active columns, h_s = h + s * ldh
__global__ void __launch_bounds__(256)
basis_update_k(int n, double *__restrict__ V, long ldv, int nc, int b,
               const double *__restrict__ h, int ldh, unsigned active) {
  const int i = blockIdx.x * 256 + threadIdx.x, s = blockIdx.y;
  if (i >= n || !((active >> s) & 1u)) return;
  double *Vs = V + (long)s * ldv;
  const double *hs = h + (long)s * ldh;
  double acc = 0.0;
  for (int c = 0; c < nc; c++) acc = fma(Vs[i + (long)c * n], hs[c], acc);
  Vs[i + (long)b * n] -= acc;
}

struct ColScales {
  double v[16];
};
// V_s(:, b) *= scale.v[s] for the active columns
__global__ void basis_scale_k(int n, double *__restrict__ V, long ldv, int b, ColScales scale,
                              unsigned active) {
  const int i = blockIdx.x * 256 + threadIdx.x, s = blockIdx.y;
  if (i >= n || !((active >> s) & 1u)) return;
  V[(long)s * ldv + (long)b * n + i] *= scale.v[s];
}

constexpr int kRows = 256;

// partial[s][i] = sum over j in slice s of op(A)(i, j) * X(j, r) for NR columns
template <int NR, bool ABS>
__global__ void __launch_bounds__(kRows)
gemv_slices_k(int n, int ncols, int nrhs, int slice, const double *__restrict__ A, long lda,
              const double *__restrict__ X, long ldx, double *__restrict__ partial) {
  __shared__ double xs[NR][256];
  const int i = blockIdx.x * kRows + threadIdx.x;
  const int s = blockIdx.y;
  const int j0 = s * slice, j1 = min(j0 + slice, ncols);
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; r++) acc[r] = 0.0;
  for (int jb = j0; jb < j1; jb += 256) {
    const int cnt = min(256, j1 - jb);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += kRows)
#pragma unroll
      for (int r = 0; r < NR; r++)
        xs[r][t] = ABS ? 1.0 : (r < nrhs ? X[(jb + t) + (long)r * ldx] : 0.0);
    __syncthreads();
    if (i < n) {
      const double *a = A + i + (long)jb * lda;
#pragma unroll 8
      for (int t = 0; t < cnt; t++) {
        double v = a[(long)t * lda];
        if (ABS) v = fabs(v);
#pragma unroll
        for (int r = 0; r < NR; r++) acc[r] = fma(v, xs[r][t], acc[r]);
      }
    }
  }
  if (i < n)
#pragma unroll
    for (int r = 0; r < NR; r++) partial[((long)s * NR + r) * n + i] = acc[r];
}

// R(i, r) = B(i, r) - sum_s partial[s][r][i]   (or the plain sum when B == 0)
template <int NR>
__global__ void gemv_reduce_k(int n, int nrhs, int slices, const double *partial, const double *B,
                              long ldb, double *R, long ldr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int r = 0; r < NR; r++) {
    if (r >= nrhs) break;
    double s = 0.0;
    for (int q = 0; q < slices; q++) s += partial[((long)q * NR + r) * n + i];
    R[i + (long)r * ldr] = B ? B[i + (long)r * ldb] - s : s;
  }
}

int g_sms = 0;

// x = hi + lo with hi = bf16(x) and lo = bf16(x - hi): about 16 significant
// bits.  Row i of dst (ld ldd, K-contiguous) receives three K-wide segments,
// each hi or lo as `pattern` says (bit s set: segment s is lo), so that a
// single K = 3 kdim product of two such operands sums hi*hi + hi*lo + lo*hi.
// x(i, k) = src[i si + k sk]; with `zero`, src is cleared behind the read.
__global__ void pack_split_k(int m, int kdim, float *src, long si, long sk,
                             __nv_bfloat16 *dst, long ldd, int pattern, int zero) {
  const long total = (long)m * kdim;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long k = e % kdim, i = e / kdim;
    float *p = src + i * si + k * sk;
    const float x = *p;
    const __nv_bfloat16 hi = __float2bfloat16_rn(x);
    const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
    __nv_bfloat16 *row = dst + i * ldd + k;
#pragma unroll
    for (int seg = 0; seg < 3; seg++) row[(long)seg * kdim] = (pattern >> seg) & 1 ? lo : hi;
    if (zero) *p = 0.f;
  }
}

}  // namespace

extern "C" int pla_k_pack_rows(int prec, int m, int kdim, const float *src, long lds, void *dst,
                               long ldd, cudaStream_t s) {
  if (m <= 0 || kdim <= 0) return 0;
  dim3 grid((m + 31) / 32, (kdim + 31) / 32), block(32, 8);
  if (prec == PLA_K_BF16)
    pack_rows_k<__nv_bfloat16><<<grid, block, 0, s>>>(m, kdim, src, lds, (__nv_bfloat16 *)dst, ldd);
  else
    pack_rows_k<__half><<<grid, block, 0, s>>>(m, kdim, src, lds, (__half *)dst, ldd);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_pack_split(int m, int kdim, float *src, long si, long sk, void *dst,
                                long ldd, int pattern, int zero, cudaStream_t s) {
  if (m <= 0 || kdim <= 0) return 0;
  const long total = (long)m * kdim;
  int grid = (int)((total + 255) / 256);
  if (grid > 148 * 16) grid = 148 * 16;
  pack_split_k<<<grid, 256, 0, s>>>(m, kdim, src, si, sk, (__nv_bfloat16 *)dst, ldd, pattern,
                                    zero);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_pack_fp8(int m, int kdim, const float *src, long si, long sk, void *dst,
                              long ldd, float *inv, cudaStream_t s) {
  if (m <= 0 || kdim <= 0) return 0;
  pack_fp8_k<<<(m + 127) / 128, 256, 0, s>>>(m, kdim, src, si, sk, (uint8_t *)dst, ldd, inv);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_sym_scale(int n, const double *A, long lda, double *d, float *dst, long ldd,
                               cudaStream_t s) {
  if (n <= 0) return 0;
  diag_rsqrt_k<<<(n + 255) / 256, 256, 0, s>>>(n, A, lda, d);
  dim3 grid((n + 1023) / 1024 < 8 ? (n + 1023) / 1024 : 8, n);
  scale_convert_k<<<grid, 256, 0, s>>>(n, A, lda, d, dst, ldd);
  pla_k_count(2);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_diag_mul(int n, int nrhs, const double *d, double *X, long ldx,
                              cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return 0;
  diag_mul_k<<<(n + 255) / 256, 256, 0, s>>>(n, nrhs, d, X, ldx);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

// R := B - A X for n x ncols A (FP64) and up to 16 columns of X; with abs_rows
// set, R(:,0) := row sums of |A| (X and B unused).  `work` must hold
// slices * nr * n doubles; pla_k_residual_work() gives the size.
extern "C" size_t pla_k_residual_work(int n, int ncols, int nrhs) {
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  int rb = (n + kRows - 1) / kRows;
  int slices = (4 * g_sms + rb - 1) / rb;
  if (slices < 1) slices = 1;
  if (slices > 64) slices = 64;
  int nr = nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : nrhs <= 8 ? 8 : 16;
  (void)ncols;
  return (size_t)slices * nr * n * sizeof(double);
}

extern "C" int pla_k_basis_dots(int n, int nrhs, const double *V, long ldv, int a0, int nc, int b,
                                 unsigned active, double *out, int ldo, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0 || nc <= 0 || nrhs > 16) return nrhs > 16 ? (int)cudaErrorInvalidValue : 0;
  basis_dots_k<<<dim3(nc, nrhs), 256, 0, s>>>(n, V, ldv, a0, nc, b, active, out, ldo);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_basis_update(int n, int nrhs, double *V, long ldv, int nc, int b,
                                  const double *h, int ldh, unsigned active, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0 || nc <= 0 || nrhs > 16) return nrhs > 16 ? (int)cudaErrorInvalidValue : 0;
  basis_update_k<<<dim3((n + 255) / 256, nrhs), 256, 0, s>>>(n, V, ldv, nc, b, h, ldh, active);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_basis_scale(int n, int nrhs, double *V, long ldv, int b, const double *scale,
                                 unsigned active, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0 || nrhs > 16) return nrhs > 16 ? (int)cudaErrorInvalidValue : 0;
  ColScales sc{};
  for (int i = 0; i < nrhs; i++) sc.v[i] = scale[i];
  basis_scale_k<<<dim3((n + 255) / 256, nrhs), 256, 0, s>>>(n, V, ldv, b, sc, active);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_gather_rows(int dt_out, int n, int nrhs, const int *perm, const double *in,
                                  long ldi, void *out, long ldo, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return 0;
  const int g = (n + 255) / 256;
  if (dt_out == MPI_FLOAT)
    gather_rows_k<double, float><<<g, 256, 0, s>>>(n, nrhs, perm, in, ldi, (float *)out, ldo);
  else if (dt_out == MPI_DOUBLE)
    gather_rows_k<double, double><<<g, 256, 0, s>>>(n, nrhs, perm, in, ldi, (double *)out, ldo);
  else
    return (int)cudaErrorInvalidValue;
  pla_k_count(1);
  return (int)cudaGetLastError();
}

extern "C" int pla_k_residual(int n, int ncols, int nrhs, const double *A, long lda,
                              const double *X, long ldx, const double *B, long ldb, double *R,
                              long ldr, int abs_rows, double *work, cudaStream_t s) {
  if (n <= 0) return 0;
  if (nrhs > 16) return (int)cudaErrorInvalidValue;
  pla_k_residual_work(n, ncols, nrhs);
  int rb = (n + kRows - 1) / kRows;
  int slices = (4 * g_sms + rb - 1) / rb;
  if (slices < 1) slices = 1;
  if (slices > 64) slices = 64;
  int slice = (ncols + slices - 1) / slices;
  slices = (ncols + slice - 1) / slice;
  if (slices < 1) slices = 1;
  dim3 grid(rb, slices);
  int rg = (n + 255) / 256;
#define RUN(NR)                                                                               \
  do {                                                                                        \
    if (abs_rows)                                                                             \
      gemv_slices_k<NR, true><<<grid, kRows, 0, s>>>(n, ncols, 1, slice, A, lda, X, ldx, work); \
    else                                                                                      \
      gemv_slices_k<NR, false><<<grid, kRows, 0, s>>>(n, ncols, nrhs, slice, A, lda, X, ldx,    \
                                                      work);                                  \
    gemv_reduce_k<NR><<<rg, 256, 0, s>>>(n, abs_rows ? 1 : nrhs, slices, work,                \
                                         abs_rows ? nullptr : B, ldb, R, ldr);                \
  } while (0)
  if (abs_rows || nrhs <= 1) RUN(1);
  else if (nrhs <= 2) RUN(2);
  else if (nrhs <= 4) RUN(4);
  else if (nrhs <= 8) RUN(8);
  else RUN(16);
#undef RUN
  pla_k_count(2);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// D := inv(L) for a unit-lower-triangular n x n fp32 L (n = 32, 64, 128 or
// 256), in one CTA of 1024 threads:
//   1. the n / 32 diagonal 32 x 32 blocks, one warp each: lane c forward-
//      substitutes column c of the block's inverse (x_c = 1, x_i = -sum_{c <=
//      j < i} L(i, j) x_j), the block and the columns in shared memory;
//   2. doubling: with D11 = inv(L11) and D22 = inv(L22) known for the two
//      h x h halves of a 2h block, D21 = -D22 (L21 D11), two h x h products
//      per pair, h = 32, 64, 128 (products in 32-wide K tiles through shared
//      memory, a 4 x 4 register tile per thread).
// D (ldd) receives the whole lower triangle, unit diagonal included; the
// strictly upper part is set to zero.  T: n * n / 2 floats of scratch.
namespace {
constexpr int kInvThreads = 1024;
// dynamic shared memory: the diagonal blocks and their inverses in phase 1,
// the product tiles in phase 2
constexpr size_t kInvSmem = 2 * 8 * 32 * 33 * sizeof(float);

// the products of one doubling level: for every pair p of h-blocks starting
// at row q = 2 h p, T_p = L21 D11 (step 0), then D21 = -D22 T_p (step 1)
__device__ void inv_products(int n, int h, const float *L, long ldl, float *D, long ldd,
                             float *T, float *sA, float *sB) {
  const int npairs = n / (2 * h), tid = threadIdx.x;
  const int tiles = (h / 4) * (h / 4);  // 4 x 4 output tiles per product
  for (int step = 0; step < 2; step++) {
    for (int p0 = 0; p0 < npairs; p0++) {
      const int q = 2 * h * p0;
      const float *Aop = step == 0 ? L + (q + h) + (long)q * ldl : D + (q + h) + (long)(q + h) * ldd;
      const long lda = step == 0 ? ldl : ldd;
      const float *Bop = step == 0 ? D + q + (long)q * ldd : T + (long)p0 * h * h;
      const long ldb = step == 0 ? ldd : h;
      float *Cop = step == 0 ? T + (long)p0 * h * h : D + (q + h) + (long)q * ldd;
      const long ldc = step == 0 ? h : ldd;
      const float alpha = step == 0 ? 1.f : -1.f;
      float acc[4][4];
      const int t = tid < tiles ? tid : 0;
      const int i0 = (t % (h / 4)) * 4, j0 = (t / (h / 4)) * 4;
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[r][c] = 0.f;
      for (int k0 = 0; k0 < h; k0 += 32) {
        // stage A[:, k0 .. k0 + 32] (h x 32) and B[k0 .. k0 + 32, :] (32 x h)
        for (int e = tid; e < h * 32; e += kInvThreads) {
          const int i = e % h, k = e / h;
          sA[i + k * h] = Aop[i + (long)(k0 + k) * lda];
          const int kk = e % 32, j = e / 32;
          sB[kk + j * 32] = Bop[(k0 + kk) + (long)j * ldb];
        }
        __syncthreads();
        if (tid < tiles)
          for (int k = 0; k < 32; k++) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; r++) a[r] = sA[(i0 + r) + k * h];
#pragma unroll
            for (int c = 0; c < 4; c++) b[c] = sB[k + (j0 + c) * 32];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
              for (int c = 0; c < 4; c++) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
          }
        __syncthreads();
      }
      if (tid < tiles)
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
          for (int c = 0; c < 4; c++) Cop[(i0 + r) + (long)(j0 + c) * ldc] = alpha * acc[r][c];
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(kInvThreads, 1)
trtri_unit_lower_k(int n, const float *__restrict__ L, long ldl, float *D, long ldd, float *T) {
  extern __shared__ __align__(16) float inv_smem[];
  auto blk = reinterpret_cast<float(*)[32][33]>(inv_smem);
  auto xs = reinterpret_cast<float(*)[32][33]>(inv_smem + 8 * 32 * 33);
  float *sA = inv_smem, *sB = inv_smem + 128 * 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // the off-diagonal blocks start at zero (the lower ones are computed below)
  for (long e = tid; e < (long)n * n; e += kInvThreads) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (i / 32 != j / 32) D[i + (long)j * ldd] = 0.f;
  }
  // 1. diagonal blocks
  const int nb32 = n / 32;
  if (warp < nb32) {
    const int q = warp * 32;
    for (int j = 0; j < 32; j++) blk[warp][lane][j] = L[(q + lane) + (long)(q + j) * ldl];
    __syncwarp();
    // column `lane` of the block's inverse: x_i for i >= lane
    for (int i = 0; i < 32; i++) {
      float x;
      if (i < lane) x = 0.f;
      else if (i == lane) x = 1.f;
      else {
        float s = 0.f;
        for (int j = lane; j < i; j++) s = fmaf(blk[warp][i][j], xs[warp][j][lane], s);
        x = -s;
      }
      xs[warp][i][lane] = x;
    }
    __syncwarp();
    for (int i = 0; i < 32; i++) D[(q + i) + (long)(q + lane) * ldd] = xs[warp][i][lane];
  }
  __syncthreads();
  // 2. doubling
  for (int h = 32; h < n; h *= 2) {
    inv_products(n, h, L, ldl, D, ldd, T, sA, sB);
    __syncthreads();
  }
}
}  // namespace

extern "C" int pla_k_trtri_unit_lower(int n, const float *L, long ldl, float *D, long ldd,
                                      float *work, cudaStream_t s) {
  if (n <= 0) return 0;
  if (n % 32 || n > 256 || (n & (n - 1))) return (int)cudaErrorInvalidValue;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(trtri_unit_lower_k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kInvSmem);
    attr = true;
  }
  trtri_unit_lower_k<<<1, kInvThreads, kInvSmem, s>>>(n, L, ldl, D, ldd, work);
  pla_k_count(1);
  return (int)cudaGetLastError();
}
