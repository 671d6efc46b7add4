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

// x = p0 + p1 + p2 with p0 = bf16(x), p1 = bf16(x - p0), p2 = bf16(x - p0 -
// p1) (each difference exact in fp32): p0 + p1 carries about 16 significant
// bits, p0 + p1 + p2 all 24.  Row i of dst (ld ldd, K-contiguous) receives
// nseg K-wide segments, segment s holding part (code >> 2 s) & 3, so that a
// single K = nseg kdim product of two such operands sums the chosen part
// products: [p0 p0 p1] x [p0 p1 p0] gives p0 p0 + p0 p1 + p1 p0 (bf16 x 3),
// [p0 p0 p1 p0 p1 p2] x [p0 p1 p0 p2 p1 p0] adds p0 p2 + p1 p1 + p2 p0 (bf16 x
// 6, the terms left out below 2^-24 relative).  x(i, k) = src[i si + k sk];
// with `zero`, src is cleared behind the read.
__device__ __forceinline__ void split_parts(float x, __nv_bfloat16 (&p)[3]) {
  p[0] = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(p[0]);
  p[1] = __float2bfloat16_rn(r1);
  p[2] = __float2bfloat16_rn(r1 - __bfloat162float(p[1]));
}

__global__ void pack_split_k(int m, int kdim, float *src, long si, long sk,
                             __nv_bfloat16 *dst, long ldd, int nseg, unsigned code, int zero) {
  const long total = (long)m * kdim;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long k = e % kdim, i = e / kdim;
    float *p = src + i * si + k * sk;
    __nv_bfloat16 part[3];
    split_parts(*p, part);
    __nv_bfloat16 *row = dst + i * ldd + k;
    for (int seg = 0; seg < nseg; seg++) row[(long)seg * kdim] = part[(code >> (2 * seg)) & 3];
    if (zero) *p = 0.f;
  }
}

// the same for a column-major source (element (i, k) at src[i + k lds]),
// transposed through shared memory so that both the reads and the writes
// are coalesced
__global__ void pack_split_rows_k(int m, int kdim, const float *src, long lds,
                                  __nv_bfloat16 *dst, long ldd, int nseg, unsigned code) {
  __shared__ float tile[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + threadIdx.x, k = k0 + r;
    tile[r][threadIdx.x] = (i < m && k < kdim) ? src[i + (long)k * lds] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, k = k0 + threadIdx.x;
    if (i < m && k < kdim) {
      __nv_bfloat16 part[3];
      split_parts(tile[threadIdx.x][r], part);
      __nv_bfloat16 *row = dst + (long)i * ldd + k;
      for (int seg = 0; seg < nseg; seg++) row[(long)seg * kdim] = part[(code >> (2 * seg)) & 3];
    }
  }
}

// out[0] = max_i |A(i, i)|, out[1] = min_i |A(i, i)| (NaN for a NaN diagonal
// entry), one CTA; the factor's diagonal range, a cheap bound from below on
// its condition number
__global__ void __launch_bounds__(1024) diag_range_k(int n, const float *A, long lda, float *out) {
  __shared__ float smax[32], smin[32];
  float hi = 0.f, lo = __int_as_float(0x7f800000);
  bool nan = false;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float a = fabsf(A[i + (long)i * lda]);
    nan |= a != a;
    hi = fmaxf(hi, a);
    lo = fminf(lo, a);
  }
  nan = __syncthreads_or(nan);
  for (int o = 16; o; o >>= 1) {
    hi = fmaxf(hi, __shfl_down_sync(0xffffffffu, hi, o));
    lo = fminf(lo, __shfl_down_sync(0xffffffffu, lo, o));
  }
  if ((threadIdx.x & 31) == 0) {
    smax[threadIdx.x >> 5] = hi;
    smin[threadIdx.x >> 5] = lo;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    hi = threadIdx.x < nw ? smax[threadIdx.x] : 0.f;
    lo = threadIdx.x < nw ? smin[threadIdx.x] : __int_as_float(0x7f800000);
    for (int o = 16; o; o >>= 1) {
      hi = fmaxf(hi, __shfl_down_sync(0xffffffffu, hi, o));
      lo = fminf(lo, __shfl_down_sync(0xffffffffu, lo, o));
    }
    if (threadIdx.x == 0) {
      out[0] = nan ? __int_as_float(0x7fc00000) : hi;
      out[1] = nan ? __int_as_float(0x7fc00000) : lo;
    }
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

extern "C" int pla_k_pack_split_ex(int m, int kdim, float *src, long si, long sk, void *dst,
                                   long ldd, int nseg, unsigned code, int zero, cudaStream_t s) {
  if (m <= 0 || kdim <= 0) return 0;
  if (nseg < 1 || nseg > 8) return (int)cudaErrorInvalidValue;
  for (int seg = 0; seg < nseg; seg++)
    if (((code >> (2 * seg)) & 3) > 2) return (int)cudaErrorInvalidValue;
  if (si == 1 && !zero) {  // column-major source: the transposing form
    dim3 grid((m + 31) / 32, (kdim + 31) / 32), block(32, 8);
    pack_split_rows_k<<<grid, block, 0, s>>>(m, kdim, src, sk, (__nv_bfloat16 *)dst, ldd, nseg,
                                             code);
  } else {
    const long total = (long)m * kdim;
    int grid = (int)((total + 255) / 256);
    if (grid > 148 * 16) grid = 148 * 16;
    pack_split_k<<<grid, 256, 0, s>>>(m, kdim, src, si, sk, (__nv_bfloat16 *)dst, ldd, nseg,
                                      code, zero);
  }
  pla_k_count(1);
  return (int)cudaGetLastError();
}

// three segments of hi (part 0) or lo (part 1): bit s of pattern set = lo
extern "C" int pla_k_pack_split(int m, int kdim, float *src, long si, long sk, void *dst,
                                long ldd, int pattern, int zero, cudaStream_t s) {
  unsigned code = 0;
  for (int seg = 0; seg < 3; seg++) code |= (unsigned)((pattern >> seg) & 1) << (2 * seg);
  return pla_k_pack_split_ex(m, kdim, src, si, sk, dst, ldd, 3, code, zero, s);
}

extern "C" int pla_k_diag_range(int n, const float *A, long lda, float *out, cudaStream_t s) {
  if (n <= 0) return 0;
  diag_range_k<<<1, 1024, 0, s>>>(n, A, lda, out);
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
// D := inv(L) for a unit-lower-triangular n x n fp32 L (n a multiple of 32, at
// most 256), by block columns: X = inv(L) solves L X = I, and block column j
// of X (32 columns) depends only on L's blocks from block row j down, so the
// block columns are independent.  CTA (j, h) computes columns 32 j + 16 h ..
// + 15 of X:
//   1. L's lower triangle from block row j down is staged in shared memory
//      (one load of everything the CTA reads); warp w inverts the diagonal
//      block j + w in place (lane c: column c by right-looking substitution,
//      the column in registers);
//   2. X_jj = inv(L_jj), then for every block row i > j: S = sum_{j <= k < i}
//      L_ik X_kj (the k range split in four quarters over warp pairs, the
//      partial sums added in a fixed order), X_ij = -inv(L_ii) S;
//   3. the CTA's columns of D written: zero above block row j and above the
//      diagonal, one on it.
// The longest chain (block column 0) is n / 32 - 1 block rows of small
// products out of shared memory, against a serial doubling over the whole
// triangle in one CTA before.
namespace {
constexpr int kInvThreads = 256;
constexpr int kInvCols = 16;         // columns of X per CTA
constexpr int kBlkStride = 32 * 33;  // one 32 x 32 block, column-major, columns padded to 33
__host__ __device__ constexpr int inv_tri_blocks(int nb) { return nb * (nb + 1) / 2; }
constexpr size_t inv_smem_bytes(int nblk) {
  return ((size_t)inv_tri_blocks(nblk) * kBlkStride + (size_t)nblk * 32 * kInvCols +
          4 * 32 * kInvCols + 32 * kInvCols) * sizeof(float);
}

__global__ void __launch_bounds__(kInvThreads, 1)
trtri_unit_lower_k(int n, const float *__restrict__ L, long ldl, float *__restrict__ D,
                   long ldd) {
  extern __shared__ __align__(16) float inv_smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = n / 32, j = blockIdx.x >> 1, h = blockIdx.x & 1;
  const int nb = nblk - j;  // block rows from j down
  // block (I, K) of the staged triangle (rows and columns relative to 32 j,
  // K <= I < nb) at (I (I + 1) / 2 + K) kBlkStride, element (r, k) at k 33 + r
  float *sL = inv_smem;
  float *sX = sL + (size_t)inv_tri_blocks(nb) * kBlkStride;  // X rows from 32 j, row-major
  float *part = sX + (size_t)nb * 32 * kInvCols;             // [quarter][column][row]
  float *sS = part + 4 * 32 * kInvCols;                       // S, row-major

  // 1. stage, then invert the diagonal blocks in place
  for (int I = 0; I < nb; I++)
    for (int K = 0; K <= I; K++) {
      float *dst = sL + (I * (I + 1) / 2 + K) * kBlkStride;
      const float *src = L + 32 * (j + I) + (long)(32 * (j + K)) * ldl;
#pragma unroll
      for (int q = 0; q < 1024 / kInvThreads; q++) {
        const int e = tid + q * kInvThreads, k = e >> 5, r = e & 31;
        dst[k * 33 + r] = src[r + (long)k * ldl];
      }
    }
  __syncthreads();
  if (warp < nb) {
    float *blk = sL + (warp * (warp + 1) / 2 + warp) * kBlkStride;
    float acc[32];
#pragma unroll
    for (int i = 0; i < 32; i++) acc[i] = i == lane ? 1.f : 0.f;
#pragma unroll
    for (int c = 0; c < 32; c++) {  // acc_i -= L(i, c) x_c for i > c, x_c = acc_c final
      const float x = acc[c];
#pragma unroll
      for (int i = c + 1; i < 32; i++) acc[i] = fmaf(-blk[c * 33 + i], x, acc[i]);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 32; i++) blk[lane * 33 + i] = i < lane ? 0.f : acc[i];
  }
  __syncthreads();

  // 2. block rows of X, from the diagonal down
  for (int e = tid; e < 32 * kInvCols; e += kInvThreads) {
    const int r = e / kInvCols, c = e % kInvCols;
    sX[e] = sL[(kInvCols * h + c) * 33 + r];  // X_jj = inv(L_jj), this CTA's columns
  }
  __syncthreads();
  const int g = warp >> 1, ch = warp & 1;  // quarter of the k range, half of the columns
  for (int I = 1; I < nb; I++) {
    const float *row = sL + (I * (I + 1) / 2) * kBlkStride;  // block (I, 0)
    float acc[8];
#pragma unroll
    for (int q = 0; q < 8; q++) acc[q] = 0.f;
    const int k0 = g * 8 * I, k1 = k0 + 8 * I;
    for (int k = k0; k < k1; k++) {
      const float a = row[(k >> 5) * kBlkStride + (k & 31) * 33 + lane];
      const float4 b0 = *reinterpret_cast<const float4 *>(sX + k * kInvCols + 8 * ch);
      const float4 b1 = *reinterpret_cast<const float4 *>(sX + k * kInvCols + 8 * ch + 4);
      acc[0] = fmaf(a, b0.x, acc[0]);
      acc[1] = fmaf(a, b0.y, acc[1]);
      acc[2] = fmaf(a, b0.z, acc[2]);
      acc[3] = fmaf(a, b0.w, acc[3]);
      acc[4] = fmaf(a, b1.x, acc[4]);
      acc[5] = fmaf(a, b1.y, acc[5]);
      acc[6] = fmaf(a, b1.z, acc[6]);
      acc[7] = fmaf(a, b1.w, acc[7]);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) part[(g * kInvCols + 8 * ch + q) * 32 + lane] = acc[q];
    __syncthreads();
    for (int e = tid; e < 32 * kInvCols; e += kInvThreads) {
      const int r = e & 31, c = e >> 5;
      const int o = c * 32 + r;
      sS[r * kInvCols + c] = ((part[o] + part[512 + o]) + part[1024 + o]) + part[1536 + o];
    }
    __syncthreads();
    {  // X_I = -inv(L_II) S: row `lane`, columns 2 warp and 2 warp + 1
      const float *dI = sL + (I * (I + 1) / 2 + I) * kBlkStride;
      float x0 = 0.f, x1 = 0.f;
#pragma unroll 8
      for (int k = 0; k < 32; k++) {
        const float a = dI[k * 33 + lane];
        const float2 s = *reinterpret_cast<const float2 *>(sS + k * kInvCols + 2 * warp);
        x0 = fmaf(a, s.x, x0);
        x1 = fmaf(a, s.y, x1);
      }
      sX[(32 * I + lane) * kInvCols + 2 * warp] = -x0;
      sX[(32 * I + lane) * kInvCols + 2 * warp + 1] = -x1;
    }
    __syncthreads();
  }

  // 3. this CTA's columns of D
  for (int e = tid; e < n * kInvCols; e += kInvThreads) {
    const int r = e % n, c = e / n;
    const int col = 32 * j + kInvCols * h + c, rr = r - 32 * j, cc = col - 32 * j;
    const float v = rr < cc ? 0.f : rr == cc ? 1.f : sX[rr * kInvCols + c];
    D[r + (long)col * ldd] = v;
  }
}
}  // namespace

extern "C" int pla_k_trtri_unit_lower(int n, const float *L, long ldl, float *D, long ldd,
                                      float *work, cudaStream_t s) {
  (void)work;  // no scratch: every intermediate stays in shared memory
  if (n <= 0) return 0;
  if (n % 32 || n > 256) return (int)cudaErrorInvalidValue;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(trtri_unit_lower_k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)inv_smem_bytes(8));
    attr = true;
  }
  const int nblk = n / 32;
  trtri_unit_lower_k<<<2 * nblk, kInvThreads, inv_smem_bytes(nblk), s>>>(n, L, ldl, D, ldd);
  pla_k_count(1);
  return (int)cudaGetLastError();
}
