// Level-1/2 kernels, copies, conversions, row interchanges and norms.
// All bandwidth-bound: grid-stride loops over column-major data with the row
// index fastest across threads so that warps read contiguous memory.
#include <atomic>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 148 * 16;

inline int blocks_for(long work) {
  long b = (work + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  return (int)(b > kMaxBlocks ? kMaxBlocks : b);
}

template <typename T>
__global__ void fill_k(int m, int n, T *A, long lda, T v) {
  long total = (long)m * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    A[i + j * lda] = v;
  }
}

template <typename T>
__global__ void axpby_k(int m, int n, T alpha, const T *X, long ldx, T beta, T *Y, long ldy) {
  long total = (long)m * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    T x = X[i + j * ldx];
    Y[i + j * ldy] = beta == T(0) ? alpha * x : alpha * x + beta * Y[i + j * ldy];
  }
}

// Y(m x n) := X' through a 32x32 shared tile so both sides stay coalesced
template <typename T>
__global__ void transpose_k(int m, int n, const T *X, long ldx, T *Y, long ldy) {
  __shared__ T tile[32][33];
  int bi = blockIdx.x * 32, bj = blockIdx.y * 32;
  // X is n x m: read X(bj + ty, bi + tx) = element (bi+tx, bj+ty) of Y
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    int xi = bj + threadIdx.x, xj = bi + ty;
    if (xi < n && xj < m) tile[ty][threadIdx.x] = X[xi + (long)xj * ldx];
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    int yi = bi + threadIdx.x, yj = bj + ty;
    if (yi < m && yj < n) Y[yi + (long)yj * ldy] = tile[threadIdx.x][ty];
  }
}

template <typename S, typename D>
__device__ inline D cvt(S v) { return (D)v; }
template <> __device__ inline __nv_bfloat16 cvt<double, __nv_bfloat16>(double v) { return __double2bfloat16(v); }
template <> __device__ inline __nv_bfloat16 cvt<float, __nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
template <> __device__ inline __half cvt<double, __half>(double v) { return __double2half(v); }
template <> __device__ inline __half cvt<float, __half>(float v) { return __float2half_rn(v); }

template <typename S, typename D>
__global__ void convert_k(const S *src, long lds, D *dst, long ldd, int m, int n) {
  long total = (long)m * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    dst[i + j * ldd] = cvt<S, D>(src[i + j * lds]);
  }
}

template <typename T>
__global__ void scal_k(int m, int n, T alpha, T *X, long ldx) {
  long total = (long)m * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    X[i + j * ldx] = alpha * X[i + j * ldx];
  }
}

template <typename T>
__global__ void swap_k(int m, int n, T *X, long ldx, T *Y, long ldy) {
  long total = (long)m * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    T a = X[i + j * ldx];
    X[i + j * ldx] = Y[i + j * ldy];
    Y[i + j * ldy] = a;
  }
}

// A := A + alpha x y' (Local_BLAS/PLA_Local_BLAS2.c:578, dger_ ordering:
// temp = alpha * y(j); A(i,j) += x(i) * temp)
template <typename T>
__global__ void ger_k(int m, int n, T alpha, const T *x, long incx, const T *y, long incy, T *A,
                      long lda) {
  long total = (long)m * n;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    T temp = alpha * y[j * incy];
    A[i + j * lda] = A[i + j * lda] + x[i * incx] * temp;
  }
}

// y := alpha A x + beta y, one thread per row, columns streamed in chunks
template <typename T>
__global__ void gemv_n_k(int m, int n, T alpha, const T *A, long lda, const T *x, T beta, T *y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  T acc = 0;
  for (int j = 0; j < n; j++) acc += A[i + (long)j * lda] * x[j];
  y[i] = beta == T(0) ? alpha * acc : alpha * acc + beta * y[i];
}

// y := alpha A' x + beta y, one warp per column
template <typename T>
__global__ void gemv_t_k(int m, int n, T alpha, const T *A, long lda, const T *x, T beta, T *y) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  if (warp >= n) return;
  const T *a = A + (long)warp * lda;
  T acc = 0;
  for (int i = lane; i < m; i += 32) acc += a[i] * x[i];
  for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) y[warp] = beta == T(0) ? alpha * acc : alpha * acc + beta * y[warp];
}

// first index of the max |x| (BLAS i?amax); one block, deterministic
template <typename T>
__global__ void iamax_k(int n, const T *x, long incx, int *idx_out, T *val_out) {
  __shared__ T sv[32];
  __shared__ int si[32];
  T best = -1;
  int bi = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    T v = fabs(x[i * incx]);
    if (v > best) { best = v; bi = i; }
  }
  for (int o = 16; o; o >>= 1) {
    T ov = __shfl_down_sync(0xffffffffu, best, o);
    int oi = __shfl_down_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
  }
  int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) { sv[w] = best; si[w] = bi; }
  __syncthreads();
  if (w == 0) {
    int nw = blockDim.x / 32;
    best = l < nw ? sv[l] : T(-1);
    bi = l < nw ? si[l] : 0;
    for (int o = 16; o; o >>= 1) {
      T ov = __shfl_down_sync(0xffffffffu, best, o);
      int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if (l == 0) {
      *idx_out = bi;
      *val_out = n > 0 ? x[bi * incx] : T(0);
    }
  }
}

// row interchanges, applied in sequence: one thread per column
template <typename T>
__global__ void laswp_k(T *A, long lda, int npiv, const int *piv, int c0, int c1, int c2,
                        int c3) {
  extern __shared__ int sp[];
  for (int i = threadIdx.x; i < npiv; i += blockDim.x) sp[i] = piv[i];
  __syncthreads();
  int w1 = c1 - c0, total = w1 + (c3 - c2);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int c = t < w1 ? c0 + t : c2 + (t - w1);
    T *col = A + (long)c * lda;
    for (int i = 0; i < npiv; i++) {
      int p = i + sp[i];
      if (p != i) {
        T a = col[i];
        col[i] = col[p];
        col[p] = a;
      }
    }
  }
}

// number of non-trivial interchanges (piv[i] != 0) in a pivot vector, added
// to *ctr: one atomic per warp
__global__ void count_interchanges_k(int npiv, const int *piv, unsigned long long *ctr) {
  unsigned c = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npiv; i += gridDim.x * blockDim.x)
    c += piv[i] != 0;
  for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(ctr, (unsigned long long)c);
}

template <typename T>
__global__ void row_abs_sums_k(int m, int n, const T *A, long lda, double *rs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double s = 0;
  for (int j = 0; j < n; j++) s += fabs((double)A[i + (long)j * lda]);
  rs[i] = s;
}

template <typename T>
__global__ void col_abs_max_k(int m, int n, const T *X, long ldx, double *out) {
  __shared__ double sm[32];
  int j = blockIdx.x;
  if (j >= n) return;
  double b = 0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) b = fmax(b, fabs((double)X[i + (long)j * ldx]));
  for (int o = 16; o; o >>= 1) b = fmax(b, __shfl_down_sync(0xffffffffu, b, o));
  if (threadIdx.x % 32 == 0) sm[threadIdx.x / 32] = b;
  __syncthreads();
  if (threadIdx.x < 32) {
    b = threadIdx.x < blockDim.x / 32 ? sm[threadIdx.x] : 0.0;
    for (int o = 16; o; o >>= 1) b = fmax(b, __shfl_down_sync(0xffffffffu, b, o));
    if (threadIdx.x == 0) out[j] = b;
  }
}

// Euclidean norm of the n elements x[0], x[inc], ... as dnrm2 / snrm2 (called
// from Local_BLAS/PLA_Local_BLAS1.c:394-441): the largest |x_i| scales the
// sum of squares, so that neither overflows nor underflows.  One CTA, FP64
// arithmetic and a fixed reduction order make the result deterministic; a NaN
// anywhere gives NaN, an infinity (and no NaN) gives infinity.
template <typename T>
__global__ void __launch_bounds__(1024) nrm2_k(long n, const T *x, long inc, double *out) {
  __shared__ double sm[32];
  __shared__ int s_nan;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) s_nan = 0;
  double mx = 0;
  bool nan = false;
  for (long i = tid; i < n; i += blockDim.x) {
    const double a = fabs((double)x[i * inc]);
    nan |= a != a;
    mx = fmax(mx, a);
  }
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __syncthreads();
  if (nan) s_nan = 1;
  if (lane == 0) sm[warp] = mx;
  __syncthreads();
  mx = lane < nw ? sm[lane] : 0.0;
  for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (s_nan || mx == 0.0 || isinf(mx)) {
    if (tid == 0) out[0] = s_nan ? __longlong_as_double(0x7ff8000000000000ll) : mx;
    return;
  }
  double ssq = 0;
  for (long i = tid; i < n; i += blockDim.x) {
    const double t = (double)x[i * inc] / mx;
    ssq = fma(t, t, ssq);
  }
  for (int o = 16; o; o >>= 1) ssq += __shfl_down_sync(0xffffffffu, ssq, o);
  __syncthreads();
  if (lane == 0) sm[warp] = ssq;
  __syncthreads();
  if (warp == 0) {
    ssq = lane < nw ? sm[lane] : 0.0;
    for (int o = 16; o; o >>= 1) ssq += __shfl_down_sync(0xffffffffu, ssq, o);
    if (lane == 0) out[0] = mx * sqrt(ssq);
  }
}

// A(i, i) += v for i < n (UTIL/PLA_Shift.c:33-86)
template <typename T>
__global__ void shift_diag_k(int n, T *A, long lda, T v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    A[(long)i + (long)i * lda] += v;
}

std::atomic<long> g_launches{0};

// every launcher below issues exactly one kernel before calling this
inline int status() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return (int)cudaGetLastError();
}

}  // namespace

extern "C" {

void pla_k_count(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long pla_k_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int pla_k_fill(int dt, int m, int n, void *A, long lda, double value, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  int g = blocks_for((long)m * n);
  if (dt == MPI_DOUBLE) fill_k<double><<<g, kThreads, 0, s>>>(m, n, (double *)A, lda, value);
  else if (dt == MPI_FLOAT) fill_k<float><<<g, kThreads, 0, s>>>(m, n, (float *)A, lda, (float)value);
  else if (dt == MPI_INT) fill_k<int><<<g, kThreads, 0, s>>>(m, n, (int *)A, lda, (int)value);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_axpby(int dt, int m, int n, double alpha, const void *X, long ldx, double beta, void *Y,
                long ldy, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  int g = blocks_for((long)m * n);
  if (dt == MPI_DOUBLE)
    axpby_k<double><<<g, kThreads, 0, s>>>(m, n, alpha, (const double *)X, ldx, beta, (double *)Y, ldy);
  else if (dt == MPI_FLOAT)
    axpby_k<float><<<g, kThreads, 0, s>>>(m, n, (float)alpha, (const float *)X, ldx, (float)beta,
                                          (float *)Y, ldy);
  else if (dt == MPI_INT)
    axpby_k<int><<<g, kThreads, 0, s>>>(m, n, (int)alpha, (const int *)X, ldx, (int)beta, (int *)Y, ldy);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_copy(int dt, int trans, int m, int n, const void *X, long ldx, void *Y, long ldy,
               cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  if (trans == PLA_NO_TRANSPOSE) {
    int es = dt == MPI_DOUBLE ? 8 : 4;
    return (int)cudaMemcpy2DAsync(Y, ldy * es, X, ldx * es, (size_t)m * es, n,
                                  cudaMemcpyDeviceToDevice, s);
  }
  dim3 grid((m + 31) / 32, (n + 31) / 32), block(32, 8);
  if (dt == MPI_DOUBLE) transpose_k<double><<<grid, block, 0, s>>>(m, n, (const double *)X, ldx, (double *)Y, ldy);
  else if (dt == MPI_FLOAT) transpose_k<float><<<grid, block, 0, s>>>(m, n, (const float *)X, ldx, (float *)Y, ldy);
  else if (dt == MPI_INT) transpose_k<int><<<grid, block, 0, s>>>(m, n, (const int *)X, ldx, (int *)Y, ldy);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_convert(int ds, const void *src, long lds, int dd, void *dst, long ldd, int m, int n,
                  cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  int g = blocks_for((long)m * n);
#define CV(S, D) convert_k<S, D><<<g, kThreads, 0, s>>>((const S *)src, lds, (D *)dst, ldd, m, n)
  if (ds == MPI_DOUBLE && dd == MPI_FLOAT) CV(double, float);
  else if (ds == MPI_FLOAT && dd == MPI_DOUBLE) CV(float, double);
  else if (ds == MPI_DOUBLE && dd == PLA_K_BF16) CV(double, __nv_bfloat16);
  else if (ds == MPI_FLOAT && dd == PLA_K_BF16) CV(float, __nv_bfloat16);
  else if (ds == MPI_DOUBLE && dd == PLA_K_FP16) CV(double, __half);
  else if (ds == MPI_FLOAT && dd == PLA_K_FP16) CV(float, __half);
  else if (ds == MPI_DOUBLE && dd == MPI_DOUBLE) CV(double, double);
  else if (ds == MPI_FLOAT && dd == MPI_FLOAT) CV(float, float);
  else return (int)cudaErrorInvalidValue;
#undef CV
  return status();
}

int pla_k_nrm2(int dt, long n, const void *x, long inc, double *out, cudaStream_t s) {
  if (dt == MPI_DOUBLE) nrm2_k<double><<<1, 1024, 0, s>>>(n, (const double *)x, inc, out);
  else if (dt == MPI_FLOAT) nrm2_k<float><<<1, 1024, 0, s>>>(n, (const float *)x, inc, out);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_shift_diag(int dt, int n, void *A, long lda, double v, cudaStream_t s) {
  if (n <= 0) return 0;
  const int g = (n + kThreads - 1) / kThreads;
  if (dt == MPI_DOUBLE) shift_diag_k<double><<<g, kThreads, 0, s>>>(n, (double *)A, lda, v);
  else if (dt == MPI_FLOAT) shift_diag_k<float><<<g, kThreads, 0, s>>>(n, (float *)A, lda, (float)v);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_scal(int dt, int m, int n, double alpha, void *X, long ldx, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  int g = blocks_for((long)m * n);
  if (dt == MPI_DOUBLE) scal_k<double><<<g, kThreads, 0, s>>>(m, n, alpha, (double *)X, ldx);
  else if (dt == MPI_FLOAT) scal_k<float><<<g, kThreads, 0, s>>>(m, n, (float)alpha, (float *)X, ldx);
  else return (int)cudaErrorInvalidValue;
  return status();
}

// x := x * (1/alpha): the reciprocal is formed once, as
// Local_BLAS/PLA_Local_BLAS1.c:256-263 does, then multiplied in
int pla_k_inv_scal(int dt, int m, int n, double alpha, void *X, long ldx, cudaStream_t s) {
  if (dt == MPI_FLOAT) return pla_k_scal(dt, m, n, (double)(1.0f / (float)alpha), X, ldx, s);
  return pla_k_scal(dt, m, n, 1.0 / alpha, X, ldx, s);
}

int pla_k_swap(int dt, int m, int n, void *X, long ldx, void *Y, long ldy, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  int g = blocks_for((long)m * n);
  if (dt == MPI_DOUBLE) swap_k<double><<<g, kThreads, 0, s>>>(m, n, (double *)X, ldx, (double *)Y, ldy);
  else if (dt == MPI_FLOAT) swap_k<float><<<g, kThreads, 0, s>>>(m, n, (float *)X, ldx, (float *)Y, ldy);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_ger(int dt, int m, int n, double alpha, const void *x, long incx, const void *y,
              long incy, void *A, long lda, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  int g = blocks_for((long)m * n);
  if (dt == MPI_DOUBLE)
    ger_k<double><<<g, kThreads, 0, s>>>(m, n, alpha, (const double *)x, incx, (const double *)y,
                                         incy, (double *)A, lda);
  else if (dt == MPI_FLOAT)
    ger_k<float><<<g, kThreads, 0, s>>>(m, n, (float)alpha, (const float *)x, incx,
                                        (const float *)y, incy, (float *)A, lda);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_gemv(int dt, int trans, int m, int n, double alpha, const void *A, long lda,
               const void *x, double beta, void *y, cudaStream_t s) {
  if (trans == PLA_NO_TRANSPOSE) {
    if (m <= 0) return 0;
    int g = (m + kThreads - 1) / kThreads;
    if (dt == MPI_DOUBLE)
      gemv_n_k<double><<<g, kThreads, 0, s>>>(m, n, alpha, (const double *)A, lda, (const double *)x,
                                              beta, (double *)y);
    else
      gemv_n_k<float><<<g, kThreads, 0, s>>>(m, n, (float)alpha, (const float *)A, lda,
                                             (const float *)x, (float)beta, (float *)y);
  } else {
    if (n <= 0) return 0;
    int g = (n * 32 + kThreads - 1) / kThreads;
    if (dt == MPI_DOUBLE)
      gemv_t_k<double><<<g, kThreads, 0, s>>>(m, n, alpha, (const double *)A, lda, (const double *)x,
                                              beta, (double *)y);
    else
      gemv_t_k<float><<<g, kThreads, 0, s>>>(m, n, (float)alpha, (const float *)A, lda,
                                             (const float *)x, (float)beta, (float *)y);
  }
  return status();
}

int pla_k_iamax(int dt, int n, const void *x, long incx, int *idx, void *val, cudaStream_t s) {
  if (dt == MPI_DOUBLE) iamax_k<double><<<1, 1024, 0, s>>>(n, (const double *)x, incx, idx, (double *)val);
  else if (dt == MPI_FLOAT) iamax_k<float><<<1, 1024, 0, s>>>(n, (const float *)x, incx, idx, (float *)val);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_laswp(int dt, void *A, long lda, int npiv, const int *piv, int c0, int c1, int c2,
                int c3, cudaStream_t s) {
  int total = (c1 - c0) + (c3 - c2);
  if (npiv <= 0 || total <= 0) return 0;
  int g = (total + 127) / 128;
  size_t sh = (size_t)npiv * sizeof(int);
  if (dt == MPI_DOUBLE) laswp_k<double><<<g, 128, sh, s>>>((double *)A, lda, npiv, piv, c0, c1, c2, c3);
  else if (dt == MPI_FLOAT) laswp_k<float><<<g, 128, sh, s>>>((float *)A, lda, npiv, piv, c0, c1, c2, c3);
  else return (int)cudaErrorInvalidValue;
  return status();
}

int pla_k_count_interchanges(int npiv, const int *piv, unsigned long long *ctr,
                              cudaStream_t s) {
  if (npiv <= 0) return 0;
  int g = (npiv + 255) / 256;
  count_interchanges_k<<<g < 148 ? g : 148, 256, 0, s>>>(npiv, piv, ctr);
  return status();
}

int pla_k_laswp_rows(int dt, void *B, long ldb, int ncols, int npiv, const int *piv,
                     cudaStream_t s) {
  // process pivots in chunks so the shared-memory copy stays small
  const int chunk = 4096;
  for (int k = 0; k < npiv; k += chunk) {
    int c = npiv - k < chunk ? npiv - k : chunk;
    char *base = (char *)B + (size_t)k * (dt == MPI_DOUBLE ? 8 : 4);
    int r = pla_k_laswp(dt, base, ldb, c, piv + k, 0, ncols, 0, 0, s);
    if (r) return r;
  }
  return 0;
}

int pla_k_row_abs_sums(int dt, int m, int n, const void *A, long lda, double *rs, cudaStream_t s) {
  if (m <= 0) return 0;
  int g = (m + kThreads - 1) / kThreads;
  if (dt == MPI_DOUBLE) row_abs_sums_k<double><<<g, kThreads, 0, s>>>(m, n, (const double *)A, lda, rs);
  else row_abs_sums_k<float><<<g, kThreads, 0, s>>>(m, n, (const float *)A, lda, rs);
  return status();
}

int pla_k_col_abs_max(int dt, int m, int n, const void *X, long ldx, double *out, cudaStream_t s) {
  if (n <= 0) return 0;
  if (dt == MPI_DOUBLE) col_abs_max_k<double><<<n, 256, 0, s>>>(m, n, (const double *)X, ldx, out);
  else col_abs_max_k<float><<<n, 256, 0, s>>>(m, n, (const float *)X, ldx, out);
  return status();
}

}  // extern "C"
