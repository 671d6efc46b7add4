// Triangular solve with one right-hand side in a single launch (fp32 with
// 128 x 128 blocks, FP64 with 64 x 64 blocks).
//
//   tri_inv_blocks_k : inverse of every TB x TB diagonal block of op(A)
//                      (computed once per factor, reused by every solve);
//   trsv_ticket_k    : x := inv(op(A)) b.  CTAs take block rows through an
//                      atomic ticket in dependency order, so a block row only
//                      ever waits for rows whose owners are already running
//                      (no co-residency assumption).  For block row i a CTA
//                      accumulates op(A)(i, j) x_j over every finished block j
//                      (waiting on j's flag with a bounded spin), multiplies by
//                      the inverse diagonal block, publishes x_i and raises
//                      flag i.  The triangle is read exactly once, so the solve
//                      is HBM-bound apart from the per-block latency chain.
//                      b and x may be the same array.
#include <cstdint>

#include "PLA.h"
#include "pla_kernels.h"

namespace {

constexpr int TB = 128, TB64 = 64, THREADS = 256;  // fp32 and FP64 block orders
constexpr long kSpin = 20000000;

template <typename T>
__device__ __forceinline__ T opA(const T *A, long lda, bool trans, long i, long j) {
  return trans ? A[j + i * lda] : A[i + j * lda];
}

// inverse of the TB x TB diagonal block `blockIdx.x` of op(A) into Dinv
// (element (r, c) of block i at Dinv[i*TB + r + c*ldd]); TB = 128 for fp32,
// 64 for FP64 (two TB x (TB + 1) blocks must fit in shared memory)
// TA: the factor's element type; T: the inverse's (an fp32 factor may have
// its inverse blocks in FP64, for solves carried out in FP64)
template <typename TA, typename T, int TB>
__global__ void __launch_bounds__(THREADS)
tri_inv_blocks_k(int n, const TA *A, long lda, bool lower_op, bool trans, bool unit, T *Dinv,
                 long ldd) {
  extern __shared__ __align__(16) unsigned char sm[];
  constexpr int L = TB + 1, NT = THREADS / TB;  // NT threads per column
  TA *D = (TA *)sm;               // TB x TB, ld TB + 1
  T *X = (T *)(sm + ((size_t)TB * L * sizeof(TA) + 15) / 16 * 16);  // TB x TB, ld TB + 1
  const int blk = blockIdx.x, r0 = blk * TB, nb = min(TB, n - r0);
  for (int t = threadIdx.x; t < TB * TB; t += THREADS) {
    int i = t % TB, j = t / TB;
    TA v = TA(0);
    if (i < nb && j < nb) v = opA(A, lda, trans, (long)r0 + i, (long)r0 + j);
    if (i == j && (unit || i >= nb)) v = TA(1);
    D[i + j * L] = v;
    X[i + j * L] = i == j ? T(1) : T(0);
  }
  __syncthreads();
  // solve D X = I; column c is handled by the NT threads with c = tid % TB
  const int c = threadIdx.x % TB, part = threadIdx.x / TB;
  for (int step = 0; step < TB; step++) {
    const int l = lower_op ? step : TB - 1 - step;
    if (part == 0) X[l + c * L] = X[l + c * L] / D[l + l * L];
    __syncthreads();
    const T xl = X[l + c * L];
    if (lower_op)
      for (int i = l + 1 + part; i < TB; i += NT) X[i + c * L] -= D[i + l * L] * xl;
    else
      for (int i = part; i < l; i += NT) X[i + c * L] -= D[i + l * L] * xl;
    __syncthreads();
  }
  for (int t = threadIdx.x; t < TB * TB; t += THREADS) {
    int i = t % TB, j = t / TB;
    Dinv[(long)(r0 + i) + (long)j * ldd] = X[i + j * L];
  }
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T>
__global__ void __launch_bounds__(THREADS)
trsv_ticket_k(int n, int nblk, const T *A, long lda, bool lower_op, bool trans, const T *Dinv,
              long ldd, const T *b, T *x, int *ticket, int *flags, int *status, bool vec_ok) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  T *Ds = reinterpret_cast<T *>(dyn_smem);  // TB x TB inverse diagonal block
  __shared__ T xs[TB];
  __shared__ T part[2][TB];
  __shared__ int s_blk, s_bad;
  const int r = threadIdx.x % TB, half = threadIdx.x / TB;
  for (;;) {
    if (threadIdx.x == 0) {
      s_blk = atomicAdd(ticket, 1);
      s_bad = 0;
    }
    __syncthreads();
    const int q = s_blk;
    if (q >= nblk) return;
    const int i = lower_op ? q : nblk - 1 - q;
    const long r0 = (long)i * TB;
    const int nbi = min(TB, n - (int)r0);
    // Each full 128 x 128 tile is read with 16 independent 16-byte loads per
    // thread (64 KB in flight per CTA).  No transpose: thread (rg, cg) owns
    // rows 4rg..4rg+3 and columns 16cg..16cg+15, so a warp reads 512
    // contiguous bytes of a column.  Transpose: op(A)(r, c) = A(c, r), thread
    // (r, half) reads 64 contiguous values of column r of A.  Ragged edge
    // tiles take a scalar path.
    const int rg = threadIdx.x & 31, cg = threadIdx.x >> 5;
    T acc4[4] = {T(0), T(0), T(0), T(0)};
    T acc = T(0);
    // the inverse diagonal block streams into shared memory while the row's
    // tiles are processed
    for (int u = threadIdx.x; u < TB * TB / 4; u += THREADS) {
      const int c = u / (TB / 4), r4 = (u % (TB / 4)) * 4;
      cp_async16(&Ds[c * TB + r4], Dinv + (r0 + r4) + (long)c * ldd);
    }
    cp_async_commit();
    for (int s = 0; s < q; s++) {
      const int j = lower_op ? s : nblk - 1 - s;
      const long c0 = (long)j * TB;
      const int nbj = min(TB, n - (int)c0);
      const bool full = nbi == TB && nbj == TB && vec_ok;
      // the tile does not depend on x_j: its loads are issued before waiting
      float4 v[16];
      if (full) {
        const T *base = trans ? A + (r0 + r) * lda + c0 + 64 * half
                              : A + (r0 + 4 * rg) + (c0 + 16 * cg) * lda;
        const long step = trans ? 4 : lda;
#pragma unroll
        for (int u = 0; u < 16; u++) v[u] = *reinterpret_cast<const float4 *>(base + u * step);
      }
      if (threadIdx.x == 0) {
        long spins = 0;
        while (ld_acquire(&flags[j]) == 0) {
          if (++spins > kSpin || *(volatile int *)status != PLA_K_OK) {
            atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
            s_bad = 1;
            break;
          }
          __nanosleep(32);
        }
      }
      __syncthreads();
      if (s_bad) return;
      if (threadIdx.x < nbj) xs[threadIdx.x] = __ldcg(&x[c0 + threadIdx.x]);
      __syncthreads();
      if (full && !trans) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const T xv = xs[16 * cg + u];
          acc4[0] += v[u].x * xv;
          acc4[1] += v[u].y * xv;
          acc4[2] += v[u].z * xv;
          acc4[3] += v[u].w * xv;
        }
      } else if (full) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int c = 64 * half + 4 * u;
          acc += v[u].x * xs[c] + v[u].y * xs[c + 1] + v[u].z * xs[c + 2] + v[u].w * xs[c + 3];
        }
      } else if (r < nbi) {
        if (!trans) {
          for (int c = half; c < nbj; c += 2) acc += A[(r0 + r) + (c0 + c) * lda] * xs[c];
        } else {
          const int cb = half * (TB / 2), ce = min(cb + TB / 2, nbj);
          const T *col = A + (r0 + r) * lda + c0;
          for (int c = cb; c < ce; c++) acc += col[c] * xs[c];
        }
      }
      __syncthreads();
    }
    // reduce: acc4 from the 8 column groups (no-transpose full tiles) plus acc
    // from the two halves (transpose or ragged tiles)
    __shared__ T red[8][TB];
#pragma unroll
    for (int e = 0; e < 4; e++) red[cg][4 * rg + e] = acc4[e];
    part[half][r] = acc;
    __syncthreads();
    if (threadIdx.x < TB) {
      T sacc = part[0][r] + part[1][r];
#pragma unroll
      for (int g = 0; g < 8; g++) sacc += red[g][r];
      xs[threadIdx.x] = r < nbi ? b[r0 + r] - sacc : T(0);
    }
    __syncthreads();
    // x_i = inv(D_i) y with the inverse block from shared memory
    cp_async_wait_all();
    __syncthreads();
    {
      T y4[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const float4 d = *reinterpret_cast<const float4 *>(&Ds[(16 * cg + u) * TB + 4 * rg]);
        const T xv = xs[16 * cg + u];
        y4[0] += d.x * xv;
        y4[1] += d.y * xv;
        y4[2] += d.z * xv;
        y4[3] += d.w * xv;
      }
#pragma unroll
      for (int e = 0; e < 4; e++) red[cg][4 * rg + e] = y4[e];
    }
    __syncthreads();
    if (threadIdx.x < nbi) {
      T y = T(0);
#pragma unroll
      for (int g = 0; g < 8; g++) y += red[g][threadIdx.x];
      x[r0 + threadIdx.x] = y;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&flags[i], 1);
  }
}

// The link blocks of the fp32 single-column solve: for every block row i
// that has a predecessor p in the solve order (p = i - 1 going forward, i + 1
// going backward), G_i = op(A)(i, p) inv(D_p), element (r, c) at
// G[i TB + r + c ldd] (the layout of Dinv).  One CTA per link, the two
// 128 x 128 factors in shared memory.
__global__ void __launch_bounds__(THREADS)
link_blocks_k(int n, int nblk, const float *A, long lda, bool lower_op, bool trans,
              const float *Dinv, long ldd, float *G) {
  extern __shared__ __align__(16) unsigned char sm[];
  float *As = reinterpret_cast<float *>(sm);  // op(A)(i, p), column-major, ld TB + 1
  float *Ds = As + TB * (TB + 1);             // inv(D_p), column-major, ld TB + 1
  constexpr int L = TB + 1;
  const int i = lower_op ? blockIdx.x + 1 : blockIdx.x, p = lower_op ? i - 1 : i + 1;
  const long r0 = (long)i * TB, c0 = (long)p * TB;
  const int nbi = min(TB, n - (int)r0), nbp = min(TB, n - (int)c0);
  for (int e = threadIdx.x; e < TB * TB; e += THREADS) {
    const int r = e % TB, c = e / TB;
    As[r + c * L] = r < nbi && c < nbp ? (trans ? A[(c0 + c) + (r0 + r) * lda]
                                                 : A[(r0 + r) + (c0 + c) * lda])
                                       : 0.f;
    Ds[r + c * L] = Dinv[(c0 + r) + (long)c * ldd];
  }
  __syncthreads();
  // thread (r, cg): row r, columns cg, cg + 2, ... (64 of them)
  const int r = threadIdx.x % TB, cg = threadIdx.x / TB;
  for (int c = cg; c < TB; c += 2) {
    float acc = 0.f;
    for (int k = 0; k < TB; k++) acc = fmaf(As[r + k * L], Ds[k + c * L], acc);
    G[r0 + r + (long)c * ldd] = acc;
  }
}

// The single-column fp32 solve with link blocks.  Block row i publishes y_i =
// b_i - sum_{j before i} op(A)(i, j) x_j before it forms x_i = inv(D_i) y_i;
// its successor s reads y_i and multiplies it by G_s = op(A)(s, i) inv(D_i)
// in place of op(A)(s, i) x_i.  y carries its own readiness: the buffer is
// filled with the bit pattern kEmpty before the launch, the producer stores
// plain values (a value with that pattern, a NaN, is stored as another NaN),
// and each consumer thread polls its own element until it changes -- no
// fence, flag or second load on the chain from one block to the next.  x_i
// is then published behind a flag (fx) for the blocks further on; every other
// detail is trsv_ticket_k's.
constexpr unsigned kEmpty = 0xffffffffu;

__device__ __forceinline__ unsigned ld_relaxed_u32(const float *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__global__ void __launch_bounds__(THREADS)
trsv_link_k(int n, int nblk, const float *A, long lda, bool lower_op, bool trans,
            const float *Dinv, long ldd, const float *G, const float *b, float *x, float *ybuf,
            int *ticket, int *fx, int *status, bool vec_ok, bool g_ok) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  float *Ds = reinterpret_cast<float *>(dyn_smem);  // TB x TB inverse diagonal block
  __shared__ float xs[TB];
  __shared__ float part[2][TB];
  __shared__ float red[8][TB];
  __shared__ int s_blk, s_bad;
  const int r = threadIdx.x % TB, half = threadIdx.x / TB;
  for (;;) {
    if (threadIdx.x == 0) {
      s_blk = atomicAdd(ticket, 1);
      s_bad = 0;
    }
    __syncthreads();
    const int q = s_blk;
    if (q >= nblk) return;
    const int i = lower_op ? q : nblk - 1 - q;
    const long r0 = (long)i * TB;
    const int nbi = min(TB, n - (int)r0);
    const int rg = threadIdx.x & 31, cg = threadIdx.x >> 5;
    float acc4[4] = {0.f, 0.f, 0.f, 0.f};
    float acc = 0.f;
    for (int u = threadIdx.x; u < TB * TB / 4; u += THREADS) {
      const int c = u / (TB / 4), r4 = (u % (TB / 4)) * 4;
      cp_async16(&Ds[c * TB + r4], Dinv + (r0 + r4) + (long)c * ldd);
    }
    cp_async_commit();
    for (int s = 0; s < q; s++) {
      const int j = lower_op ? s : nblk - 1 - s;
      const bool link = s == q - 1;  // the block solved just before i: G_i and y_j
      const long c0 = (long)j * TB;
      const int nbj = min(TB, n - (int)c0);
      const bool full = nbi == TB && nbj == TB && (link ? g_ok : vec_ok);
      const bool ntr = link || !trans;  // G is stored untransposed
      float4 v[16];
      if (full) {
        const float *base = link ? G + (r0 + 4 * rg) + (long)(16 * cg) * ldd
                            : trans ? A + (r0 + r) * lda + c0 + 64 * half
                                    : A + (r0 + 4 * rg) + (c0 + 16 * cg) * lda;
        const long step = link ? ldd : trans ? 4 : lda;
#pragma unroll
        for (int u = 0; u < 16; u++) v[u] = *reinterpret_cast<const float4 *>(base + u * step);
      }
      if (link) {  // each thread waits for its own element of y_j
        if (threadIdx.x < nbj) {
          long spins = 0;
          unsigned u;
          while ((u = ld_relaxed_u32(&ybuf[c0 + threadIdx.x])) == kEmpty) {
            if (++spins > kSpin || *(volatile int *)status != PLA_K_OK) {
              atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
              s_bad = 1;
              break;
            }
            __nanosleep(32);
          }
          xs[threadIdx.x] = __uint_as_float(u);
        }
        __syncthreads();
        if (s_bad) return;
      } else {
        if (threadIdx.x == 0) {
          long spins = 0;
          while (ld_acquire(&fx[j]) == 0) {
            if (++spins > kSpin || *(volatile int *)status != PLA_K_OK) {
              atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
              s_bad = 1;
              break;
            }
            __nanosleep(32);
          }
        }
        __syncthreads();
        if (s_bad) return;
        if (threadIdx.x < nbj) xs[threadIdx.x] = __ldcg(&x[c0 + threadIdx.x]);
        __syncthreads();
      }
      if (full && ntr) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const float xv = xs[16 * cg + u];
          acc4[0] += v[u].x * xv;
          acc4[1] += v[u].y * xv;
          acc4[2] += v[u].z * xv;
          acc4[3] += v[u].w * xv;
        }
      } else if (full) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int c = 64 * half + 4 * u;
          acc += v[u].x * xs[c] + v[u].y * xs[c + 1] + v[u].z * xs[c + 2] + v[u].w * xs[c + 3];
        }
      } else if (r < nbi) {
        if (link) {
          for (int c = half; c < nbj; c += 2) acc += G[(r0 + r) + (long)c * ldd] * xs[c];
        } else if (!trans) {
          for (int c = half; c < nbj; c += 2) acc += A[(r0 + r) + (c0 + c) * lda] * xs[c];
        } else {
          const int cb = half * (TB / 2), ce = min(cb + TB / 2, nbj);
          const float *col = A + (r0 + r) * lda + c0;
          for (int c = cb; c < ce; c++) acc += col[c] * xs[c];
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int e = 0; e < 4; e++) red[cg][4 * rg + e] = acc4[e];
    part[half][r] = acc;
    __syncthreads();
    if (threadIdx.x < TB) {
      float sacc = part[0][r] + part[1][r];
#pragma unroll
      for (int g = 0; g < 8; g++) sacc += red[g][r];
      const float y = r < nbi ? b[r0 + r] - sacc : 0.f;
      xs[threadIdx.x] = y;
      if (r < nbi)  // the successor may start
        ybuf[r0 + r] = __float_as_uint(y) == kEmpty ? __uint_as_float(0x7fffffffu) : y;
    }
    __syncthreads();
    // x_i = inv(D_i) y_i, for the blocks further on
    cp_async_wait_all();
    __syncthreads();
    {
      float y4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const float4 d = *reinterpret_cast<const float4 *>(&Ds[(16 * cg + u) * TB + 4 * rg]);
        const float xv = xs[16 * cg + u];
        y4[0] += d.x * xv;
        y4[1] += d.y * xv;
        y4[2] += d.z * xv;
        y4[3] += d.w * xv;
      }
#pragma unroll
      for (int e = 0; e < 4; e++) red[cg][4 * rg + e] = y4[e];
    }
    __syncthreads();
    if (threadIdx.x < nbi) {
      float y = 0.f;
#pragma unroll
      for (int g = 0; g < 8; g++) y += red[g][threadIdx.x];
      x[r0 + threadIdx.x] = y;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&fx[i], 1);
  }
}

// The same solve for several right-hand sides (fp32): X := inv(op(A)) B, B
// and X n x nrhs.  The columns form groups of NR (blockIdx.y); each group is
// an independent ticket chain with its own counter and flags, and the groups'
// CTAs run side by side.  Within a group every tile of A is loaded once and
// multiplied into NR accumulators per thread; the reduction buffers and the
// group's block of right-hand sides are in dynamic shared memory (Ds TB x TB
// | red NR x 8 x TB | xs NR x TB | part 2 x NR x TB), so a block row costs the
// single-column number of barriers.  Groups of 4 keep each chain's serial
// step (the last tile, the reduction and the inverse block, per column) short:
// at n = 32768, 16 columns as one chain took 2.73 ms, as four chains 1.81 ms.
// T: the right-hand sides' and the arithmetic's type, float or double (the
// factor A is fp32 either way; Dinv is of type T)
template <typename T>
struct Four {
  T x, y, z, w;
};
template <typename T>
__device__ __forceinline__ Four<T> ld_four(const T *p) {
  if constexpr (sizeof(T) == 4) {
    const float4 f = *reinterpret_cast<const float4 *>(p);
    return {f.x, f.y, f.z, f.w};
  } else {
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    const double2 b = reinterpret_cast<const double2 *>(p)[1];
    return {a.x, a.y, b.x, b.y};
  }
}

template <int NR, typename T>
__global__ void __launch_bounds__(THREADS)
trsv_ticket_nr_k(int n, int nblk, int nrhs, const float *A, long lda, bool lower_op, bool trans,
                 const T *Dinv, long ldd, const T *B, long ldb, T *X, long ldx,
                 int *ticket, int *flags, int *status, bool vec_ok) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  T *Ds = reinterpret_cast<T *>(dyn_smem);
  T *red = Ds + TB * TB;
  T *xs = red + NR * 8 * TB;
  T *part = xs + NR * TB;
  __shared__ int s_blk, s_bad;
  const int r = threadIdx.x % TB, half = threadIdx.x / TB;
  const int rg = threadIdx.x & 31, cg = threadIdx.x >> 5;
  {  // this CTA's group of columns and its chain
    const int grp = blockIdx.y;
    B += (long)grp * NR * ldb;
    X += (long)grp * NR * ldx;
    nrhs -= grp * NR;
    ticket += grp;
    flags += (long)grp * nblk;
  }
  for (;;) {
    if (threadIdx.x == 0) {
      s_blk = atomicAdd(ticket, 1);
      s_bad = 0;
    }
    __syncthreads();
    const int q = s_blk;
    if (q >= nblk) return;
    const int i = lower_op ? q : nblk - 1 - q;
    const long r0 = (long)i * TB;
    const int nbi = min(TB, n - (int)r0);
    T acc4[NR][4], acc[NR];
#pragma unroll
    for (int k = 0; k < NR; k++) {
      acc[k] = T(0);
#pragma unroll
      for (int e = 0; e < 4; e++) acc4[k][e] = T(0);
    }
    constexpr int kv = 16 / sizeof(T);  // elements per 16-byte copy
    for (int u = threadIdx.x; u < TB * TB / kv; u += THREADS) {
      const int c = u / (TB / kv), rk = (u % (TB / kv)) * kv;
      cp_async16(&Ds[c * TB + rk], Dinv + (r0 + rk) + (long)c * ldd);
    }
    cp_async_commit();
    for (int s = 0; s < q; s++) {
      const int j = lower_op ? s : nblk - 1 - s;
      const long c0 = (long)j * TB;
      const int nbj = min(TB, n - (int)c0);
      const bool full = nbi == TB && nbj == TB && vec_ok;
      float4 v[16];
      if (full) {
        const float *base = trans ? A + (r0 + r) * lda + c0 + 64 * half
                                  : A + (r0 + 4 * rg) + (c0 + 16 * cg) * lda;
        const long step = trans ? 4 : lda;
#pragma unroll
        for (int u = 0; u < 16; u++) v[u] = *reinterpret_cast<const float4 *>(base + u * step);
      }
      if (threadIdx.x == 0) {
        long spins = 0;
        while (ld_acquire(&flags[j]) == 0) {
          if (++spins > kSpin || *(volatile int *)status != PLA_K_OK) {
            atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
            s_bad = 1;
            break;
          }
          __nanosleep(32);
        }
      }
      __syncthreads();
      if (s_bad) return;
      for (int t = threadIdx.x; t < NR * TB; t += THREADS) {
        const int k = t / TB, c = t % TB;
        xs[t] = k < nrhs && c < nbj ? __ldcg(&X[c0 + c + (long)k * ldx]) : T(0);
      }
      __syncthreads();
      if (full && !trans) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
#pragma unroll
          for (int k = 0; k < NR; k++) {
            const T xv = xs[k * TB + 16 * cg + u];
            acc4[k][0] += v[u].x * xv;
            acc4[k][1] += v[u].y * xv;
            acc4[k][2] += v[u].z * xv;
            acc4[k][3] += v[u].w * xv;
          }
        }
      } else if (full) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int c = 64 * half + 4 * u;
#pragma unroll
          for (int k = 0; k < NR; k++) {
            const T *xk = xs + k * TB + c;
            acc[k] += v[u].x * xk[0] + v[u].y * xk[1] + v[u].z * xk[2] + v[u].w * xk[3];
          }
        }
      } else if (r < nbi) {
        if (!trans) {
          for (int c = half; c < nbj; c += 2) {
            const float a = A[(r0 + r) + (c0 + c) * lda];
#pragma unroll
            for (int k = 0; k < NR; k++) acc[k] += a * xs[k * TB + c];
          }
        } else {
          const int cb = half * (TB / 2), ce = min(cb + TB / 2, nbj);
          const float *col = A + (r0 + r) * lda + c0;
          for (int c = cb; c < ce; c++) {
            const float a = col[c];
#pragma unroll
            for (int k = 0; k < NR; k++) acc[k] += a * xs[k * TB + c];
          }
        }
      }
      __syncthreads();
    }
    // reduce the 8 column groups and the two halves, then y = b - sum
#pragma unroll
    for (int k = 0; k < NR; k++) {
#pragma unroll
      for (int e = 0; e < 4; e++) red[(k * 8 + cg) * TB + 4 * rg + e] = acc4[k][e];
      part[(half * NR + k) * TB + r] = acc[k];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NR * TB; t += THREADS) {
      const int k = t / TB, row = t % TB;
      T sacc = part[k * TB + row] + part[(NR + k) * TB + row];
#pragma unroll
      for (int g = 0; g < 8; g++) sacc += red[(k * 8 + g) * TB + row];
      xs[t] = row < nbi && k < nrhs ? B[r0 + row + (long)k * ldb] - sacc : T(0);
    }
    cp_async_wait_all();
    __syncthreads();
    // x_i = inv(D_i) y for every column, with the inverse block from shared memory
    {
      T y4[NR][4];
#pragma unroll
      for (int k = 0; k < NR; k++)
#pragma unroll
        for (int e = 0; e < 4; e++) y4[k][e] = T(0);
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const Four<T> d = ld_four(&Ds[(16 * cg + u) * TB + 4 * rg]);
#pragma unroll
        for (int k = 0; k < NR; k++) {
          const T xv = xs[k * TB + 16 * cg + u];
          y4[k][0] += d.x * xv;
          y4[k][1] += d.y * xv;
          y4[k][2] += d.z * xv;
          y4[k][3] += d.w * xv;
        }
      }
#pragma unroll
      for (int k = 0; k < NR; k++)
#pragma unroll
        for (int e = 0; e < 4; e++) red[(k * 8 + cg) * TB + 4 * rg + e] = y4[k][e];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NR * TB; t += THREADS) {
      const int k = t / TB, row = t % TB;
      if (k >= nrhs || row >= nbi) continue;
      T y = T(0);
#pragma unroll
      for (int g = 0; g < 8; g++) y += red[(k * 8 + g) * TB + row];
      X[r0 + row + (long)k * ldx] = y;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&flags[i], 1);
  }
}

// The FP64 form: 64 x 64 blocks (a 64 x 64 FP64 inverse is 32 KB), each tile
// read as 8 independent 16-byte loads per thread.  No transpose: thread
// (rg, cg) owns rows 2rg, 2rg+1 and columns 8cg .. 8cg+7; transpose: thread
// (r, quarter) reads 16 contiguous values of column r of A.
__global__ void __launch_bounds__(THREADS)
trsv_ticket64_k(int n, int nblk, const double *A, long lda, bool lower_op, bool trans,
                const double *Dinv, long ldd, const double *b, double *x, int *ticket, int *flags,
                int *status, bool vec_ok) {
  constexpr int T64 = TB64;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  double *Ds = reinterpret_cast<double *>(dyn_smem);  // T64 x T64 inverse diagonal block
  __shared__ double xs[T64];
  __shared__ double part[4][T64];
  __shared__ double red[8][T64];
  __shared__ int s_blk, s_bad;
  const int r = threadIdx.x % T64, quarter = threadIdx.x / T64;
  const int rg = threadIdx.x & 31, cg = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) {
      s_blk = atomicAdd(ticket, 1);
      s_bad = 0;
    }
    __syncthreads();
    const int q = s_blk;
    if (q >= nblk) return;
    const int i = lower_op ? q : nblk - 1 - q;
    const long r0 = (long)i * T64;
    const int nbi = min(T64, n - (int)r0);
    double acc2[2] = {0.0, 0.0};
    double acc = 0.0;
    for (int u = threadIdx.x; u < T64 * T64 / 2; u += THREADS) {
      const int c = u / (T64 / 2), r2 = (u % (T64 / 2)) * 2;
      cp_async16(&Ds[c * T64 + r2], Dinv + (r0 + r2) + (long)c * ldd);
    }
    cp_async_commit();
    for (int s2 = 0; s2 < q; s2++) {
      const int j = lower_op ? s2 : nblk - 1 - s2;
      const long c0 = (long)j * T64;
      const int nbj = min(T64, n - (int)c0);
      const bool full = nbi == T64 && nbj == T64 && vec_ok;
      // the tile does not depend on x_j: its loads are issued before waiting
      double2 v[8];
      if (full) {
        const double *base = trans ? A + (r0 + r) * lda + c0 + 16 * quarter
                                   : A + (r0 + 2 * rg) + (c0 + 8 * cg) * lda;
        const long step = trans ? 2 : lda;
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = *reinterpret_cast<const double2 *>(base + u * step);
      }
      if (threadIdx.x == 0) {
        long spins = 0;
        while (ld_acquire(&flags[j]) == 0) {
          if (++spins > kSpin || *(volatile int *)status != PLA_K_OK) {
            atomicCAS(status, PLA_K_OK, PLA_K_TIMEOUT);
            s_bad = 1;
            break;
          }
          __nanosleep(32);
        }
      }
      __syncthreads();
      if (s_bad) return;
      if (threadIdx.x < nbj) xs[threadIdx.x] = __ldcg(&x[c0 + threadIdx.x]);
      __syncthreads();
      if (full && !trans) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const double xv = xs[8 * cg + u];
          acc2[0] += v[u].x * xv;
          acc2[1] += v[u].y * xv;
        }
      } else if (full) {
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const int c = 16 * quarter + 2 * u;
          acc += v[u].x * xs[c] + v[u].y * xs[c + 1];
        }
      } else if (r < nbi) {
        if (!trans) {
          for (int c = quarter; c < nbj; c += 4) acc += A[(r0 + r) + (c0 + c) * lda] * xs[c];
        } else {
          const int cb = quarter * (T64 / 4), ce = min(cb + T64 / 4, nbj);
          const double *col = A + (r0 + r) * lda + c0;
          for (int c = cb; c < ce; c++) acc += col[c] * xs[c];
        }
      }
      __syncthreads();
    }
    red[cg][2 * rg] = acc2[0];
    red[cg][2 * rg + 1] = acc2[1];
    part[quarter][r] = acc;
    __syncthreads();
    if (threadIdx.x < T64) {
      double sacc = part[0][r] + part[1][r] + part[2][r] + part[3][r];
#pragma unroll
      for (int g = 0; g < 8; g++) sacc += red[g][r];
      xs[threadIdx.x] = r < nbi ? b[r0 + r] - sacc : 0.0;
    }
    __syncthreads();
    cp_async_wait_all();
    __syncthreads();
    {
      double y2[2] = {0.0, 0.0};
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const double2 d = *reinterpret_cast<const double2 *>(&Ds[(8 * cg + u) * T64 + 2 * rg]);
        const double xv = xs[8 * cg + u];
        y2[0] += d.x * xv;
        y2[1] += d.y * xv;
      }
      red[cg][2 * rg] = y2[0];
      red[cg][2 * rg + 1] = y2[1];
    }
    __syncthreads();
    if (threadIdx.x < nbi) {
      double y = 0.0;
#pragma unroll
      for (int g = 0; g < 8; g++) y += red[g][threadIdx.x];
      x[r0 + threadIdx.x] = y;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) st_release(&flags[i], 1);
  }
}

void *g_flags = nullptr;
size_t g_flags_bytes = 0;

int *flags_for(int nblk) {
  size_t need = (size_t)(nblk + 8) * sizeof(int);
  if (g_flags_bytes < need) {
    if (g_flags) cudaFree(g_flags);
    g_flags = nullptr;
    g_flags_bytes = 0;
    if (cudaMalloc(&g_flags, need) != cudaSuccess) return nullptr;
    g_flags_bytes = need;
  }
  return (int *)g_flags;
}

int g_sms = 0;

template <typename TA, typename T, int TBK>
int inv_blocks(char uplo, char trans, char diag, int n, const void *A, long lda, void *Dinv,
               long ldd, cudaStream_t s) {
  const bool tr = trans != 'N', lower_op = (uplo == 'L') != tr, unit = diag == 'U';
  const int nblk = (n + TBK - 1) / TBK;
  const size_t sm = ((size_t)TBK * (TBK + 1) * sizeof(TA) + 15) / 16 * 16 +
                    (size_t)TBK * (TBK + 1) * sizeof(T);
  cudaFuncSetAttribute(tri_inv_blocks_k<TA, T, TBK>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  tri_inv_blocks_k<TA, T, TBK><<<nblk, THREADS, sm, s>>>(n, (const TA *)A, lda, lower_op, tr,
                                                         unit, (T *)Dinv, ldd);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

template <typename T>
int ticket_solve(char uplo, char trans, int n, const void *A, long lda, const void *Dinv,
                 long ldd, const void *b, void *x, int *status, cudaStream_t s) {
  const bool tr = trans != 'N', lower_op = (uplo == 'L') != tr;
  const int nblk = (n + TB - 1) / TB;
  int *fl = flags_for(nblk);
  if (!fl) return (int)cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemsetAsync(fl, 0, (size_t)(nblk + 8) * sizeof(int), s);
  if (e) return (int)e;
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  if (ldd % TB || (uintptr_t)Dinv % 16) return (int)cudaErrorMisalignedAddress;
  const bool vec_ok = lda % 4 == 0 && (uintptr_t)A % 16 == 0;
  int grid = nblk < 3 * g_sms ? nblk : 3 * g_sms;
  const size_t dyn = (size_t)TB * TB * sizeof(T);
  cudaFuncSetAttribute(trsv_ticket_k<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  trsv_ticket_k<T><<<grid, THREADS, dyn, s>>>(n, nblk, (const T *)A, lda, lower_op, tr,
                                            (const T *)Dinv, ldd, (const T *)b, (T *)x,
                                            fl + nblk, fl, status, vec_ok);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

template <int NR, typename T>
int ticket_solve_nr(char uplo, char trans, int n, int nrhs, const float *A, long lda,
                    const T *Dinv, long ldd, const T *B, long ldb, T *X, long ldx,
                    int *status, cudaStream_t s) {
  const bool tr = trans != 'N', lower_op = (uplo == 'L') != tr;
  const int nblk = (n + TB - 1) / TB, groups = (nrhs + NR - 1) / NR;
  // flags of group g at [g nblk, (g + 1) nblk), its ticket at groups nblk + g
  int *fl = flags_for(groups * nblk + groups);
  if (!fl) return (int)cudaErrorMemoryAllocation;
  cudaError_t e =
      cudaMemsetAsync(fl, 0, (size_t)(groups * nblk + groups + 8) * sizeof(int), s);
  if (e) return (int)e;
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  if (ldd % TB || (uintptr_t)Dinv % 16) return (int)cudaErrorMisalignedAddress;
  const bool vec_ok = lda % 4 == 0 && (uintptr_t)A % 16 == 0;
  // two CTAs per SM fit in fp32, one in FP64 (the ticket order needs no
  // co-residency either way)
  int per = (sizeof(T) == 4 ? 2 : 1) * g_sms / groups;
  if (per < 1) per = 1;
  const dim3 grid(nblk < per ? nblk : per, groups);
  const size_t dyn = ((size_t)TB * TB + (size_t)NR * 8 * TB + (size_t)NR * TB + 2 * NR * TB) *
                     sizeof(T);
  cudaFuncSetAttribute(trsv_ticket_nr_k<NR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)dyn);
  trsv_ticket_nr_k<NR, T><<<grid, THREADS, dyn, s>>>(n, nblk, nrhs, A, lda, lower_op, tr, Dinv,
                                                     ldd, B, ldb, X, ldx, fl + groups * nblk, fl,
                                                     status, vec_ok);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

int ticket_solve64(char uplo, char trans, int n, const void *A, long lda, const void *Dinv,
                   long ldd, const void *b, void *x, int *status, cudaStream_t s) {
  const bool tr = trans != 'N', lower_op = (uplo == 'L') != tr;
  const int nblk = (n + TB64 - 1) / TB64;
  int *fl = flags_for(nblk);
  if (!fl) return (int)cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemsetAsync(fl, 0, (size_t)(nblk + 8) * sizeof(int), s);
  if (e) return (int)e;
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  if (ldd % TB64 || (uintptr_t)Dinv % 16) return (int)cudaErrorMisalignedAddress;
  const bool vec_ok = lda % 2 == 0 && (uintptr_t)A % 16 == 0;
  int grid = nblk < 3 * g_sms ? nblk : 3 * g_sms;
  const size_t dyn = (size_t)TB64 * TB64 * sizeof(double);
  trsv_ticket64_k<<<grid, THREADS, dyn, s>>>(n, nblk, (const double *)A, lda, lower_op, tr,
                                             (const double *)Dinv, ldd, (const double *)b,
                                             (double *)x, fl + nblk, fl, status, vec_ok);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

int link_blocks(char uplo, char trans, int n, const float *A, long lda, const float *Dinv,
                long ldd, float *G, cudaStream_t s) {
  const bool tr = trans != 'N', lower_op = (uplo == 'L') != tr;
  const int nblk = (n + TB - 1) / TB;
  if (nblk < 2) return 0;
  if (ldd % TB) return (int)cudaErrorMisalignedAddress;
  const size_t sm = (size_t)2 * TB * (TB + 1) * sizeof(float);
  cudaFuncSetAttribute(link_blocks_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  link_blocks_k<<<nblk - 1, THREADS, sm, s>>>(n, nblk, A, lda, lower_op, tr, Dinv, ldd, G);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

int ticket_solve_link(char uplo, char trans, int n, const float *A, long lda, const float *Dinv,
                      long ldd, const float *G, const float *b, float *x, int *status,
                      cudaStream_t s) {
  const bool tr = trans != 'N', lower_op = (uplo == 'L') != tr;
  const int nblk = (n + TB - 1) / TB;
  // fx, the ticket, then y (n floats, filled with the bit pattern kEmpty)
  const int nflags = nblk + 8;
  int *fl = flags_for(nflags + n);
  if (!fl) return (int)cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemsetAsync(fl, 0, (size_t)nflags * sizeof(int), s);
  if (e) return (int)e;
  e = cudaMemsetAsync(fl + nflags, 0xff, (size_t)n * sizeof(float), s);
  if (e) return (int)e;
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  if (ldd % TB || (uintptr_t)Dinv % 16 || (uintptr_t)G % 16) return (int)cudaErrorMisalignedAddress;
  const bool vec_ok = lda % 4 == 0 && (uintptr_t)A % 16 == 0;
  int grid = nblk < 3 * g_sms ? nblk : 3 * g_sms;
  const size_t dyn = (size_t)TB * TB * sizeof(float);
  cudaFuncSetAttribute(trsv_link_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  trsv_link_k<<<grid, THREADS, dyn, s>>>(n, nblk, A, lda, lower_op, tr, Dinv, ldd, G, b, x,
                                         reinterpret_cast<float *>(fl + nflags), fl + nblk, fl,
                                         status, vec_ok, true);
  pla_k_count(1);
  return (int)cudaGetLastError();
}

}  // namespace

// Dinv must hold ldd x TB elements with ldd >= n rounded up to TB (TB = 128
// for fp32, 64 for FP64).
extern "C" int pla_k_trsv_inv_blocks(int dt, char uplo, char trans, char diag, int n,
                                     const void *A, long lda, void *Dinv, long ldd,
                                     cudaStream_t s) {
  if (n <= 0) return 0;
  if (dt == MPI_FLOAT)
    return inv_blocks<float, float, TB>(uplo, trans, diag, n, A, lda, Dinv, ldd, s);
  if (dt == MPI_DOUBLE)
    return inv_blocks<double, double, TB64>(uplo, trans, diag, n, A, lda, Dinv, ldd, s);
  return (int)cudaErrorInvalidValue;
}

// FP64 inverses (128 x 128 blocks, ldd a multiple of 128) of an fp32 factor's
// diagonal blocks, for pla_k_trsv_ticket_multi_f64
extern "C" int pla_k_trsv_inv_blocks_f64(char uplo, char trans, char diag, int n,
                                         const float *A, long lda, double *Dinv, long ldd,
                                         cudaStream_t s) {
  if (n <= 0) return 0;
  return inv_blocks<float, double, TB>(uplo, trans, diag, n, A, lda, Dinv, ldd, s);
}

extern "C" int pla_k_trsv_ticket(int dt, char uplo, char trans, int n, const void *A, long lda,
                                 const void *Dinv, long ldd, const void *b, void *x, int *status,
                                 cudaStream_t s) {
  if (n <= 0) return 0;
  if (dt == MPI_FLOAT)
    return ticket_solve<float>(uplo, trans, n, A, lda, Dinv, ldd, b, x, status, s);
  if (dt == MPI_DOUBLE) return ticket_solve64(uplo, trans, n, A, lda, Dinv, ldd, b, x, status, s);
  return (int)cudaErrorInvalidValue;
}

// X := inv(op(A)) B for nrhs <= 16 fp32 right-hand sides in one launch (B and
// X may be the same array); Dinv as for pla_k_trsv_ticket
extern "C" int pla_k_trsv_ticket_multi(char uplo, char trans, int n, int nrhs, const float *A,
                                       long lda, const float *Dinv, long ldd, const float *B,
                                       long ldb, float *X, long ldx, int *status,
                                       cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return 0;
  if (nrhs > 16) return (int)cudaErrorInvalidValue;
  return ticket_solve_nr<4, float>(uplo, trans, n, nrhs, A, lda, Dinv, ldd, B, ldb, X, ldx,
                                   status, s);
}

// The same with FP64 right-hand sides and arithmetic on the fp32 factor
// (the factor read once, 4 bytes an element): X := inv(op(A)) B for nrhs <=
// 16, Dinv from pla_k_trsv_inv_blocks_f64
extern "C" int pla_k_trsv_ticket_multi_f64(char uplo, char trans, int n, int nrhs,
                                           const float *A, long lda, const double *Dinv,
                                           long ldd, const double *B, long ldb, double *X,
                                           long ldx, int *status, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return 0;
  if (nrhs > 16) return (int)cudaErrorInvalidValue;
  return ticket_solve_nr<4, double>(uplo, trans, n, nrhs, A, lda, Dinv, ldd, B, ldb, X, ldx,
                                    status, s);
}

// The link blocks G of an fp32 triangle (ldd x TB floats, the layout of its
// Dinv), for pla_k_trsv_ticket_link
extern "C" int pla_k_trsv_link_blocks(char uplo, char trans, int n, const float *A, long lda,
                                      const float *Dinv, long ldd, float *G, cudaStream_t s) {
  if (n <= 0) return 0;
  return link_blocks(uplo, trans, n, A, lda, Dinv, ldd, G, s);
}

// x := inv(op(A)) b (fp32, one column, b and x may be the same array) with the
// link blocks: the chain between consecutive blocks skips the inverse-block
// product
extern "C" int pla_k_trsv_ticket_link(char uplo, char trans, int n, const float *A, long lda,
                                      const float *Dinv, long ldd, const float *G,
                                      const float *b, float *x, int *status, cudaStream_t s) {
  if (n <= 0) return 0;
  return ticket_solve_link(uplo, trans, n, A, lda, Dinv, ldd, G, b, x, status, s);
}

extern "C" void pla_trsv_release(void) {
  if (g_flags) cudaFree(g_flags);
  g_flags = nullptr;
  g_flags_bytes = 0;
}
