// Out-of-core matrices and the out-of-core Cholesky factorization.
//
// The reference keeps an out-of-core matrix in a file: PLA_File_create /
// open / close / unlink (IO/PLA_File.c:25-75), an object without a buffer
// (OBJ/PLA_Obj_ooc.c:50-72) to which the file is attached
// (OBJ/PLA_Obj_management.c:146-166), and PLA_Copy moving tiles between the
// file and in-core objects.  PLA_OOC_Chol factors such a matrix with the
// left-looking tile algorithm of POOCLAPACK (Reiley and van de Geijn,
// "POOCLAPACK: Parallel Out-of-Core Linear Algebra Package", 1999):
//
//   for each diagonal tile A11 (nb_tile rows):
//     A11 <- A11 - L10 L10'            L10: the tile's rows left of it
//     A11 <- L11 = chol(A11)
//     for each tile A21 below it:
//       A21 <- A21 - L20 L10'          L20: that tile's rows left of it
//       A21 <- L21 = A21 inv(L11')
//
// Here the file (or a file in host memory, such as one under /dev/shm) is
// the slow memory and the GPU's HBM the fast one.  Tiles and K-chunks of L10
// and L20 move file -> pinned host buffer -> HBM; the products run on the
// device GEMM, the tile factorization on the in-core Cholesky and the solve
// on the device TRSM.  L10 stays resident in HBM for the whole tile column
// when it fits a budget (otherwise it is streamed with L20).  While the GPU
// multiplies chunk c the host reads chunk c + 1 from the file and queues its
// copy on the copy stream: two pinned staging buffers and two device chunk
// buffers alternate, each reused only after the event of its last use.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "pla_internal.h"
#include "pla_kernels.h"

using namespace pla;

namespace pla {
int chol_on_device(int dt, int n, char *A, long lda, int nb, int *info_host);
int trsm_device(int dt, char side, char uplo, char trans, char diag, int nt, int other,
                double alpha, const char *T, long ldt, char *B, long ldb);
}  // namespace pla

namespace {

// IO/PLA_File_stats.c: bytes and seconds of file reads and writes while
// collection is on
struct IoStats {
  bool on = false;
  double read_bytes = 0, read_s = 0, write_bytes = 0, write_s = 0;
};
IoStats g_io;

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// one contiguous range; false on an error
bool pread_all(int fd, char *dst, size_t bytes, off_t off) {
  size_t done = 0;
  while (done < bytes) {
    const ssize_t r = pread(fd, dst + done, bytes - done, off + (off_t)done);
    if (r < 0) return false;
    if (r == 0) {  // past the end of the file: never written, reads as zero
      std::memset(dst + done, 0, bytes - done);
      break;
    }
    done += (size_t)r;
  }
  return true;
}
bool pwrite_all(int fd, const char *src, size_t bytes, off_t off) {
  size_t done = 0;
  while (done < bytes) {
    const ssize_t r = pwrite(fd, src + done, bytes - done, off + (off_t)done);
    if (r <= 0) return false;
    done += (size_t)r;
  }
  return true;
}

// A file region of `count` pieces of `piece` bytes, piece k at file offset
// off + k * stride and at buffer offset k * piece, moved by up to kIoThreads
// host threads: one thread copies from the page cache (or tmpfs) at a few
// GB/s, several at the host's memory bandwidth.
constexpr int kIoThreads = 8;
constexpr size_t kIoSplit = size_t(4) << 20;  // bytes below which one thread moves it all

template <typename Op>
bool io_pieces(long count, size_t piece, off_t off, off_t stride, Op op) {
  const size_t total = (size_t)count * piece;
  int nt = (int)std::min<size_t>(kIoThreads, total / kIoSplit);
  if (nt <= 1) {
    for (long k = 0; k < count; k++)
      if (!op(k * piece, piece, off + (off_t)k * stride)) return false;
    return true;
  }
  // split the pieces, or, for one large piece, its bytes
  std::atomic<bool> ok{true};
  std::vector<std::thread> th;
  if (count >= nt) {
    for (int w = 0; w < nt; w++)
      th.emplace_back([&, w] {
        for (long k = count * w / nt; k < count * (w + 1) / nt && ok; k++)
          if (!op(k * piece, piece, off + (off_t)k * stride)) ok = false;
      });
  } else {
    for (long k = 0; k < count; k++) {
      const size_t part = (piece + nt - 1) / nt;
      for (int w = 0; w < nt; w++) {
        const size_t b0 = (size_t)w * part, b1 = std::min(piece, b0 + part);
        if (b0 >= b1) break;
        th.emplace_back([&, k, b0, b1] {
          if (!op(k * piece + b0, b1 - b0, off + (off_t)k * stride + (off_t)b0)) ok = false;
        });
      }
      for (std::thread &t : th) t.join();
      th.clear();
    }
  }
  for (std::thread &t : th) t.join();
  return ok;
}

// The file of the current out-of-core call mapped into memory (MapScope):
// parallel writes through pwrite queue on the file's inode lock, copies into
// a shared mapping only take page locks.  Ranges outside it use pread/pwrite.
struct FileMap {
  int fd = -1;
  char *base = nullptr;
  size_t len = 0;
};
FileMap g_map;

struct MapScope {
  bool mine = false;
  explicit MapScope(int fd) {
    if (g_map.fd != -1) return;
    struct stat st;
    if (fstat(fd, &st) != 0 || st.st_size <= 0) return;
    void *p = mmap(nullptr, (size_t)st.st_size, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    if (p == MAP_FAILED) return;
    g_map.fd = fd;
    g_map.base = (char *)p;
    g_map.len = (size_t)st.st_size;
    mine = true;
  }
  ~MapScope() {
    if (!mine) return;
    munmap(g_map.base, g_map.len);
    g_map = FileMap();
  }
};

bool mapped(int fd, off_t off, size_t bytes) {
  return fd == g_map.fd && off >= 0 && (size_t)off + bytes <= g_map.len;
}

int io_read(int fd, char *dst, long count, size_t piece, off_t off, off_t stride) {
  const double t = now_s();
  const size_t span = count > 0 ? (size_t)(count - 1) * stride + piece : 0;
  if (mapped(fd, off, span)) {
    io_pieces(count, piece, off, stride, [&](size_t at, size_t n, off_t fo) {
      std::memcpy(dst + at, g_map.base + fo, n);
      return true;
    });
  } else if (!io_pieces(count, piece, off, stride, [&](size_t at, size_t n, off_t fo) {
               return pread_all(fd, dst + at, n, fo);
             })) {
    PLA_FAIL("error reading file");
  }
  if (g_io.on) {
    g_io.read_bytes += (double)count * piece;
    g_io.read_s += now_s() - t;
  }
  return PLA_SUCCESS;
}

int io_write(int fd, const char *src, long count, size_t piece, off_t off, off_t stride) {
  const double t = now_s();
  const size_t span = count > 0 ? (size_t)(count - 1) * stride + piece : 0;
  if (mapped(fd, off, span)) {
    io_pieces(count, piece, off, stride, [&](size_t at, size_t n, off_t fo) {
      std::memcpy(g_map.base + fo, src + at, n);
      return true;
    });
  } else if (!io_pieces(count, piece, off, stride, [&](size_t at, size_t n, off_t fo) {
               return pwrite_all(fd, src + at, n, fo);
             })) {
    PLA_FAIL("error writing file");
  }
  if (g_io.on) {
    g_io.write_bytes += (double)count * piece;
    g_io.write_s += now_s() - t;
  }
  return PLA_SUCCESS;
}

#define R(call)         \
  do {                  \
    int r_ = (call);    \
    if (r_) return r_;  \
  } while (0)

// pinned staging buffers and the events of their last copy
constexpr size_t kStageBytes = size_t(64) << 20;
struct Staging {
  char *buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
};
Staging g_stage;

int staging() {
  for (int i = 0; i < 2; i++) {
    if (!g_stage.buf[i]) PLA_CUDA(cudaHostAlloc((void **)&g_stage.buf[i], kStageBytes, 0));
    if (!g_stage.done[i])
      PLA_CUDA(cudaEventCreateWithFlags(&g_stage.done[i], cudaEventDisableTiming));
  }
  return PLA_SUCCESS;
}

// file offset of element (i, j) of an out-of-core view
off_t file_off(PLA_Obj v, long i, long j) {
  return (off_t)(((long)v->row0 + i) + ((long)v->col0 + j) * v->base->ldim) * v->base->esize;
}

// Read the m x n block at (i0, j0) of out-of-core view v into device memory
// dst (leading dimension ldd), in chunks of whole columns through the two
// staging buffers; each chunk's copy is queued on stream s.  The copies may
// still be running on return.
int read_block(PLA_Obj v, long i0, long j0, long m, long n, char *dst, long ldd,
               cudaStream_t s) {
  if (m <= 0 || n <= 0) return PLA_SUCCESS;
  const int es = v->base->esize;
  const long per = std::max(1L, (long)(kStageBytes / ((size_t)m * es)));
  if ((size_t)m * es > kStageBytes) PLA_FAIL("out-of-core tile taller than the staging buffer");
  static int next = 0;
  for (long c0 = 0; c0 < n; c0 += per) {
    const long nc = std::min(per, n - c0);
    const int b = next;
    next ^= 1;
    PLA_CUDA(cudaEventSynchronize(g_stage.done[b]));
    char *h = g_stage.buf[b];
    if (m == v->base->ldim && v->row0 == 0 && i0 == 0) {
      // whole columns of the file: one range
      R(io_read(v->base->fd, h, 1, (size_t)m * nc * es, file_off(v, 0, j0 + c0), 0));
    } else {
      R(io_read(v->base->fd, h, nc, (size_t)m * es, file_off(v, i0, j0 + c0),
                (off_t)v->base->ldim * es));
    }
    PLA_CUDA(cudaMemcpy2DAsync(dst + (size_t)c0 * ldd * es, (size_t)ldd * es, h, (size_t)m * es,
                               (size_t)m * es, nc, cudaMemcpyHostToDevice, s));
    PLA_CUDA(cudaEventRecord(g_stage.done[b], s));
  }
  return PLA_SUCCESS;
}

// Write the m x n device block src (leading dimension lds) to the block at
// (i0, j0) of out-of-core view v, after everything queued on stream s.  The
// copy of chunk c + 1 to the host overlaps the file write of chunk c.
int write_block(PLA_Obj v, long i0, long j0, long m, long n, const char *src, long lds,
                cudaStream_t s) {
  if (m <= 0 || n <= 0) return PLA_SUCCESS;
  const int es = v->base->esize;
  if ((size_t)m * es > kStageBytes) PLA_FAIL("out-of-core tile taller than the staging buffer");
  const long per = std::max(1L, (long)(kStageBytes / ((size_t)m * es)));
  long pending = -1, pending_n = 0;
  int pb = 0;
  auto flush = [&]() -> int {
    if (pending < 0) return PLA_SUCCESS;
    PLA_CUDA(cudaEventSynchronize(g_stage.done[pb]));
    R(io_write(v->base->fd, g_stage.buf[pb], pending_n, (size_t)m * es,
               file_off(v, i0, j0 + pending), (off_t)v->base->ldim * es));
    pending = -1;
    return PLA_SUCCESS;
  };
  int b = 0;
  for (long c0 = 0; c0 < n; c0 += per) {
    const long nc = std::min(per, n - c0);
    PLA_CUDA(cudaEventSynchronize(g_stage.done[b]));
    PLA_CUDA(cudaMemcpy2DAsync(g_stage.buf[b], (size_t)m * es, src + (size_t)c0 * lds * es,
                               (size_t)lds * es, (size_t)m * es, nc, cudaMemcpyDeviceToHost, s));
    PLA_CUDA(cudaEventRecord(g_stage.done[b], s));
    int r = flush();
    if (r) return r;
    pending = c0;
    pending_n = nc;
    pb = b;
    b ^= 1;
  }
  return flush();
}

struct DevBuf {
  char *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int alloc(size_t bytes) {
    PLA_CUDA(cudaMalloc((void **)&p, std::max(bytes, (size_t)16)));
    return PLA_SUCCESS;
  }
};

struct Events {
  cudaEvent_t e[4] = {};
  ~Events() {
    for (cudaEvent_t x : e)
      if (x) cudaEventDestroy(x);
  }
  int create() {
    for (cudaEvent_t &x : e) PLA_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    return PLA_SUCCESS;
  }
};

#define K(call)                                                    \
  do {                                                             \
    int r_ = (call);                                               \
    if (r_) return cuda_fail((cudaError_t)r_, __LINE__, __FILE__); \
  } while (0)
// HBM held for the resident L10 block of one tile column: 16 GB, or the
// bytes in PLA_B200_OOC_RESIDENT_BYTES (0 streams L10 with L20 always)
size_t resident_budget() {
  const char *e = std::getenv("PLA_B200_OOC_RESIDENT_BYTES");
  return e ? (size_t)std::strtoull(e, nullptr, 10) : (size_t(16) << 30);
}

}  // namespace

namespace pla {

// PLA_Copy between an out-of-core view and a device object of the same shape
int ooc_copy(PLA_Obj from, PLA_Obj to) {
  if (from->base->ooc && to->base->ooc) PLA_FAIL("copy between two out-of-core objects");
  PLA_Obj f = from->base->ooc ? from : to, d = from->base->ooc ? to : from;
  if (f->base->fd < 0) PLA_FAIL("out-of-core object without a file");
  if (d->base->on_host) PLA_FAIL("copy between an out-of-core object and a multiscalar");
  if (from->base->datatype != to->base->datatype) PLA_FAIL("datatype mismatch");
  if (from->length != to->length || from->width != to->width) PLA_FAIL("objects do not conform");
  R(staging());
  MapScope map(f->base->fd);
  cudaStream_t s = stream();
  if (from->base->ooc)
    R(read_block(f, 0, 0, f->length, f->width, at(d, 0, 0), ld(d), s));
  else
    R(write_block(f, 0, 0, f->length, f->width, at(d, 0, 0), ld(d), s));
  PLA_CUDA(cudaStreamSynchronize(s));
  return PLA_SUCCESS;
}

void release_ooc() {
  for (int i = 0; i < 2; i++) {
    if (g_stage.done[i]) cudaEventSynchronize(g_stage.done[i]);
    if (g_stage.buf[i]) cudaFreeHost(g_stage.buf[i]);
    if (g_stage.done[i]) cudaEventDestroy(g_stage.done[i]);
    g_stage.buf[i] = nullptr;
    g_stage.done[i] = nullptr;
  }
}

}  // namespace pla

namespace {

// C(m x t) -= X Y' over k columns, X the m x k block of A at (xr, 0) and Y the
// t x k block at (yr, 0).  Y comes from HBM when `yres` holds it (ld t), else
// it is streamed with X; X == Y (the diagonal tile, lower triangle only) when
// xr == yr and uplo == 'L'.  K-chunks of width kc alternate between two
// device buffers; chunk c + 1 is read and copied on the copy stream while the
// GEMM of chunk c runs on the library stream.
int ooc_update(PLA_Obj A, long xr, long yr, int m, int t, long k, const char *yres, char *C,
               long ldc, int uplo, char *dx[2], char *dy[2], long kc, Events &ev) {
  if (k <= 0) return PLA_SUCCESS;
  const int dt = A->base->datatype;
  cudaStream_t s0 = stream(), cs = copy_stream();
  const bool same = xr == yr && uplo == 'L';
  // ev.e[0..1]: chunk in buffer b copied; ev.e[2..3]: GEMM on buffer b done
  for (int b = 0; b < 2; b++) PLA_CUDA(cudaEventRecord(ev.e[2 + b], s0));
  int b = 0;
  const size_t es = A->base->esize;
  for (long p = 0; p < k; p += kc, b ^= 1) {
    const long w = std::min(kc, k - p);
    const char *x, *y;
    if (same && yres) {  // the diagonal tile's L10 is the resident block itself
      x = y = yres + (size_t)p * t * es;
    } else {
      PLA_CUDA(cudaStreamWaitEvent(cs, ev.e[2 + b], 0));
      R(read_block(A, xr, p, m, w, dx[b], m, cs));
      if (!yres && !same) R(read_block(A, yr, p, t, w, dy[b], t, cs));
      PLA_CUDA(cudaEventRecord(ev.e[b], cs));
      PLA_CUDA(cudaStreamWaitEvent(s0, ev.e[b], 0));
      x = dx[b];
      y = yres ? yres + (size_t)p * t * es : same ? dx[b] : dy[b];
    }
    K(pla_k_gemm(dt, PLA_NO_TRANSPOSE, PLA_TRANSPOSE, m, t, (int)w, -1.0, x, m, y, t, 1.0, C, ldc,
                 uplo, nullptr, s0));
    PLA_CUDA(cudaEventRecord(ev.e[2 + b], s0));
  }
  return PLA_SUCCESS;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- files ---
// IO/PLA_File.c:25-45: create (truncate) a file for size elements of datatype
int PLA_File_create(char *filename, MPI_Datatype datatype, int size, int *fd) {
  if (!filename || !fd) PLA_FAIL("PLA_File_create: null argument");
  const int es = esize_of(datatype);
  if (es == 0) PLA_FAIL("PLA_File_create: unsupported datatype");
  *fd = open(filename, O_RDWR | O_CREAT | O_TRUNC, 0700);
  if (*fd == -1) {
    char msg[300];
    std::snprintf(msg, sizeof msg, "Cannot open file %s", filename);
    PLA_FAIL(msg);
  }
  if (size > 0 && ftruncate(*fd, (off_t)size * es) != 0) PLA_FAIL("PLA_File_create: cannot size the file");
  return PLA_SUCCESS;
}

// IO/PLA_File.c:47-58
int PLA_File_open(char *filename, MPI_Datatype datatype, int size, int *fd) {
  (void)datatype;
  (void)size;
  if (!filename || !fd) PLA_FAIL("PLA_File_open: null argument");
  *fd = open(filename, O_RDWR);
  if (*fd == -1) {
    char msg[300];
    std::snprintf(msg, sizeof msg, "Cannot open file %s", filename);
    PLA_FAIL(msg);
  }
  return PLA_SUCCESS;
}

// IO/PLA_File.c:61-70
int PLA_File_close(int fd) {
  if (close(fd) == -1) PLA_FAIL("Trouble closing file");
  return PLA_SUCCESS;
}

// IO/PLA_File.c:72-82
int PLA_File_unlink(char *filename) {
  if (!filename || unlink(filename) == -1) PLA_FAIL("Trouble unlinking file");
  return PLA_SUCCESS;
}

// IO/PLA_File_stats.c:21-90: collect, then print the totals as the reference
int PLA_File_stats_start(void) {
  g_io = IoStats();
  g_io.on = true;
  return PLA_SUCCESS;
}

int PLA_File_stats_stop(void) {
  g_io.on = false;
  const double rm = g_io.read_bytes / 1e6, wm = g_io.write_bytes / 1e6;
  if (g_io.read_s > 0.0)
    std::printf("READ : size(MB)=%4.2lf  time(s)=%4.2lf MB/s=%4.2lf\n", rm, g_io.read_s,
                rm / g_io.read_s);
  if (g_io.write_s > 0.0)
    std::printf("WRITE: size(MB)=%4.2lf time(s)=%4.2lf MB/s=%4.2lf\n", wm, g_io.write_s,
                wm / g_io.write_s);
  if (g_io.read_s + g_io.write_s > 0.0)
    std::printf("BOTH : size(MB)=%4.2lf time(s)=%4.2lf MB/s=%4.2lf\n", rm + wm,
                g_io.read_s + g_io.write_s, (rm + wm) / (g_io.read_s + g_io.write_s));
  return PLA_SUCCESS;
}

int PLA_B200_file_stats(double *read_bytes, double *read_seconds, double *write_bytes,
                        double *write_seconds) {
  if (read_bytes) *read_bytes = g_io.read_bytes;
  if (read_seconds) *read_seconds = g_io.read_s;
  if (write_bytes) *write_bytes = g_io.write_bytes;
  if (write_seconds) *write_seconds = g_io.write_s;
  return PLA_SUCCESS;
}

// ------------------------------------------------------- out-of-core Chol ---
// POOCLAPACK/OOC_Cholesky/PLA_OOC_Chol.c:13: the lower triangle of the
// out-of-core matrix A is overwritten with L.  Returns 0, or (unlike the
// reference, which discards PLA_Chol's value) the global 1-based column whose
// diagonal was not positive, as PLA_Chol does; the factorization stops there.
int PLA_OOC_Chol(int nb_ooc, int nb_tile, PLA_Obj A) {
  if (!valid_any(A) || !A->base->ooc) PLA_FAIL("PLA_OOC_Chol: A must be an out-of-core matrix");
  if (A->base->fd < 0) PLA_FAIL("PLA_OOC_Chol: A has no file attached");
  if (A->length != A->width) PLA_FAIL("PLA_OOC_Chol: A must be square");
  if (A->base->datatype != MPI_DOUBLE && A->base->datatype != MPI_FLOAT)
    PLA_FAIL("PLA_OOC_Chol: datatype not yet supported");
  if (nb_tile <= 0 || nb_ooc <= 0) PLA_FAIL("PLA_OOC_Chol: block sizes must be positive");
  const int n = A->length, dt = A->base->datatype, es = A->base->esize;
  if (n == 0) return PLA_SUCCESS;
  int nb;
  PLA_Environ_nb_alg(PLA_OP_PAN_PAN, A->templ, &nb);
  const int T = std::min(nb_tile, n);
  // K-chunks: a whole number of nb_ooc panels, about 512 MB of a T-row chunk
  long kc = std::max<long>(nb_ooc, ((size_t(512) << 20) / ((size_t)T * es)) / nb_ooc * nb_ooc);
  kc = std::min<long>(kc, std::max(n - T, 1));
  if ((size_t)T * es > kStageBytes) PLA_FAIL("PLA_OOC_Chol: nb_tile too large");
  R(staging());
  DevBuf d11, d21, cx0, cx1, cy0, cy1, res;
  R(d11.alloc((size_t)T * T * es));
  R(d21.alloc((size_t)T * T * es));
  R(cx0.alloc((size_t)T * kc * es));
  R(cx1.alloc((size_t)T * kc * es));
  // L10 of any tile column is at most T x n
  const bool resident = (size_t)T * n * es <= resident_budget();
  if (resident) {
    R(res.alloc((size_t)T * n * es));
  } else {
    R(cy0.alloc((size_t)T * kc * es));
    R(cy1.alloc((size_t)T * kc * es));
  }
  char *dx[2] = {cx0.p, cx1.p}, *dy[2] = {cy0.p, cy1.p};
  Events ev;
  R(ev.create());
  MapScope map(A->base->fd);
  cudaStream_t s0 = stream();
  for (int j0 = 0; j0 < n; j0 += T) {
    const int t = std::min(T, n - j0);
    // L10 (t x j0) resident for this tile column
    const char *yres = nullptr;
    if (resident && j0 > 0) {
      R(read_block(A, j0, 0, t, j0, res.p, t, s0));
      yres = res.p;
    }
    // A11 <- chol(A11 - L10 L10')
    R(read_block(A, j0, j0, t, t, d11.p, t, s0));
    R(ooc_update(A, j0, j0, t, t, j0, yres, d11.p, t, 'L', dx, dy, kc, ev));
    int info = 0;
    R(chol_on_device(dt, t, d11.p, t, nb, &info));
    if (info) {
      PLA_CUDA(cudaStreamSynchronize(copy_stream()));
      return j0 + info;
    }
    R(write_block(A, j0, j0, t, t, d11.p, t, s0));
    // A21 <- (A21 - L20 L10') inv(L11'), one tile of rows at a time
    for (int i0 = j0 + t; i0 < n; i0 += T) {
      const int m = std::min(T, n - i0);
      R(read_block(A, i0, j0, m, t, d21.p, m, s0));
      R(ooc_update(A, i0, j0, m, t, j0, yres, d21.p, m, 0, dx, dy, kc, ev));
      R(trsm_device(dt, 'R', 'L', 'T', 'N', t, m, 1.0, d11.p, t, d21.p, m));
      R(write_block(A, i0, j0, m, t, d21.p, m, s0));
    }
  }
  PLA_CUDA(cudaStreamSynchronize(s0));
  PLA_CUDA(cudaStreamSynchronize(copy_stream()));
  return PLA_SUCCESS;
}

}  // extern "C"
