// Library state, templates, block sizes, diagnostics, objects, views and
// their inquiry functions: the object layer of the reference (OBJ/, TEMPLATE/,
// INCLUDE/PLA_Obj.h) on a 1x1 template with device-resident buffers.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "pla_internal.h"
#include "pla_kernels.h"

namespace pla {

State &state() {
  static State s;
  return s;
}

int esize_of(MPI_Datatype dt) {
  switch (dt) {
    case MPI_CHAR: return 1;
    case MPI_INT: return 4;
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_COMPLEX: return 8;
    case MPI_DOUBLE_COMPLEX: return 16;
    default: return 0;
  }
}

bool valid_any(PLA_Obj o) {
  return o != nullptr && o->magic == kObjMagic && o->base != nullptr;
}
// an object whose data is in device (or pinned host) memory: everything that
// reads or writes the data refuses out-of-core objects, which have none
bool valid(PLA_Obj o) { return valid_any(o) && !o->base->ooc; }
bool valid(PLA_Template t) { return t != nullptr && t->magic == kTempMagic; }

cudaStream_t stream() {
  State &s = state();
  if (s.override_stream) return s.override_stream;
  if (s.stream) return s.stream;
  if (!s.own_stream) cudaStreamCreateWithFlags(&s.own_stream, cudaStreamNonBlocking);
  return s.own_stream;
}

// ------------------------------------------------------- host memory ---
// OBJ/PLA_Memory.c: malloc with running totals of the bytes held.  Each block
// carries its size in a 16-byte header in front of the pointer returned, so
// that PLA_free can subtract it.  A failed allocation returns NULL and sets
// the last error; the reference prints and exits.
std::atomic<long long> g_host_bytes{0}, g_host_bytes_max{0};

void *host_alloc(size_t size, bool zero) {
  void *p = zero ? std::calloc(1, size + 16) : std::malloc(size + 16);
  if (!p) {
    fail("malloc failed in PLA_malloc", __LINE__, __FILE__);
    return nullptr;
  }
  *(size_t *)p = size;
  const long long now = g_host_bytes += (long long)size;
  long long m = g_host_bytes_max.load();
  while (now > m && !g_host_bytes_max.compare_exchange_weak(m, now)) {
  }
  return (char *)p + 16;
}

int lookahead_ctas(int dt) {
  static const int f32 = [] {
    const char *e = std::getenv("PLA_B200_LOOKAHEAD_CTAS_F32");
    const int v = e ? std::atoi(e) : 0;
    return v > 0 ? v : kLookaheadCtasF32Default;
  }();
  static const int f64 = [] {
    const char *e = std::getenv("PLA_B200_LOOKAHEAD_CTAS_F64");
    const int v = e ? std::atoi(e) : 0;
    return v > 0 ? v : kLookaheadCtasF64Default;
  }();
  return dt == MPI_DOUBLE ? f64 : f32;
}

cudaStream_t lookahead_stream() {
  State &s = state();
  if (!s.la_stream) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStreamCreateWithPriority(&s.la_stream, cudaStreamNonBlocking, hi);
  }
  return s.la_stream;
}

cudaStream_t copy_stream() {
  State &s = state();
  if (!s.copy_stream) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStreamCreateWithPriority(&s.copy_stream, cudaStreamNonBlocking, lo);
  }
  return s.copy_stream;
}

cudaStream_t replay_stream() {
  State &s = state();
  if (!s.replay_stream) {
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaStreamCreateWithPriority(&s.replay_stream, cudaStreamNonBlocking, lo);
  }
  return s.replay_stream;
}

cudaEvent_t lookahead_event(int i) {
  State &s = state();
  if (!s.la_events[i]) cudaEventCreateWithFlags(&s.la_events[i], cudaEventDisableTiming);
  return s.la_events[i];
}

OnStream::OnStream(cudaStream_t st) : saved(state().override_stream) {
  state().override_stream = st;
}
OnStream::~OnStream() { state().override_stream = saved; }

int fail(const char *message, int line, const char *file) {
  State &s = state();
  char buf[512];
  snprintf(buf, sizeof buf, "PLAPACK error: %s (line %d of %s)", message, line, file);
  s.last_message = buf;
  s.last_error = PLA_ERROR;
  if (getenv("PLA_B200_VERBOSE")) fprintf(stderr, "%s\n", buf);
  return PLA_ERROR;
}

int cuda_fail(cudaError_t e, int line, const char *file) {
  char buf[256];
  snprintf(buf, sizeof buf, "CUDA error %d: %s", (int)e, cudaGetErrorString(e));
  return fail(buf, line, file);
}

void warn(const char *message) {
  if (getenv("PLA_B200_VERBOSE")) fprintf(stderr, "PLAPACK warning: %s\n", message);
}

double scalar_value(PLA_Obj s) {
  double v = 0.0;
  char tmp[16];
  const char *p = at(s, 0, 0);
  if (!s->base->on_host) {
    d2h(tmp, p, s->base->esize);
    p = tmp;
  }
  switch (s->base->datatype) {
    case MPI_DOUBLE: v = *(const double *)p; break;
    case MPI_FLOAT: v = *(const float *)p; break;
    case MPI_INT: v = *(const int *)p; break;
    default: v = 0.0;
  }
  return v;
}

namespace {
struct Scratch {
  void *ptr = nullptr;
  size_t bytes = 0;
};
constexpr int kScratchSlots = 40;
Scratch g_scratch[kScratchSlots];
}  // namespace

cudaError_t d2h(void *dst, const void *src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, stream());
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(stream());
}

void *scratch(int slot, size_t bytes) {
  if (slot < 0 || slot >= kScratchSlots) return nullptr;
  Scratch &s = g_scratch[slot];
  if (s.bytes >= bytes && s.ptr) return s.ptr;
  if (s.ptr) {
    cudaStreamSynchronize(stream());
    cudaFree(s.ptr);
    s.ptr = nullptr;
    s.bytes = 0;
  }
  size_t want = bytes < 256 ? 256 : bytes;
  if (cudaMalloc(&s.ptr, want) != cudaSuccess) {
    s.ptr = nullptr;
    return nullptr;
  }
  s.bytes = want;
  return s.ptr;
}

void release_scratch() {
  for (auto &s : g_scratch) {
    if (s.ptr) cudaFree(s.ptr);
    s.ptr = nullptr;
    s.bytes = 0;
  }
}

namespace {
struct Pending {
  double *acc;
  cudaEvent_t a, b;
};
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_event_pool;

cudaEvent_t take_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

PhaseTimer::PhaseTimer(double *target) : acc(target), on(state().phase_timing != 0) {
  if (!on) return;
  e0 = take_event();
  e1 = take_event();
  cudaEventRecord(e0, stream());
}

PhaseTimer::~PhaseTimer() {
  if (!on) return;
  cudaEventRecord(e1, stream());
  g_pending.push_back({acc, e0, e1});
}

namespace {
unsigned long long *g_interchanges = nullptr;  // device counter, phase timing only
bool g_interchanges_pending = false;
}  // namespace

void count_interchanges(int npiv, const int *piv) {
  if (!state().phase_timing || npiv <= 0) return;
  if (!g_interchanges) {
    if (cudaMalloc(&g_interchanges, sizeof(unsigned long long)) != cudaSuccess) {
      g_interchanges = nullptr;
      return;
    }
    cudaMemsetAsync(g_interchanges, 0, sizeof(unsigned long long), stream());
  }
  if (pla_k_count_interchanges(npiv, piv, g_interchanges, stream()) == 0)
    g_interchanges_pending = true;
}

void release_interchange_counter() {
  if (g_interchanges) cudaFree(g_interchanges);
  g_interchanges = nullptr;
  g_interchanges_pending = false;
}

void resolve_phases() {
  if (g_interchanges_pending) {
    unsigned long long v = 0;
    cudaStream_t s = stream();
    if (cudaMemcpyAsync(&v, g_interchanges, sizeof v, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
        cudaStreamSynchronize(s) == cudaSuccess)
      state().phases.interchanges += (long long)v;
    cudaMemsetAsync(g_interchanges, 0, sizeof(unsigned long long), s);
    g_interchanges_pending = false;
  }
  for (Pending &p : g_pending) {
    cudaEventSynchronize(p.b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    *p.acc += ms;
    g_event_pool.push_back(p.a);
    g_event_pool.push_back(p.b);
  }
  g_pending.clear();
}

}  // namespace pla

using namespace pla;

// ---------------------------------------------------------------- objects --
static pla_base *new_base(MPI_Datatype dt, int length, int width, bool on_host, int *err) {
  *err = PLA_SUCCESS;
  int es = esize_of(dt);
  if (es == 0) {
    *err = fail("unsupported datatype", __LINE__, __FILE__);
    return nullptr;
  }
  if (length < 0 || width < 0) {
    *err = fail("negative object dimension", __LINE__, __FILE__);
    return nullptr;
  }
  pla_base *b = new pla_base();
  b->datatype = dt;
  b->esize = es;
  b->length = length;
  b->width = width;
  // leading dimension = global length, as OBJ/PLA_Obj.c:368 attaches it
  b->ldim = length > 0 ? length : 1;
  b->views = 0;
  b->user_buffer = 0;
  b->on_host = on_host ? 1 : 0;
  size_t bytes = (size_t)b->ldim * (size_t)(width > 0 ? width : 1) * es;
  cudaError_t e;
  if (on_host)
    e = cudaHostAlloc((void **)&b->buf, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
  else
    e = cudaMalloc((void **)&b->buf, bytes);
  if (e != cudaSuccess) {
    delete b;
    *err = cuda_fail(e, __LINE__, __FILE__);
    return nullptr;
  }
  // objects start as zero (OBJ/PLA_Obj.c:370)
  if (on_host)
    memset(b->buf, 0, bytes);
  else
    cudaMemsetAsync(b->buf, 0, bytes, stream());
  return b;
}

// a matrix whose data will live in a file (OBJ/PLA_Obj_ooc.c:50-72): no
// buffer, no file until PLA_Obj_attach_fd
static pla_base *new_ooc_base(MPI_Datatype dt, int length, int width, int *err) {
  *err = PLA_SUCCESS;
  const int es = esize_of(dt);
  if (es == 0 || dt == MPI_INT) {
    *err = fail("unsupported datatype", __LINE__, __FILE__);
    return nullptr;
  }
  if (length < 0 || width < 0) {
    *err = fail("negative object dimension", __LINE__, __FILE__);
    return nullptr;
  }
  pla_base *b = new pla_base();
  b->datatype = dt;
  b->esize = es;
  b->length = length;
  b->width = width;
  b->ldim = length > 0 ? length : 1;
  b->ooc = 1;
  b->fd = -1;
  return b;
}

static PLA_Obj new_view(pla_base *b, int objtype, PLA_Template templ) {
  PLA_Obj v = new PLA_Obj_view_struct();
  v->magic = kObjMagic;
  v->objtype = objtype;
  v->fixed = 0;
  v->length = b->length;
  v->width = b->width;
  v->row0 = v->col0 = 0;
  v->align_row = v->align_col = 0;
  v->owner_row = v->owner_col = 0;
  v->proj_onto = PLA_PROJ_ONTO_COL;
  v->templ = templ;
  v->base = b;
  b->views++;
  return v;
}

static PLA_Obj copy_view(PLA_Obj src) {
  PLA_Obj v = new PLA_Obj_view_struct(*src);
  v->base->views++;
  return v;
}

static void drop_view(PLA_Obj v) {
  if (!v) return;
  pla_base *b = v->base;
  v->magic = 0;
  delete v;
  if (b && --b->views == 0) {
    if (!b->user_buffer && b->buf) {
      if (b->on_host) {
        cudaFreeHost(b->buf);
      } else {
        cudaStreamSynchronize(stream());
        cudaFree(b->buf);
      }
    }
    delete b;
  }
}

static int create(MPI_Datatype dt, int objtype, int length, int width, PLA_Template templ,
                  bool on_host, PLA_Obj *out) {
  if (!out) PLA_FAIL("null output handle");
  if (state().check_parameters && !valid(templ)) PLA_FAIL("invalid template");
  int err;
  pla_base *b = new_base(dt, length, width, on_host, &err);
  if (!b) return err;
  PLA_Obj v = new_view(b, objtype, templ);
  if (*out && valid(*out)) drop_view(*out);
  *out = v;
  return PLA_SUCCESS;
}

extern "C" {

// ------------------------------------------------------ init and templates --
int PLA_Init(MPI_Comm comm) {
  State &s = state();
  if (s.initialized) PLA_FAIL("PLA_Init called more than once");
  if (comm == MPI_COMM_NULL) PLA_FAIL("Null communicator");
  int dev = 0;
  PLA_CUDA(cudaGetDevice(&dev));
  PLA_CUDA(cudaFree(nullptr));  // create the context now
  s.initialized = 1;
  (void)stream();
  return PLA_SUCCESS;
}

int PLA_Finalize(void) {
  State &s = state();
  if (!s.initialized) PLA_FAIL("PLAPACK not yet initialized");
  cudaStreamSynchronize(stream());
  release_scratch();
  release_ooc();
  release_interchange_counter();
  pla_kernels_release();
  for (cudaStream_t *st : {&s.la_stream, &s.copy_stream, &s.replay_stream})
    if (*st) {
      cudaStreamSynchronize(*st);
      cudaStreamDestroy(*st);
      *st = nullptr;
    }
  for (auto &e : s.la_events)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  if (s.own_stream) {
    cudaStreamDestroy(s.own_stream);
    s.own_stream = nullptr;
  }
  s.initialized = 0;
  return PLA_SUCCESS;
}

int PLA_Initialized(int *initialized) {
  if (initialized) *initialized = state().initialized;
  return state().initialized;
}

int PLA_Comm_1D_to_2D(MPI_Comm comm1d, int nprows, int npcols, MPI_Comm *comm2d) {
  if (nprows * npcols != 1) PLA_FAIL("only a 1 x 1 mesh drives one GPU");
  if (comm2d) *comm2d = comm1d;
  return PLA_SUCCESS;
}

int PLA_Comm_1D_to_2D_ratio(MPI_Comm comm1d, float ratio, MPI_Comm *comm2d) {
  (void)ratio;
  if (comm2d) *comm2d = comm1d;
  return PLA_SUCCESS;
}

int PLA_Temp_create(int nb, int zero_or_one, PLA_Template *templ) {
  if (!templ) PLA_FAIL("null template handle");
  if (nb <= 0) PLA_FAIL("template block size must be positive");
  if (zero_or_one != 0 && zero_or_one != 1) PLA_FAIL("zero_or_one must be 0 or 1");
  PLA_Template t = new PLA_Template_struct();
  t->magic = kTempMagic;
  t->nb = nb;
  t->zero_or_one = zero_or_one;
  t->refs = 1;
  *templ = t;
  return PLA_SUCCESS;
}

int PLA_Temp_free(PLA_Template *templ) {
  if (!templ || !*templ) return PLA_SUCCESS;
  if (!valid(*templ)) PLA_FAIL("invalid template");
  (*templ)->magic = 0;
  delete *templ;
  *templ = nullptr;
  return PLA_SUCCESS;
}

int PLA_Temp_nb(PLA_Template t, int *nb) {
  if (!valid(t)) PLA_FAIL("invalid template");
  *nb = t->nb;
  return PLA_SUCCESS;
}
int PLA_Temp_zero_or_one(PLA_Template t, int *z) {
  if (!valid(t)) PLA_FAIL("invalid template");
  *z = t->zero_or_one;
  return PLA_SUCCESS;
}
int PLA_Temp_comm_all_size(PLA_Template t, int *n) {
  (void)t;
  *n = 1;
  return PLA_SUCCESS;
}
int PLA_Temp_comm_all_rank(PLA_Template t, int *r) {
  (void)t;
  *r = 0;
  return PLA_SUCCESS;
}

// TEMPLATE/PLA_Environ.c:54-127: one algorithmic block size per operation class
static int op_slot(int op) {
  int k = op - PLA_OP_OFFSET - 1;
  return (k >= 0 && k < 6) ? k : -1;
}

int pla_Environ_set_nb_alg(int op, int nb_alg) {
  if (nb_alg <= 0) PLA_FAIL("nb_alg must be positive");
  State &s = state();
  if (op == PLA_OP_ALL_ALG) {
    for (int &v : s.nb_alg) v = nb_alg;
    return PLA_SUCCESS;
  }
  int k = op_slot(op);
  if (k < 0) PLA_FAIL("unknown operation class");
  s.nb_alg[k] = nb_alg;
  return PLA_SUCCESS;
}

int PLA_Environ_nb_alg(int op, PLA_Template templ, int *nb_alg) {
  (void)templ;
  int k = op_slot(op);
  *nb_alg = state().nb_alg[k < 0 ? 2 : k];
  return PLA_SUCCESS;
}

// ------------------------------------------------------------- diagnostics --
int PLA_Set_error_checking(int error, int parameters, int sequential, int r12) {
  State &s = state();
  s.error_checking = error;
  // with error checking off every other check is off (PLA_Diagnostics.c:413)
  s.check_parameters = error ? parameters : 0;
  s.check_sequential = error ? sequential : 0;
  s.check_r12 = error ? r12 : 0;
  return PLA_SUCCESS;
}

int PLA_Get_error_checking(int *error, int *parameters, int *sequential, int *r12) {
  State &s = state();
  if (error) *error = s.error_checking;
  if (parameters) *parameters = s.check_parameters;
  if (sequential) *sequential = s.check_sequential;
  if (r12) *r12 = s.check_r12;
  return PLA_SUCCESS;
}

int PLA_Abort(char *message, int line, char *file) { return fail(message, line, file); }

int PLA_Warning(char *message) {
  warn(message);
  return PLA_SUCCESS;
}

int PLA_Last_error(char *buf, int len) {
  State &s = state();
  if (buf && len > 0) {
    strncpy(buf, s.last_message.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return s.last_error;
}

int PLA_Clear_error(void) {
  state().last_error = 0;
  state().last_message.clear();
  return PLA_SUCCESS;
}

int PLA_B200_set_stream(void *s) {
  state().stream = (cudaStream_t)s;
  return PLA_SUCCESS;
}
void *PLA_B200_get_stream(void) { return (void *)stream(); }

int PLA_B200_phase_times(PLA_Phase_times *t) {
  resolve_phases();
  PLA_Phase_times &p = state().phases;
  p.total_ms = p.panel_ms + p.swap_ms + p.trsm_ms + p.update_ms + p.solve_ms + p.refine_ms +
               p.convert_ms;
  if (t) *t = p;
  return PLA_SUCCESS;
}
int PLA_B200_set_phase_timing(int on) {
  state().phase_timing = on;
  return PLA_SUCCESS;
}
int PLA_B200_reset_phase_times(void) {
  resolve_phases();
  state().phases = PLA_Phase_times{};
  return PLA_SUCCESS;
}
long PLA_B200_kernel_launches(void) { return pla_k_launches(); }

// ---------------------------------------------------------------- creation --
int PLA_OOC_Matrix_create_without_fd(MPI_Datatype datatype, int global_length,
                                     int global_width, PLA_Template templ,
                                     int global_align_row, int global_align_col,
                                     PLA_Obj *new_obj) {
  if (!new_obj) PLA_FAIL("null output handle");
  if (state().check_parameters && !valid(templ)) PLA_FAIL("invalid template");
  int err;
  pla_base *b = new_ooc_base(datatype, global_length, global_width, &err);
  if (!b) return err;
  PLA_Obj v = new_view(b, PLA_MATRIX, templ);
  v->align_row = global_align_row;
  v->align_col = global_align_col;
  if (*new_obj && valid_any(*new_obj)) drop_view(*new_obj);
  *new_obj = v;
  return PLA_SUCCESS;
}

// OBJ/PLA_Obj_management.c:146-166: the file and its leading dimension (in
// elements); the reference exits when a file is already attached
int PLA_Obj_attach_fd(PLA_Obj obj, int fd, int local_ldim, int user_buffer) {
  if (!valid_any(obj) || !obj->base->ooc) PLA_FAIL("PLA_Obj_attach_fd: not an out-of-core object");
  if (obj->base->fd != -1) PLA_FAIL("PLA_Obj_attach_fd: object already has file descriptor");
  if (fd < 0) PLA_FAIL("PLA_Obj_attach_fd: invalid file descriptor");
  if (local_ldim < std::max(obj->base->length, 1))
    PLA_FAIL("PLA_Obj_attach_fd: leading dimension smaller than the object's length");
  obj->base->fd = fd;
  obj->base->ldim = local_ldim;
  obj->base->user_buffer = user_buffer;
  return PLA_SUCCESS;
}

int PLA_Matrix_create(MPI_Datatype dt, int length, int width, PLA_Template templ,
                      int align_row, int align_col, PLA_Obj *obj) {
  int r = create(dt, PLA_MATRIX, length, width, templ, false, obj);
  if (r == PLA_SUCCESS) {
    (*obj)->align_row = align_row == PLA_ALIGN_FIRST ? 0 : align_row;
    (*obj)->align_col = align_col == PLA_ALIGN_FIRST ? 0 : align_col;
  }
  return r;
}

int PLA_Mvector_create(MPI_Datatype dt, int length, int width, PLA_Template templ, int align,
                       PLA_Obj *obj) {
  int r = create(dt, PLA_MVECTOR, length, width, templ, false, obj);
  if (r == PLA_SUCCESS) (*obj)->align_row = align == PLA_ALIGN_FIRST ? 0 : align;
  return r;
}

int PLA_Mscalar_create(MPI_Datatype dt, int owner_row, int owner_col, int length, int width,
                       PLA_Template templ, PLA_Obj *obj) {
  // duplicated multiscalars hold small host-side data (constants, pivot
  // blocks): keep them in pinned, device-mapped host memory
  bool small = (long)length * (long)width <= 4096;
  int r = create(dt, PLA_MSCALAR, length, width, templ, small, obj);
  if (r == PLA_SUCCESS) {
    (*obj)->owner_row = owner_row;
    (*obj)->owner_col = owner_col;
  }
  return r;
}

int PLA_Pmvector_create(MPI_Datatype dt, int project_onto, int owner, int length, int width,
                        PLA_Template templ, int align, PLA_Obj *obj) {
  // a projected multivector of a 1x1 mesh is an ordinary column-major block
  int r = create(dt, PLA_PMVECTOR, length, width, templ, false, obj);
  if (r == PLA_SUCCESS) {
    (*obj)->proj_onto = project_onto;
    (*obj)->owner_row = owner;
    (*obj)->align_row = align == PLA_ALIGN_FIRST ? 0 : align;
  }
  return r;
}

int PLA_Matrix_create_conf_to(PLA_Obj o, PLA_Obj *obj) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  return PLA_Matrix_create(o->base->datatype, o->length, o->width, o->templ, o->align_row,
                           o->align_col, obj);
}

int PLA_Mvector_create_conf_to(PLA_Obj o, int width, PLA_Obj *obj) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  // conformal to the object's length (a row projection already stores the
  // matrix's row dimension as its length)
  return PLA_Mvector_create(o->base->datatype, o->length, width, o->templ, o->align_row, obj);
}

int PLA_Mscalar_create_conf_to(PLA_Obj o, int owner_row, int owner_col, PLA_Obj *obj) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  return PLA_Mscalar_create(o->base->datatype, owner_row, owner_col, o->length, o->width,
                            o->templ, obj);
}

int PLA_Pmvector_create_conf_to(PLA_Obj o, int project_onto, int owner, int width,
                                PLA_Obj *obj) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  int length = project_onto == PLA_PROJ_ONTO_COL ? o->length : o->width;
  int r = PLA_Pmvector_create(o->base->datatype, project_onto, owner, length, width, o->templ,
                              o->align_row, obj);
  return r;
}

int PLA_Create_constants_conf_to(PLA_Obj o, PLA_Obj *minus_one, PLA_Obj *zero,
                                 PLA_Obj *one) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  MPI_Datatype dt = o->base->datatype;
  if (dt == MPI_INT) dt = MPI_DOUBLE;
  const double vals[3] = {-1.0, 0.0, 1.0};
  PLA_Obj *outs[3] = {minus_one, zero, one};
  for (int k = 0; k < 3; k++) {
    if (!outs[k]) continue;
    int r = PLA_Mscalar_create(dt, PLA_ALL_ROWS, PLA_ALL_COLS, 1, 1, o->templ, outs[k]);
    if (r != PLA_SUCCESS) return r;
    r = PLA_Obj_set(*outs[k], MPI_DOUBLE, (void *)&vals[k]);
    if (r != PLA_SUCCESS) return r;
    (*outs[k])->fixed = 1;
  }
  return PLA_SUCCESS;
}

int PLA_Obj_free(PLA_Obj *obj) {
  if (!obj || !*obj) return PLA_SUCCESS;
  if (!valid_any(*obj)) PLA_FAIL("invalid object");
  drop_view(*obj);
  *obj = nullptr;
  return PLA_SUCCESS;
}

// ------------------------------------------------------------------- views --
static void assign(PLA_Obj *out, PLA_Obj v) {
  if (!out) {
    drop_view(v);
    return;
  }
  PLA_Obj old = *out;
  *out = v;
  if (old && valid_any(old)) drop_view(old);
}

int PLA_Obj_view(PLA_Obj o, int length, int width, int disp_row, int disp_col, PLA_Obj *view) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  if (length == PLA_DIM_ALL) length = o->length - disp_row;
  if (width == PLA_DIM_ALL) width = o->width - disp_col;
  if (disp_row < 0 || disp_col < 0 || length < 0 || width < 0 ||
      disp_row + length > o->length || disp_col + width > o->width)
    PLA_FAIL("view out of range");
  PLA_Obj v = copy_view(o);
  v->row0 += disp_row;
  v->col0 += disp_col;
  v->length = length;
  v->width = width;
  v->align_row += disp_row;
  v->align_col += disp_col;
  v->fixed = 0;
  assign(view, v);
  return PLA_SUCCESS;
}

int PLA_Obj_view_all(PLA_Obj o, PLA_Obj *view) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  PLA_Obj v = copy_view(o);
  v->fixed = 0;
  assign(view, v);
  return PLA_SUCCESS;
}

int PLA_Obj_split_4(PLA_Obj o, int length, int width, PLA_Obj *tl, PLA_Obj *tr, PLA_Obj *bl,
                    PLA_Obj *br) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  // sign selects which block the size describes (OBJ/PLA_Obj.c:2078-2088)
  int top = length >= 0 ? length : o->length + length;
  int left = width >= 0 ? width : o->width + width;
  if (top < 0) top = 0;
  if (top > o->length) top = o->length;
  if (left < 0) left = 0;
  if (left > o->width) left = o->width;
  const int rows[2] = {top, o->length - top}, cols[2] = {left, o->width - left};
  const int r0[2] = {0, top}, c0[2] = {0, left};
  PLA_Obj *outs[4] = {tl, tr, bl, br};
  PLA_Obj made[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int q = 0; q < 4; q++) {
    if (!outs[q]) continue;
    int i = q / 2, j = q % 2;
    PLA_Obj v = copy_view(o);
    v->row0 += r0[i];
    v->col0 += c0[j];
    v->align_row += r0[i];
    v->align_col += c0[j];
    v->length = rows[i];
    v->width = cols[j];
    v->fixed = 0;
    made[q] = v;
  }
  for (int q = 0; q < 4; q++)
    if (outs[q]) assign(outs[q], made[q]);
  return PLA_SUCCESS;
}

int PLA_Obj_horz_split_2(PLA_Obj o, int length, PLA_Obj *top, PLA_Obj *bottom) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  return PLA_Obj_split_4(o, length, o->width, top, nullptr, bottom, nullptr);
}

int PLA_Obj_vert_split_2(PLA_Obj o, int width, PLA_Obj *left, PLA_Obj *right) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  return PLA_Obj_split_4(o, o->length, width, left, right, nullptr, nullptr);
}

// positive moves a boundary down / right (OBJ/PLA_Obj.c:3189-3201)
int PLA_Obj_view_shift(PLA_Obj o, int shift_top, int shift_left, int shift_right,
                       int shift_bottom) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  int row0 = o->row0 + shift_top, col0 = o->col0 + shift_left;
  int length = o->length - shift_top + shift_bottom;
  int width = o->width - shift_left + shift_right;
  if (row0 < 0 || col0 < 0 || length < 0 || width < 0 || row0 + length > o->base->length ||
      col0 + width > o->base->width)
    PLA_FAIL("view shift leaves the base object");
  o->row0 = row0;
  o->col0 = col0;
  o->align_row += shift_top;
  o->align_col += shift_left;
  o->length = length;
  o->width = width;
  return PLA_SUCCESS;
}

int PLA_Obj_view_swap(PLA_Obj *a, PLA_Obj *b) {
  PLA_Obj t = *a;
  *a = *b;
  *b = t;
  return PLA_SUCCESS;
}

// ----------------------------------------------------------------- inquiry --
#define INQ(name, expr)                          \
  int name(PLA_Obj o, int *out) {                \
    if (!valid_any(o)) PLA_FAIL("invalid object");   \
    *out = (expr);                               \
    return PLA_SUCCESS;                          \
  }
INQ(PLA_Obj_objtype, o->objtype)
INQ(PLA_Obj_global_length, o->length)
INQ(PLA_Obj_global_width, o->width)
INQ(PLA_Obj_global_name, 0)
INQ(PLA_Obj_global_align_row, o->align_row)
INQ(PLA_Obj_global_align_col, o->align_col)
INQ(PLA_Obj_local_length, o->length)
INQ(PLA_Obj_local_width, o->width)
INQ(PLA_Obj_local_ldim, (int)o->base->ldim)
INQ(PLA_Obj_local_stride, 1)
INQ(PLA_Obj_owner_row, o->owner_row)
INQ(PLA_Obj_owner_col, o->owner_col)
INQ(PLA_Obj_project_onto, o->proj_onto)
#undef INQ

int PLA_Obj_datatype(PLA_Obj o, MPI_Datatype *dt) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  *dt = o->base->datatype;
  return PLA_SUCCESS;
}

int PLA_Obj_template(PLA_Obj o, PLA_Template *t) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  *t = o->templ;
  return PLA_SUCCESS;
}

int PLA_Obj_local_buffer(PLA_Obj o, void **buffer) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  // an out-of-core object has no buffer (OBJ/PLA_Obj_management.c:161-163)
  *buffer = o->base->ooc ? nullptr : at(o, 0, 0);
  return PLA_SUCCESS;
}

int PLA_Obj_set_orientation(PLA_Obj o, int project_onto) {
  if (!valid_any(o)) PLA_FAIL("invalid object");
  o->proj_onto = project_onto;
  return PLA_SUCCESS;
}

// ---------------------------------------------------------------- contents --
int PLA_Obj_set(PLA_Obj o, MPI_Datatype dt, void *value) {
  if (!valid(o)) PLA_FAIL("invalid object");
  double v;
  if (dt == MPI_DOUBLE) v = *(double *)value;
  else if (dt == MPI_FLOAT) v = *(float *)value;
  else if (dt == MPI_INT) v = *(int *)value;
  else PLA_FAIL("unsupported datatype of value");
  if (o->length == 0 || o->width == 0) return PLA_SUCCESS;
  if (o->base->on_host) {
    for (int j = 0; j < o->width; j++)
      for (int i = 0; i < o->length; i++) {
        char *p = at(o, i, j);
        switch (o->base->datatype) {
          case MPI_DOUBLE: *(double *)p = v; break;
          case MPI_FLOAT: *(float *)p = (float)v; break;
          case MPI_INT: *(int *)p = (int)v; break;
          default: break;
        }
      }
    return PLA_SUCCESS;
  }
  int r = pla_k_fill(o->base->datatype, o->length, o->width, at(o, 0, 0), ld(o), v, stream());
  if (r) PLA_FAIL("fill kernel failed");
  PLA_CUDA(cudaStreamSynchronize(stream()));
  return PLA_SUCCESS;
}

int PLA_Obj_set_to_zero(PLA_Obj o) {
  double z = 0.0;
  return PLA_Obj_set(o, MPI_DOUBLE, &z);
}
int PLA_Obj_set_to_one(PLA_Obj o) {
  double z = 1.0;
  return PLA_Obj_set(o, MPI_DOUBLE, &z);
}
int PLA_Obj_set_to_minus_one(PLA_Obj o) {
  double z = -1.0;
  return PLA_Obj_set(o, MPI_DOUBLE, &z);
}

int PLA_Obj_set_to_identity(PLA_Obj o) {
  int r = PLA_Obj_set_to_zero(o);
  if (r) return r;
  int k = o->length < o->width ? o->length : o->width;
  double one = 1.0;
  for (int i = 0; i < k; i++) {
    PLA_Obj e = nullptr;
    PLA_Obj_view(o, 1, 1, i, i, &e);
    PLA_Obj_set(e, MPI_DOUBLE, &one);
    PLA_Obj_free(&e);
  }
  return PLA_SUCCESS;
}

// copy between a host buffer (column-major, ldim_buf, element stride) and the
// object; trans = PLA_TRANSPOSE stores the transpose (OBJ/PLA_Obj.c)
static int local_contents(bool to_obj, PLA_Obj o, int trans, void *buf, int ldim_buf,
                          int stride_buf) {
  const int m = o->length, n = o->width, es = o->base->esize;
  if (m == 0 || n == 0) return PLA_SUCCESS;
  if (stride_buf != 1) PLA_FAIL("only unit stride host buffers are supported");
  if (trans == PLA_NO_TRANSPOSE) {
    if (ldim_buf < m) PLA_FAIL("host leading dimension too small");
    if (o->base->on_host) {
      for (int j = 0; j < n; j++) {
        char *d = at(o, 0, j), *h = (char *)buf + (size_t)j * ldim_buf * es;
        if (to_obj) memcpy(d, h, (size_t)m * es);
        else memcpy(h, d, (size_t)m * es);
      }
      return PLA_SUCCESS;
    }
    if (to_obj)
      PLA_CUDA(cudaMemcpy2DAsync(at(o, 0, 0), ld(o) * es, buf, (size_t)ldim_buf * es,
                                 (size_t)m * es, n, cudaMemcpyHostToDevice, stream()));
    else
      PLA_CUDA(cudaMemcpy2DAsync(buf, (size_t)ldim_buf * es, at(o, 0, 0), ld(o) * es,
                                 (size_t)m * es, n, cudaMemcpyDeviceToHost, stream()));
    PLA_CUDA(cudaStreamSynchronize(stream()));
    return PLA_SUCCESS;
  }
  // transposed: element (i, j) of the object <-> buf[j + i * ldim_buf]
  if (ldim_buf < n) PLA_FAIL("host leading dimension too small");
  std::vector<char> tmp((size_t)m * n * es);
  if (to_obj) {
    for (int j = 0; j < n; j++)
      for (int i = 0; i < m; i++)
        memcpy(&tmp[((size_t)i + (size_t)j * m) * es],
               (char *)buf + ((size_t)j + (size_t)i * ldim_buf) * es, es);
    return local_contents(true, o, PLA_NO_TRANSPOSE, tmp.data(), m, 1);
  }
  int r = local_contents(false, o, PLA_NO_TRANSPOSE, tmp.data(), m, 1);
  if (r) return r;
  for (int j = 0; j < n; j++)
    for (int i = 0; i < m; i++)
      memcpy((char *)buf + ((size_t)j + (size_t)i * ldim_buf) * es,
             &tmp[((size_t)i + (size_t)j * m) * es], es);
  return PLA_SUCCESS;
}

int PLA_Obj_get_local_contents(PLA_Obj o, int trans, int *rows_in_buf, int *cols_in_buf,
                               void *buf, int ldim_buf, int stride_buf) {
  if (!valid(o)) PLA_FAIL("invalid object");
  if (rows_in_buf) *rows_in_buf = trans == PLA_NO_TRANSPOSE ? o->length : o->width;
  if (cols_in_buf) *cols_in_buf = trans == PLA_NO_TRANSPOSE ? o->width : o->length;
  return local_contents(false, o, trans, buf, ldim_buf, stride_buf);
}

static int device_contents(bool to_obj, PLA_Obj o, void *dev, int ldim) {
  if (!valid(o)) PLA_FAIL("invalid object");
  const int m = o->length, n = o->width, es = o->base->esize;
  if (m == 0 || n == 0) return PLA_SUCCESS;
  if (ldim < m) PLA_FAIL("device leading dimension too small");
  if (to_obj)
    PLA_CUDA(cudaMemcpy2DAsync(at(o, 0, 0), ld(o) * es, dev, (size_t)ldim * es, (size_t)m * es, n,
                               cudaMemcpyDefault, stream()));
  else
    PLA_CUDA(cudaMemcpy2DAsync(dev, (size_t)ldim * es, at(o, 0, 0), ld(o) * es, (size_t)m * es, n,
                               cudaMemcpyDefault, stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));
  return PLA_SUCCESS;
}

int PLA_Obj_set_local_contents_device(const void *dev_buf, int ldim, PLA_Obj obj) {
  return device_contents(true, obj, const_cast<void *>(dev_buf), ldim);
}

int PLA_Obj_get_local_contents_device(PLA_Obj obj, void *dev_buf, int ldim) {
  return device_contents(false, obj, dev_buf, ldim);
}

int PLA_Obj_set_local_contents(int trans, int rows_in_buf, int cols_in_buf, void *buf,
                               int ldim_buf, int stride_buf, PLA_Obj o) {
  if (!valid(o)) PLA_FAIL("invalid object");
  int m = trans == PLA_NO_TRANSPOSE ? rows_in_buf : cols_in_buf;
  int n = trans == PLA_NO_TRANSPOSE ? cols_in_buf : rows_in_buf;
  if (m != o->length || n != o->width) PLA_FAIL("buffer does not conform to the object");
  return local_contents(true, o, trans, buf, ldim_buf, stride_buf);
}

}  // extern "C"

extern "C" {
void *PLA_malloc(size_t size) { return pla::host_alloc(size, false); }
void *PLA_calloc(size_t size, size_t typesize) {
  if (typesize && size > (~(size_t)0 - 16) / typesize) {
    pla::fail("PLA_calloc: size overflows", __LINE__, __FILE__);
    return nullptr;
  }
  return pla::host_alloc(size * typesize, true);
}
void *PLA_free(void *buffer) {
  if (buffer) {
    char *p = (char *)buffer - 16;
    pla::g_host_bytes -= (long long)*(size_t *)p;
    std::free(p);
  }
  return nullptr;
}
int PLA_Total_size_malloced(void) { return (int)pla::g_host_bytes.load(); }
int PLA_Max_size_malloced(void) { return (int)pla::g_host_bytes_max.load(); }
}  // extern "C"

// OBJ/PLA_Timings.c:17-140: the reference's per-operation timers.  Here they
// are the library's phase timers: initialize resets and starts them, print
// writes each nonzero phase as the reference writes each timer, average (a
// reduction over ranks) has nothing to combine on one GPU.
extern "C" {
int PLA_Timings_initialize(void) {
  PLA_B200_reset_phase_times();
  return PLA_B200_set_phase_timing(1);
}
int PLA_Timings_print(void) {
  PLA_Phase_times t;
  int r = PLA_B200_phase_times(&t);
  if (r) return r;
  const struct {
    const char *name;
    double ms;
  } rows[] = {{"panel  ", t.panel_ms},  {"swap   ", t.swap_ms},  {"trsm   ", t.trsm_ms},
              {"update ", t.update_ms}, {"solve  ", t.solve_ms}, {"refine ", t.refine_ms},
              {"convert", t.convert_ms}};
  for (const auto &row : rows)
    if (row.ms != 0) std::printf("%s time = %f\n", row.name, row.ms / 1e3);
  return PLA_SUCCESS;
}
int PLA_Timings_average(void) { return PLA_SUCCESS; }
}  // extern "C"
