// Internal declarations shared by the host-side translation units of
// libplapack_b200.  Not installed; the public surface is include/PLA.h.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "PLA.h"

// A base object owns one device (or, for multiscalars, pinned host) buffer;
// views share it and count references, like PLA_Obj_base_struct in the
// reference (INCLUDE/PLA_Obj.h:15-44, OBJ/PLA_Obj_management.c:63-110).
struct pla_base {
  MPI_Datatype datatype;
  int esize;           // bytes per element
  char *buf;           // device pointer (host pinned for PLA_MSCALAR)
  long ldim;           // leading dimension in elements (column-major)
  int length, width;   // size of the base object
  int views;           // number of live views
  int user_buffer;     // buffer not owned by the library
  int on_host;         // buf is pinned host memory (duplicated multiscalars)
  int ooc;             // out-of-core: the data lives in file fd (buf is null)
  int fd;              // file of an out-of-core object, -1 until attached
};

// A view: a rectangular window into a base object (INCLUDE/PLA_Obj.h:49-82).
// On a 1x1 template every view is entirely local.
struct PLA_Obj_view_struct {
  unsigned magic;
  int objtype;
  int fixed;           // constants created by PLA_Create_constants_conf_to
  int length, width;   // global (== local) size
  int row0, col0;      // displacement inside the base
  int align_row, align_col;
  int owner_row, owner_col;
  int proj_onto;
  PLA_Template templ;
  pla_base *base;
};

struct PLA_Template_struct {
  unsigned magic;
  int nb;
  int zero_or_one;
  int refs;
};

namespace pla {

constexpr unsigned kObjMagic = 0x504c414fu;   // "PLAO"
constexpr unsigned kTempMagic = 0x504c4154u;  // "PLAT"

// library state (TEMPLATE/PLA_Init.c, TEMPLATE/PLA_Environ.c:46-52,
// OBJ/PLA_Diagnostics.c:16-19)
struct State {
  int initialized = 0;
  int nb_alg[8] = {128, 128, 128, 128, 128, 128, 128, 128};
  int error_checking = 1;
  int check_parameters = 1;
  int check_sequential = 0;
  int check_r12 = 0;
  int api_active = 0;
  int last_error = 0;
  std::string last_message;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t override_stream = nullptr;  // set by OnStream while a scope queues elsewhere
  cudaStream_t la_stream = nullptr;        // high-priority stream of the lookahead panels
  cudaStream_t copy_stream = nullptr;      // host-to-device copies of a streamed solve
  cudaStream_t replay_stream = nullptr;    // a streamed solve's catch-up of arrived columns
  cudaEvent_t la_events[2] = {nullptr, nullptr};
  int phase_timing = 0;
  PLA_Phase_times phases{};
};
State &state();

int esize_of(MPI_Datatype dt);
bool valid(PLA_Obj obj);      // a live object with its data in memory
bool valid_any(PLA_Obj obj);  // a live object, out-of-core ones included
bool valid(PLA_Template t);
cudaStream_t stream();

// Lookahead: panels run on a second, high-priority stream while the trailing
// update of the previous step runs on stream(); two events order them.
// CTAs of a panel that runs beside a trailing update: few enough to leave the
// update most SMs, enough that a 32-column sub-panel of 32768 rows still fits
// in their shared memory.  Measured at n = 32768 (CTAs: mixed / FP64 solve):
// 32: 0.358 / 1.148 s, 48: 0.331 / 1.143 s, 72: 0.310 / 1.159 s,
// 100: 0.316 / 1.177 s.  The fp32 panel of the mixed LU runs beside a short
// HBM-bound update and wants more CTAs; the FP64 panel beside the long DGEMM
// fewer.  With the faster DGEMM the FP64 solve measured 32: 0.843, 48: 0.824,
// 64: 0.829, 96: 0.830 s.
// The environment variables PLA_B200_LOOKAHEAD_CTAS_F32 / _F64 (read once)
// override the defaults, for tuning on other parts.
constexpr int kLookaheadCtasF32Default = 72;
constexpr int kLookaheadCtasF64Default = 48;
int lookahead_ctas(int dt);
cudaStream_t lookahead_stream();
cudaEvent_t lookahead_event(int i);
cudaStream_t copy_stream();
cudaStream_t replay_stream();
// while alive, stream() returns `s` (host code is sequential, so the switch
// only affects the calls made inside the scope)
struct OnStream {
  cudaStream_t saved;
  explicit OnStream(cudaStream_t s);
  ~OnStream();
};

// typed pointer to element (i, j) of a view (device pointer unless on_host)
inline char *at(PLA_Obj v, long i, long j) {
  return v->base->buf + ((long)(v->row0 + i) + (long)(v->col0 + j) * v->base->ldim) *
                            v->base->esize;
}
inline long ld(PLA_Obj v) { return v->base->ldim; }
inline bool is_double(PLA_Obj v) { return v->base->datatype == MPI_DOUBLE; }
inline bool is_float(PLA_Obj v) { return v->base->datatype == MPI_FLOAT; }

// value of a 1x1 scalar object as double (reads host or device memory)
double scalar_value(PLA_Obj s);

// error handling: records the message, returns PLA_ERROR; never exits
int fail(const char *message, int line, const char *file);
int cuda_fail(cudaError_t e, int line, const char *file);
void warn(const char *message);

// device -> host copy ordered after everything queued on the library stream
// (which is non-blocking: a plain cudaMemcpy would not wait for it)
cudaError_t d2h(void *dst, const void *src, size_t bytes);

// device scratch owned by the library (grown on demand, freed at PLA_Finalize)
void *scratch(int slot, size_t bytes);
void release_scratch();

// out-of-core objects (pla_ooc.cpp): PLA_Copy between a file-backed view and
// a device object, and the pinned staging buffers released at PLA_Finalize
int ooc_copy(PLA_Obj from, PLA_Obj to);
void release_ooc();

// phase timing: events recorded on the library stream, resolved later
struct PhaseTimer {
  cudaEvent_t e0{}, e1{};
  double *acc;
  bool on;
  explicit PhaseTimer(double *target);
  ~PhaseTimer();
};
void resolve_phases();
// with phase timing on: add the non-trivial interchanges of piv[0..npiv) to
// PLA_Phase_times.interchanges (a device count, read when the times are)
void count_interchanges(int npiv, const int *piv);
void release_interchange_counter();

}  // namespace pla

#define PLA_CUDA(call)                                                   \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return pla::cuda_fail(e_, __LINE__, __FILE__); \
  } while (0)

#define PLA_FAIL(msg) return pla::fail((msg), __LINE__, __FILE__)
