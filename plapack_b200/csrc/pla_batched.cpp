// Batched factor-and-solve: plan (sort, bucket, autotune, upload, capture a
// CUDA graph), execute (replay the graph), and the per-instance launch loop
// of the plain kernels that the batched launch is measured against.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>

#include "pla_internal.h"
#include "pla_kernels.h"

using namespace pla;

extern "C" size_t pla_k_batched_smem(int dt, int n_smem_max);
extern "C" size_t pla_k_batched_blocked_smem(int dt, int n, int pw);
extern "C" int pla_k_batched(int dt, const void *inst, const int *order, const void *tasks,
                             int ntasks, int *queue, int *info, int grid, size_t smem,
                             cudaStream_t s);

namespace pla {
int lu_async(int dt, int m, int n, char *A, long lda, int *piv, int nb);
int chol_async(int dt, int n, char *A, long lda, int nb);
}

struct PLA_Batch_plan_struct {
  int dt = 0, count = 0, ntasks = 0, grid = 0, n_smem = 0, n_pw32 = 0;
  size_t smem = 0;
  void *inst = nullptr;   // device Inst<T>[count]
  int *order = nullptr;   // device
  void *tasks = nullptr;  // device Task[ntasks]
  int *queue = nullptr;   // device counter
  int *info = nullptr;    // device, caller's
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

struct InstRec {  // layout of Inst<T> in k_batched.cu
  int n, nrhs, kind, pad;
  void *A, *B;
  int *piv;
};
struct TaskRec {
  int first, count, mode, pad;
};

int g_sms = 0;
int sms() {
  if (!g_sms) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, d);
  }
  return g_sms;
}

// largest order that fits the shared-memory budget of a mode-1 CTA
int smem_limit(int dt, size_t budget) {
  int n = 32;
  while (pla_k_batched_smem(dt, n + 1) <= budget) n++;
  return n;
}

// Tasks, largest instances first: up to 8 instances of order <= 32 per task
// (a warp each), then one instance per task -- in shared memory up to order
// n_smem, else in global memory with panels of 32 columns from order n_pw32
// on (mode 3) or of 16 below it (mode 2).
void build_tasks(const std::vector<PLA_Batch_instance> &v, int n_smem, int n_pw32,
                 std::vector<int> &order, std::vector<TaskRec> &tasks) {
  order.resize(v.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return v[a].n > v[b].n; });
  tasks.clear();
  size_t i = 0;
  while (i < order.size()) {
    const PLA_Batch_instance &in = v[order[i]];
    if (in.n <= 32 && in.nrhs <= 4) {
      TaskRec t{(int)i, 0, 0, 0};
      while (i < order.size() && t.count < 8 && v[order[i]].n <= 32 && v[order[i]].nrhs <= 4) {
        t.count++;
        i++;
      }
      tasks.push_back(t);
    } else {
      int mode = (in.n <= n_smem && in.nrhs <= 4) ? 1 : (in.n >= n_pw32 ? 3 : 2);
      tasks.push_back(TaskRec{(int)i, 1, mode, 0});
      i++;
    }
  }
}

// dynamic shared memory of a launch: the shared-memory form up to n_smem and
// the blocked form of the largest instance in global memory, within the
// device's per-CTA limit (an instance whose panel does not fit runs the column
// algorithm in place)
size_t launch_smem(int dt, const std::vector<PLA_Batch_instance> &v, int n_smem, int n_pw32) {
  static int optin = 0;
  if (!optin) {
    int d;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d);
  }
  size_t s = pla_k_batched_smem(dt, n_smem);
  for (auto &in : v) {
    if (in.n <= n_smem || in.n <= 32) continue;
    const size_t b = pla_k_batched_blocked_smem(dt, in.n, in.n >= n_pw32 ? 32 : 16);
    if (b <= (size_t)optin - 4096 && b > s) s = b;
  }
  return s;
}

int upload(PLA_Batch_plan p, const std::vector<PLA_Batch_instance> &v,
           const std::vector<int> &order, const std::vector<TaskRec> &tasks) {
  std::vector<InstRec> recs(v.size());
  for (size_t k = 0; k < v.size(); k++)
    recs[k] = InstRec{v[k].n, v[k].nrhs, v[k].kind, 0, v[k].A, v[k].B, v[k].pivots};
  if (p->inst) cudaFree(p->inst);
  if (p->order) cudaFree(p->order);
  if (p->tasks) cudaFree(p->tasks);
  if (!p->queue) PLA_CUDA(cudaMalloc(&p->queue, 256));
  PLA_CUDA(cudaMalloc(&p->inst, recs.size() * sizeof(InstRec) + 16));
  PLA_CUDA(cudaMalloc((void **)&p->order, order.size() * sizeof(int) + 16));
  PLA_CUDA(cudaMalloc(&p->tasks, tasks.size() * sizeof(TaskRec) + 16));
  PLA_CUDA(cudaMemcpy(p->inst, recs.data(), recs.size() * sizeof(InstRec), cudaMemcpyHostToDevice));
  PLA_CUDA(cudaMemcpy(p->order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
  PLA_CUDA(cudaMemcpy(p->tasks, tasks.data(), tasks.size() * sizeof(TaskRec),
                      cudaMemcpyHostToDevice));
  p->ntasks = (int)tasks.size();
  return PLA_SUCCESS;
}

int launch(PLA_Batch_plan p, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(p->queue, 0, sizeof(int), s);
  if (e) return (int)e;
  return pla_k_batched(p->dt, p->inst, p->order, p->tasks, p->ntasks, p->queue, p->info, p->grid,
                       p->smem, s);
}

// Autotuner.  Per size bucket it picks the form each range of orders runs in
// -- shared memory up to n_smem, blocked panels of 16 or 32 columns above it
// (32 from n_pw32 on) -- and the persistent CTAs per SM, by timing every
// candidate on a sample of the batch itself: every k-th instance (about an
// eighth of them, the size mix kept), with the caller's own matrices copied
// into scratch memory (pivoting included), restored before each run.  The
// result is cached per (datatype, size histogram) for the life of the process.
struct Tuned {
  int n_smem, n_pw32, per_sm;
};
std::map<std::vector<int>, Tuned> g_tuned;

// without autotuning: 16-column panels in FP64 (74 KB of shared memory at
// n = 512, so two CTAs share an SM) and 32-column panels in fp32 from order
// 192 on (the same footprint)
Tuned default_tuning(int dt) {
  return Tuned{smem_limit(dt, 110 * 1024), dt == MPI_DOUBLE ? (1 << 30) : 192, 2};
}

Tuned autotune(int dt, const std::vector<PLA_Batch_instance> &v) {
  std::vector<int> key{dt};
  {
    int hist[10] = {0};
    for (auto &in : v) hist[std::min(9, (int)std::log2(std::max(1, in.n)))]++;
    for (int h : hist) key.push_back(h > 0 ? (int)std::log2(h) + 1 : 0);
  }
  auto it = g_tuned.find(key);
  if (it != g_tuned.end()) return it->second;
  const int es = dt == MPI_DOUBLE ? 8 : 4;
  const int nmax_smem = smem_limit(dt, 110 * 1024);
  Tuned best = default_tuning(dt);
  const int stride = std::max<int>(1, (int)v.size() / 2048);
  std::vector<PLA_Batch_instance> smp;
  size_t bytes = 0;
  for (size_t k = 0; k < v.size(); k += stride) {
    smp.push_back(v[k]);
    bytes += ((size_t)v[k].n * v[k].n + (size_t)v[k].n * v[k].nrhs) * es + (size_t)v[k].n * 4 + 64;
  }
  bytes = (bytes + 255) / 256 * 256;
  char *pool = (char *)scratch(14, 2 * bytes + 256);
  int *info = (int *)scratch(15, smp.size() * sizeof(int) + 64);
  if (!pool || !info) return best;
  char *pristine = pool + bytes;
  size_t off = 0;
  for (auto &in : smp) {
    const size_t a = (size_t)in.n * in.n * es, b = (size_t)in.n * in.nrhs * es;
    if (a) cudaMemcpyAsync(pristine + off, in.A, a, cudaMemcpyDeviceToDevice, stream());
    in.A = pool + off;
    off += a;
    if (b) cudaMemcpyAsync(pristine + off, in.B, b, cudaMemcpyDeviceToDevice, stream());
    in.B = pool + off;
    off += b;
    in.pivots = (int *)(pool + off);
    off += (size_t)in.n * 4 + 64;
    off = (off + 15) / 16 * 16;
  }
  PLA_Batch_plan_struct p;
  p.dt = dt;
  p.info = info;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  const int cands_smem[3] = {std::min(64, nmax_smem), std::min(96, nmax_smem), nmax_smem};
  const int cands_pw32[3] = {0, 192, 1 << 30};
  for (int cs : cands_smem)
    for (int c32 : cands_pw32)
      for (int per_sm : {1, 2}) {
        std::vector<int> order;
        std::vector<TaskRec> tasks;
        build_tasks(smp, cs, c32, order, tasks);
        if (upload(&p, smp, order, tasks)) continue;
        p.smem = launch_smem(dt, smp, cs, c32);
        p.grid = sms() * per_sm;
        float ms_best_run = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
          cudaMemcpyAsync(pool, pristine, bytes, cudaMemcpyDeviceToDevice, stream());
          cudaEventRecord(e0, stream());
          int r = launch(&p, stream());
          cudaEventRecord(e1, stream());
          if (cudaEventSynchronize(e1) != cudaSuccess || r) break;
          float ms;
          cudaEventElapsedTime(&ms, e0, e1);
          ms_best_run = std::min(ms_best_run, ms);
        }
        if (ms_best_run < best_ms) {
          best_ms = ms_best_run;
          best = Tuned{cs, c32, per_sm};
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(p.inst);
  cudaFree(p.order);
  cudaFree(p.tasks);
  cudaFree(p.queue);
  g_tuned[key] = best;
  return best;
}

}  // namespace

extern "C" {

int PLA_Batch_plan_create(int datatype, int count, const PLA_Batch_instance *instances,
                          int *info, int autotune_on, PLA_Batch_plan *plan) {
  if (!plan) PLA_FAIL("null plan handle");
  if (datatype != MPI_DOUBLE && datatype != MPI_FLOAT) PLA_FAIL("datatype not supported");
  if (count < 0 || (count > 0 && (!instances || !info))) PLA_FAIL("invalid batch");
  std::vector<PLA_Batch_instance> v(instances, instances + count);
  for (auto &in : v) {
    if (in.n < 0 || in.nrhs < 0 || (in.kind != 0 && in.kind != 1)) PLA_FAIL("invalid instance");
    if (in.n > 0 && !in.A) PLA_FAIL("instance without a matrix");
    if (in.nrhs > 0 && !in.B) PLA_FAIL("instance without right-hand sides");
    if (in.kind == 0 && in.n > 0 && !in.pivots) PLA_FAIL("LU instance without a pivot vector");
  }
  PLA_Batch_plan p = new PLA_Batch_plan_struct();
  p->dt = datatype;
  p->count = count;
  p->info = info;
  Tuned t = autotune_on ? autotune(datatype, v) : default_tuning(datatype);
  p->n_smem = t.n_smem;
  p->n_pw32 = t.n_pw32;
  p->smem = launch_smem(datatype, v, t.n_smem, t.n_pw32);
  p->grid = sms() * t.per_sm;
  std::vector<int> order;
  std::vector<TaskRec> tasks;
  build_tasks(v, t.n_smem, t.n_pw32, order, tasks);
  int r = upload(p, v, order, tasks);
  if (r) {
    PLA_Batch_plan_free(&p);
    return r;
  }
  // capture the launch (queue reset + persistent kernel) in a CUDA graph
  cudaStream_t cs;
  PLA_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  PLA_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int lr = launch(p, cs);
  cudaError_t ce = cudaStreamEndCapture(cs, &p->graph);
  cudaStreamDestroy(cs);
  if (lr || ce != cudaSuccess) {
    PLA_Batch_plan_free(&p);
    PLA_FAIL("cannot capture the batched launch");
  }
  PLA_CUDA(cudaGraphInstantiate(&p->exec, p->graph, 0));
  *plan = p;
  return PLA_SUCCESS;
}

int PLA_Batch_plan_execute(PLA_Batch_plan plan) {
  if (!plan) PLA_FAIL("null plan");
  if (plan->ntasks == 0) return PLA_SUCCESS;
  PLA_CUDA(cudaGraphLaunch(plan->exec, stream()));
  PLA_CUDA(cudaStreamSynchronize(stream()));
  return PLA_SUCCESS;
}

int PLA_Batch_plan_free(PLA_Batch_plan *plan) {
  if (!plan || !*plan) return PLA_SUCCESS;
  PLA_Batch_plan p = *plan;
  cudaStreamSynchronize(stream());
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->inst) cudaFree(p->inst);
  if (p->order) cudaFree(p->order);
  if (p->tasks) cudaFree(p->tasks);
  if (p->queue) cudaFree(p->queue);
  delete p;
  *plan = nullptr;
  return PLA_SUCCESS;
}

int PLA_Batched_factor_solve(int datatype, int count, const PLA_Batch_instance *instances,
                             int *info) {
  PLA_Batch_plan p = nullptr;
  int r = PLA_Batch_plan_create(datatype, count, instances, info, 0, &p);
  if (r) return r;
  r = PLA_Batch_plan_execute(p);
  PLA_Batch_plan_free(&p);
  return r;
}

// The baseline: every instance through the plain single-matrix kernels
// (blocked LU / Cholesky, then the blocked triangular solves), one after the
// other on the library stream; info is not collected.
int PLA_Batched_factor_solve_loop(int datatype, int count, const PLA_Batch_instance *instances) {
  if (datatype != MPI_DOUBLE && datatype != MPI_FLOAT) PLA_FAIL("datatype not supported");
  for (int k = 0; k < count; k++) {
    const PLA_Batch_instance &in = instances[k];
    if (in.n == 0) continue;
    int r = in.kind == 0 ? lu_async(datatype, in.n, in.n, (char *)in.A, in.n, in.pivots, 64)
                         : chol_async(datatype, in.n, (char *)in.A, in.n, 64);
    if (r) return r;
    if (in.nrhs == 0) continue;
    if (in.kind == 0) {
      int e = pla_k_laswp_rows(datatype, in.B, in.n, in.nrhs, in.n, in.pivots, stream());
      if (!e) e = pla_k_trsv_blocked(datatype, 'L', 'N', 'U', in.n, in.nrhs, in.A, in.n, in.B,
                                     in.n, stream());
      if (!e) e = pla_k_trsv_blocked(datatype, 'U', 'N', 'N', in.n, in.nrhs, in.A, in.n, in.B,
                                     in.n, stream());
      if (e) return cuda_fail((cudaError_t)e, __LINE__, __FILE__);
    } else {
      int e = pla_k_trsv_blocked(datatype, 'L', 'N', 'N', in.n, in.nrhs, in.A, in.n, in.B, in.n,
                                 stream());
      if (!e) e = pla_k_trsv_blocked(datatype, 'L', 'T', 'N', in.n, in.nrhs, in.A, in.n, in.B,
                                     in.n, stream());
      if (e) return cuda_fail((cudaError_t)e, __LINE__, __FILE__);
    }
  }
  PLA_CUDA(cudaStreamSynchronize(stream()));
  return PLA_SUCCESS;
}

}  // extern "C"
