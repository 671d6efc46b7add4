/*
 * Single-rank MPI stand-in (see mpi.h).  Test infrastructure only: it lets the
 * upstream PLAPACK hot-path sources run as a CPU oracle on one process.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SHIM_MAX_TYPES 256
static int type_size[SHIM_MAX_TYPES] = {
    0, /* NULL */ 1, /* CHAR */ 1, /* BYTE */ (int)sizeof(int),
    (int)sizeof(float), (int)sizeof(double), 2 * (int)sizeof(float),
    2 * (int)sizeof(double), (int)sizeof(long), (int)sizeof(unsigned),
    (int)sizeof(short), 1};
static int next_type = 32;
static int next_comm = 16;

static void shim_fail(const char *what) {
  fprintf(stderr, "mpi shim: %s\n", what);
  abort();
}

static int tsize(MPI_Datatype t) {
  if (t <= 0 || t >= SHIM_MAX_TYPES || type_size[t] <= 0)
    shim_fail("unknown datatype");
  return type_size[t];
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Initialized(int *flag) { *flag = 1; return 0; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return 0; }

double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  if (comm == MPI_COMM_NULL) shim_fail("rank of MPI_COMM_NULL");
  *rank = 0;
  return 0;
}
int MPI_Comm_size(MPI_Comm comm, int *size) {
  if (comm == MPI_COMM_NULL) shim_fail("size of MPI_COMM_NULL");
  *size = 1;
  return 0;
}
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm) {
  (void)comm;
  *newcomm = next_comm++;
  return 0;
}
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return 0; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm) {
  (void)comm; (void)key;
  *newcomm = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : next_comm++;
  return 0;
}
int MPI_Cart_create(MPI_Comm comm, int ndims, int *dims, int *periods,
                    int reorder, MPI_Comm *newcomm) {
  int i, p = 1;
  (void)comm; (void)periods; (void)reorder;
  for (i = 0; i < ndims; i++) p *= dims[i];
  if (p != 1) shim_fail("only a 1x1 mesh is available on one rank");
  *newcomm = next_comm++;
  return 0;
}
int MPI_Cart_get(MPI_Comm comm, int maxdims, int *dims, int *periods,
                 int *coords) {
  int i;
  (void)comm;
  for (i = 0; i < maxdims; i++) {
    dims[i] = 1;
    periods[i] = 0;
    coords[i] = 0;
  }
  return 0;
}
int MPI_Cart_sub(MPI_Comm comm, int *remain_dims, MPI_Comm *newcomm) {
  (void)comm; (void)remain_dims;
  *newcomm = next_comm++;
  return 0;
}

int MPI_Type_size(MPI_Datatype type, int *size) {
  *size = tsize(type);
  return 0;
}
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype) {
  if (next_type >= SHIM_MAX_TYPES) shim_fail("too many derived types");
  type_size[next_type] = count * tsize(old);
  *newtype = next_type++;
  return 0;
}
int MPI_Type_commit(MPI_Datatype *type) { (void)type; return 0; }
int MPI_Type_free(MPI_Datatype *type) { *type = MPI_DATATYPE_NULL; return 0; }

/* ---- point-to-point to self: a FIFO of copied messages ------------------ */
typedef struct shim_msg {
  struct shim_msg *next;
  MPI_Comm comm;
  int tag;
  int bytes;
  char data[];
} shim_msg;
static shim_msg *queue_head = NULL, *queue_tail = NULL;

typedef struct {
  int used, is_recv, done;
  void *buf;
  int bytes, tag;
  MPI_Comm comm;
  MPI_Status st;
} shim_req;
#define SHIM_MAX_REQ 4096
static shim_req reqs[SHIM_MAX_REQ];

static void enqueue(const void *buf, int bytes, int tag, MPI_Comm comm) {
  shim_msg *m = (shim_msg *)malloc(sizeof(shim_msg) + (size_t)bytes);
  if (!m) shim_fail("out of memory");
  m->next = NULL;
  m->comm = comm;
  m->tag = tag;
  m->bytes = bytes;
  if (bytes) memcpy(m->data, buf, (size_t)bytes);
  if (queue_tail) queue_tail->next = m; else queue_head = m;
  queue_tail = m;
}

static shim_msg *find(int tag, MPI_Comm comm, int take) {
  shim_msg *prev = NULL, *m;
  for (m = queue_head; m; prev = m, m = m->next) {
    if (m->comm == comm && (tag == MPI_ANY_TAG || m->tag == tag)) {
      if (take) {
        if (prev) prev->next = m->next; else queue_head = m->next;
        if (queue_tail == m) queue_tail = prev;
      }
      return m;
    }
  }
  return NULL;
}

static int deliver(void *buf, int max_bytes, int tag, MPI_Comm comm,
                   MPI_Status *st) {
  shim_msg *m = find(tag, comm, 1);
  if (!m) return 0;
  if (m->bytes > max_bytes) shim_fail("message truncated");
  if (m->bytes) memcpy(buf, m->data, (size_t)m->bytes);
  if (st) {
    st->MPI_SOURCE = 0;
    st->MPI_TAG = m->tag;
    st->MPI_ERROR = 0;
    st->count_bytes = m->bytes;
  }
  free(m);
  return 1;
}

static int new_req(void) {
  int i;
  for (i = 1; i < SHIM_MAX_REQ; i++)
    if (!reqs[i].used) { memset(&reqs[i], 0, sizeof reqs[i]); reqs[i].used = 1; return i; }
  shim_fail("too many outstanding requests");
  return 0;
}

int MPI_Send(void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm) {
  if (dest != 0) shim_fail("send to a rank other than self");
  enqueue(buf, count * tsize(type), tag, comm);
  return 0;
}
int MPI_Isend(void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req) {
  int r;
  MPI_Send(buf, count, type, dest, tag, comm);
  r = new_req();
  reqs[r].done = 1;
  *req = r;
  return 0;
}
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status) {
  (void)source;
  if (!deliver(buf, count * tsize(type), tag, comm, status))
    shim_fail("receive with no matching message (would deadlock)");
  return 0;
}
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req) {
  int r = new_req();
  (void)source;
  reqs[r].is_recv = 1;
  reqs[r].buf = buf;
  reqs[r].bytes = count * tsize(type);
  reqs[r].tag = tag;
  reqs[r].comm = comm;
  *req = r;
  return 0;
}
static int progress(int r) {
  if (reqs[r].done) return 1;
  if (reqs[r].is_recv &&
      deliver(reqs[r].buf, reqs[r].bytes, reqs[r].tag, reqs[r].comm, &reqs[r].st))
    reqs[r].done = 1;
  return reqs[r].done;
}
int MPI_Wait(MPI_Request *req, MPI_Status *status) {
  int r = *req;
  if (r <= 0 || r >= SHIM_MAX_REQ || !reqs[r].used) return 0;
  if (!progress(r)) shim_fail("wait on a receive with no matching message");
  if (status) *status = reqs[r].st;
  reqs[r].used = 0;
  *req = MPI_REQUEST_NULL;
  return 0;
}
int MPI_Test(MPI_Request *req, int *flag, MPI_Status *status) {
  int r = *req;
  if (r <= 0 || r >= SHIM_MAX_REQ || !reqs[r].used) { *flag = 1; return 0; }
  *flag = progress(r);
  if (*flag) {
    if (status) *status = reqs[r].st;
    reqs[r].used = 0;
    *req = MPI_REQUEST_NULL;
  }
  return 0;
}
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int *flag,
               MPI_Status *status) {
  shim_msg *m = find(tag, comm, 0);
  (void)source;
  *flag = m != NULL;
  if (m && status) {
    status->MPI_SOURCE = 0;
    status->MPI_TAG = m->tag;
    status->MPI_ERROR = 0;
    status->count_bytes = m->bytes;
  }
  return 0;
}
int MPI_Get_count(MPI_Status *status, MPI_Datatype type, int *count) {
  *count = status->count_bytes / tsize(type);
  return 0;
}

/* ---- collectives over one rank: copies ------------------------------------ */
static void copy_bytes(void *dst, const void *src, size_t n) {
  if (src == MPI_IN_PLACE || dst == src || n == 0) return;
  memmove(dst, src, n);
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
              MPI_Comm comm) {
  (void)buf; (void)count; (void)type; (void)root; (void)comm;
  return 0;
}
int MPI_Reduce(void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm) {
  (void)op; (void)root; (void)comm;
  copy_bytes(recvbuf, sendbuf, (size_t)count * tsize(type));
  return 0;
}
int MPI_Allreduce(void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm) {
  (void)op; (void)comm;
  copy_bytes(recvbuf, sendbuf, (size_t)count * tsize(type));
  return 0;
}
int MPI_Reduce_scatter(void *sendbuf, void *recvbuf, int *recvcounts,
                       MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
  (void)op; (void)comm;
  copy_bytes(recvbuf, sendbuf, (size_t)recvcounts[0] * tsize(type));
  return 0;
}
int MPI_Allgather(void *sendbuf, int sendcount, MPI_Datatype sendtype,
                  void *recvbuf, int recvcount, MPI_Datatype recvtype,
                  MPI_Comm comm) {
  (void)recvcount; (void)recvtype; (void)comm;
  copy_bytes(recvbuf, sendbuf, (size_t)sendcount * tsize(sendtype));
  return 0;
}
int MPI_Allgatherv(void *sendbuf, int sendcount, MPI_Datatype sendtype,
                   void *recvbuf, int *recvcounts, int *displs,
                   MPI_Datatype recvtype, MPI_Comm comm) {
  (void)recvcounts; (void)comm;
  copy_bytes((char *)recvbuf + (size_t)displs[0] * tsize(recvtype), sendbuf,
             (size_t)sendcount * tsize(sendtype));
  return 0;
}
int MPI_Gatherv(void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, int *recvcounts, int *displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm) {
  (void)recvcounts; (void)root; (void)comm;
  copy_bytes((char *)recvbuf + (size_t)displs[0] * tsize(recvtype), sendbuf,
             (size_t)sendcount * tsize(sendtype));
  return 0;
}
int MPI_Scatterv(void *sendbuf, int *sendcounts, int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm) {
  (void)recvcount; (void)recvtype; (void)root; (void)comm;
  copy_bytes(recvbuf, (char *)sendbuf + (size_t)displs[0] * tsize(sendtype),
             (size_t)sendcounts[0] * tsize(sendtype));
  return 0;
}
