/*
 * Single-rank MPI stand-in used ONLY to compile the upstream PLAPACK sources
 * into the CPU oracle (oracle/_ref).  Test infrastructure, not product code.
 *
 * Every communicator has exactly one rank (rank 0).  Collectives copy the
 * send buffer to the receive buffer; point-to-point messages to self are
 * queued and matched by (communicator, tag).  This is enough for PLAPACK on a
 * 1x1 template, where every redistribution is a copy to self.
 */
#ifndef PLA_ORACLE_MPI_SHIM_H
#define PLA_ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;

typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)

/* predefined datatypes (handles index a size table in the shim) */
#define MPI_DATATYPE_NULL   0
#define MPI_CHAR            1
#define MPI_BYTE            2
#define MPI_INT             3
#define MPI_FLOAT           4
#define MPI_DOUBLE          5
#define MPI_COMPLEX         6
#define MPI_DOUBLE_COMPLEX  7
#define MPI_LONG            8
#define MPI_UNSIGNED        9
#define MPI_SHORT          10
#define MPI_PACKED         11

/* communicators */
#define MPI_COMM_NULL   0
#define MPI_COMM_WORLD  1
#define MPI_COMM_SELF   2

/* reduction operators */
#define MPI_OP_NULL 0
#define MPI_SUM     1
#define MPI_MAX     2
#define MPI_MIN     3
#define MPI_PROD    4
#define MPI_MAXLOC  5
#define MPI_MINLOC  6

#define MPI_ANY_SOURCE  (-1)
#define MPI_ANY_TAG     (-1)
#define MPI_PROC_NULL   (-2)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_IN_PLACE    ((void *) 1)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Initialized(int *flag);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int MPI_Barrier(MPI_Comm comm);

int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Cart_create(MPI_Comm comm, int ndims, int *dims, int *periods,
                    int reorder, MPI_Comm *newcomm);
int MPI_Cart_get(MPI_Comm comm, int maxdims, int *dims, int *periods,
                 int *coords);
int MPI_Cart_sub(MPI_Comm comm, int *remain_dims, MPI_Comm *newcomm);

int MPI_Type_size(MPI_Datatype type, int *size);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);

int MPI_Send(void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm);
int MPI_Isend(void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Test(MPI_Request *req, int *flag, MPI_Status *status);
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int *flag,
               MPI_Status *status);
int MPI_Get_count(MPI_Status *status, MPI_Datatype type, int *count);

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root,
              MPI_Comm comm);
int MPI_Reduce(void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
               MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Reduce_scatter(void *sendbuf, void *recvbuf, int *recvcounts,
                       MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(void *sendbuf, int sendcount, MPI_Datatype sendtype,
                  void *recvbuf, int recvcount, MPI_Datatype recvtype,
                  MPI_Comm comm);
int MPI_Allgatherv(void *sendbuf, int sendcount, MPI_Datatype sendtype,
                   void *recvbuf, int *recvcounts, int *displs,
                   MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Gatherv(void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, int *recvcounts, int *displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Scatterv(void *sendbuf, int *sendcounts, int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
