/*
 * A stand-in <mpi.h> with MPICH's handle style, for the ABI tests: handles are
 * ints that encode a kind and a size, none equal to the library's own datatype
 * and communicator codes.  Single process; no communication.
 */
#ifndef MOCK_MPICH_MPI_H
#define MOCK_MPICH_MPI_H

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

typedef int MPI_Datatype;
typedef int MPI_Comm;

#define MPI_DATATYPE_NULL  ((MPI_Datatype)0x0c000000)
#define MPI_CHAR           ((MPI_Datatype)0x4c000101)
#define MPI_INT            ((MPI_Datatype)0x4c000405)
#define MPI_FLOAT          ((MPI_Datatype)0x4c00040a)
#define MPI_LONG           ((MPI_Datatype)0x4c000807)
#define MPI_DOUBLE         ((MPI_Datatype)0x4c00080b)
#define MPI_COMPLEX        ((MPI_Datatype)0x4c00081e)
#define MPI_DOUBLE_COMPLEX ((MPI_Datatype)0x4c001022)
#define MPI_COMM_NULL      ((MPI_Comm)0x04000000)
#define MPI_COMM_WORLD     ((MPI_Comm)0x44000000)
#define MPI_SUCCESS 0

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm) {
  *newcomm = comm == MPI_COMM_NULL ? MPI_COMM_NULL : (MPI_Comm)(0x84000000 | (comm & 0xff));
  return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

#endif
