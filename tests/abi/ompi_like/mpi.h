/*
 * A stand-in <mpi.h> with Open MPI's handle style, for the ABI tests: handles
 * are pointers to predefined objects, 8 bytes wide where the library's codes
 * are 4-byte ints.  Single process; no communication.
 */
#ifndef MOCK_OMPI_MPI_H
#define MOCK_OMPI_MPI_H

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

typedef struct mock_ompi_datatype_t *MPI_Datatype;
typedef struct mock_ompi_communicator_t *MPI_Comm;
struct mock_ompi_datatype_t { int size; };
struct mock_ompi_communicator_t { int id; };

static struct mock_ompi_datatype_t mock_ompi_char __attribute__((unused)) = {1};
static struct mock_ompi_datatype_t mock_ompi_int __attribute__((unused)) = {4};
static struct mock_ompi_datatype_t mock_ompi_float __attribute__((unused)) = {4};
static struct mock_ompi_datatype_t mock_ompi_long __attribute__((unused)) = {8};
static struct mock_ompi_datatype_t mock_ompi_double __attribute__((unused)) = {8};
static struct mock_ompi_datatype_t mock_ompi_complex __attribute__((unused)) = {8};
static struct mock_ompi_datatype_t mock_ompi_dcomplex __attribute__((unused)) = {16};
static struct mock_ompi_datatype_t mock_ompi_dt_null __attribute__((unused)) = {0};
static struct mock_ompi_communicator_t mock_ompi_comm_world __attribute__((unused)) = {1};
static struct mock_ompi_communicator_t mock_ompi_comm_dup __attribute__((unused)) = {2};
static struct mock_ompi_communicator_t mock_ompi_comm_null __attribute__((unused)) = {0};

#define MPI_DATATYPE_NULL  (&mock_ompi_dt_null)
#define MPI_CHAR           (&mock_ompi_char)
#define MPI_INT            (&mock_ompi_int)
#define MPI_FLOAT          (&mock_ompi_float)
#define MPI_LONG           (&mock_ompi_long)
#define MPI_DOUBLE         (&mock_ompi_double)
#define MPI_COMPLEX        (&mock_ompi_complex)
#define MPI_DOUBLE_COMPLEX (&mock_ompi_dcomplex)
#define MPI_COMM_NULL      (&mock_ompi_comm_null)
#define MPI_COMM_WORLD     (&mock_ompi_comm_world)
#define MPI_SUCCESS 0

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm) {
  *newcomm = comm == MPI_COMM_NULL ? MPI_COMM_NULL : &mock_ompi_comm_dup;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

#endif
