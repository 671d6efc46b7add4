/*
 * pla_mpi_compat.h — the caller's MPI handles translated to the library's
 * codes.  Included by PLA.h when an MPI header is present (PLA_B200_WITH_MPI);
 * never include it directly.
 *
 * The reference's objects carry real MPI datatypes and its template a real
 * communicator (INCLUDE/PLA.h:14, TEMPLATE/PLA_Init.c:20-82).  This library
 * runs one process per GPU on a 1x1 template and needs neither, but a driver
 * written against the reference passes its MPI's handles: MPI_DOUBLE is
 * 0x4c00080b in MPICH and the address of a global object in Open MPI.  The
 * entry points that take or return a datatype or a communicator are therefore
 * macros here: each maps the caller's handle to the code the library takes
 * (PLA_B200_DT_*, PLA_B200_COMM_*) and, for outputs, back.  A datatype the
 * library does not handle maps to -1, which every entry point rejects with
 * PLA_ERROR.  Taking a function's address (no call) bypasses the macro and
 * yields the code-taking function.
 *
 * Communicators: PLA_Comm_1D_to_2D on a 1 x 1 mesh returns a duplicate of the
 * caller's communicator (MPI_Comm_dup), which the caller may free as it would
 * the reference's Cartesian communicator; PLA_Init accepts any communicator
 * but MPI_COMM_NULL.  Several ranks each drive their own GPU with their own
 * 1x1 template; no data moves between them.
 */
#ifndef PLA_B200_MPI_COMPAT_H
#define PLA_B200_MPI_COMPAT_H

#if !defined(PLA_B200_BUILDING_LIBRARY)

static inline PLA_B200_Datatype pla_b200_datatype_code(MPI_Datatype dt) {
  if (dt == MPI_DOUBLE) return PLA_B200_DT_DOUBLE;
  if (dt == MPI_FLOAT) return PLA_B200_DT_FLOAT;
  if (dt == MPI_INT) return PLA_B200_DT_INT;
  if (dt == MPI_CHAR) return PLA_B200_DT_CHAR;
#ifdef MPI_COMPLEX
  if (dt == MPI_COMPLEX) return PLA_B200_DT_COMPLEX;
#endif
#ifdef MPI_DOUBLE_COMPLEX
  if (dt == MPI_DOUBLE_COMPLEX) return PLA_B200_DT_DOUBLE_COMPLEX;
#endif
  return -1;
}

static inline MPI_Datatype pla_b200_datatype_handle(PLA_B200_Datatype code) {
  switch (code) {
    case PLA_B200_DT_DOUBLE: return MPI_DOUBLE;
    case PLA_B200_DT_FLOAT: return MPI_FLOAT;
    case PLA_B200_DT_INT: return MPI_INT;
    case PLA_B200_DT_CHAR: return MPI_CHAR;
#ifdef MPI_COMPLEX
    case PLA_B200_DT_COMPLEX: return MPI_COMPLEX;
#endif
#ifdef MPI_DOUBLE_COMPLEX
    case PLA_B200_DT_DOUBLE_COMPLEX: return MPI_DOUBLE_COMPLEX;
#endif
    default: return MPI_DATATYPE_NULL;
  }
}

static inline PLA_B200_Comm pla_b200_comm_code(MPI_Comm comm) {
  return comm == MPI_COMM_NULL ? PLA_B200_COMM_NULL : PLA_B200_COMM_WORLD;
}

static inline int pla_b200_obj_datatype(PLA_Obj obj, MPI_Datatype *datatype) {
  PLA_B200_Datatype code = -1;
  int r = (PLA_Obj_datatype)(obj, &code);
  if (datatype) *datatype = pla_b200_datatype_handle(code);
  return r;
}

static inline int pla_b200_comm_1d_to_2d(MPI_Comm comm1d, int nprows, int npcols,
                                         MPI_Comm *comm2d) {
  PLA_B200_Comm out = PLA_B200_COMM_NULL;
  int r = (PLA_Comm_1D_to_2D)(pla_b200_comm_code(comm1d), nprows, npcols, &out);
  if (comm2d) {
    *comm2d = MPI_COMM_NULL;
    if (r == PLA_SUCCESS && out != PLA_B200_COMM_NULL) MPI_Comm_dup(comm1d, comm2d);
  }
  return r;
}

static inline int pla_b200_comm_1d_to_2d_ratio(MPI_Comm comm1d, float ratio, MPI_Comm *comm2d) {
  PLA_B200_Comm out = PLA_B200_COMM_NULL;
  int r = (PLA_Comm_1D_to_2D_ratio)(pla_b200_comm_code(comm1d), ratio, &out);
  if (comm2d) {
    *comm2d = MPI_COMM_NULL;
    if (r == PLA_SUCCESS && out != PLA_B200_COMM_NULL) MPI_Comm_dup(comm1d, comm2d);
  }
  return r;
}

#define PLA_Init(comm) (PLA_Init)(pla_b200_comm_code(comm))
#define PLA_Comm_1D_to_2D(comm1d, nprows, npcols, comm2d) \
  pla_b200_comm_1d_to_2d((comm1d), (nprows), (npcols), (comm2d))
#define PLA_Comm_1D_to_2D_ratio(comm1d, ratio, comm2d) \
  pla_b200_comm_1d_to_2d_ratio((comm1d), (ratio), (comm2d))
#define PLA_Matrix_create(dt, length, width, templ, align_row, align_col, obj) \
  (PLA_Matrix_create)(pla_b200_datatype_code(dt), (length), (width), (templ), (align_row), \
                      (align_col), (obj))
#define PLA_Mvector_create(dt, length, width, templ, align, obj) \
  (PLA_Mvector_create)(pla_b200_datatype_code(dt), (length), (width), (templ), (align), (obj))
#define PLA_Mscalar_create(dt, owner_row, owner_col, length, width, templ, obj)               \
  (PLA_Mscalar_create)(pla_b200_datatype_code(dt), (owner_row), (owner_col), (length), (width), \
                       (templ), (obj))
#define PLA_Pmvector_create(dt, project_onto, owner, length, width, templ, align, obj)         \
  (PLA_Pmvector_create)(pla_b200_datatype_code(dt), (project_onto), (owner), (length), (width), \
                        (templ), (align), (obj))
#define PLA_Obj_datatype(obj, dt) pla_b200_obj_datatype((obj), (dt))
#define PLA_Obj_set(obj, dt, value) (PLA_Obj_set)((obj), pla_b200_datatype_code(dt), (value))
#define PLA_Shift(obj, dt, value) (PLA_Shift)((obj), pla_b200_datatype_code(dt), (value))
#define PLA_OOC_Matrix_create_without_fd(dt, length, width, templ, align_row, align_col, obj) \
  (PLA_OOC_Matrix_create_without_fd)(pla_b200_datatype_code(dt), (length), (width), (templ), \
                                     (align_row), (align_col), (obj))
#define PLA_File_create(name, dt, size, fd) \
  (PLA_File_create)((name), pla_b200_datatype_code(dt), (size), (fd))
#define PLA_File_open(name, dt, size, fd) \
  (PLA_File_open)((name), pla_b200_datatype_code(dt), (size), (fd))
#define PLA_B200_lu_panel_noalloc(dt, m, w, A, lda, pivots, status, stream)                    \
  (PLA_B200_lu_panel_noalloc)(pla_b200_datatype_code(dt), (m), (w), (A), (lda), (pivots), \
                              (status), (stream))
#define PLA_Batch_plan_create(dt, count, instances, info, autotune, plan) \
  (PLA_Batch_plan_create)(pla_b200_datatype_code(dt), (count), (instances), (info), (autotune), \
                          (plan))
#define PLA_Batched_factor_solve(dt, count, instances, info) \
  (PLA_Batched_factor_solve)(pla_b200_datatype_code(dt), (count), (instances), (info))
#define PLA_Batched_factor_solve_loop(dt, count, instances) \
  (PLA_Batched_factor_solve_loop)(pla_b200_datatype_code(dt), (count), (instances))

#endif /* !PLA_B200_BUILDING_LIBRARY */

#endif /* PLA_B200_MPI_COMPAT_H */
