/*
 * PLA.h — drop-in C interface of the B200 dense direct-solve library.
 *
 * A caller of PLAPACK's dense solvers includes this header instead of the
 * reference's INCLUDE/PLA.h and links libplapack_b200.so.  Names, argument
 * order and meaning, constant values and return conventions follow the
 * reference (INCLUDE/PLA_define.h, INCLUDE/PLA_Obj_prototypes.h,
 * INCLUDE/PLA_API_prototypes.h and the solver sources cited below).  The
 * template is always 1x1: one process drives one GPU, and every object's data
 * lives in device memory (PLA_Obj_local_buffer returns a device pointer).
 *
 * Differences a caller may notice, all deliberate:
 *   - no MPI is needed: without an MPI header the MPI handle names below are
 *     plain int codes and MPI_COMM_WORLD names the single rank; with one, the
 *     caller's own MPI handles are translated at each call (pla_mpi_compat.h);
 *   - fatal errors never call exit(): PLA_Abort records the message and the
 *     failing call returns PLA_ERROR (see PLA_Last_error in pla_b200.h);
 *   - fill and extract go through PLA_API_axpy_* or PLA_Obj_set/get_local_contents
 *     (host buffers), since the local buffer is not host-addressable.
 */
#ifndef PLA_B200_PLA_H
#define PLA_B200_PLA_H

#include <stddef.h> /* size_t */

#ifdef __cplusplus
extern "C" {
#endif

/* ---- MPI -------------------------------------------------------------------
 * The library needs no MPI: one process drives one GPU on a 1x1 template.  Its
 * entry points take datatype and communicator CODES, plain ints with the
 * values below (PLA_B200_Datatype, PLA_B200_Comm).
 *  - Without an MPI header, the MPI_* names are those codes, so a caller
 *    writes MPI_DOUBLE or MPI_COMM_WORLD as it would against the reference.
 *  - With an MPI header -- included before this one, or found on the include
 *    path, as the reference's INCLUDE/PLA.h:14 includes <mpi.h> -- MPI_* are
 *    that MPI's own handles (ints in MPICH, pointers in Open MPI).  The entry
 *    points that take or return a datatype or a communicator are then macros
 *    over the inline translators at the end of this header
 *    (pla_mpi_compat.h), which map the caller's handles to the codes and back.
 *    Define PLA_B200_NO_MPI to keep MPI out even when <mpi.h> is reachable. */
#if !defined(PLA_B200_NO_MPI) && !defined(MPI_VERSION) && !defined(MPI_DOUBLE) && \
    defined(__has_include)
#if __has_include(<mpi.h>)
#include <mpi.h>
#endif
#endif
#if !defined(PLA_B200_NO_MPI) && (defined(MPI_VERSION) || defined(MPI_DOUBLE))
#define PLA_B200_WITH_MPI 1
#endif

typedef int PLA_B200_Datatype; /* datatype code */
typedef int PLA_B200_Comm;     /* communicator code */
#define PLA_B200_DT_CHAR           1
#define PLA_B200_DT_INT            3
#define PLA_B200_DT_FLOAT          4
#define PLA_B200_DT_DOUBLE         5
#define PLA_B200_DT_COMPLEX        6
#define PLA_B200_DT_DOUBLE_COMPLEX 7
#define PLA_B200_COMM_NULL         0
#define PLA_B200_COMM_WORLD        1

#ifndef PLA_B200_WITH_MPI
typedef PLA_B200_Datatype MPI_Datatype;
typedef PLA_B200_Comm MPI_Comm;
#define MPI_COMM_NULL       PLA_B200_COMM_NULL
#define MPI_COMM_WORLD      PLA_B200_COMM_WORLD
#define MPI_CHAR            PLA_B200_DT_CHAR
#define MPI_INT             PLA_B200_DT_INT
#define MPI_FLOAT           PLA_B200_DT_FLOAT
#define MPI_DOUBLE          PLA_B200_DT_DOUBLE
#define MPI_COMPLEX         PLA_B200_DT_COMPLEX
#define MPI_DOUBLE_COMPLEX  PLA_B200_DT_DOUBLE_COMPLEX
#endif

/* ---- constants: same names and values as INCLUDE/PLA_define.h:11-101 ---- */
#define PLA_OBJTYPE_OFFSET 10
#define PLA_VECTOR      (PLA_OBJTYPE_OFFSET + 1)
#define PLA_MVECTOR     (PLA_OBJTYPE_OFFSET + 2)
#define PLA_MATRIX      (PLA_OBJTYPE_OFFSET + 3)
#define PLA_MSCALAR     (PLA_OBJTYPE_OFFSET + 4)
#define PLA_PVECTOR     (PLA_OBJTYPE_OFFSET + 5)
#define PLA_PMVECTOR    (PLA_OBJTYPE_OFFSET + 6)

#define PLA_TRANSPOSE_OFFSET 20
#define PLA_NO_TRANSPOSE        (PLA_TRANSPOSE_OFFSET + 1)
#define PLA_NO_TRANS            (PLA_TRANSPOSE_OFFSET + 1)
#define PLA_TRANSPOSE           (PLA_TRANSPOSE_OFFSET + 2)
#define PLA_TRANS               (PLA_TRANSPOSE_OFFSET + 2)
#define PLA_CONJUGATE_TRANSPOSE (PLA_TRANSPOSE_OFFSET + 3)
#define PLA_CONJ_TRANS          (PLA_TRANSPOSE_OFFSET + 3)
#define PLA_CONJUGATE           (PLA_TRANSPOSE_OFFSET + 4)
#define PLA_CONJ                (PLA_TRANSPOSE_OFFSET + 4)

#define PLA_OWNER_OFFSET -30
#define PLA_ALL_ROWS    (PLA_OWNER_OFFSET - 1)
#define PLA_ALL_COLS    (PLA_OWNER_OFFSET - 2)

#define PLA_SIDE_OFFSET 40
#define PLA_SIDE_TOP    (PLA_SIDE_OFFSET + 1)
#define PLA_SIDE_BOTTOM (PLA_SIDE_OFFSET + 2)
#define PLA_SIDE_LEFT   (PLA_SIDE_OFFSET + 3)
#define PLA_SIDE_RIGHT  (PLA_SIDE_OFFSET + 4)

#define PLA_SHAPE_OFFSET 50
#define PLA_UPPER_TRIANGULAR        (PLA_SHAPE_OFFSET + 1)
#define PLA_UP_TRIAN                (PLA_SHAPE_OFFSET + 1)
#define PLA_LOWER_TRIANGULAR        (PLA_SHAPE_OFFSET + 2)
#define PLA_LOWER_TRIAN             (PLA_SHAPE_OFFSET + 2)
#define PLA_SHAPE_GENERAL           (PLA_SHAPE_OFFSET + 3)
#define PLA_SHAPE_LOWER_TRAPEZOIDAL (PLA_SHAPE_OFFSET + 4)
#define PLA_SHAPE_LOW_TRAP          (PLA_SHAPE_OFFSET + 4)
#define PLA_SHAPE_UPPER_TRAPEZOIDAL (PLA_SHAPE_OFFSET + 5)
#define PLA_SHAPE_UP_TRAP           (PLA_SHAPE_OFFSET + 5)

#define PLA_API_OFFSET 70
#define PLA_MODE_CLOSED      (PLA_API_OFFSET + 1)
#define PLA_MODE_OPEN        (PLA_API_OFFSET + 2)
#define PLA_STATE_API_ACTIVE (PLA_API_OFFSET + 3)
#define PLA_STATE_NORMAL     (PLA_API_OFFSET + 4)

#define PLA_OP_OFFSET 80
#define PLA_OP_MAT_PAN       (PLA_OP_OFFSET + 1)
#define PLA_OP_PAN_MAT       (PLA_OP_OFFSET + 2)
#define PLA_OP_PAN_PAN       (PLA_OP_OFFSET + 3)
/* INCLUDE/PLA_Versions.h:11-13: the stationary operand of PLA_Gemm_x */
#define PLA_VERSION_A        100
#define PLA_VERSION_B        200
#define PLA_VERSION_C        300
#define PLA_OP_PAN_TRIAN_MAT (PLA_OP_OFFSET + 4)
#define PLA_OP_SYM_PAN_PAN   (PLA_OP_OFFSET + 5)
#define PLA_OP_TRIAN_MAT_PAN (PLA_OP_OFFSET + 6)
#define PLA_OP_ALL_ALG       (PLA_OP_OFFSET + 7)

#define PLA_PROJ_OFFSET 90
#define PLA_PROJ_ONTO_COL (PLA_PROJ_OFFSET + 1)
#define PLA_PROJ_ONTO_ROW (PLA_PROJ_OFFSET + 2)

#define PLA_DIAG_OFFSET 100
#define PLA_UNIT_DIAG    (PLA_DIAG_OFFSET + 1)
#define PLA_NONUNIT_DIAG (PLA_DIAG_OFFSET + 2)
#define PLA_ZERO_DIAG    (PLA_DIAG_OFFSET + 3)

#define PLA_DUMMY        0
#define PLA_SUCCESS      0
#define PLA_ALIGN_FIRST  -200
#define PLA_DIM_ALL      -201
#define PLA_INHERIT      -202
#define PLA_UNDEFINED    -203

/* returned by a call that failed a fatal check (the reference exits instead) */
#define PLA_ERROR        -1000

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

/* ---- opaque handles (INCLUDE/PLA_Obj.h:82, INCLUDE/PLA_Template.h:31) ---- */
typedef struct PLA_Obj_view_struct *PLA_Obj;
typedef struct PLA_Template_struct *PLA_Template;

/* ---- library and template (TEMPLATE/PLA_Init.c, TEMPLATE/PLA_Temp.c) ---- */
int PLA_Init(PLA_B200_Comm comm);                                  /* PLA_Init.c:85 */
int PLA_Finalize(void);                                       /* PLA_Init.c:132 */
int PLA_Initialized(int *initialized);                        /* PLA_Init.c:113 */
int PLA_Comm_1D_to_2D(PLA_B200_Comm comm1d, int nprows, int npcols,
                      PLA_B200_Comm *comm2d);                      /* PLA_Init.c:20 */
int PLA_Comm_1D_to_2D_ratio(PLA_B200_Comm comm1d, float ratio,
                            PLA_B200_Comm *comm2d);                /* PLA_Init.c:38 */
int PLA_Temp_create(int nb, int zero_or_one, PLA_Template *templ); /* PLA_Temp.c:19 */
int PLA_Temp_free(PLA_Template *templ);                       /* PLA_Temp.c:136 */
int PLA_Temp_nb(PLA_Template templ, int *nb);                 /* PLA_Temp.c:176 */
int PLA_Temp_zero_or_one(PLA_Template templ, int *zero_or_one);
int PLA_Temp_comm_all_size(PLA_Template templ, int *nprocs);  /* PLA_Temp.c:169 */
int PLA_Temp_comm_all_rank(PLA_Template templ, int *rank);    /* PLA_Temp.c:205 */

/* algorithmic block size (TEMPLATE/PLA_Environ.c:54, :88) */
int pla_Environ_set_nb_alg(int op, int nb_alg);
int PLA_Environ_nb_alg(int op, PLA_Template templ, int *nb_alg);

/* diagnostics (OBJ/PLA_Diagnostics.c:402-432, :108-151) */
int PLA_Set_error_checking(int error, int parameters, int sequential, int r12);
int PLA_Get_error_checking(int *error, int *parameters, int *sequential, int *r12);
int PLA_Abort(char *message, int line, char *file);
int PLA_Warning(char *message);

/* ---- object creation (OBJ/PLA_Obj.c) ---------------------------------- */
int PLA_Matrix_create(PLA_B200_Datatype datatype, int length, int width,
                      PLA_Template templ, int align_row, int align_col,
                      PLA_Obj *new_obj);                      /* PLA_Obj.c:323 */
int PLA_Mvector_create(PLA_B200_Datatype datatype, int length, int width,
                       PLA_Template templ, int align, PLA_Obj *new_obj); /* :149 */
int PLA_Mscalar_create(PLA_B200_Datatype datatype, int owner_row, int owner_col,
                       int length, int width, PLA_Template templ,
                       PLA_Obj *new_obj);                     /* PLA_Obj.c:497 */
int PLA_Pmvector_create(PLA_B200_Datatype datatype, int project_onto, int owner,
                        int length, int width, PLA_Template templ, int align,
                        PLA_Obj *new_obj);                    /* PLA_Obj.c:740 */
int PLA_Matrix_create_conf_to(PLA_Obj obj, PLA_Obj *new_obj);
int PLA_Mvector_create_conf_to(PLA_Obj obj, int width, PLA_Obj *new_obj);
int PLA_Mscalar_create_conf_to(PLA_Obj obj, int owner_row, int owner_col,
                               PLA_Obj *new_obj);
int PLA_Pmvector_create_conf_to(PLA_Obj obj, int project_onto, int owner,
                                int width, PLA_Obj *new_obj);
int PLA_Create_constants_conf_to(PLA_Obj obj, PLA_Obj *minus_one,
                                 PLA_Obj *zero, PLA_Obj *one); /* PLA_Obj.c:4189 */
int PLA_Obj_free(PLA_Obj *obj);                               /* PLA_Obj.c:803 */

/* ---- views (OBJ/PLA_Obj.c:1929-3702) ------------------------------------ */
int PLA_Obj_view(PLA_Obj obj, int length, int width, int disp_row,
                 int disp_col, PLA_Obj *view);                /* :1929 */
int PLA_Obj_view_all(PLA_Obj obj, PLA_Obj *view);             /* :1981 */
int PLA_Obj_split_4(PLA_Obj obj, int length, int width, PLA_Obj *tl,
                    PLA_Obj *tr, PLA_Obj *bl, PLA_Obj *br);   /* :2063 */
int PLA_Obj_horz_split_2(PLA_Obj obj, int length, PLA_Obj *top,
                         PLA_Obj *bottom);                    /* :3122 */
int PLA_Obj_vert_split_2(PLA_Obj obj, int width, PLA_Obj *left,
                         PLA_Obj *right);                     /* :3156 */
int PLA_Obj_view_shift(PLA_Obj obj, int shift_top, int shift_left,
                       int shift_right, int shift_bottom);    /* :3189 */
int PLA_Obj_view_swap(PLA_Obj *obj1, PLA_Obj *obj2);

/* ---- inquiry (OBJ/PLA_Obj.c:831-1436) ------------------------------------ */
int PLA_Obj_objtype(PLA_Obj obj, int *objtype);
int PLA_Obj_datatype(PLA_Obj obj, PLA_B200_Datatype *datatype);
int PLA_Obj_template(PLA_Obj obj, PLA_Template *templ);
int PLA_Obj_global_length(PLA_Obj obj, int *length);
int PLA_Obj_global_width(PLA_Obj obj, int *width);
int PLA_Obj_global_name(PLA_Obj obj, int *name);
int PLA_Obj_global_align_row(PLA_Obj obj, int *align);
int PLA_Obj_global_align_col(PLA_Obj obj, int *align);
int PLA_Obj_local_length(PLA_Obj obj, int *length);
int PLA_Obj_local_width(PLA_Obj obj, int *width);
int PLA_Obj_local_ldim(PLA_Obj obj, int *ldim);
int PLA_Obj_local_stride(PLA_Obj obj, int *stride);
int PLA_Obj_local_buffer(PLA_Obj obj, void **buffer);   /* device pointer */
int PLA_Obj_owner_row(PLA_Obj obj, int *owner);
int PLA_Obj_owner_col(PLA_Obj obj, int *owner);
int PLA_Obj_project_onto(PLA_Obj obj, int *project_onto);
int PLA_Obj_set_orientation(PLA_Obj obj, int project_onto);

/* ---- contents (OBJ/PLA_Obj.c, host buffers) ------------------------------ */
int PLA_Obj_set_to_zero(PLA_Obj obj);
int PLA_Obj_set_to_one(PLA_Obj obj);
int PLA_Obj_set_to_minus_one(PLA_Obj obj);
int PLA_Obj_set_to_identity(PLA_Obj obj);
int PLA_Obj_set(PLA_Obj obj, PLA_B200_Datatype datatype, void *value);
int PLA_Obj_get_local_contents(PLA_Obj obj, int trans, int *rows_in_buf,
                               int *cols_in_buf, void *buf, int ldim_buf,
                               int stride_buf);
int PLA_Obj_set_local_contents(int trans, int rows_in_buf, int cols_in_buf,
                               void *buf, int ldim_buf, int stride_buf,
                               PLA_Obj obj);
int PLA_Copy(PLA_Obj from, PLA_Obj to);                       /* COPY/PLA_Copy.c:18 */

/* ---- application interface (API/PLA_API.c) -------------------------------- */
int PLA_API_begin(void);                                      /* :24 */
int PLA_API_end(void);                                        /* :61 */
int PLA_Obj_API_open(PLA_Obj obj);                            /* :126 */
int PLA_Obj_API_close(PLA_Obj obj);                           /* :166 */
int PLA_Obj_API_sync(PLA_Obj obj);                            /* :916 */
int PLA_API_axpy_vector_to_global(int size, void *alpha, void *local_vector,
                                  int local_stride, PLA_Obj obj,
                                  int global_displacement);   /* :220 */
int PLA_API_axpy_global_to_vector(int size, void *alpha, PLA_Obj obj,
                                  int global_displacement, void *local_vector,
                                  int local_stride);          /* :257 */
int PLA_API_axpy_matrix_to_global(int m, int n, void *alpha, void *local_matrix,
                                  int local_ldim, PLA_Obj obj, int disp_row,
                                  int disp_col);              /* :390 */
int PLA_API_axpy_global_to_matrix(int m, int n, void *alpha, PLA_Obj obj,
                                  int disp_row, int disp_col, void *local_matrix,
                                  int local_ldim);            /* :593 */

/* ---- timings (OBJ/PLA_Timings.c): the library's phase timers -------------- */
int PLA_Timings_initialize(void);                    /* OBJ/PLA_Timings.c:17 */
int PLA_Timings_print(void);                         /* OBJ/PLA_Timings.c:41 */
int PLA_Timings_average(void);                       /* OBJ/PLA_Timings.c:127 */

/* ---- host memory (OBJ/PLA_Memory.c; INCLUDE/PLA_Memory_prototypes.h) ------ */
/* as the reference: malloc / calloc with running totals of the bytes held.
 * Where the reference prints and exits on failure these return NULL and set
 * PLA_Last_error.  PLA_free returns NULL. */
void *PLA_malloc(size_t size);                       /* OBJ/PLA_Memory.c:18 */
void *PLA_calloc(size_t size, size_t typesize);      /* OBJ/PLA_Memory.c:51 */
void *PLA_free(void *buffer);                        /* OBJ/PLA_Memory.c:68 */
int PLA_Total_size_malloced(void);                   /* OBJ/PLA_Memory.c:87 */
int PLA_Max_size_malloced(void);                     /* OBJ/PLA_Memory.c:100 */

/* ---- out-of-core matrices (IO/PLA_File.c, OBJ/PLA_Obj_ooc.c) --------------- */
/* an out-of-core matrix keeps its data in a file (column-major, leading
 * dimension local_ldim elements); PLA_Copy moves blocks between its views and
 * in-core objects.  Errors return PLA_ERROR where the reference aborts. */
int PLA_OOC_Matrix_create_without_fd(PLA_B200_Datatype datatype, int global_length,
                                     int global_width, PLA_Template templ,
                                     int global_align_row, int global_align_col,
                                     PLA_Obj *new_obj);   /* OBJ/PLA_Obj_ooc.c:50 */
int PLA_Obj_attach_fd(PLA_Obj obj, int fd, int local_ldim,
                      int user_buffer);       /* OBJ/PLA_Obj_management.c:146 */
int PLA_File_create(char *filename, PLA_B200_Datatype datatype, int size, int *fd); /* IO/PLA_File.c:25 */
int PLA_File_open(char *filename, PLA_B200_Datatype datatype, int size, int *fd);   /* :47 */
int PLA_File_close(int fd);                          /* IO/PLA_File.c:61 */
int PLA_File_unlink(char *filename);                 /* IO/PLA_File.c:72 */
int PLA_File_stats_start(void);                      /* IO/PLA_File_stats.c:21 */
int PLA_File_stats_stop(void);                       /* IO/PLA_File_stats.c:53 */
/* left-looking tile Cholesky of the lower triangle of an out-of-core matrix;
 * returns 0 or the global 1-based failing column (the reference discards it) */
int PLA_OOC_Chol(int nb_ooc, int nb_tile, PLA_Obj A); /* POOCLAPACK/OOC_Cholesky/PLA_OOC_Chol.c:13 */

/* ---- solvers and parallel BLAS on the dense-solve path ------------------------ */
int PLA_LU(PLA_Obj A, PLA_Obj pivots);               /* SOLVERS/LU/PLA_LU.c:13 */
int PLA_LU_right(int nb_alg, PLA_Obj A, PLA_Obj pivots); /* SOLVERS/LU/PLA_LU.c:37 */
/* the unblocked panel factorization; A_11_msc receives the factored top block */
int PLA_LU_right_mv(PLA_Obj A_mv, PLA_Obj A_11_msc, PLA_Obj pivots_msc); /* PLA_LU_mv.c:13 */
/* the blocked LU whose interchanges skip the columns left of each panel */
int PLA_LU_linpack(PLA_Obj A, PLA_Obj pivots);       /* SOLVERS/LINPACK/PLA_LU_linpack.c:13 */
int PLA_LU_linpack_right(int nb_alg, PLA_Obj A, PLA_Obj pivots); /* :30 */
int PLA_Apply_pivots_to_rows(PLA_Obj A, PLA_Obj pivots); /* PLA_Apply_pivots_new.c:13 */
int PLA_Apply_pivots_to_columns_in_reverse(PLA_Obj A, PLA_Obj pivots); /* :309 */
int PLA_General_solve(PLA_Obj A, PLA_Obj pivots, PLA_Obj B); /* PLA_General.c:67 */
int PLA_Chol(int uplo, PLA_Obj A);                   /* SOLVERS/Cholesky/PLA_Chol.c:13 */
int PLA_Pos_def_solve(PLA_Obj A, PLA_Obj B);         /* PLA_Pos_def.c:44 */
int PLA_Trsv(int uplo, int trans, int diag, PLA_Obj A, PLA_Obj x); /* BLAS2/PLA_Trsv.c:15 */
int PLA_Trsm(int side, int uplo, int trans, int diag, PLA_Obj alpha, PLA_Obj A,
             PLA_Obj B);                             /* BLAS3/PLA_Trsm.c:13 */
int PLA_Gemm(int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B,
             PLA_Obj beta, PLA_Obj C);               /* BLAS3/PLA_Gemm.c:13 */
int PLA_Gemm_x(int version, int transa, int transb, PLA_Obj alpha, PLA_Obj A,
               PLA_Obj B, PLA_Obj beta, PLA_Obj C);  /* BLAS3/PLA_Gemm_x.c:13 */
int PLA_Gemv(int trans, PLA_Obj alpha, PLA_Obj A, PLA_Obj x, PLA_Obj beta,
             PLA_Obj y);                             /* BLAS2/PLA_Gemv.c */
int PLA_Iamax(PLA_Obj x, PLA_Obj k, PLA_Obj xmax);   /* BLAS1/PLA_Iamax.c:37 */
int PLA_Axpy(PLA_Obj alpha, PLA_Obj x, PLA_Obj y);   /* BLAS1/PLA_Axpy.c:13 */
int PLA_Nrm2(PLA_Obj x, PLA_Obj alpha);              /* BLAS1/PLA_Nrm2.c:13 */
int PLA_Shift(PLA_Obj obj, PLA_B200_Datatype datatype, void *value); /* UTIL/PLA_Shift.c:15 */
int PLA_Syrk_perform_local_part(int uplo, PLA_Obj alpha, PLA_Obj X,
                                PLA_Obj X_trans, PLA_Obj beta,
                                PLA_Obj A);  /* BLAS3/PLA_Syrk_perform_local_part.c:13 */

/* ---- node-local kernels (Local_BLAS/); on a 1x1 template local = global ---- */
int PLA_Local_gemm(int transa, int transb, PLA_Obj alpha, PLA_Obj A, PLA_Obj B,
                   PLA_Obj beta, PLA_Obj C);         /* PLA_Local_gemm.c:13 */
int PLA_Local_trsm(int side, int uplo, int trans, int diag, PLA_Obj alpha,
                   PLA_Obj A, PLA_Obj B);            /* PLA_Local_trsm.c:13 */
int PLA_Local_syrk(int uplo, int trans, PLA_Obj alpha, PLA_Obj A, PLA_Obj beta,
                   PLA_Obj C);                       /* PLA_Local_syrk.c:13 */
int PLA_Local_iamax(PLA_Obj x, int *index, void *value); /* PLA_Local_iamax.c:17 */
int PLA_Local_scal(PLA_Obj alpha, PLA_Obj x);        /* PLA_Local_BLAS1.c:68 */
int PLA_Local_axpy(PLA_Obj alpha, PLA_Obj x, PLA_Obj y); /* PLA_Local_BLAS1.c:327 */
int PLA_Local_nrm2(PLA_Obj x, PLA_Obj alpha);        /* PLA_Local_BLAS1.c:394 */
int PLA_Local_inv_scal(PLA_Obj alpha, PLA_Obj x);    /* PLA_Local_BLAS1.c:173 */
int PLA_Local_swap(PLA_Obj x, PLA_Obj y);            /* PLA_Local_BLAS1.c:562 */
int PLA_Local_copy(PLA_Obj from, PLA_Obj to);        /* PLA_Local_BLAS1.c:17 */
int PLA_Local_ger(PLA_Obj alpha, PLA_Obj x, PLA_Obj y, PLA_Obj A); /* PLA_Local_BLAS2.c:578 */
int PLA_Local_gemv(int trans, PLA_Obj alpha, PLA_Obj A, PLA_Obj x, PLA_Obj beta,
                   PLA_Obj y);                       /* PLA_Local_BLAS2.c:15 */
int PLA_Local_trsv(int uplo, int trans, int diag, PLA_Obj A,
                   PLA_Obj x);                       /* PLA_Local_BLAS2.c:478 */
int PLA_Local_chol(int uplo, PLA_Obj A);   /* SOLVERS/Cholesky/PLA_Local_chol.c:15 */

#ifdef __cplusplus
}
#endif

#include "pla_b200.h"

#ifdef PLA_B200_WITH_MPI
#include "pla_mpi_compat.h"
#endif

#endif /* PLA_B200_PLA_H */
