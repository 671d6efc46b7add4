/*
 * pla_b200.h — additions of the B200 library that have no counterpart in the
 * reference's headers.  Included by PLA.h.
 */
#ifndef PLA_B200_EXT_H
#define PLA_B200_EXT_H

#ifdef __cplusplus
extern "C" {
#endif

/* Copy the message of the last fatal error into buf (NUL-terminated, at most
 * len bytes).  Returns PLA_SUCCESS when no error has been recorded, else the
 * PLA_ERROR code of that error.  The reference prints and exits instead
 * (OBJ/PLA_Diagnostics.c:108-128). */
int PLA_Last_error(char *buf, int len);
int PLA_Clear_error(void);

/* PLA_LU plus a LAPACK-style info: 0, or the 1-based index of the first exact
 * zero pivot (the factorization still completes, as PLA_LU does). */
int PLA_LU_info(PLA_Obj A, PLA_Obj pivots, int *info);

/* The CUDA stream all library work is queued on (a cudaStream_t, passed as
 * void*).  NULL selects the library's own stream.  Every PLA_* call returns
 * after its work has completed on the device. */
int PLA_B200_set_stream(void *stream);
void *PLA_B200_get_stream(void);

/* Fill or extract an object from a DEVICE buffer (column-major, ldim >= the
 * object's length), for callers whose data is already in GPU memory.  The
 * host-buffer forms are PLA_Obj_set/get_local_contents. */
int PLA_Obj_set_local_contents_device(const void *dev_buf, int ldim, PLA_Obj obj);
int PLA_Obj_get_local_contents_device(PLA_Obj obj, void *dev_buf, int ldim);

/* Device time of the last solver call, in milliseconds, by phase. */
typedef struct {
  double total_ms;
  double panel_ms;   /* panel factorization (iamax, swap, scale, rank-1)  */
  double swap_ms;    /* row interchanges outside the panel                */
  double trsm_ms;    /* triangular solves with the diagonal block         */
  double update_ms;  /* trailing GEMM / SYRK                              */
  double solve_ms;   /* triangular solves with the right-hand sides       */
  double refine_ms;  /* residuals and corrections of iterative refinement */
  double convert_ms; /* precision conversions and operand packing         */
  int update_launches; /* trailing-update kernels timed in update_ms      */
  long long interchanges; /* LU row interchanges that moved rows (pivot
                             offset != 0), summed over the factorizations
                             timed; each costs a read and a write of two
                             elements in every column outside its panel   */
} PLA_Phase_times;
/* Phase timing uses CUDA events recorded on the library stream without
 * synchronizing; the times are collected when PLA_B200_phase_times is
 * called.  Timing stays on until switched off and accumulates across calls
 * until PLA_B200_reset_phase_times. */
int PLA_B200_phase_times(PLA_Phase_times *t);
int PLA_B200_set_phase_timing(int on);
int PLA_B200_reset_phase_times(void);

/* Number of CUDA kernels the library has launched since it was loaded. */
long PLA_B200_kernel_launches(void);

/* ---- mixed-precision solve with FP64 iterative refinement ------------------
 * Factor a low-precision copy of A (trailing updates on the tensor cores),
 * then refine x in FP64 until the normwise backward error
 *     ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
 * reaches tol.  A is read, never overwritten; B (n x nrhs) is overwritten by
 * X.  LU-IR corrects with the low-precision factors; GMRES-IR runs restarted
 * GMRES on A preconditioned by them (FP64 residual, orthogonalisation and
 * update).  The result is the same contract as PLA_General_solve /
 * PLA_Pos_def_solve: X overwrites B. */
#define PLA_B200_PREC_BF16   1   /* trailing update in bf16, fp32 accumulate */
#define PLA_B200_PREC_FP16   2   /* trailing update in fp16, fp32 accumulate */
#define PLA_B200_PREC_FP32   3   /* fp32 throughout                          */
#define PLA_B200_PREC_FP64   4   /* FP64 factors (the plain PLA_LU / PLA_Chol) */
#define PLA_B200_PREC_FP8    5   /* trailing update in fp8 E4M3 with one power-of-two
                                    scale per 128-row tile, fp32 accumulate; the
                                    Cholesky factors D A D, D = diag(A)^-1/2, and
                                    refines with M^-1 = D (L L')^-1 D */
#define PLA_B200_PREC_BF16X6 6   /* trailing update on the tensor cores with both
                                    operands split three ways into bf16 (x = p0 +
                                    p1 + p2) and six of the nine part products
                                    summed in fp32: fp32-level factors at about
                                    six times the bf16 tensor work */
#define PLA_B200_PREC_BF16X3 7   /* the same split, two ways (x = p0 + p1, about 16
                                    significant bits) and three part products: the
                                    trailing update and U12 at three times the bf16
                                    tensor work, factors about 2^-16 accurate */
#define PLA_B200_IR_LU       1   /* classic iterative refinement             */
#define PLA_B200_IR_GMRES    2   /* GMRES-IR                                 */
/* pivoting of the low-precision LU's fp32 panels (the FP64 PLA_LU always uses
 * the reference's partial pivoting) */
#define PLA_B200_PIVOT_PARTIAL    0 /* one pivot search over the panel per column */
#define PLA_B200_PIVOT_TOURNAMENT 1 /* tournament pivoting (CALU): each block of
                                       rows picks its pivot candidates on its own,
                                       the candidate sets meet in a reduction tree;
                                       the pivots differ from partial pivoting's */

typedef struct {
  int precision;        /* PLA_B200_PREC_*                                  */
  int refinement;       /* PLA_B200_IR_*                                    */
  int max_iterations;   /* outer refinement steps (default 50)              */
  int gmres_restart;    /* inner GMRES iterations per step (default 30)     */
  int nb;               /* block size of the low-precision factorization; 0 = nb_alg */
  int escalate;         /* 1 (default): when the refinement stagnates (a GMRES-IR
                           step, or two LU-IR steps in a row, that fail to halve
                           the backward error; a non-finite iterate;
                           max_iterations reached) or the low-precision
                           Cholesky breaks down, refactor one precision higher
                           (FP8 -> BF16 -> BF16X6 -> FP64; FP16, BF16X3 ->
                           BF16X6 -> FP64; FP32 -> FP64) and continue from the current
                           iterate.  Right after a low-precision factorization,
                           a diagonal range of its factors (max / min |u_ii|,
                           squared for a Cholesky factor) above 1e4 over the
                           precision's unit roundoff escalates one level at
                           once, without refining                           */
  double tol;           /* target backward error; <= 0 selects n * 2^-53    */
  int panel_pivoting;   /* PLA_B200_PIVOT_* of the fp32 LU panels (default
                           TOURNAMENT)                                       */
} PLA_Mixed_params;

typedef struct {
  int converged;          /* 1 when backward_error <= tol for every column */
  int iterations;         /* outer steps taken                              */
  int inner_iterations;   /* total GMRES iterations                         */
  int info;               /* LU: first zero pivot (1-based) or 0; Chol: failing column */
  double backward_error;  /* max over columns                               */
  double factor_ms;       /* device time of the factorization               */
  double refine_ms;       /* device time of the refinement                  */
  int precision_used;     /* PLA_B200_PREC_* of the factors that finished   */
  int factorizations;     /* 1 + the number of escalations                  */
} PLA_Mixed_report;

void PLA_Mixed_params_default(PLA_Mixed_params *p);
int PLA_General_solve_mixed(PLA_Obj A, PLA_Obj B, const PLA_Mixed_params *params,
                            PLA_Mixed_report *report);
int PLA_Pos_def_solve_mixed(PLA_Obj A, PLA_Obj B, const PLA_Mixed_params *params,
                            PLA_Mixed_report *report);
/* PLA_General_solve_mixed for a matrix that is still in host memory: A_host
 * (n x n FP64, column-major, leading dimension ldh >= n) is copied into the
 * device object A during the call.  For n >= 4096 and bf16 / fp16 / fp8
 * factors the copy overlaps the factorization: A travels in groups of
 * columns and each group joins the right-looking loop when it has arrived,
 * replaying the steps it missed, so the result does not depend on the
 * copy's timing.  A_host in page-locked memory (cudaHostAlloc) lets the copy
 * run asynchronously; pageable memory works, without the overlap. */
int PLA_General_solve_mixed_host(PLA_Obj A, const void *A_host, int ldh, PLA_Obj B,
                                 const PLA_Mixed_params *params, PLA_Mixed_report *report);

/* ---- panel factorization that allocates nothing ---------------------------
 * No counterpart in the reference.  Factors the m x w panel A (device memory,
 * column-major, lda >= m, w <= m) in place with partial pivoting, the column
 * loop PLA_LU runs on each panel: pivots[j] receives the reference's offset
 * encoding (row j was swapped with row j + pivots[j]), the swaps cover the
 * panel's own columns only.  status points to two device ints, both 0 on
 * entry: status[0] is set to 1 if a bounded wait in the kernel gave up,
 * status[1] to the 1-based column of the first exact zero pivot (the
 * factorization still completes, dividing by that zero, as PLA_LU does).
 * For callers that cannot let the library call cudaMalloc -- programs whose
 * GPU memory belongs to another allocator, or services that forbid allocation
 * while running: the kernel's workspace is a fixed array of about 667 KB in
 * device memory, present on every GPU that loads the library until the
 * process exits, instead of memory the library allocates.  Limit: w <= 128
 * (larger panels return PLA_ERROR with a message in PLA_Last_error).
 * The call is asynchronous on `stream` (a cudaStream_t, NULL for the default
 * stream).  The first call on a device, and the first after the device's
 * context was replaced (cudaDeviceReset), looks up the array's device address
 * and queues a clear of the array; make that call before any stream capture.
 * The array is cleared again once every 2^24 panel launches.  All calls share
 * the one array, so calls whose kernels overlap on the GPU (other streams,
 * other host threads) race: serialise them on one stream or synchronise
 * between them. */
int PLA_B200_lu_panel_noalloc(PLA_B200_Datatype datatype, int m, int w, void *A, int lda, int *pivots,
                              int *status, void *stream);

/* ---- batched factor-and-solve ------------------------------------------------
 * Many independent systems of uneven order, each factored in place (LU with
 * partial pivoting, or lower Cholesky) and solved for its right-hand sides, in
 * ONE persistent kernel launch replayed from a CUDA graph.  All pointers are
 * device pointers; A is n x n and B n x nrhs, column-major with leading
 * dimension n.  info (device, one int per instance) receives 0, the first
 * exact zero pivot (LU) or the failing column (Cholesky), 1-based. */
typedef struct {
  int n;
  int nrhs;
  int kind;       /* 0 = LU with partial pivoting, 1 = Cholesky (lower) */
  void *A;
  void *B;
  int *pivots;    /* LU only: n offsets in the reference's encoding */
} PLA_Batch_instance;

typedef struct PLA_Batch_plan_struct *PLA_Batch_plan;
/* Sort and bucket the instances, optionally autotune the schedule on a
 * synthetic sample of the same sizes, upload the descriptors and capture the
 * launch in a CUDA graph.  The instances' buffers must stay valid. */
int PLA_Batch_plan_create(PLA_B200_Datatype datatype, int count, const PLA_Batch_instance *instances,
                          int *info, int autotune, PLA_Batch_plan *plan);
int PLA_Batch_plan_execute(PLA_Batch_plan plan);
int PLA_Batch_plan_free(PLA_Batch_plan *plan);
/* create + execute + free, without autotuning */
int PLA_Batched_factor_solve(PLA_B200_Datatype datatype, int count,
                             const PLA_Batch_instance *instances, int *info);
/* the same work as a loop of per-instance launches of the single-matrix
 * kernels (the baseline the batched launch is measured against) */
int PLA_Batched_factor_solve_loop(PLA_B200_Datatype datatype, int count,
                                  const PLA_Batch_instance *instances);

/* The counters of PLA_File_stats_start/stop: bytes and seconds of the file
 * reads and writes since the last PLA_File_stats_start. */
int PLA_B200_file_stats(double *read_bytes, double *read_seconds, double *write_bytes,
                        double *write_seconds);

#ifdef __cplusplus
}
#endif

#endif
