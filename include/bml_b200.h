/*
 * bml_b200.h -- public C ABI of libbml_b200.so, a B200 (sm_100a) implementation
 * of bml's thresholded sparse matrix path (ELLPACK-R and ELLBLOCK) that links in
 * place of the reference libbml for that path.
 *
 * Every function below that carries a bml_ name has the reference's name,
 * signature, argument meaning and ownership rules; the citation beside each one
 * is the reference declaration it replaces (paths relative to the bml tree,
 * src/C-interface/).  Matrices live in device memory; every computing call runs
 * hand-written CUDA kernels on the current device and returns when its result is
 * complete.  There is no CPU fallback: without a usable GPU a call fails.
 *
 * Errors.  The reference logs, prints a backtrace and exit()s on any error
 * (bml_logger.c:92-116).  This library never exits or traps: it prints the same
 * kind of message to stderr, records a status that bml_b200_last_error() returns,
 * and leaves its outputs in a defined state (see each call).  Row overflow
 * (a result row wider than the output's M) is detected before anything is
 * written past M; the reference writes into the next row first
 * (ellpack/bml_multiply_ellpack_typed.c:301-330).
 *
 * Types and precisions.  ELLPACK and ELLBLOCK matrices in single_real and
 * double_real are supported.  Other types and precisions set
 * BML_B200_ERR_UNSUPPORTED and return NULL/0.
 */
#ifndef BML_B200_H
#define BML_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BML_B200_API __attribute__((visibility("default")))
#else
#define BML_B200_API
#endif

/* ---- types: same enumerators, same order, same struct layouts as the
 * reference (bml_types.h:7-129), so callers compiled against bml.h link
 * unchanged. ---------------------------------------------------------------- */
typedef enum
{
    type_uninitialized,
    dense,
    ellpack,
    ellblock,
    csr,
    distributed2d
} bml_matrix_type_t;

typedef enum
{
    precision_uninitialized,
    single_real,
    double_real,
    single_complex,
    double_complex
} bml_matrix_precision_t;

typedef enum
{
    dense_row_major,
    dense_column_major
} bml_dense_order_t;

typedef void bml_vector_t;
typedef void bml_matrix_t;

typedef struct
{
    int N_rows;
    int N_cols;
    int N_nz_max;
    int *bsizes;
    int NB;
} bml_matrix_dimension_t;

typedef enum
{
    sequential,
    distributed,
    graph_distributed
} bml_distribution_mode_t;

struct bml_domain_t
{
    int totalProcs;
    int totalRows;
    int totalCols;
    int globalRowMin;
    int globalRowMax;
    int globalRowExtent;
    int maxLocalExtent;
    int minLocalExtent;
    int *localRowMin;
    int *localRowMax;
    int *localRowExtent;
    int *localElements;
    int *localDispl;
};
typedef struct bml_domain_t bml_domain_t;

typedef enum
{
    BML_LOG_DEBUG,
    BML_LOG_INFO,
    BML_LOG_WARNING,
    BML_LOG_ERROR
} bml_log_level_t;

/* ---- allocation (bml_allocate.h) ---------------------------------------- */
BML_B200_API void *bml_allocate_memory(size_t s);                 /* bml_allocate.h:13 */
BML_B200_API void *bml_noinit_allocate_memory(size_t s);          /* bml_allocate.h:16 */
BML_B200_API void bml_free_memory(void *ptr);                     /* bml_allocate.h:23 */
BML_B200_API void bml_free_ptr(void **ptr);                       /* bml_allocate.h:26 */
BML_B200_API int bml_allocated(bml_matrix_t *A);                  /* bml_allocate.h:10 */
BML_B200_API void bml_deallocate(bml_matrix_t **A);               /* bml_allocate.h:29 */
BML_B200_API void bml_deallocate_domain(bml_domain_t *D);         /* bml_allocate.h:32 */
BML_B200_API void bml_clear(bml_matrix_t *A);                     /* bml_allocate.h:35 */
BML_B200_API bml_matrix_t *bml_noinit_matrix(bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, int N, int M,
    bml_distribution_mode_t distrib_mode);                        /* bml_allocate.h:44 */
BML_B200_API bml_matrix_t *bml_zero_matrix(bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, int N, int M,
    bml_distribution_mode_t distrib_mode);                        /* bml_allocate.h:51 */
BML_B200_API bml_matrix_t *bml_random_matrix(bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, int N, int M,
    bml_distribution_mode_t distrib_mode);                        /* bml_allocate.h:58 */
BML_B200_API bml_matrix_t *bml_banded_matrix(bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, int N, int M,
    bml_distribution_mode_t distrib_mode);                        /* bml_allocate.h:65 */
BML_B200_API bml_matrix_t *bml_identity_matrix(bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, int N, int M,
    bml_distribution_mode_t distrib_mode);                        /* bml_allocate.h:72 */
BML_B200_API bml_domain_t *bml_default_domain(int N, int M,
    bml_distribution_mode_t distrib_mode);                        /* bml_allocate.h:79 */

/* ---- introspection (bml_introspection.h) -------------------------------- */
BML_B200_API bml_matrix_type_t bml_get_type(bml_matrix_t *A);               /* :8  */
BML_B200_API bml_matrix_type_t bml_get_deep_type(bml_matrix_t *A);          /* :11 */
BML_B200_API bml_matrix_precision_t bml_get_precision(bml_matrix_t *A);     /* :14 */
BML_B200_API int bml_get_N(bml_matrix_t *A);                                /* :17 */
BML_B200_API int bml_get_M(bml_matrix_t *A);                                /* :20 */
BML_B200_API int bml_get_NB(bml_matrix_t *A);                               /* :23 */
BML_B200_API int bml_get_row_bandwidth(bml_matrix_t *A, int i);             /* :26 */
BML_B200_API int bml_get_bandwidth(bml_matrix_t *A);                        /* :30 */
BML_B200_API double bml_get_sparsity(bml_matrix_t *A, double threshold);    /* :33 */
BML_B200_API bml_distribution_mode_t bml_get_distribution_mode(bml_matrix_t *A); /* :37 */

/* ---- copy / convert / import / export / elements ------------------------ */
BML_B200_API bml_matrix_t *bml_copy_new(bml_matrix_t *A);                   /* bml_copy.h:8  */
BML_B200_API void bml_copy(bml_matrix_t *A, bml_matrix_t *B);               /* bml_copy.h:11 */
BML_B200_API bml_matrix_t *bml_convert(bml_matrix_t *A, bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, int M,
    bml_distribution_mode_t distrib_mode);                                  /* bml_convert.h:8 */
BML_B200_API bml_matrix_t *bml_import_from_dense(bml_matrix_type_t matrix_type,
    bml_matrix_precision_t matrix_precision, bml_dense_order_t order, int N, int M,
    void *A, double threshold, bml_distribution_mode_t distrib_mode);      /* bml_import.h:8 */
BML_B200_API void *bml_export_to_dense(bml_matrix_t *A, bml_dense_order_t order); /* bml_export.h:8 */
BML_B200_API void *bml_get_element(bml_matrix_t *A, int i, int j);          /* bml_getters.h:8  */
BML_B200_API void *bml_get_row(bml_matrix_t *A, int i);                     /* bml_getters.h:13 */
BML_B200_API void *bml_get_diagonal(bml_matrix_t *A);                       /* bml_getters.h:17 */
BML_B200_API void bml_set_element_new(bml_matrix_t *A, int i, int j, void *value); /* bml_setters.h:8  */
BML_B200_API void bml_set_element(bml_matrix_t *A, int i, int j, void *value);     /* bml_setters.h:14 */
BML_B200_API void bml_set_row(bml_matrix_t *A, int i, void *row, double threshold); /* bml_setters.h:20 */
BML_B200_API void bml_set_diagonal(bml_matrix_t *A, void *diagonal, double threshold); /* bml_setters.h:26 */

/* ---- the thresholded sparse path ---------------------------------------- */
/* C <- alpha*A*B + beta*C, thresholded (bml_multiply.h:9; bml_multiply.c:27-59). */
BML_B200_API void bml_multiply(bml_matrix_t *A, bml_matrix_t *B, bml_matrix_t *C,
    double alpha, double beta, double threshold);
/* X2 <- X*X thresholded; returns malloc'd double[2] = {tr X, tr X2}, released
 * with bml_free_memory() (bml_multiply.h:18; bml_multiply.c:71-101). */
BML_B200_API void *bml_multiply_x2(bml_matrix_t *X, bml_matrix_t *X2, double threshold);
/* C <- A*B thresholded, diagonal kept (bml_multiply.h:24; bml_multiply.c:114-144). */
BML_B200_API void bml_multiply_AB(bml_matrix_t *A, bml_matrix_t *B, bml_matrix_t *C,
    double threshold);
/* As bml_multiply_AB, doubling the threshold until every row fits in C's M
 * (bml_multiply.h:31; ellpack/bml_multiply_ellpack_typed.c:566-707). */
BML_B200_API void bml_multiply_adjust_AB(bml_matrix_t *A, bml_matrix_t *B,
    bml_matrix_t *C, double threshold);
/* A <- alpha*A + beta*B thresholded (bml_add.h:8; bml_add.c:26-57). */
BML_B200_API void bml_add(bml_matrix_t *A, bml_matrix_t *B, double alpha, double beta,
    double threshold);
/* A <- A + beta*I (bml_add.h:22); A <- alpha*A + beta*I (bml_add.h:27). */
BML_B200_API void bml_add_identity(bml_matrix_t *A, double beta, double threshold);
BML_B200_API void bml_scale_add_identity(bml_matrix_t *A, double alpha, double beta,
    double threshold);
/* In-place and copying threshold (bml_threshold.h:8-12; bml_threshold.c:30-89). */
BML_B200_API bml_matrix_t *bml_threshold_new(bml_matrix_t *A, double threshold);
BML_B200_API void bml_threshold(bml_matrix_t *A, double threshold);
/* tr A and tr(A*B) (bml_trace.h:9-13; bml_trace.c:20-88). */
BML_B200_API double bml_trace(bml_matrix_t *A);
BML_B200_API double bml_trace_mult(bml_matrix_t *A, bml_matrix_t *B);
/* Transpose (bml_transpose.h:9-12; bml_transpose.c:21-85). */
BML_B200_API bml_matrix_t *bml_transpose_new(bml_matrix_t *A);
BML_B200_API void bml_transpose(bml_matrix_t *A);
/* Norms (bml_norm.h:8-45), ELLPACK.  bml_fnorm2 is ||A - B||_F with the
 * reference's rule for entries of B that A lacks or holds as 0. */
BML_B200_API double bml_sum_squares(bml_matrix_t *A);                      /* bml_norm.h:9  */
BML_B200_API double bml_fnorm(bml_matrix_t *A);                            /* bml_norm.h:35 */
BML_B200_API double bml_fnorm2(bml_matrix_t *A, bml_matrix_t *B);          /* bml_norm.h:39 */

/* Scaling (bml_scale.h:8-17). scale_factor points to a value of A's precision. */
BML_B200_API bml_matrix_t *bml_scale_new(void *scale_factor, bml_matrix_t *A);
BML_B200_API void bml_scale(void *scale_factor, bml_matrix_t *A, bml_matrix_t *B);
BML_B200_API void bml_scale_inplace(void *scale_factor, bml_matrix_t *A);
/* Gershgorin bounds -> malloc'd double[2] = {emin, emax}; normalisation to
 * (emax*I - A)/(emax - emin) (bml_normalize.h:9-15). */
BML_B200_API void *bml_gershgorin(bml_matrix_t *A);
BML_B200_API void bml_normalize(bml_matrix_t *A, double mineval, double maxeval);

/* ---- ELLBLOCK block partition (ellblock/bml_allocate_ellblock.h:199-210) -- */
BML_B200_API void bml_set_block_sizes(int *bsize, int nb, int mb);
BML_B200_API int *bml_get_block_sizes(int N, int M);
BML_B200_API int bml_get_nb(void);
BML_B200_API int bml_get_mb(void);

/* Forget the process-wide block partition so that another can be set (the
 * reference allows one per process; no counterpart there). */
BML_B200_API void bml_b200_reset_block_sizes(void);

/* ---- init / shutdown / logging / printing -------------------------------- */
BML_B200_API void bml_init(void);                                  /* bml_init.h:12 (non-MPI form) */
BML_B200_API void bml_shutdown(void);                              /* bml_shutdown.h:8 */
/* one process per library context: rank 0 of 1 (the reference's non-MPI build) */
BML_B200_API int bml_getNRanks(void);                              /* bml_parallel.h:22 */
BML_B200_API int bml_getMyRank(void);                              /* bml_parallel.h:26 */
BML_B200_API int bml_printRank(void);                              /* bml_parallel.h:38 */
BML_B200_API void bml_log(bml_log_level_t log_level, char *format, ...);  /* bml_logger.h:24 */
BML_B200_API void bml_log_location(bml_log_level_t log_level, char *filename,
    int linenumber, char *format, ...);                            /* bml_logger.h:29 */
BML_B200_API char *bml_version(void);                              /* bml_logger.h:36 */
BML_B200_API void bml_print_version(void);                         /* bml_logger.h:39 */
BML_B200_API void bml_print_dense_matrix(int N, bml_matrix_precision_t matrix_precision,
    bml_dense_order_t order, void *A, int i_l, int i_u, int j_l, int j_u); /* bml_utilities.h:9 */
BML_B200_API void bml_print_bml_matrix(bml_matrix_t *A, int i_l, int i_u, int j_l,
    int j_u);                                                      /* bml_utilities.h:31 */
BML_B200_API void bml_read_bml_matrix(bml_matrix_t *A, char *filename);   /* bml_utilities.h:38 */
BML_B200_API void bml_write_bml_matrix(bml_matrix_t *A, char *filename);  /* bml_utilities.h:42 */
BML_B200_API int bml_sqrtint(const int x);                         /* bml_utilities.h:46 */

/* ======================================================================== *
 * B200 extensions.  None of these exists in the reference; they give callers
 * status codes, raw-array transfer and the SP2 solver that consumers of the
 * reference write themselves.
 * ======================================================================== */
enum
{
    BML_B200_OK = 0,
    BML_B200_ERR_NO_DEVICE = 1,    /* no CUDA device, or the kernels do not load */
    BML_B200_ERR_CUDA = 2,         /* a CUDA call failed */
    BML_B200_ERR_INVALID = 3,      /* bad argument (NULL, size mismatch, index out of range) */
    BML_B200_ERR_UNSUPPORTED = 4,  /* matrix type or precision outside this library */
    BML_B200_ERR_ROW_OVERFLOW = 5, /* a result row needs more than M entries */
    BML_B200_ERR_ALLOC = 6,        /* device or host allocation failed */
    BML_B200_ERR_TIMEOUT = 7       /* a bounded device-side wait ran out */
};

/* Status of the most recent failing call on this thread (0 if none since the
 * last clear), its text, and a reset. */
BML_B200_API int bml_b200_last_error(void);
BML_B200_API const char *bml_b200_error_string(int status);
BML_B200_API void bml_b200_clear_error(void);
/* Suppress (0) or enable (1, default) the stderr message printed on error. */
BML_B200_API void bml_b200_set_verbose(int on);

/* Status-returning X^2: same semantics as bml_multiply_x2, traces written to
 * trace[0..1].  On ROW_OVERFLOW each overflowing row keeps its first M entries
 * (in the reference's first-touch order) and the traces are still exact. */
BML_B200_API int bml_b200_multiply_x2(bml_matrix_t *X, bml_matrix_t *X2,
    double threshold, double *trace);
/* Largest row width that the last X^2 / multiply on this thread needed before
 * truncation to M (lets a caller size M exactly after ROW_OVERFLOW). */
BML_B200_API int bml_b200_last_required_M(void);

/* Row-sharded SP2 (no reference counterpart; the reference distributes rows
 * over MPI ranks).  bml_b200_multiply_x2_rows forms rows [r0, r1) of X^2
 * from all of X (X2's other rows are left as they are; overflow is reported
 * on the thresholded width as for X^2) and returns those rows' partial
 * traces.  bml_b200_sp2_update_rows applies the SP2 step to rows [r0, r1):
 * X <- X2 (branch 0) or X <- 2X - X2 thresholded (branch 1).  A caller on
 * several GPUs sums the partial traces over ranks, chooses the branch, then
 * gathers every rank's rows of X before the next X^2. */
BML_B200_API int bml_b200_multiply_x2_rows(bml_matrix_t *X, bml_matrix_t *X2, double threshold,
    int r0, int r1, double *trace);
BML_B200_API int bml_b200_sp2_update_rows(bml_matrix_t *X, bml_matrix_t *X2, double threshold,
    int branch, int r0, int r1);

/* Diagnostics of the last ELLPACK multiply: rows per kernel tier, in the
 * order A (one warp, 1024-slot table), W8, B1 (four warps, 2048 slots,
 * TMA-staged rows), W16 (8/16 warps per row, each warp owning a share of the
 * column classes k % 32 with a 256-slot table), K4, K8 (8 warps, bitmap-ranked
 * accumulator of up to 4096/8192 columns), C (dense accumulator in device
 * memory).  Returns the tier count. */
BML_B200_API int bml_b200_last_tier_counts(int *counts, int n);

/* Selects the multiply tiers later ELLPACK multiplies may use: bit t enables
 * tier t in the order of bml_b200_last_tier_counts; the dense tier C is
 * always enabled; 0 restores the default (A and C).  Any choice gives the same result
 * (the tiers differ only in speed), and rows a tier cannot hold move on to the
 * next enabled one.  Also discards the per-row width estimates kept from the
 * last multiply.  Returns the previous mask.  No reference counterpart. */
BML_B200_API int bml_b200_set_x2_tiers(int mask);

/* Chooses how later ELLPACK products (bml_multiply_x2, bml_multiply,
 * bml_multiply_AB and the SP2 drivers) sum.  exact = 0 (the default): the
 * unordered kernel, which forms the same products and applies the same keep
 * rule but adds the products of one entry in no fixed order (each still a
 * separately rounded multiply and add), so an entry differs from the
 * reference's by at most (n-1) u sum|a_ij b_jk| for n products, and writes a
 * row's kept entries in ascending column order.  exact = 1: the ordered tiers
 * above, bit-identical to the reference, rows in its first-touch order.
 * Rows wider than the unordered kernel holds (M above about 8000) always use
 * the ordered tiers.  Returns the previous choice.  No reference counterpart. */
BML_B200_API int bml_b200_set_x2_exact(int exact);

/* The unordered X^2 of an exactly symmetric matrix (each entry's mirror holds
 * the same bits, checked on the device every call) forms only the columns
 * k >= i of each row and mirrors them: half the products, the same result
 * bound, and an exactly symmetric X^2.  set_x2_symmetric(0) forbids that form
 * (the full product runs); returns the previous setting (default 1).
 * last_x2_symmetric() is 1 when the last unordered product took it.  No
 * reference counterpart. */
BML_B200_API int bml_b200_set_x2_symmetric(int allow);
BML_B200_API int bml_b200_last_x2_symmetric(void);

/* Diagnostics: with set_kernel_timing(1), later unordered products time
 * their product kernel (the kernel that forms and sums the products) with
 * CUDA events on the library stream; last_x2_kernel_ms() returns that time
 * for the last product, or -1.  set_kernel_timing returns the previous
 * setting.  No reference counterpart. */
/* The dense tier of the unordered product: when both operands' rows fill at
 * least 40 % of their columns on average (and the dense images fit 64 GiB),
 * A and B are scattered into dense images, multiplied by a register-tiled
 * GEMM and compacted with the same keep rule, rows in ascending column
 * order.  set_dense_tier(0) forbids it (default 1; returns the previous
 * setting); last_x2_dense() is 1 when the last unordered product ran on it.
 * No reference counterpart. */
BML_B200_API int bml_b200_set_dense_tier(int allow);
BML_B200_API int bml_b200_last_x2_dense(void);
BML_B200_API int bml_b200_set_kernel_timing(int on);
BML_B200_API double bml_b200_last_x2_kernel_ms(void);

/* Device-memory budget, in bytes, for the accumulator slabs of the exact
 * ELLBLOCK products (bml_multiply_x2, bml_multiply_AB, bml_multiply): every
 * CTA holds a slot for each block column a row can touch, NB of them, when
 * that fits the budget; otherwise it first holds MB + 1 slots and a call
 * whose rows touch more runs again with NB slots on fewer CTAs.  0 restores
 * the default of 24 GiB.  Results do not depend on it.  Returns the previous
 * budget.  No reference counterpart. */
BML_B200_API long long bml_b200_set_ellblock_slab_budget(long long bytes);

/* Raw ELLPACK transfer between the device matrix and caller host arrays laid
 * out like the reference (row-major value[N*M], index[N*M], nnz[N]).  Only
 * the columns up to the widest row are transferred: entries past a row's nnz
 * are neither read from the device nor written to the caller's arrays.
 * Upload rejects an nnz outside [0, M] (BML_B200_ERR_INVALID). */
BML_B200_API int bml_b200_ellpack_upload(bml_matrix_t *A, const void *value,
    const int *index, const int *nnz);
BML_B200_API int bml_b200_ellpack_download(bml_matrix_t *A, void *value, int *index,
    int *nnz);
/* Device pointers and row stride (elements) of an ELLPACK matrix. */
BML_B200_API int bml_b200_ellpack_device_arrays(bml_matrix_t *A, void **d_value,
    int **d_index, int **d_nnz, int *ld);
/* Number of non-zeros of a matrix (sum of nnz), computed on the device. */
BML_B200_API long long bml_b200_nnz(bml_matrix_t *A);
/* Wait for all work this library queued. */
BML_B200_API int bml_b200_synchronize(void);
/* Select the CUDA device the library starts on (before its first call; one
 * process per GPU).  Default: the thread's current device. */
BML_B200_API int bml_b200_set_device(int device);
/* Number of kernels this library has launched so far in this process. */
BML_B200_API unsigned long long bml_b200_launch_count(void);
/* CUDA events on the library's stream (slots 0..63), for timing its work on
 * the device: record, then milliseconds between two recorded slots. */
BML_B200_API int bml_b200_event_record(int slot);
BML_B200_API int bml_b200_event_elapsed(int a, int b, float *ms);
/* Device properties this library uses: SM count, device ordinal. */
BML_B200_API int bml_b200_device_info(int *sm_count, int *device);

/* Trace of an ELLPACK matrix without allocating memory.  No counterpart in
 * the reference: for callers that may not have the library allocate -- an
 * application that owns all device memory through its own fixed pool, or a
 * latency-critical loop where cudaMalloc/cudaFree (which synchronise the
 * device) are not acceptable.  Inputs are the matrix's device arrays (as
 * bml_b200_ellpack_device_arrays returns them, or the caller's own):
 * row-major value[N*ld] of the given precision (single_real or double_real),
 * index[N*ld], nnz[N]; the trace is written to *d_trace, one double in device
 * memory owned by the caller; the kernels run on `stream` (NULL: the default
 * stream) and the call returns without waiting for them.  Scratch is a fixed
 * array of 2^19 doubles (4 MiB) compiled into the library, held on every GPU
 * that loads it until the process exits: N above 2^19 is rejected with
 * BML_B200_ERR_INVALID.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress, with the device current); make that
 * first call before any stream capture.  All calls share the array and it
 * keeps the last call's contents, so calls that overlap on the GPU race on
 * it; calls on one stream are safe.  No cudaMalloc, cudaFree or allocating
 * library routine is called. */
BML_B200_API int bml_b200_ellpack_trace_noalloc(const void *d_value, const int *d_index,
    const int *d_nnz, int N, int ld, int precision, double *d_trace, void *stream);

/* SP2 density-matrix purification (Niklasson, PRB 66, 155115 (2002)), the
 * consumer loop around bml_multiply_x2 that PROGRESS/LATTE write on top of bml:
 *   X0 = (emax I - H)/(emax - emin) with Gershgorin bounds of H;
 *   repeat: X2 = X*X (thresholded), t = tr X, t2 = tr X2;
 *           X <- X2        if |t2 - occ| <= |2t - t2 - occ|,
 *           X <- 2X - X2   otherwise (thresholded add);
 *   stop when |t - t2| < tol, when the idempotency error |t - t2| has not
 *   decreased for `stall` iterations (stall <= 0 disables), or at maxiter.
 * H is not modified.  D receives the final X and must have H's type and
 * precision (its M bounds every iterate; overflow stops the solve with
 * ROW_OVERFLOW).  info (may be NULL) receives: [0] iterations run, [1] stop
 * rule (1 tol, 2 stall, 3 maxiter, 4 error), [2] tr D, [3] last |t - t2|,
 * [4] max row width seen, [5] seconds spent in X^2 calls. */
BML_B200_API int bml_b200_sp2(bml_matrix_t *H, bml_matrix_t *D, double threshold,
    double occupation, int maxiter, double tol, int stall, double *info);

/* SP2 in mixed precision (no reference counterpart).  H and D are
 * double_real ELLPACK.  The Gershgorin bounds and X0 are formed in FP64; the
 * first iterations (up to maxiter - nclose, with the tol/stall rules of
 * bml_b200_sp2) run on an FP32 copy of X: FP32 products and sums in X^2, FP32
 * adds, with the traces summed in FP64 and the branch choice and stop tests
 * made in FP64.  The last nclose iterations run in FP64 on X converted back,
 * as a closing refinement (they always run).  info (may be NULL) receives
 * the eight values [0] iterations run in all, [1] stop rule of the FP32
 * phase, [2] tr D, [3] last |t - t2|, [4] max row width, [5] seconds in all
 * X^2 calls, [6] FP32 iterations, [7] seconds in the FP32 X^2 calls. */
BML_B200_API int bml_b200_sp2_mixed(bml_matrix_t *H, bml_matrix_t *D, double threshold,
    double occupation, int maxiter, double tol, int stall, int nclose, double *info);

/* ELLBLOCK X^2 on the tensor cores (no reference counterpart): X is scaled
 * by a power of two, each 32x32 block x is split as hi = fp16(x), lo =
 * fp16(x - hi), and the block products are formed as hi*hi + hi*lo + lo*hi
 * on tcgen05 with FP32 accumulation, scaled back and written in X2's
 * precision; blocks are kept as by bml_multiply_x2 (kb == ib
 * or max |x| > threshold).  trace (may be NULL) receives {tr X, tr X2}.  Every
 * block of X and X2 must be 32 x 32 (bml_set_block_sizes); otherwise
 * UNSUPPORTED; so are NB > 65536, MB > 32767, and inputs whose per-group
 * tables would take more than 16 GiB of device memory.  Blocks of a row come
 * out in ascending block column. */
BML_B200_API int bml_b200_ellblock_multiply_x2_tc(bml_matrix_t *X, bml_matrix_t *X2, double threshold,
    double *trace);

/* Chooses the split of bml_b200_ellblock_multiply_x2_tc (no reference
 * counterpart) and returns the previous choice.  0 (the default): FP16 hi/lo
 * halves, three products per block pair, FP32 accumulation in tensor memory
 * (about 1e-5 of the product magnitudes per entry).  1: each entry as five
 * signed 8-bit slices of its row's (left operand) or column's (right
 * operand) power-of-two scale, the fifteen slice products of order <= 6 per
 * block pair on kind::i8 with exact INT32 accumulation, recombined in FP64:
 * within about 2^-33 of the row and column scales per product term, with no
 * accumulation error.  Takes NB <= 24576 and groups of four block rows with
 * at most 3276 block columns (else UNSUPPORTED). */
BML_B200_API int bml_b200_set_tc_split(int mode);

/* SP2 on ELLBLOCK matrices in mixed precision (no reference counterpart):
 * bulk iterations use bml_b200_ellblock_multiply_x2_tc, the last nclose
 * iterations the matrix-precision X^2 of bml_multiply_x2; adds, copies, the
 * branch choice and the stop tests as bml_b200_sp2.  A bulk iteration that
 * the tensor-core X^2 rejects as UNSUPPORTED (blocks other than 32 x 32, or
 * a partition beyond its limits) runs on the exact X^2.
 * info as for bml_b200_sp2_mixed ([4] is 0; [6] and [7] count the
 * iterations that ran on the tensor cores). */
BML_B200_API int bml_b200_ellblock_sp2_mixed(bml_matrix_t *H, bml_matrix_t *D, double threshold,
    double occupation, int maxiter, double tol, int stall, int nclose, double *info);

/* Density-matrix response of SP2 (no reference counterpart): the gradient of
 * L = sum_ij D_ij V_ij with respect to the stored entries of H, where D is X
 * after `iters` iterations of bml_b200_sp2's loop from H (fixed count, no stop
 * test).  Thresholds and branch choices are held fixed; the Gershgorin bounds'
 * dependence on H is included.  The forward pass keeps X every `every`
 * iterations and recomputes the iterates in between on the way back, so at
 * most iters/every + every iterates are held.  Iterates have M entries per
 * row.  H, V, dH: ELLPACK of one precision and N; dH receives the gradient on
 * H's pattern (H's order) and must be distinct from H and V.  *loss (may be
 * NULL) receives L. */
BML_B200_API int bml_b200_sp2_adjoint(bml_matrix_t *H, bml_matrix_t *V, double threshold,
    double occupation, int iters, int every, int M, bml_matrix_t *dH, double *loss);

/* Synthetic Hamiltonians (host arrays in the reference ELLPACK layout), seeded
 * splitmix64 + Box-Muller, symmetric.  Used to give the oracle and this
 * library byte-identical inputs.
 *   kind 1: 1-D chain, H_ii ~ U[-1,1], H_ij = u exp(-|i-j|/4), 0<|i-j|<=16.
 *   kind 2: L^3 cubic lattice (x fastest), neighbours with |r| <= radius,
 *           H_ij = -exp(-d)(1 + 0.1 g), H_ii ~ N(0,1); first N sites kept.
 * Returns the number of rows written, or -1 if a row needs more than M. */
BML_B200_API int bml_b200_gen_chain(int N, int M, unsigned long long seed,
    double *value, int *index, int *nnz);
BML_B200_API int bml_b200_gen_lattice(int L, int radius, int N, int M,
    unsigned long long seed, double *value, int *index, int *nnz);

/* ELLBLOCK Hamiltonian on a block lattice: L^3 block sites (x fastest),
 * block (a, b) present when the sites are within `radius`, entries
 * N(0,1) exp(-d), symmetric, seeded splitmix64 + Box-Muller.  The block
 * partition must already be L^3 blocks of bs with MB at least the number of
 * neighbours (bml_set_block_sizes).  Returns a new matrix or NULL. */
BML_B200_API bml_matrix_t *bml_b200_gen_block_lattice(int L, double radius, int bs,
    unsigned long long seed, bml_matrix_precision_t precision);

#ifdef __cplusplus
}
#endif
#endif /* BML_B200_H */
