// Internal declarations shared by the libbml_b200 translation units.
#pragma once

#include "../../include/bml_b200.h"

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstddef>

// ---------------------------------------------------------------------------
// Matrix structs.  The leading fields are bml's own (same names, types and
// order as ellpack/bml_types_ellpack.h:11-46 and ellblock/bml_types_ellblock.h:
// 11-54 without the optional MPI/mempool/cuSPARSE members); the device-side
// members follow them, the way the reference appends its csr* mirrors.
// ---------------------------------------------------------------------------

// Where the current contents of a matrix live.
enum MirrorState
{
    MIRROR_SYNCED = 0,    // host and device hold the same matrix
    MIRROR_HOST_NEWER = 1,  // host arrays were written; device is stale
    MIRROR_DEVICE_NEWER = 2 // a kernel wrote the device arrays; host is stale
};

struct bml_matrix_ellpack_t
{
    bml_matrix_type_t matrix_type;
    bml_matrix_precision_t matrix_precision;
    bml_distribution_mode_t distribution_mode;
    int N;
    int M;
    void *value;          // host mirror, row-major value[N*M]
    int *index;           // host mirror, row-major index[N*M]
    int *nnz;             // host mirror, nnz[N]
    bml_domain_t *domain;
    bml_domain_t *domain2;
    // device side
    void *d_value;        // value[N*ld]
    int *d_index;         // index[N*ld]
    int *d_nnz;           // nnz[N]
    int ld;               // device row stride in elements: M rounded up to 32
    int mirror;           // MirrorState
};

struct bml_matrix_ellblock_t
{
    bml_matrix_type_t matrix_type;
    bml_matrix_precision_t matrix_precision;
    bml_distribution_mode_t distribution_mode;
    int N;
    int M;
    int NB;
    int MB;
    void **ptr_value;     // host: pointer to block (ib, jp) at [ib*MB + jp] or NULL
    int *indexb;          // host mirror, indexb[NB*MB]
    int *nnzb;            // host mirror, nnzb[NB]
    int *bsize;           // block sizes, bsize[NB]
    bml_domain_t *domain;
    bml_domain_t *domain2;
    // host block pool: slot (ib*MB + jp) holds block (ib, jp) as a row-major
    // bsize[ib] x bsize[jb] array at h_pool + slot*slot_elems
    void *h_pool;
    // device side: the same slot layout
    void *d_pool;
    int *d_indexb;
    int *d_nnzb;
    int *d_bsize;
    int *d_boff;          // first scalar row of each block row, boff[NB+1]
    int maxbs;            // largest block size
    long long slot_elems; // maxbs*maxbs
    int mirror;
};

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
void b200_set_error(int status, const char *fmt, ...);
int b200_get_error();
// Sets whether errors are printed as they are recorded; returns the previous
// setting (a caller that expects and handles an error mutes it around the call).
int b200_swap_verbose(int on);

// Evaluates a CUDA runtime call; on failure records ERR_CUDA and yields false.
bool b200_cuda_ok(cudaError_t err, const char *what, const char *file, int line);
#define CUDA_OK(call) b200_cuda_ok((call), #call, __FILE__, __LINE__)
void b200_count_launch();
#define LAUNCH_OK(what) (b200_count_launch(), b200_cuda_ok(cudaGetLastError(), what, __FILE__, __LINE__))

// ---------------------------------------------------------------------------
// Device context: one CUDA stream per process on the current device, a
// growable scratch arena, and a small pinned host buffer for results that
// come back to the caller (traces, bounds, counters).
// ---------------------------------------------------------------------------
struct B200Context
{
    int device;
    int sm_count;
    size_t smem_optin;     // max dynamic shared memory per block (opt-in)
    cudaStream_t stream;
    void *scratch;
    size_t scratch_bytes;
    void *pinned;          // 64 KiB pinned host buffer
    void *d_small;         // 64 KiB device buffer for counters/flags
};

// Returns the context, initialising it on first use; nullptr (with
// ERR_NO_DEVICE recorded) when no usable GPU is present.
B200Context *b200_ctx();
// Device scratch of at least `bytes`, valid until the next call that grows it.
void *b200_scratch(size_t bytes);
// Synchronise the library stream; false (error recorded) on failure.
bool b200_sync();

// ---------------------------------------------------------------------------
// Matrix helpers (matrix.cu)
// ---------------------------------------------------------------------------
bool ell_is_supported(const bml_matrix_ellpack_t *A);
size_t prec_size(bml_matrix_precision_t p);
bml_matrix_ellpack_t *ell_alloc(bml_matrix_precision_t prec, int N, int M,
                                bml_distribution_mode_t mode, bool zero);
void ell_free(bml_matrix_ellpack_t *A);
bool ell_to_device(bml_matrix_ellpack_t *A);   // upload if host is newer
bool ell_to_host(bml_matrix_ellpack_t *A);     // download if device is newer
inline void ell_mark_device(bml_matrix_ellpack_t *A) { A->mirror = MIRROR_DEVICE_NEWER; }
inline void ell_mark_host(bml_matrix_ellpack_t *A) { A->mirror = MIRROR_HOST_NEWER; }

bml_domain_t *b200_default_domain(int N, int M, bml_distribution_mode_t mode);
void b200_free_domain(bml_domain_t *D);

// ---------------------------------------------------------------------------
// ELLPACK kernels (ellpack_*.cu).  All return false with an error recorded.
// ---------------------------------------------------------------------------
// C <- A*B (A==B allowed) thresholded with the diagonal kept, in the
// reference's first-touch column order.  trace (nullable) receives
// {sum of A's diagonal entries, sum of C's diagonal entries}.
// FP32 products may use the dense tier's f32 reduction at L2, which
// flushes subnormal sums to zero (used by mixed-precision SP2; off by default).
void ell_set_f32_reduce(bool on);
bool ell_multiply_AB(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B,
                     bml_matrix_ellpack_t *C, double threshold, double *trace,
                     int *required_M, int x2_rows = 0);
// The unordered product (ellpack_x2_fast.cu): the same products and keep
// rule, sums in no fixed order, rows written in ascending column order.
// ell_multiply_AB uses it unless the ordered (bit-identical) form is selected
// (bml_b200_set_x2_exact) or the row width exceeds what it holds.
bool ell_x2_exact();
bool ell_unordered_fits(const bml_matrix_ellpack_t *A);
bool ell_multiply_unordered(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C,
                            double threshold, double *trace, int *required_M, bool check_pre);
// C = A*B at P's pattern (the masked form of the unordered product): row i
// of C lists P's row i columns in P's order with the sums of their products
// (0 where there are none), no threshold.  *taken is false, with no status
// set, where the form does not apply (the ordered form selected, rows too
// wide for the kernel, or operands the dense tier takes); C needs P's M.
bool ell_multiply_masked(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *P,
                         bml_matrix_ellpack_t *C, bool *taken);
// The dense tier of the unordered product (ellpack_dense.cu): a GEMM on dense
// images when both operands' rows fill at least 40 % of their columns.
bool ell_dense_fits(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C, double threshold);
// Runs the dense tier when it applies (*taken); the result is the product's
// status then.
bool ell_multiply_dense_tier(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C,
                             double threshold, double *trace, int *required_M, bool *taken);
bool ell_multiply_dense(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C, double threshold,
                        double *trace, int *required_M);
// Wide-row forms (ellpack_wide.cu) of the operations whose shared-memory
// hash cannot hold a row: through a dense image of one operand.
bool ell_add_wide(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double alpha, double beta, double threshold);
bool ell_trace_mult_wide(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *trace);
bool ell_fnorm2_wide(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *result);
bool ell_restrict_wide(bml_matrix_ellpack_t *S, bml_matrix_ellpack_t *P, bml_matrix_ellpack_t *O);
// A view of rows [r0, r1) of A: the same storage, N = r1 - r0 (columns keep
// their global numbering).  Operations on the view touch only those rows.
bml_matrix_ellpack_t ell_row_view(const bml_matrix_ellpack_t *A, int r0, int r1);
bool ell_add(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double alpha,
             double beta, double threshold);
bool ell_add_identity(bml_matrix_ellpack_t *A, double beta, double threshold);
bool ell_scale(const void *scale, bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B);
bool ell_threshold(bml_matrix_ellpack_t *A, double threshold);
bool ell_threshold_new(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double threshold);
bool ell_trace(bml_matrix_ellpack_t *A, double *trace);
bool ell_trace_mult(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *trace);
bool ell_transpose_new(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B);
bool ell_copy(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B);
bool ell_gershgorin(bml_matrix_ellpack_t *A, double *bounds);
bool ell_sum_squares(bml_matrix_ellpack_t *A, double *result);
bool ell_fnorm2(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *result);
bool ell_convert(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B); // any precisions, same entries
// O <- S's values on P's pattern (P's order; 0 where S lacks the column); O may be P.
bool ell_restrict(bml_matrix_ellpack_t *S, bml_matrix_ellpack_t *P, bml_matrix_ellpack_t *O);
bool ell_import_dense(bml_matrix_ellpack_t *A, const void *dense, bml_dense_order_t order,
                      double threshold);
bool ell_export_dense(bml_matrix_ellpack_t *A, void *dense, bml_dense_order_t order);
bool ell_nnz_total(bml_matrix_ellpack_t *A, long long *total, int *maxrow);

// ---------------------------------------------------------------------------
// Small device utilities
// ---------------------------------------------------------------------------
#define B200_EMPTY_KEY (-1)

__host__ __device__ inline int b200_ceil_div(long long a, long long b)
{
    return (int) ((a + b - 1) / b);
}
__host__ __device__ inline int b200_round_up(int a, int b)
{
    return ((a + b - 1) / b) * b;
}
