// ELLBLOCK (block ELLPACK) matrices: storage, host mirror, constructors,
// element access, and the block-row kernels of the thresholded path.
//
// Device layout: one pool of NB*MB slots of maxbs*maxbs elements; block
// (ib, jp) (the jp-th block of block row ib, column block indexb[ib*MB+jp])
// is a row-major bsize[ib] x bsize[jb] array at slot ib*MB + jp.  The host
// mirror uses the same slots, and ptr_value[ib*MB + jp] points at them for
// jp < nnzb[ib] (the reference's per-block pointers, bml_types_ellblock.h:36).
//
// Every kernel works on whole block rows (one CTA per block row), follows the
// reference loop's block order and element arithmetic, and keeps or drops
// whole blocks by their max-norm as the reference does.
#include "ellblock.h"
#include "device_util.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace b200;

extern "C" void bml_b200_reset_block_sizes(void);

namespace {

inline size_t eb_pool_elems(const bml_matrix_ellblock_t *A)
{
    return (size_t) A->NB * A->MB * A->slot_elems;
}

template <typename T> struct EbView
{
    T *pool;
    int *indexb;
    int *nnzb;
    const int *bsize;
    const int *boff;
    int NB, MB;
    long long slot;
    __device__ T *blk(int ib, int jp) const { return pool + ((size_t) ib * MB + jp) * slot; }
};

template <typename T> EbView<T> view(bml_matrix_ellblock_t *A)
{
    return EbView<T>{static_cast<T *>(A->d_pool), A->d_indexb, A->d_nnzb, A->d_bsize, A->d_boff,
                     A->NB, A->MB, A->slot_elems};
}

void host_pointers(bml_matrix_ellblock_t *A)
{
    const size_t sz = prec_size(A->matrix_precision);
    for (int ib = 0; ib < A->NB; ib++)
        for (int jp = 0; jp < A->MB; jp++)
        {
            const size_t ind = (size_t) ib * A->MB + jp;
            A->ptr_value[ind] =
                jp < A->nnzb[ib] ? static_cast<char *>(A->h_pool) + ind * A->slot_elems * sz : nullptr;
        }
}

} // namespace

// ---------------------------------------------------------------------------
// storage
// ---------------------------------------------------------------------------
bml_matrix_ellblock_t *eb_alloc_blocks(bml_matrix_precision_t prec, int NB, int MB, int M,
                                       const int *bsize, bml_distribution_mode_t mode)
{
    const size_t sz = prec_size(prec);
    if (sz == 0)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "ELLBLOCK precision %d", (int) prec);
        return nullptr;
    }
    if (NB <= 0 || MB <= 0 || !bsize)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK NB=%d MB=%d", NB, MB);
        return nullptr;
    }
    B200Context *c = b200_ctx();
    if (!c)
        return nullptr;
    auto *A = static_cast<bml_matrix_ellblock_t *>(calloc(1, sizeof(bml_matrix_ellblock_t)));
    if (!A)
        return nullptr;
    A->matrix_type = ellblock;
    A->matrix_precision = prec;
    A->distribution_mode = mode;
    A->NB = NB;
    A->MB = MB;
    A->M = M;
    A->bsize = static_cast<int *>(malloc(sizeof(int) * NB));
    memcpy(A->bsize, bsize, sizeof(int) * NB);
    int N = 0, maxbs = 0;
    std::vector<int> boff(NB + 1, 0);
    for (int ib = 0; ib < NB; ib++)
    {
        boff[ib] = N;
        N += bsize[ib];
        maxbs = bsize[ib] > maxbs ? bsize[ib] : maxbs;
    }
    boff[NB] = N;
    A->N = N;
    A->maxbs = maxbs;
    A->slot_elems = (long long) maxbs * maxbs;
    A->indexb = static_cast<int *>(malloc(sizeof(int) * (size_t) NB * MB));
    for (size_t q = 0; q < (size_t) NB * MB; q++)
        A->indexb[q] = -1;
    A->nnzb = static_cast<int *>(calloc(NB, sizeof(int)));
    A->ptr_value = static_cast<void **>(calloc((size_t) NB * MB, sizeof(void *)));
    A->h_pool = calloc(eb_pool_elems(A), sz);
    A->domain = b200_default_domain(N, M, mode);
    A->domain2 = b200_default_domain(N, M, mode);
    bool ok = A->bsize && A->indexb && A->nnzb && A->ptr_value && A->h_pool;
    if (ok)
    {
        cudaError_t e1 = cudaMallocAsync(&A->d_pool, eb_pool_elems(A) * sz, c->stream);
        cudaError_t e2 = cudaMallocAsync(reinterpret_cast<void **>(&A->d_indexb), sizeof(int) * (size_t) NB * MB, c->stream);
        cudaError_t e3 = cudaMallocAsync(reinterpret_cast<void **>(&A->d_nnzb), sizeof(int) * NB, c->stream);
        cudaError_t e4 = cudaMallocAsync(reinterpret_cast<void **>(&A->d_bsize), sizeof(int) * NB, c->stream);
        cudaError_t e5 = cudaMallocAsync(reinterpret_cast<void **>(&A->d_boff), sizeof(int) * (NB + 1), c->stream);
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess ||
            e5 != cudaSuccess)
        {
            cudaGetLastError();
            b200_set_error(BML_B200_ERR_ALLOC, "ELLBLOCK device arrays NB=%d MB=%d maxbs=%d", NB, MB, maxbs);
            ok = false;
        }
    }
    ok = ok && CUDA_OK(cudaMemcpyAsync(A->d_bsize, bsize, sizeof(int) * NB, cudaMemcpyHostToDevice, c->stream)) &&
         CUDA_OK(cudaMemcpyAsync(A->d_boff, boff.data(), sizeof(int) * (NB + 1), cudaMemcpyHostToDevice,
                                 c->stream)) &&
         CUDA_OK(cudaMemcpyAsync(A->d_indexb, A->indexb, sizeof(int) * (size_t) NB * MB,
                                 cudaMemcpyHostToDevice, c->stream)) &&
         CUDA_OK(cudaMemsetAsync(A->d_nnzb, 0, sizeof(int) * NB, c->stream)) &&
         CUDA_OK(cudaMemsetAsync(A->d_pool, 0, eb_pool_elems(A) * sz, c->stream)) && b200_sync();
    if (!ok)
    {
        eb_free(A);
        return nullptr;
    }
    A->mirror = MIRROR_SYNCED;
    // the first matrix defines the process-wide partition (reference
    // bml_allocate_ellblock_typed.c:237-240)
    if (bml_get_mb() == 0)
        bml_set_block_sizes(A->bsize, NB, MB);
    return A;
}

void eb_free(bml_matrix_ellblock_t *A)
{
    if (!A)
        return;
    B200Context *c = b200_ctx();
    if (c)
    {
        // freed in stream order, after the kernels queued on these arrays
        for (void *p : {static_cast<void *>(A->d_pool), static_cast<void *>(A->d_indexb),
                        static_cast<void *>(A->d_nnzb), static_cast<void *>(A->d_bsize),
                        static_cast<void *>(A->d_boff)})
            if (p)
                cudaFreeAsync(p, c->stream);
    }
    free(A->h_pool);
    free(A->ptr_value);
    free(A->indexb);
    free(A->nnzb);
    free(A->bsize);
    b200_free_domain(A->domain);
    b200_free_domain(A->domain2);
    free(A);
}

bool eb_to_device(bml_matrix_ellblock_t *A)
{
    if (A->mirror != MIRROR_HOST_NEWER)
        return true;
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const size_t sz = prec_size(A->matrix_precision);
    // only the first w slots of every block row, w the widest row
    int w = 0;
    for (int ib = 0; ib < A->NB; ib++)
        w = A->nnzb[ib] > w ? A->nnzb[ib] : w;
    const size_t slot = (size_t) A->slot_elems * sz, pitch = slot * A->MB;
    if ((w > 0 && !CUDA_OK(cudaMemcpy2DAsync(A->d_pool, pitch, A->h_pool, pitch, slot * w, A->NB,
                                             cudaMemcpyHostToDevice, c->stream))) ||
        !CUDA_OK(cudaMemcpyAsync(A->d_indexb, A->indexb, sizeof(int) * (size_t) A->NB * A->MB,
                                 cudaMemcpyHostToDevice, c->stream)) ||
        !CUDA_OK(cudaMemcpyAsync(A->d_nnzb, A->nnzb, sizeof(int) * A->NB, cudaMemcpyHostToDevice,
                                 c->stream)) ||
        !b200_sync())
        return false;
    A->mirror = MIRROR_SYNCED;
    return true;
}

bool eb_to_host(bml_matrix_ellblock_t *A)
{
    if (A->mirror != MIRROR_DEVICE_NEWER)
        return true;
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const size_t sz = prec_size(A->matrix_precision);
    // the row widths first, then only the first w slots of every block row
    if (!CUDA_OK(cudaMemcpyAsync(A->nnzb, A->d_nnzb, sizeof(int) * A->NB, cudaMemcpyDeviceToHost,
                                 c->stream)) ||
        !b200_sync())
        return false;
    int w = 0;
    for (int ib = 0; ib < A->NB; ib++)
        w = A->nnzb[ib] > w ? A->nnzb[ib] : w;
    const size_t slot = (size_t) A->slot_elems * sz, pitch = slot * A->MB;
    if ((w > 0 && !CUDA_OK(cudaMemcpy2DAsync(A->h_pool, pitch, A->d_pool, pitch, slot * w, A->NB,
                                             cudaMemcpyDeviceToHost, c->stream))) ||
        !CUDA_OK(cudaMemcpyAsync(A->indexb, A->d_indexb, sizeof(int) * (size_t) A->NB * A->MB,
                                 cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    host_pointers(A);
    A->mirror = MIRROR_SYNCED;
    return true;
}

static void eb_mark_device(bml_matrix_ellblock_t *A) { A->mirror = MIRROR_DEVICE_NEWER; }
static void eb_mark_host(bml_matrix_ellblock_t *A) { A->mirror = MIRROR_HOST_NEWER; }

void eb_clear(bml_matrix_ellblock_t *A)
{
    B200Context *c = b200_ctx();
    if (!c)
        return;
    if (CUDA_OK(cudaMemsetAsync(A->d_nnzb, 0, sizeof(int) * A->NB, c->stream)))
    {
        if (A->mirror == MIRROR_HOST_NEWER)
            A->mirror = MIRROR_SYNCED;
        eb_mark_device(A);
    }
}

// ---------------------------------------------------------------------------
// constructors: filled on the host in the reference's order, then uploaded
// (ellblock/bml_allocate_ellblock_typed.c:245-443)
// ---------------------------------------------------------------------------
template <typename T> static T *hblk(bml_matrix_ellblock_t *A, int ib, int jp)
{
    return static_cast<T *>(A->h_pool) + ((size_t) ib * A->MB + jp) * A->slot_elems;
}

template <typename T> static void eb_set_element_host(bml_matrix_ellblock_t *A, int i, int j, T v, bool append_new)
{
    (void) append_new;
    int ib = 0, jb = 0, ii = i, jj = j;
    while (ii >= A->bsize[ib])
    {
        ii -= A->bsize[ib];
        ib++;
    }
    while (jj >= A->bsize[jb])
    {
        jj -= A->bsize[jb];
        jb++;
    }
    for (int jp = 0; jp < A->nnzb[ib]; jp++)
        if (A->indexb[(size_t) ib * A->MB + jp] == jb)
        {
            hblk<T>(A, ib, jp)[ii * A->bsize[jb] + jj] = v;
            return;
        }
    if (A->nnzb[ib] == A->MB)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "Number of non-zeroes blocks per row > MB, Increase MB");
        return;
    }
    const int jp = A->nnzb[ib];
    T *b = hblk<T>(A, ib, jp);
    memset(b, 0, sizeof(T) * A->bsize[ib] * A->bsize[jb]);
    b[ii * A->bsize[jb] + jj] = v;
    A->indexb[(size_t) ib * A->MB + jp] = jb;
    A->nnzb[ib]++;
}

template <typename T> static void fill_eb(bml_matrix_ellblock_t *A, int kind)
{
    const int NB = A->NB, MB = A->MB;
    const int *bsize = A->bsize;
    if (kind == 1) // random (bml_allocate_ellblock_typed.c:336-393)
    {
        std::vector<int> marker(NB, -1), pos(MB);
        for (int ib = 0; ib < NB; ib++)
        {
            int bcol = ib, n = 0;
            for (int jb = 0; jb < MB; jb++)
            {
                if (marker[bcol] == -1)
                {
                    T *b = hblk<T>(A, ib, n);
                    for (int ii = 0; ii < bsize[ib]; ii++)
                        for (int jj = 0; jj < bsize[bcol]; jj++)
                            b[ii * bsize[bcol] + jj] = rand() / (T) RAND_MAX;
                    A->indexb[(size_t) ib * MB + n] = bcol;
                    pos[n] = bcol;
                    marker[bcol] = 1;
                    n++;
                }
                bcol = rand() % NB;
            }
            A->nnzb[ib] = n;
            for (int q = 0; q < n; q++)
                marker[pos[q]] = -1;
        }
    }
    else if (kind == 2) // banded through set_element_new (:171-187)
    {
        const int N = A->N, M = A->M;
        for (int i = 0; i < N; i++)
            for (int j = (i - M / 2 >= 0 ? i - M / 2 : 0); j < (i - M / 2 + M <= N ? i - M / 2 + M : N); j++)
                eb_set_element_host<T>(A, i, j, rand() / (T) RAND_MAX, true);
    }
    else if (kind == 3) // identity (:421-443)
    {
        for (int ib = 0; ib < NB; ib++)
        {
            T *b = hblk<T>(A, ib, 0);
            memset(b, 0, sizeof(T) * bsize[ib] * bsize[ib]);
            for (int ii = 0; ii < bsize[ib]; ii++)
                b[ii * bsize[ib] + ii] = (T) 1.0;
            A->nnzb[ib] = 1;
            A->indexb[(size_t) ib * MB] = ib;
        }
    }
}

bml_matrix_ellblock_t *eb_constructor(int kind, bml_matrix_precision_t prec, int N, int M,
                                      bml_distribution_mode_t mode)
{
    if (N <= 0)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK N=%d", N);
        return nullptr;
    }
    int *bsize = bml_get_block_sizes(N, M);
    bml_matrix_ellblock_t *A = eb_alloc_blocks(prec, bml_get_nb(), bml_get_mb(), M, bsize, mode);
    if (!A || kind == 0 || kind == 4)
        return A;
    if (prec == double_real)
        fill_eb<double>(A, kind);
    else
        fill_eb<float>(A, kind);
    eb_mark_host(A);
    if (!eb_to_device(A))
    {
        eb_free(A);
        return nullptr;
    }
    return A;
}

// ---------------------------------------------------------------------------
// host-side element access on the mirror
// ---------------------------------------------------------------------------
void eb_set_element(bml_matrix_ellblock_t *A, int i, int j, const void *value, bool append_new)
{
    if (!A || !value || i < 0 || j < 0 || i >= A->N || j >= A->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK set_element (%d, %d)", i, j);
        return;
    }
    if (!eb_to_host(A))
        return;
    if (A->matrix_precision == double_real)
        eb_set_element_host<double>(A, i, j, *static_cast<const double *>(value), append_new);
    else
        eb_set_element_host<float>(A, i, j, *static_cast<const float *>(value), append_new);
    host_pointers(A);
    eb_mark_host(A);
}

// ---------------------------------------------------------------------------
// Matrix Market I/O (ellblock/bml_utilities_ellblock_typed.c:25-256)
// ---------------------------------------------------------------------------
// Writes every element of every stored block, block rows in order, blocks in
// list order, elements row-major, 1-based, "%d %d %20.15e" (:174-256).
bool eb_write_mm(bml_matrix_ellblock_t *A, FILE *f)
{
    if (!eb_to_host(A))
        return false;
    std::vector<int> off(A->NB + 1, 0);
    for (int ib = 0; ib < A->NB; ib++)
        off[ib + 1] = off[ib] + A->bsize[ib];
    long long msum = 0;
    for (int ib = 0; ib < A->NB; ib++)
        for (int jp = 0; jp < A->nnzb[ib]; jp++)
            msum += (long long) A->bsize[ib] * A->bsize[A->indexb[(size_t) ib * A->MB + jp]];
    fprintf(f, "%%%%%%MatrixMarket matrix coordinate real general\n");
    fprintf(f, "%d %d %lld\n", A->N, A->N, msum);
    const bool dbl = A->matrix_precision == double_real;
    for (int ib = 0; ib < A->NB; ib++)
        for (int jp = 0; jp < A->nnzb[ib]; jp++)
        {
            const int jb = A->indexb[(size_t) ib * A->MB + jp];
            for (int ii = 0; ii < A->bsize[ib]; ii++)
                for (int jj = 0; jj < A->bsize[jb]; jj++)
                {
                    const int e = ii * A->bsize[jb] + jj;
                    const double v = dbl ? (double) hblk<double>(A, ib, jp)[e] : (double) hblk<float>(A, ib, jp)[e];
                    fprintf(f, "%d %d %20.15e\n", off[ib] + 1 + ii, off[jb] + 1 + jj, v);
                }
        }
    return true;
}

// Reads `ne` entries "%d %d value" (1-based) into A: each entry is written
// into its block, a block the row lacks is appended zeroed (existing blocks
// and entries are kept, as the reference reads into the matrix it is given);
// with a symmetric header the transposed entry is set too (:25-167; where
// the reference's symmetric branch appends a block it writes the column
// index at slot nnzb[jb] of block row 0 and leaves the block unallocated,
// :148-156, here the block goes to its own row, zeroed).  Values are parsed
// in the matrix precision (%e / %le).
template <typename T> static bool eb_read_mm_typed(bml_matrix_ellblock_t *A, FILE *f, long long ne, bool symmetric)
{
    for (long long e = 0; e < ne; e++)
    {
        int i, j;
        T v;
        const int got = sizeof(T) == 8 ? fscanf(f, "%d %d %le", &i, &j, reinterpret_cast<double *>(&v))
                                       : fscanf(f, "%d %d %e", &i, &j, reinterpret_cast<float *>(&v));
        if (got != 3)
        {
            b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: entry %lld of %lld unreadable", e + 1, ne);
            return false;
        }
        i--;
        j--;
        if (i < 0 || j < 0 || i >= A->N || j >= A->N)
        {
            b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: entry (%d, %d) outside N=%d", i + 1, j + 1, A->N);
            return false;
        }
        eb_set_element_host<T>(A, i, j, v, true);
        if (symmetric && i != j)
            eb_set_element_host<T>(A, j, i, v, true);
        if (b200_get_error() == BML_B200_ERR_ROW_OVERFLOW)
            return false;
    }
    return true;
}

bool eb_read_mm(bml_matrix_ellblock_t *A, FILE *f, long long ne, bool symmetric)
{
    if (!eb_to_host(A))
        return false;
    bml_b200_clear_error();
    const bool ok = A->matrix_precision == double_real ? eb_read_mm_typed<double>(A, f, ne, symmetric)
                                                       : eb_read_mm_typed<float>(A, f, ne, symmetric);
    host_pointers(A);
    eb_mark_host(A);
    return ok;
}

// Row i <- the entries of row[0..N) with |row[k]| > threshold, written into
// their blocks (a missing block is appended zeroed); entries already in the
// row are kept (ellblock/bml_setters_ellblock_typed.c:131-198).
template <typename T> static void eb_set_row_host(bml_matrix_ellblock_t *A, int i, const T *row, double threshold)
{
    for (int k = 0; k < A->N; k++)
        if (fabs((double) row[k]) > threshold)
        {
            eb_set_element_host<T>(A, i, k, row[k], true);
            if (b200_get_error() == BML_B200_ERR_ROW_OVERFLOW)
                return;
        }
}

void eb_set_row(bml_matrix_ellblock_t *A, int i, const void *row, double threshold)
{
    if (!A || !row || i < 0 || i >= A->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK set_row %d", i);
        return;
    }
    if (!eb_to_host(A))
        return;
    if (A->matrix_precision == double_real)
        eb_set_row_host<double>(A, i, static_cast<const double *>(row), threshold);
    else
        eb_set_row_host<float>(A, i, static_cast<const float *>(row), threshold);
    host_pointers(A);
    eb_mark_host(A);
}

// Diagonal <- diagonal[0..N): per block row, when the max |d| of the block's
// segment exceeds threshold the diagonal block's diagonal takes the segment
// (the block is appended zeroed if missing), otherwise an existing diagonal
// block's diagonal is zeroed (ellblock/bml_setters_ellblock_typed.c:209-284).
template <typename T> static void eb_set_diagonal_host(bml_matrix_ellblock_t *A, const T *d, double threshold)
{
    int off = 0;
    for (int ib = 0; ib < A->NB; ib++)
    {
        const int bs = A->bsize[ib];
        double norm = 0.0;
        for (int ii = 0; ii < bs; ii++)
            norm = fmax(norm, (double) fabs((double) d[off + ii]));
        bool found = false;
        for (int jp = 0; jp < A->nnzb[ib]; jp++)
            if (A->indexb[(size_t) ib * A->MB + jp] == ib)
            {
                T *b = hblk<T>(A, ib, jp);
                for (int ii = 0; ii < bs; ii++)
                    b[ii * bs + ii] = norm > threshold ? d[off + ii] : T(0);
                found = true;
            }
        if (!found && norm > threshold)
        {
            if (A->nnzb[ib] == A->MB)
            {
                b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "set_diagonal: block row %d is full (MB=%d)", ib, A->MB);
                return;
            }
            const int jp = A->nnzb[ib];
            T *b = hblk<T>(A, ib, jp);
            memset(b, 0, sizeof(T) * bs * bs);
            for (int ii = 0; ii < bs; ii++)
                b[ii * bs + ii] = d[off + ii];
            A->indexb[(size_t) ib * A->MB + jp] = ib;
            A->nnzb[ib]++;
        }
        off += bs;
    }
}

void eb_set_diagonal(bml_matrix_ellblock_t *A, const void *diagonal, double threshold)
{
    if (!A || !diagonal)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK set_diagonal: NULL argument");
        return;
    }
    if (!eb_to_host(A))
        return;
    if (A->matrix_precision == double_real)
        eb_set_diagonal_host<double>(A, static_cast<const double *>(diagonal), threshold);
    else
        eb_set_diagonal_host<float>(A, static_cast<const float *>(diagonal), threshold);
    host_pointers(A);
    eb_mark_host(A);
}

template <typename T> static T eb_get_host(bml_matrix_ellblock_t *A, int i, int j, bool &found, T **where)
{
    int ib = 0, jb = 0, ii = i, jj = j;
    while (ii >= A->bsize[ib])
    {
        ii -= A->bsize[ib];
        ib++;
    }
    while (jj >= A->bsize[jb])
    {
        jj -= A->bsize[jb];
        jb++;
    }
    for (int jp = 0; jp < A->nnzb[ib]; jp++)
        if (A->indexb[(size_t) ib * A->MB + jp] == jb)
        {
            found = true;
            *where = hblk<T>(A, ib, jp) + ii * A->bsize[jb] + jj;
            return **where;
        }
    found = false;
    return T(0);
}

void *eb_get_element(bml_matrix_ellblock_t *A, int i, int j)
{
    static double zd = 0.0, md = -1.0;
    static float zf = 0.0f, mf = -1.0f;
    const bool dbl = A && A->matrix_precision == double_real;
    if (!A || i < 0 || j < 0 || i >= A->N || j >= A->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK get_element (%d, %d)", i, j);
        return dbl ? (void *) &md : (void *) &mf;
    }
    if (!eb_to_host(A))
        return nullptr;
    bool found = false;
    if (dbl)
    {
        double *w = nullptr;
        eb_get_host<double>(A, i, j, found, &w);
        return found ? (void *) w : (void *) &zd;
    }
    float *w = nullptr;
    eb_get_host<float>(A, i, j, found, &w);
    return found ? (void *) w : (void *) &zf;
}

void *eb_get_row(bml_matrix_ellblock_t *A, int i)
{
    if (!A || !eb_to_host(A))
        return nullptr;
    const size_t sz = prec_size(A->matrix_precision);
    char *row = static_cast<char *>(calloc(A->N, sz));
    if (!row || i < 0 || i >= A->N)
        return row;
    for (int j = 0; j < A->N; j++)
    {
        void *e = eb_get_element(A, i, j);
        memcpy(row + j * sz, e, sz);
    }
    return row;
}

void *eb_get_diagonal(bml_matrix_ellblock_t *A)
{
    if (!A || !eb_to_host(A))
        return nullptr;
    const size_t sz = prec_size(A->matrix_precision);
    char *d = static_cast<char *>(calloc(A->N, sz));
    for (int i = 0; d && i < A->N; i++)
        memcpy(d + i * sz, eb_get_element(A, i, i), sz);
    return d;
}

int eb_row_bandwidth(bml_matrix_ellblock_t *A, int i)
{
    if (!A || !eb_to_host(A) || i < 0 || i >= A->N)
        return -1;
    int ib = 0, ii = i;
    while (ii >= A->bsize[ib])
    {
        ii -= A->bsize[ib];
        ib++;
    }
    int w = 0;
    for (int jp = 0; jp < A->nnzb[ib]; jp++)
        w += A->bsize[A->indexb[(size_t) ib * A->MB + jp]];
    return w;
}

int eb_bandwidth(bml_matrix_ellblock_t *A)
{
    if (!A || !eb_to_host(A))
        return -1;
    int best = 0;
    for (int ib = 0, i0 = 0; ib < A->NB; i0 += A->bsize[ib], ib++)
    {
        const int w = eb_row_bandwidth(A, i0);
        best = w > best ? w : best;
    }
    return best;
}

double eb_sparsity(bml_matrix_ellblock_t *A, double threshold)
{
    if (!A || !eb_to_host(A))
        return -1.0;
    long long nz = 0;
    const bool dbl = A->matrix_precision == double_real;
    for (int ib = 0; ib < A->NB; ib++)
        for (int jp = 0; jp < A->nnzb[ib]; jp++)
        {
            const int jb = A->indexb[(size_t) ib * A->MB + jp];
            const int ne = A->bsize[ib] * A->bsize[jb];
            for (int e = 0; e < ne; e++)
            {
                const double v = dbl ? hblk<double>(A, ib, jp)[e] : hblk<float>(A, ib, jp)[e];
                if (fabs(v) > threshold)
                    nz++;
            }
        }
    return 1.0 - (double) nz / ((double) A->N * A->N);
}

long long eb_nnz(bml_matrix_ellblock_t *A)
{
    if (!A || !eb_to_host(A))
        return -1;
    long long n = 0;
    for (int ib = 0; ib < A->NB; ib++)
        for (int jp = 0; jp < A->nnzb[ib]; jp++)
            n += (long long) A->bsize[ib] * A->bsize[A->indexb[(size_t) ib * A->MB + jp]];
    return n;
}

// ---------------------------------------------------------------------------
// device kernels, one block row per CTA
// ---------------------------------------------------------------------------
namespace {

// max |x| over a block, as the double the reference's bml_norm_inf returns
template <typename T> __device__ double block_norm_inf(const T *x, int ne, double *red)
{
    double m = 0.0;
    for (int e = threadIdx.x; e < ne; e += blockDim.x)
        m = fmax(m, (double) fabs(x[e]));
    for (int o = 16; o; o >>= 1)
        m = fmax(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = m;
    __syncthreads();
    double r = 0.0;
    for (int w = 0; w < (int) (blockDim.x >> 5); ++w)
        r = fmax(r, red[w]);
    __syncthreads();
    return r;
}

// copy B <- A (same partition)
template <typename T> __global__ void eb_copy_kernel(EbView<T> A, EbView<T> B, int *overflow)
{
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
    {
        const int n = A.nnzb[ib];
        if (n > B.MB)
        {
            if (threadIdx.x == 0)
                atomicExch(overflow, 1);
            continue;
        }
        for (int jp = 0; jp < n; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const int ne = A.bsize[ib] * A.bsize[jb];
            const T *src = A.blk(ib, jp);
            T *dst = B.blk(ib, jp);
            for (int e = threadIdx.x; e < ne; e += blockDim.x)
                dst[e] = src[e];
            if (threadIdx.x == 0)
                B.indexb[(size_t) ib * B.MB + jp] = jb;
        }
        if (threadIdx.x == 0)
            B.nnzb[ib] = n;
    }
}

// scale every stored element: x <- s*x (ellblock/bml_scale_ellblock_typed.c:66-87)
template <typename T> __global__ void eb_scale_kernel(EbView<T> A, T s)
{
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
        for (int jp = 0; jp < A.nnzb[ib]; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const int ne = A.bsize[ib] * A.bsize[jb];
            T *x = A.blk(ib, jp);
            for (int e = threadIdx.x; e < ne; e += blockDim.x)
                x[e] = mul_rn(s, x[e]);
        }
}

// A <- alpha*A + beta*B, block kept if max|x| > thr (norm rounded to the
// matrix precision, as `REAL_T normx = bml_norm_inf(...)` does)
// (ellblock/bml_add_ellblock_typed.c:35-197).  Blocks: A's in order, then
// B's new ones in order.  Thread 0 of each CTA merges the two block lists of
// a block row into the CTA's scratch (mark[NB] | list[cap] | src_a[cap] |
// src_b[cap], cap = A.MB + B.MB, so a merged row of any width fits); the
// sums are then written in place (see below).
template <typename T>
__global__ void eb_add_kernel(EbView<T> A, EbView<T> B, double alpha, double beta, double thr, int *scr,
                              int cap, int *overflow)
{
    __shared__ int nl;
    __shared__ double red[32];
    const bool use_a = alpha > 0.0 || alpha < 0.0;
    const bool use_b = beta > 0.0 || beta < 0.0;
    int *mark = scr + (size_t) blockIdx.x * (A.NB + 3 * (size_t) cap);
    int *list = mark + A.NB;   // merged column-block list
    int *src_a = list + cap;   // position in A or -1
    int *src_b = src_a + cap;  // position in B or -1
    const T thr_t = (T) thr;
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
    {
        if (threadIdx.x == 0)
        {
            int n = 0;
            const int na = use_a ? A.nnzb[ib] : 0, nb = use_b ? B.nnzb[ib] : 0;
            for (int p = 0; p < na; ++p)
            {
                const int jb = A.indexb[(size_t) ib * A.MB + p];
                mark[jb] = n + 1;
                list[n] = jb;
                src_a[n] = p;
                src_b[n] = -1;
                n++;
            }
            for (int p = 0; p < nb; ++p)
            {
                const int jb = B.indexb[(size_t) ib * B.MB + p];
                if (mark[jb])
                    src_b[mark[jb] - 1] = p;
                else
                {
                    mark[jb] = n + 1;
                    list[n] = jb;
                    src_a[n] = -1;
                    src_b[n] = p;
                    n++;
                }
            }
            for (int q = 0; q < n; ++q)
                mark[list[q]] = 0;
            nl = n;
        }
        __syncthreads();
        // The sum of list entry q is written straight into A at position
        // kept <= q: A's blocks sit at positions 0..na-1 in list order, so
        // every block of A still to be read is at a position above kept, and
        // a block that is dropped is overwritten by the next one kept.  The
        // max-norm is taken in the same pass.
        const int n = nl;
        int kept = 0;
        for (int q = 0; q < n; ++q)
        {
            const int jb = list[q];
            const int ne = A.bsize[ib] * A.bsize[jb];
            const T *a = src_a[q] >= 0 ? A.blk(ib, src_a[q]) : nullptr;
            const T *b = src_b[q] >= 0 ? B.blk(ib, src_b[q]) : nullptr;
            T *x = kept < A.MB ? A.blk(ib, kept) : nullptr;
            double m = 0.0;
            for (int e = threadIdx.x; e < ne; e += blockDim.x)
            {
                T v = T(0);
                if (a)
                    v = axpy_d(v, alpha, a[e]);
                if (b)
                    v = axpy_d(v, beta, b[e]);
                if (x)
                    x[e] = v;
                m = fmax(m, (double) fabs(v));
            }
            for (int o = 16; o; o >>= 1)
                m = fmax(m, __shfl_xor_sync(FULL, m, o));
            if ((threadIdx.x & 31) == 0)
                red[threadIdx.x >> 5] = m;
            __syncthreads();
            double r = 0.0;
            for (int w = 0; w < (int) (blockDim.x >> 5); ++w)
                r = fmax(r, red[w]);
            const T normx = (T) r;
            if (fabs(normx) > thr_t)
            {
                if (threadIdx.x == 0 && kept < A.MB)
                    A.indexb[(size_t) ib * A.MB + kept] = jb;
                kept++;
            }
            __syncthreads(); // red is rewritten, and the kept block's writes land before the next q reads
        }
        if (kept > A.MB)
        {
            if (threadIdx.x == 0)
                atomicExch(overflow, 1);
            kept = A.MB;
        }
        if (threadIdx.x == 0)
            A.nnzb[ib] = kept;
        __syncthreads();
    }
}

// threshold: drop blocks with max|x| <= thr (order kept), zero the elements
// with |x| <= thr in the others (ellblock/bml_threshold_ellblock_typed.c:95-140)
template <typename T> __global__ void __launch_bounds__(256) eb_threshold_kernel(EbView<T> A, EbView<T> B, double thr)
{
    // one read of every block: each thread holds its (at most 16) elements
    // in registers across the max-norm reduction (blocks of at most 64 x 64,
    // 256 threads); B may be A (kept blocks move down, out <= jp)
    constexpr int PER = 64 * 64 / 256;
    __shared__ double red[8];
    const T thr_t = (T) thr;
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
    {
        int out = 0;
        const int n = A.nnzb[ib];
        for (int jp = 0; jp < n; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const int ne = A.bsize[ib] * A.bsize[jb];
            const T *x = A.blk(ib, jp);
            T v[PER];
            double m = 0.0;
#pragma unroll
            for (int u = 0; u < PER; ++u)
            {
                const int e = u * 256 + threadIdx.x;
                v[u] = e < ne ? x[e] : T(0);
                m = fmax(m, (double) fabs(v[u]));
            }
            for (int o = 16; o; o >>= 1)
                m = fmax(m, __shfl_xor_sync(FULL, m, o));
            if ((threadIdx.x & 31) == 0)
                red[threadIdx.x >> 5] = m;
            __syncthreads();
            double r = 0.0;
#pragma unroll
            for (int w = 0; w < 8; ++w)
                r = fmax(r, red[w]);
            const T normx = (T) r;
            if (fabs(normx) > thr_t)
            {
                T *y = B.blk(ib, out);
#pragma unroll
                for (int u = 0; u < PER; ++u)
                {
                    const int e = u * 256 + threadIdx.x;
                    if (e < ne)
                        y[e] = fabs(v[u]) > thr_t ? v[u] : T(0);
                }
                if (threadIdx.x == 0)
                    B.indexb[(size_t) ib * B.MB + out] = jb;
                out++;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0)
            B.nnzb[ib] = out;
        __syncthreads();
    }
}

// per-block-row diagonal sums: first diagonal block of the row
// (ellblock/bml_trace_ellblock_typed.c:27-58)
template <typename T> __global__ void eb_diag_kernel(EbView<T> A, double *d)
{
    for (int ib = blockIdx.x * blockDim.x + threadIdx.x; ib < A.NB; ib += gridDim.x * blockDim.x)
    {
        double s = 0.0;
        T acc = T(0);
        for (int jp = 0; jp < A.nnzb[ib]; ++jp)
            if (A.indexb[(size_t) ib * A.MB + jp] == ib)
            {
                const T *x = A.blk(ib, jp);
                for (int ii = 0; ii < A.bsize[ib]; ++ii)
                    acc = add_rn(acc, x[ii * A.bsize[ib] + ii]);
                break;
            }
        s = (double) acc;
        d[ib] = s;
    }
}

// trace(A*B) = sum over ib, A's blocks (ib, jb), B's blocks (jb, ib) of
// sum_ii sum_jj A[ii][jj] B[jj][ii] (ellblock/bml_trace_ellblock_typed.c:69-122)
template <typename T> __global__ void eb_trace_mult_kernel(EbView<T> A, EbView<T> B, double *part)
{
    __shared__ double red[32];
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
    {
        double s = 0.0;
        for (int jp = 0; jp < A.nnzb[ib]; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const T *a = A.blk(ib, jp);
            for (int kp = 0; kp < B.nnzb[jb]; ++kp)
                if (B.indexb[(size_t) jb * B.MB + kp] == ib)
                {
                    const T *b = B.blk(jb, kp);
                    const int bi = A.bsize[ib], bj = A.bsize[jb];
                    for (int e = threadIdx.x; e < bi * bj; e += blockDim.x)
                    {
                        const int ii = e / bj, jj = e % bj;
                        s += (double) mul_rn(a[ii * bj + jj], b[jj * bi + ii]);
                    }
                }
        }
        for (int o = 16; o; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        if ((threadIdx.x & 31) == 0)
            red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double t = 0.0;
            for (int w = 0; w < (int) (blockDim.x >> 5); ++w)
                t += red[w];
            part[ib] = t;
        }
        __syncthreads();
    }
}

// Gershgorin per scalar row (ellblock/bml_normalize_ellblock_typed.c:97-150):
// dval = the diagonal element, rad += (double)|a| over all other elements of
// the row, in block order; hi/lo = dval +/- rad in the matrix precision.
template <typename T> __global__ void eb_gersh_kernel(EbView<T> A, double *hi, double *lo)
{
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
        for (int ii = threadIdx.x; ii < A.bsize[ib]; ii += blockDim.x)
        {
            T rad = T(0), dval = T(0);
            for (int jp = 0; jp < A.nnzb[ib]; ++jp)
            {
                const int jb = A.indexb[(size_t) ib * A.MB + jp];
                const T *x = A.blk(ib, jp) + ii * A.bsize[jb];
                for (int jj = 0; jj < A.bsize[jb]; ++jj)
                {
                    if (ib == jb && ii == jj)
                        dval = x[jj];
                    else
                        rad = (T) __dadd_rn((double) rad, (double) fabs(x[jj]));
                }
            }
            const int i = A.boff[ib] + ii;
            hi[i] = (double) add_rn(dval, rad);
            lo[i] = (double) add_rn(dval, (T) -rad);
        }
}

// transpose: block (ib, jb) -> (jb, ib) transposed, appended to block row jb
// in ascending ib (the serial order of ellblock/bml_transpose_ellblock_typed.c:
// 29-70).  One thread per destination block row gathers its blocks in order.
// Transpose, in two passes.  Block row jb of B = A^T lists the blocks
// (ib, jb) of A in ascending ib, the order of the reference's loop over
// block rows (ellblock/bml_transpose_ellblock_typed.c:29-70).
// Pass 1: every block (ib, jp) of A takes a slot in its target row jb
// (atomic count) and records its source there (ib*MB + jp).
__global__ void eb_tr_scatter_kernel(const int *indexb, const int *nnzb, int NB, int MBa, int MBb, int *cnt,
                                     int *src, int *overflow)
{
    for (long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x; e < (long long) NB * MBa;
         e += (long long) gridDim.x * blockDim.x)
    {
        const int ib = (int) (e / MBa), jp = (int) (e % MBa);
        if (jp >= nnzb[ib])
            continue;
        const int jb = indexb[e];
        const int slot = atomicAdd(&cnt[jb], 1);
        if (slot < MBb)
            src[(size_t) jb * MBb + slot] = (int) e;
        else
            atomicExch(overflow, 1);
    }
}

// Pass 2: one CTA per row jb of B ranks its sources by ib (they are
// distinct) and writes each block transposed at its rank, through a padded
// shared-memory tile.
// Shared memory: ids[MBb] (source slots) | rank[MBb] | tile[maxbs][maxbs+1]
template <typename T> __global__ void eb_tr_place_kernel(EbView<T> A, EbView<T> B, const int *cnt, const int *src)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int maxbs = (int) sqrtf((float) A.slot + 0.5f);
    int *ids = reinterpret_cast<int *>(smem);
    int *rank = ids + B.MB;
    T *tile = reinterpret_cast<T *>(smem + (((size_t) 2 * B.MB * sizeof(int) + 15) & ~size_t(15)));
    const int ld = maxbs + 1;
    for (int jb = blockIdx.x; jb < A.NB; jb += gridDim.x)
    {
        const int n = min(cnt[jb], B.MB);
        for (int q = threadIdx.x; q < n; q += blockDim.x)
            ids[q] = src[(size_t) jb * B.MB + q];
        __syncthreads();
        for (int q = threadIdx.x; q < n; q += blockDim.x)
        {
            const int ib = ids[q] / A.MB;
            int r = 0;
            for (int u = 0; u < n; ++u)
                r += ids[u] / A.MB < ib;
            rank[q] = r;
        }
        __syncthreads();
        const int bj = A.bsize[jb];
        for (int q = 0; q < n; ++q)
        {
            const int e = ids[q], ib = e / A.MB, bi = A.bsize[ib];
            const T *a = A.pool + (size_t) e * A.slot; // block (ib, jp): bi x bj, row-major
            for (int x = threadIdx.x; x < bi * bj; x += blockDim.x)
                tile[(x / bj) * ld + x % bj] = a[x];
            __syncthreads();
            T *b = B.blk(jb, rank[q]); // bj x bi, row-major
            for (int x = threadIdx.x; x < bi * bj; x += blockDim.x)
                b[x] = tile[(x % bi) * ld + x / bi];
            if (threadIdx.x == 0)
                B.indexb[(size_t) jb * B.MB + rank[q]] = ib;
            __syncthreads();
        }
        if (threadIdx.x == 0)
            B.nnzb[jb] = n;
        __syncthreads();
    }
}

// dense import/export (ellblock/bml_import_ellblock_typed.c, bml_export_ellblock_typed.c)
template <typename T>
__global__ void eb_import_kernel(EbView<T> A, const T *D, int N, int colmajor, double thr, int *overflow)
{
    __shared__ double red[32];
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
    {
        int n = 0;
        for (int jb = 0; jb < A.NB; ++jb)
        {
            const int bi = A.bsize[ib], bj = A.bsize[jb];
            const int r0 = A.boff[ib], c0 = A.boff[jb];
            double m = 0.0;
            for (int e = threadIdx.x; e < bi * bj; e += blockDim.x)
            {
                const int ii = e / bj, jj = e % bj;
                const T v = colmajor ? D[(size_t) (c0 + jj) * N + r0 + ii] : D[(size_t) (r0 + ii) * N + c0 + jj];
                m = fmax(m, (double) fabs(v));
            }
            for (int o = 16; o; o >>= 1)
                m = fmax(m, __shfl_xor_sync(FULL, m, o));
            if ((threadIdx.x & 31) == 0)
                red[threadIdx.x >> 5] = m;
            __syncthreads();
            double norm = 0.0;
            for (int w = 0; w < (int) (blockDim.x >> 5); ++w)
                norm = fmax(norm, red[w]);
            __syncthreads();
            if (norm > thr)
            {
                if (n < A.MB)
                {
                    T *x = A.blk(ib, n);
                    for (int e = threadIdx.x; e < bi * bj; e += blockDim.x)
                    {
                        const int ii = e / bj, jj = e % bj;
                        x[e] = colmajor ? D[(size_t) (c0 + jj) * N + r0 + ii] : D[(size_t) (r0 + ii) * N + c0 + jj];
                    }
                    if (threadIdx.x == 0)
                        A.indexb[(size_t) ib * A.MB + n] = jb;
                }
                else if (threadIdx.x == 0)
                    atomicExch(overflow, 1);
                n++;
            }
        }
        if (threadIdx.x == 0)
            A.nnzb[ib] = n < A.MB ? n : A.MB;
        __syncthreads();
    }
}

template <typename T> __global__ void eb_export_kernel(EbView<T> A, T *D, int N, int colmajor)
{
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
        for (int jp = 0; jp < A.nnzb[ib]; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const int bi = A.bsize[ib], bj = A.bsize[jb];
            const int r0 = A.boff[ib], c0 = A.boff[jb];
            const T *x = A.blk(ib, jp);
            for (int e = threadIdx.x; e < bi * bj; e += blockDim.x)
            {
                const int ii = e / bj, jj = e % bj;
                if (colmajor)
                    D[(size_t) (c0 + jj) * N + r0 + ii] = x[e];
                else
                    D[(size_t) (r0 + ii) * N + c0 + jj] = x[e];
            }
        }
}

// ---------------------------------------------------------------------------
// X^2 / A*B, exact form (ellblock/bml_multiply_ellblock_typed.c:246-442 and
// :455-621).  One CTA per block row ib.  For every (jp, kp) in order the
// block product X[ib,jb] X[jb,kb] is added into the accumulator of kb (first
// touch: kb appended to the row's list, accumulator zeroed), element (ii, jj)
// as x = x + s with s = a0*b0 + a1*b1 + ... summed left to right, exactly the
// reference micro-kernel's expression.  Accumulators live in a per-CTA slab
// in device memory (MB_out slots); each thread owns fixed elements of every
// accumulator, so the only barriers are around the staging of the two
// blocks in shared memory.  Kept blocks (kb == ib or max|x| > thr) are copied
// to C in first-touch order.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) eb_mul_kernel(EbView<T> A, EbView<T> B, EbView<T> C, double thr,
                                                     int use_norm_inf_fast, int cap, T *slab, int *lists,
                                                     int *marks, double *dA, double *dC, int *flags)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int maxbs = (int) sqrtf((float) A.slot + 0.5f);
    T *sL = reinterpret_cast<T *>(smem);
    T *sR = sL + (size_t) maxbs * maxbs;
    __shared__ int lb, firstflag, slotq, stopflag;
    __shared__ double red[32];
    // cap slab slots and list entries per CTA (first-touch order)
    T *myslab = slab + (size_t) blockIdx.x * cap * A.slot;
    int *list = lists + (size_t) blockIdx.x * cap;
    int *mark = marks + (size_t) blockIdx.x * B.NB;
    for (int ib = blockIdx.x; ib < A.NB; ib += gridDim.x)
    {
        // (no further rows once a row has outgrown the slots: the call runs again)
        if (threadIdx.x == 0)
        {
            lb = 0;
            stopflag = *reinterpret_cast<volatile int *>(&flags[4]);
        }
        __syncthreads();
        if (stopflag)
            break;
        T trA = T(0);
        const int bi = A.bsize[ib];
        for (int jp = 0; jp < A.nnzb[ib]; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const int bj = A.bsize[jb];
            const T *L = A.blk(ib, jp);
            for (int e = threadIdx.x; e < bi * bj; e += blockDim.x)
                sL[e] = L[e];
            if (jb == ib)
                for (int kk = 0; kk < bi; ++kk)
                    trA = add_rn(trA, L[kk * (1 + bi)]);
            for (int kp = 0; kp < B.nnzb[jb]; ++kp)
            {
                const int kb = B.indexb[(size_t) jb * B.MB + kp];
                const int bk = B.bsize[kb];
                const T *R = B.blk(jb, kp);
                if (threadIdx.x == 0)
                {
                    const int m = mark[kb];
                    if (m == 0)
                    {
                        firstflag = 1;
                        slotq = lb;
                        if (lb < cap)
                            list[lb] = kb;
                        mark[kb] = lb + 1;
                        lb++;
                        if (lb > cap)
                            atomicExch(&flags[4], 1);
                    }
                    else
                    {
                        firstflag = 0;
                        slotq = m - 1;
                    }
                }
                for (int e = threadIdx.x; e < bj * bk; e += blockDim.x)
                    sR[e] = R[e];
                __syncthreads();
                const int q = slotq;
                const bool first = firstflag;
                if (q < cap)
                {
                    T *x = myslab + (size_t) q * A.slot;
                    for (int e = threadIdx.x; e < bi * bk; e += blockDim.x)
                    {
                        const int ii = e / bk, jj = e % bk;
                        T s = mul_rn(sL[ii * bj], sR[jj]);
                        for (int l = 1; l < bj; ++l)
                            s = add_rn(s, mul_rn(sL[ii * bj + l], sR[l * bk + jj]));
                        x[e] = add_rn(first ? T(0) : x[e], s);
                    }
                }
                __syncthreads();
            }
        }
        // keep and copy out in first-touch order
        const int n = lb;
        int kept = 0;
        T trC = T(0);
        for (int q = 0; q < min(n, cap); ++q)
        {
            const int kb = list[q];
            const int bk = B.bsize[kb];
            if (threadIdx.x == 0)
                mark[kb] = 0;
            const T *x = myslab + (size_t) q * A.slot;
            const double normx = block_norm_inf(x, bi * bk, red);
            const bool keep = kb == ib || (use_norm_inf_fast ? normx > thr : (T) normx > (T) thr);
            if (keep)
            {
                if (kb == ib)
                    for (int kk = 0; kk < bi; ++kk)
                        trC = add_rn(trC, x[kk * (1 + bi)]);
                if (kept < C.MB)
                {
                    T *dst = C.blk(ib, kept);
                    for (int e = threadIdx.x; e < bi * bk; e += blockDim.x)
                        dst[e] = x[e];
                    if (threadIdx.x == 0)
                        C.indexb[(size_t) ib * C.MB + kept] = kb;
                }
                kept++;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            C.nnzb[ib] = kept < C.MB ? kept : C.MB;
            atomicMax(&flags[1], kept);
            if (kept > C.MB)
                atomicExch(&flags[0], 1);
            if (n > cap)
                atomicExch(&flags[4], 1);
            if (dA)
                dA[ib] = (double) trA;
            if (dC)
                dC[ib] = (double) trC;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// The same exact X^2 / A*B for a uniform partition of 32 x 32 blocks, with
// the block products register-tiled.  Same arithmetic (every element
// x = x + s, s = a0*b0 + a1*b1 + ... left to right, separately rounded), same
// first-touch slot order, same keep rule, so the results are bit-identical to
// eb_mul_kernel's.
//
// Four warps per CTA.  Lane r holds row r of the left block X[ib,jb] in
// registers (staged once per left block through a padded transpose in
// shared memory); warp w forms columns 8w..8w+7 of each block product, so a
// broadcast 16-byte load of a right-block row feeds 16 / sizeof(T)
// multiply-adds and the left block is not re-read per product.  Thread 0
// copies the right blocks X[jb,kb] with cp.async.bulk through a ring of
// EB32_STAGES buffers ahead of use, completing on mbarriers (bounded waits;
// a wait that runs out raises flags[2]).  At the start of every left block
// (in segments of EB32_SEG right blocks) all threads assign the slots of its
// right blocks at once: a ballot prefix in kp order appends first touches to
// the row's list.  Accumulators stay in the per-CTA slab, column-major
// within a slot so that every access is coalesced, each element owned by one
// thread; kept blocks are transposed back to row-major through shared memory
// on the way out.
// Shared memory: EbS32<T> (41 KB for double, four CTAs per SM).
// ---------------------------------------------------------------------------
#ifndef B200_EB32_STAGES
#define B200_EB32_STAGES 3
#endif
constexpr int EB32_STAGES = B200_EB32_STAGES, EB32_THREADS = 128, EB32_SEG = 1024;

template <typename T> struct EbS32
{
    uint64_t full_r[EB32_STAGES];
    __align__(16) T R[EB32_STAGES][1024]; // right blocks; after a row's products, transpose scratch
    T Lt[32 * 33];                         // left block transposed, padded: Lt[l*33 + r] = L[r][l]
    int slotq[EB32_SEG]; // per kp of the segment: slot, or -(slot + 1) on first touch; then, per
                         // chunk of EB32_SEG slots, output position (-1 when dropped)
    int cnt[EB32_THREADS / 32];
    int kept;
    int row;
};

template <typename T> struct Vec16;
template <> struct Vec16<double>
{
    using type = double2;
    static constexpr int n = 2;
    __device__ static double at(const double2 &v, int q) { return q ? v.y : v.x; }
};
template <> struct Vec16<float>
{
    using type = float4;
    static constexpr int n = 4;
    __device__ static float at(const float4 &v, int q) { return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w; }
};

__device__ __forceinline__ unsigned eb_su32(const void *p) { return (unsigned) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void eb_bulk(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(eb_su32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     eb_su32(dst)),
                 "l"(src), "r"(bytes), "r"(eb_su32(bar))
                 : "memory");
}

__device__ __forceinline__ bool eb_test(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(eb_su32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Wait for phase `parity` of bar, at most about 2 s; false on timeout.
__device__ bool eb_wait2s(uint64_t *bar, unsigned parity)
{
    unsigned long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (;;)
    {
        if (eb_test(bar, parity))
            return true;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > 2000000000ull)
            return false;
    }
}

// The same, raising *flag on timeout.  Once the flag is up the kernel's
// result is void, and later waits return at once.
__device__ __forceinline__ void eb_wait(uint64_t *bar, unsigned parity, int *flag)
{
    if (eb_test(bar, parity) || *reinterpret_cast<volatile int *>(flag))
        return;
    if (!eb_wait2s(bar, parity))
        atomicExch(flag, 1);
}

// FUSED: each block product's inner sums by fused multiply-adds (one
// rounding per step, half the FP64 instructions; the unordered form of the
// library), or, as the restatement and the reference's -std=c99 build, by a
// separately rounded product and sum (the ordered form, bit for bit).
template <typename T, bool FUSED>
__global__ void __launch_bounds__(EB32_THREADS, 4) eb_mul32_kernel(EbView<T> A, EbView<T> B, EbView<T> C, double thr,
                                                                  int use_norm_inf_fast, int cap, T *slab,
                                                                  int *lists, int *marks, double *dA, double *dC,
                                                                  int *flags)
{
    using V = Vec16<T>;
    using VT = typename V::type;
    constexpr int NV = V::n;
    constexpr unsigned BLK = 1024 * sizeof(T);
    extern __shared__ __align__(128) unsigned char smem[];
    EbS32<T> &S = *reinterpret_cast<EbS32<T> *>(smem);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // cap slab slots and list entries (kb per slot, first-touch order) per CTA
    T *myslab = slab + (size_t) blockIdx.x * cap * 1024;
    int *list = lists + (size_t) blockIdx.x * cap;
    int *mark = marks + (size_t) blockIdx.x * B.NB;
    int *tflag = &flags[2];

    if (tid == 0)
    {
        for (int s = 0; s < EB32_STAGES; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(eb_su32(&S.full_r[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    unsigned consumed = 0; // right blocks consumed over every row of this CTA (uniform)
    // producer state (thread 0): copies issued, and the next pair (pj, pk)
    unsigned issued = 0;
    int pj = 0, pk = 0, pnk = 0, pjb = 0;

    for (;;)
    {
        // block rows are claimed from a counter (rows differ in cost), by
        // one thread for the whole CTA
        // (none once a row has outgrown the slots: the call runs again)
        if (tid == 0)
            S.row = *reinterpret_cast<volatile int *>(&flags[4]) ? A.NB : atomicAdd(&flags[3], 1);
        __syncthreads();
        const int ib = S.row;
        if (ib >= A.NB)
            break;
        const int na = A.nnzb[ib];
        const int *arow = A.indexb + (size_t) ib * A.MB;
        // left blocks whose block row of B is empty have no pairs
        auto prod_skip = [&]() {
            while (pj < na)
            {
                pjb = arow[pj];
                pnk = B.nnzb[pjb];
                if (pnk > 0)
                    return;
                ++pj;
            }
        };
        auto produce = [&]() {
            // generic-proxy accesses of the buffers being refilled are
            // ordered before the bulk copies by the barrier and this fence
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            while (pj < na && issued - consumed < (unsigned) EB32_STAGES)
            {
                const unsigned s = issued % EB32_STAGES;
                eb_bulk(S.R[s], B.blk(pjb, pk), BLK, &S.full_r[s]);
                ++issued;
                if (++pk == pnk)
                {
                    pk = 0;
                    ++pj;
                    prod_skip();
                }
            }
        };
        if (tid == 0)
        {
            pj = 0;
            pk = 0;
            prod_skip();
            produce();
        }

        int lb = 0; // slots in use (uniform)
        T trA = T(0);
        for (int jp = 0; jp < na; ++jp)
        {
            const int jb = arow[jp];
            const int nk = B.nnzb[jb];
            const T *L = A.blk(ib, jp);
            if (jb == ib && tid == 0)
                for (int kk = 0; kk < 32; ++kk)
                    trA = add_rn(trA, L[kk * 33]);
            if (nk == 0)
                continue;
            // the left block, transposed into shared memory (ordered before
            // its reads by the barriers of the slot assignment)
#pragma unroll
            for (int u = 0; u < 1024 / EB32_THREADS; ++u)
            {
                const int e = u * EB32_THREADS + tid;
                S.Lt[(e & 31) * 33 + (e >> 5)] = L[e];
            }
            const int *brow = B.indexb + (size_t) jb * B.MB;
            for (int seg0 = 0; seg0 < nk; seg0 += EB32_SEG)
            {
                const int ns = min(EB32_SEG, nk - seg0);
                // slots of this segment's right blocks, first touches appended in kp order
                for (int c0 = 0; c0 < ns; c0 += EB32_THREADS)
                {
                    const int q = c0 + tid;
                    bool isnew = false;
                    int sl = 0, kb = 0;
                    if (q < ns)
                    {
                        kb = brow[seg0 + q];
                        const int m = mark[kb];
                        isnew = m == 0;
                        sl = m - 1;
                    }
                    const unsigned bal = __ballot_sync(FULL, isnew);
                    if (lane == 0)
                        S.cnt[warp] = __popc(bal);
                    __syncthreads();
                    int pre = 0, tot = 0;
#pragma unroll
                    for (int w = 0; w < EB32_THREADS / 32; ++w)
                    {
                        const int cw = S.cnt[w];
                        pre += w < warp ? cw : 0;
                        tot += cw;
                    }
                    if (isnew)
                    {
                        sl = lb + pre + __popc(bal & lanemask_lt());
                        mark[kb] = sl + 1;
                        if (sl < cap)
                            list[sl] = kb;
                    }
                    if (q < ns)
                        S.slotq[q] = isnew ? -(sl + 1) : sl;
                    lb += tot;
                    if (tid == 0 && lb > cap)
                        atomicExch(&flags[4], 1);
                    __syncthreads();
                }
                // this lane's row of the left block
                T lrow[32];
#pragma unroll
                for (int l = 0; l < 32; ++l)
                    lrow[l] = S.Lt[l * 33 + lane];
                for (int q = 0; q < ns; ++q)
                {
                    const unsigned st = consumed % EB32_STAGES;
                    eb_wait(&S.full_r[st], (consumed / EB32_STAGES) & 1, tflag);
                    const int code = S.slotq[q];
                    const bool first = code < 0;
                    const int sl = first ? -code - 1 : code;
                    if (sl < cap)
                    {
                        // element (r, c) of a slot at c*32 + r
                        T *x = myslab + (size_t) sl * 1024 + warp * 8 * 32 + lane;
                        T xo[8];
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            xo[c] = first ? T(0) : x[c * 32];
                        const VT *rb = reinterpret_cast<const VT *>(S.R[st] + warp * 8);
                        T s[8];
#pragma unroll
                        for (int l = 0; l < 32; ++l)
                        {
                            VT bv[8 / NV];
#pragma unroll
                            for (int u = 0; u < 8 / NV; ++u)
                                bv[u] = rb[l * (32 / NV) + u];
#pragma unroll
                            for (int c = 0; c < 8; ++c)
                            {
                                if (FUSED)
                                    s[c] = l == 0 ? lrow[l] * V::at(bv[c / NV], c % NV)
                                                  : fma(lrow[l], V::at(bv[c / NV], c % NV), s[c]);
                                else
                                {
                                    const T p = mul_rn(lrow[l], V::at(bv[c / NV], c % NV));
                                    s[c] = l == 0 ? p : add_rn(s[c], p);
                                }
                            }
                        }
#pragma unroll
                        for (int c = 0; c < 8; ++c)
                            x[c * 32] = add_rn(xo[c], s[c]);
                    }
                    __syncthreads();
                    ++consumed;
                    if (tid == 0)
                        produce();
                }
            }
        }
        __syncthreads();

        // keep (kb == ib or max|x| > thr) and copy out in first-touch order,
        // EB32_SEG slots at a time
        const int n = lb;
        const int nl = min(n, cap);
        // each warp transposes its blocks back to row-major, 16 columns at a
        // time, through 32 x 17 elements of the (idle) right-block ring
        T *tp = &S.R[0][0] + warp * (32 * 17);
        int kept = 0; // uniform
        for (int q0 = 0; q0 < nl; q0 += EB32_SEG)
        {
            const int qn = min(EB32_SEG, nl - q0);
            for (int q = warp; q < qn; q += EB32_THREADS / 32)
            {
                const VT *x = reinterpret_cast<const VT *>(myslab + (size_t) (q0 + q) * 1024);
                double m = 0.0;
                for (int e = lane; e < 1024 / NV; e += 32)
                {
                    const VT v = x[e];
#pragma unroll
                    for (int u = 0; u < NV; ++u)
                        m = fmax(m, (double) fabs(V::at(v, u)));
                }
                for (int o = 16; o; o >>= 1)
                    m = fmax(m, __shfl_xor_sync(FULL, m, o));
                const int kb = list[q0 + q];
                const bool keep = kb == ib || (use_norm_inf_fast ? m > thr : (T) m > (T) thr);
                if (lane == 0)
                    S.slotq[q] = keep;
            }
            __syncthreads();
            if (warp == 0)
            {
                int base = kept;
                for (int c0 = 0; c0 < qn; c0 += 32)
                {
                    const int q = c0 + lane;
                    const bool f = q < qn && S.slotq[q];
                    const unsigned bal = __ballot_sync(FULL, f);
                    if (q < qn)
                        S.slotq[q] = f ? base + __popc(bal & lanemask_lt()) : -1;
                    base += __popc(bal);
                }
                if (lane == 0)
                    S.kept = base;
            }
            __syncthreads();
            kept = S.kept;
            for (int q = warp; q < qn; q += EB32_THREADS / 32)
            {
                const int d = S.slotq[q];
                if (d < 0 || d >= C.MB)
                    continue;
                const T *src = myslab + (size_t) (q0 + q) * 1024;
                T *dst = C.blk(ib, d);
                for (int h = 0; h < 2; ++h)
                {
#pragma unroll
                    for (int c = 0; c < 16; ++c)
                        tp[lane * 17 + c] = src[(h * 16 + c) * 32 + lane];
                    __syncwarp();
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                    {
                        const int e = u * 32 + lane, r = e >> 4, c = e & 15;
                        dst[r * 32 + h * 16 + c] = tp[r * 17 + c];
                    }
                    __syncwarp();
                }
                if (lane == 0)
                    C.indexb[(size_t) ib * C.MB + d] = list[q0 + q];
            }
            __syncthreads(); // slotq and S.kept are rewritten by the next chunk
        }
        if (tid == 0)
        {
            // the diagonal block is always kept; its trace in row order
            T trC = T(0);
            const int dq = mark[ib] - 1;
            if (dq >= 0 && dq < nl)
            {
                const T *x = myslab + (size_t) dq * 1024;
                for (int kk = 0; kk < 32; ++kk)
                    trC = add_rn(trC, x[kk * 33]);
            }
            C.nnzb[ib] = kept < C.MB ? kept : C.MB;
            atomicMax(&flags[1], kept);
            if (kept > C.MB)
                atomicExch(&flags[0], 1);
            if (n > cap)
                atomicExch(&flags[4], 1);
            if (dA)
                dA[ib] = (double) trA;
            if (dC)
                dC[ib] = (double) trC;
        }
        __syncthreads();
        for (int q = tid; q < nl; q += EB32_THREADS)
            mark[list[q]] = 0;
        __syncthreads();
    }
    // after a timeout, copies still in flight land before the CTA leaves:
    // the last fill of every buffer, each wait bounded
    if (tid == 0 && *reinterpret_cast<volatile int *>(tflag))
        for (unsigned b = 0; b < (unsigned) EB32_STAGES && b < issued; ++b)
        {
            const unsigned u = issued - 1 - b;
            eb_wait2s(&S.full_r[u % EB32_STAGES], (u / EB32_STAGES) & 1);
        }
}

template <typename T> int eb_grid(B200Context *c, int NB, int per_sm) { return max(1, min(NB, c->sm_count * per_sm)); }

constexpr long long EB_SLAB_BUDGET_DEFAULT = 24ll << 30;
long long g_eb_slab_budget = EB_SLAB_BUDGET_DEFAULT;

int *eb_flags(B200Context *c)
{
    int *f = reinterpret_cast<int *>(static_cast<unsigned char *>(c->d_small) + 4096);
    if (!CUDA_OK(cudaMemsetAsync(f, 0, 32, c->stream)))
        return nullptr;
    return f;
}

bool eb_read_flags(B200Context *c, int *f, int *out, int n)
{
    int *pin = reinterpret_cast<int *>(static_cast<unsigned char *>(c->pinned) + 4096);
    if (!CUDA_OK(cudaMemcpyAsync(pin, f, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    for (int q = 0; q < n; q++)
        out[q] = pin[q];
    return true;
}

bool same_partition(const bml_matrix_ellblock_t *A, const bml_matrix_ellblock_t *B, const char *op)
{
    if (!A || !B)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK %s: NULL matrix", op);
        return false;
    }
    if (A->NB != B->NB || A->matrix_precision != B->matrix_precision ||
        memcmp(A->bsize, B->bsize, sizeof(int) * A->NB) != 0)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK %s: block partitions or precisions differ", op);
        return false;
    }
    return true;
}

template <typename T>
bool eb_multiply_typed(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C,
                       double thr, bool fast_norm, double *trace)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    if (A->maxbs > 64)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "ELLBLOCK multiply: blocks larger than 64");
        return false;
    }
    // uniform 32 x 32 blocks: the register-tiled kernel (same bits)
    bool bs32 = A->maxbs == 32 && B->maxbs == 32 && C->maxbs == 32;
    for (int ib = 0; bs32 && ib < A->NB; ib++)
        bs32 = A->bsize[ib] == 32 && B->bsize[ib] == 32;
    const int grid0 = bs32 ? eb_grid<T>(c, A->NB, 4) : eb_grid<T>(c, A->NB, 2);
    const size_t slot_bytes = (size_t) A->slot_elems * sizeof(T);
    // Accumulator slots per CTA: room for all NB block columns (the
    // reference's accumulator) when the slabs of a full grid fit the budget
    // (bml_b200_set_ellblock_slab_budget, 24 GiB by default); otherwise first room for the output's width plus one, and a row
    // that touches more block columns before thresholding stops the launch
    // early and makes the call run again with room for all NB (on fewer CTAs
    // if need be).
    const size_t budget = (size_t) g_eb_slab_budget;
    const auto per_cta = [&](int cp) {
        return (size_t) cp * (slot_bytes + sizeof(int)) + (size_t) B->NB * sizeof(int);
    };
    int cap = (size_t) grid0 * per_cta(B->NB) <= budget ? B->NB : std::min(C->MB + 1, B->NB);
    int hf[8];
    for (int attempt = 0; attempt < 2; ++attempt)
    {
        const int grid = (int) std::max<size_t>(1, std::min<size_t>((size_t) grid0, budget / per_cta(cap)));
        const size_t slab = (size_t) grid * cap * slot_bytes;
        const size_t lists = (size_t) grid * cap * sizeof(int);
        const size_t marks = (size_t) grid * B->NB * sizeof(int);
        const size_t diag = (size_t) 2 * A->NB * sizeof(double);
        unsigned char *scr = static_cast<unsigned char *>(b200_scratch(slab + lists + marks + diag + 1024));
        if (!scr)
            return false;
        T *dslab = reinterpret_cast<T *>(scr);
        int *dlists = reinterpret_cast<int *>(scr + slab);
        int *dmarks = dlists + (size_t) grid * cap;
        double *dA = reinterpret_cast<double *>(scr + ((slab + lists + marks + 255) & ~size_t(255)));
        double *dC = dA + A->NB;
        int *flags = eb_flags(c);
        if (!flags || !CUDA_OK(cudaMemsetAsync(dmarks, 0, marks, c->stream)))
            return false;
        if (bs32)
        {
            const size_t smem = sizeof(EbS32<T>);
            auto k = ell_x2_exact() ? eb_mul32_kernel<T, false> : eb_mul32_kernel<T, true>;
            if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
                return false;
            k<<<grid, EB32_THREADS, smem, c->stream>>>(view<T>(A), view<T>(B), view<T>(C), thr, fast_norm ? 1 : 0,
                                                       cap, dslab, dlists, dmarks, trace ? dA : nullptr,
                                                       trace ? dC : nullptr, flags);
            if (!LAUNCH_OK("eb_mul32_kernel"))
                return false;
        }
        else
        {
            const size_t smem = 2 * slot_bytes;
            auto k = eb_mul_kernel<T>;
            if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
                return false;
            k<<<grid, 256, smem, c->stream>>>(view<T>(A), view<T>(B), view<T>(C), thr, fast_norm ? 1 : 0, cap,
                                             dslab, dlists, dmarks, trace ? dA : nullptr, trace ? dC : nullptr,
                                             flags);
            if (!LAUNCH_OK("eb_mul_kernel"))
                return false;
        }
        if (trace)
        {
            // the traces, summed over block rows, land after the flags
            double *out = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(flags) + 64);
            b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(dA, dC, A->NB, out);
            if (!LAUNCH_OK("b200_sum_rows_kernel"))
                return false;
        }
        unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 4096;
        if (!CUDA_OK(cudaMemcpyAsync(pin, flags, 64 + 16, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
            return false;
        memcpy(hf, pin, sizeof(hf));
        if (trace)
            memcpy(trace, pin + 64, 2 * sizeof(double));
        if (hf[4] && !hf[2] && cap < B->NB)
        {
            cap = B->NB;
            continue;
        }
        break;
    }
    eb_mark_device(C);
    if (hf[2])
    {
        b200_set_error(BML_B200_ERR_TIMEOUT, "ELLBLOCK multiply: a block copy did not complete");
        return false;
    }
    if (hf[0])
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW,
                       "Number of non-zeroes blocks per row > MB, Increase MB (need %d, MB = %d)", hf[1], C->MB);
        return false;
    }
    return true;
}

} // namespace

// ---------------------------------------------------------------------------
// entry points used by the C API
// ---------------------------------------------------------------------------
#define EB_DISPATCH(A, call) ((A)->matrix_precision == double_real ? call<double> : call<float>)

bool eb_copy(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B)
{
    if (!same_partition(A, B, "copy"))
        return false;
    if (A == B)
        return true;
    B200Context *c = b200_ctx();
    if (!c || !eb_to_device(A))
        return false;
    if (B->mirror == MIRROR_HOST_NEWER)
        B->mirror = MIRROR_SYNCED;
    int *f = eb_flags(c);
    if (!f)
        return false;
    const int grid = A->matrix_precision == double_real ? eb_grid<double>(c, A->NB, 8) : eb_grid<float>(c, A->NB, 8);
    if (A->matrix_precision == double_real)
        eb_copy_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), view<double>(B), f);
    else
        eb_copy_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), view<float>(B), f);
    if (!LAUNCH_OK("eb_copy_kernel"))
        return false;
    eb_mark_device(B);
    int hf = 0;
    if (!eb_read_flags(c, f, &hf, 1))
        return false;
    if (hf)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "ELLBLOCK copy: a block row of A exceeds B's MB");
        return false;
    }
    return true;
}

bml_matrix_ellblock_t *eb_copy_new(bml_matrix_ellblock_t *A)
{
    if (!A)
        return nullptr;
    bml_matrix_ellblock_t *B = eb_alloc_blocks(A->matrix_precision, A->NB, A->MB, A->M, A->bsize,
                                               A->distribution_mode);
    if (B && !eb_copy(A, B))
    {
        eb_free(B);
        return nullptr;
    }
    return B;
}

bool eb_scale(const void *scale, bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B)
{
    if (!scale || !same_partition(A, B, "scale"))
        return false;
    if (A != B && !eb_copy(A, B))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !eb_to_device(B))
        return false;
    const int grid = eb_grid<double>(c, B->NB, 8);
    if (B->matrix_precision == double_real)
        eb_scale_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(B), *static_cast<const double *>(scale));
    else
        eb_scale_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(B), *static_cast<const float *>(scale));
    if (!LAUNCH_OK("eb_scale_kernel"))
        return false;
    eb_mark_device(B);
    return true;
}

bool eb_add(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, double alpha, double beta, double threshold)
{
    if (!same_partition(A, B, "add"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !eb_to_device(A) || !eb_to_device(B))
        return false;
    if (A == B)
    {
        bml_matrix_ellblock_t *T0 = eb_copy_new(A);
        if (!T0)
            return false;
        const bool ok = eb_add(A, T0, alpha, beta, threshold);
        eb_free(T0);
        return ok;
    }
    const int grid = eb_grid<double>(c, A->NB, 4);
    const int cap = A->MB + B->MB;
    const size_t marks = (size_t) grid * (A->NB + 3 * (size_t) cap) * sizeof(int);
    int *dmarks = static_cast<int *>(b200_scratch(marks + 256));
    int *f = eb_flags(c);
    if (!dmarks || !f || !CUDA_OK(cudaMemsetAsync(dmarks, 0, marks, c->stream)))
        return false;
    if (A->matrix_precision == double_real)
        eb_add_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), view<double>(B), alpha, beta, threshold,
                                                           dmarks, cap, f);
    else
        eb_add_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), view<float>(B), alpha, beta, threshold,
                                                          dmarks, cap, f);
    if (!LAUNCH_OK("eb_add_kernel"))
        return false;
    eb_mark_device(A);
    int hf = 0;
    if (!eb_read_flags(c, f, &hf, 1))
        return false;
    if (hf)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "ELLBLOCK add: a block row of the sum exceeds MB=%d", A->MB);
        return false;
    }
    return true;
}

// A + beta*I through an identity matrix and add, as the reference does
// (ellblock/bml_add_ellblock_typed.c:355-368).
bool eb_add_identity(bml_matrix_ellblock_t *A, double beta, double threshold)
{
    if (!A)
        return false;
    bml_matrix_ellblock_t *I = eb_alloc_blocks(A->matrix_precision, A->NB, A->MB, A->M, A->bsize,
                                               A->distribution_mode);
    if (!I)
        return false;
    if (A->matrix_precision == double_real)
        fill_eb<double>(I, 3);
    else
        fill_eb<float>(I, 3);
    eb_mark_host(I);
    const bool ok = eb_to_device(I) && eb_add(A, I, 1.0, beta, threshold);
    eb_free(I);
    return ok;
}

bool eb_scale_add_identity(bml_matrix_ellblock_t *A, double alpha, double beta, double threshold)
{
    if (!A)
        return false;
    float af = (float) alpha;
    return eb_scale(A->matrix_precision == double_real ? (void *) &alpha : (void *) &af, A, A) &&
           eb_add_identity(A, beta, threshold);
}

static bool eb_threshold_fits(const bml_matrix_ellblock_t *A)
{
    if (A->maxbs <= 64)
        return true;
    b200_set_error(BML_B200_ERR_UNSUPPORTED, "ELLBLOCK threshold: blocks larger than 64");
    return false;
}

bml_matrix_ellblock_t *eb_threshold_new(bml_matrix_ellblock_t *A, double threshold)
{
    if (!A || !eb_threshold_fits(A))
        return nullptr;
    bml_matrix_ellblock_t *B = eb_alloc_blocks(A->matrix_precision, A->NB, A->MB, A->M, A->bsize,
                                               A->distribution_mode);
    B200Context *c = b200_ctx();
    if (!B || !c || !eb_to_device(A))
    {
        eb_free(B);
        return nullptr;
    }
    const int grid = eb_grid<double>(c, A->NB, 8);
    if (A->matrix_precision == double_real)
        eb_threshold_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), view<double>(B), threshold);
    else
        eb_threshold_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), view<float>(B), threshold);
    if (!LAUNCH_OK("eb_threshold_kernel"))
    {
        eb_free(B);
        return nullptr;
    }
    eb_mark_device(B);
    return B;
}

bool eb_threshold(bml_matrix_ellblock_t *A, double threshold)
{
    B200Context *c = b200_ctx();
    if (!A || !c || !eb_threshold_fits(A) || !eb_to_device(A))
        return false;
    // in place: each block row's surviving blocks move to lower positions only
    const int grid = eb_grid<double>(c, A->NB, 8);
    if (A->matrix_precision == double_real)
        eb_threshold_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), view<double>(A), threshold);
    else
        eb_threshold_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), view<float>(A), threshold);
    if (!LAUNCH_OK("eb_threshold_kernel"))
        return false;
    eb_mark_device(A);
    return true;
}

static bool eb_sum_to_host(B200Context *c, double *d, int n, double *out2)
{
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 4096 + 128);
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(d, nullptr, n, out);
    if (!LAUNCH_OK("b200_sum_rows_kernel"))
        return false;
    double *pin = reinterpret_cast<double *>(static_cast<unsigned char *>(c->pinned) + 4096 + 128);
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    out2[0] = pin[0];
    return true;
}

bool eb_trace(bml_matrix_ellblock_t *A, double *trace)
{
    B200Context *c = b200_ctx();
    if (!A || !c || !eb_to_device(A))
        return false;
    double *d = static_cast<double *>(b200_scratch((size_t) A->NB * sizeof(double)));
    if (!d)
        return false;
    const int grid = max(1, min(b200_ceil_div(A->NB, 256), c->sm_count * 4));
    if (A->matrix_precision == double_real)
        eb_diag_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), d);
    else
        eb_diag_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), d);
    if (!LAUNCH_OK("eb_diag_kernel"))
        return false;
    return eb_sum_to_host(c, d, A->NB, trace);
}

bool eb_trace_mult(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, double *trace)
{
    if (!same_partition(A, B, "trace_mult"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !eb_to_device(A) || !eb_to_device(B))
        return false;
    double *d = static_cast<double *>(b200_scratch((size_t) A->NB * sizeof(double)));
    if (!d)
        return false;
    const int grid = eb_grid<double>(c, A->NB, 8);
    if (A->matrix_precision == double_real)
        eb_trace_mult_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), view<double>(B), d);
    else
        eb_trace_mult_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), view<float>(B), d);
    if (!LAUNCH_OK("eb_trace_mult_kernel"))
        return false;
    return eb_sum_to_host(c, d, A->NB, trace);
}

bml_matrix_ellblock_t *eb_transpose_new(bml_matrix_ellblock_t *A)
{
    B200Context *c = b200_ctx();
    if (!A || !c || !eb_to_device(A))
        return nullptr;
    bml_matrix_ellblock_t *B = eb_alloc_blocks(A->matrix_precision, A->NB, A->MB, A->M, A->bsize,
                                               A->distribution_mode);
    int *f = eb_flags(c);
    if (!B || !f)
    {
        eb_free(B);
        return nullptr;
    }
    const size_t smem = (((size_t) 2 * B->MB * sizeof(int) + 15) & ~size_t(15)) +
                        (size_t) A->maxbs * (A->maxbs + 1) * prec_size(A->matrix_precision);
    if (smem > (size_t) c->smem_optin)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "ELLBLOCK transpose: MB=%d too large", B->MB);
        eb_free(B);
        return nullptr;
    }
    // per row of B: a count and the source slot of every block
    int *cnt = static_cast<int *>(b200_scratch((size_t) A->NB * (1 + (size_t) B->MB) * sizeof(int)));
    if (!cnt || !CUDA_OK(cudaMemsetAsync(cnt, 0, sizeof(int) * A->NB, c->stream)))
    {
        eb_free(B);
        return nullptr;
    }
    int *src = cnt + A->NB;
    const long long entries = (long long) A->NB * A->MB;
    const int sgrid = (int) std::min<long long>((entries + 255) / 256, (long long) c->sm_count * 8);
    eb_tr_scatter_kernel<<<sgrid, 256, 0, c->stream>>>(A->d_indexb, A->d_nnzb, A->NB, A->MB, B->MB, cnt, src, f);
    const int grid = eb_grid<double>(c, A->NB, 8);
    bool launched = LAUNCH_OK("eb_tr_scatter_kernel");
    if (launched && A->matrix_precision == double_real)
    {
        launched = CUDA_OK(cudaFuncSetAttribute(eb_tr_place_kernel<double>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        if (launched)
            eb_tr_place_kernel<double><<<grid, 128, smem, c->stream>>>(view<double>(A), view<double>(B), cnt, src);
    }
    else if (launched)
    {
        launched = CUDA_OK(cudaFuncSetAttribute(eb_tr_place_kernel<float>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        if (launched)
            eb_tr_place_kernel<float><<<grid, 128, smem, c->stream>>>(view<float>(A), view<float>(B), cnt, src);
    }
    int hf = 0;
    if (!launched || !LAUNCH_OK("eb_tr_place_kernel") || !eb_read_flags(c, f, &hf, 1))
    {
        eb_free(B);
        return nullptr;
    }
    eb_mark_device(B);
    if (hf)
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "ELLBLOCK transpose: a block column exceeds MB");
    return B;
}

bool eb_transpose(bml_matrix_ellblock_t *A)
{
    bml_matrix_ellblock_t *B = eb_transpose_new(A);
    if (!B)
        return false;
    const bool ok = eb_copy(B, A);
    eb_free(B);
    return ok;
}

bool eb_gershgorin(bml_matrix_ellblock_t *A, double *bounds)
{
    B200Context *c = b200_ctx();
    if (!A || !c || !eb_to_device(A))
        return false;
    double *hi = static_cast<double *>(b200_scratch((size_t) 2 * A->N * sizeof(double)));
    if (!hi)
        return false;
    double *lo = hi + A->N;
    const int grid = eb_grid<double>(c, A->NB, 8);
    if (A->matrix_precision == double_real)
        eb_gersh_kernel<double><<<grid, 64, 0, c->stream>>>(view<double>(A), hi, lo);
    else
        eb_gersh_kernel<float><<<grid, 64, 0, c->stream>>>(view<float>(A), hi, lo);
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 4096 + 192);
    b200_count_launch();
    b200_maxmin_rows_kernel<<<1, 1024, 0, c->stream>>>(hi, lo, A->N, DBL_MIN, DBL_MAX, out);
    if (!LAUNCH_OK("eb gershgorin"))
        return false;
    double *pin = reinterpret_cast<double *>(static_cast<unsigned char *>(c->pinned) + 4096 + 192);
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    bounds[0] = pin[1];
    bounds[1] = pin[0];
    return true;
}

bool eb_normalize(bml_matrix_ellblock_t *A, double mineval, double maxeval)
{
    const double mm = maxeval - mineval;
    double sd = -1.0 / mm;
    float sf = (float) (-1.0 / mm);
    return A && eb_scale(A->matrix_precision == double_real ? (void *) &sd : (void *) &sf, A, A) &&
           eb_add_identity(A, maxeval / mm, 0.0);
}

// ---------------------------------------------------------------------------
// ELLPACK <-> ELLBLOCK on the device (bml_convert,
// ellblock/bml_convert_ellblock_typed.c:16-73, ellpack/bml_convert_ellpack_typed.c:13-36).
// The reference builds the ELLBLOCK matrix with every one of the NB x NB
// blocks, filled element by element through bml_get_element; here each
// block row holds the blocks its rows have entries in, in ascending block
// column, with the same values (the dense forms are identical), and the
// slots per block row are sized to the widest block row.
// ---------------------------------------------------------------------------
namespace {

// Block columns touched by the rows of block row ib, as a bitmap over NB in
// shared memory (NB/32 words); one CTA per block row.
// Entries with a column outside [0, N) or a row length outside [0, ldE]
// raise *bad and are skipped.
template <typename Tin>
__device__ void conv_bitmap(const int *En, const int *Ei, int ldE, int N, const int *colblk, int r0, int r1,
                            unsigned *bits, int words, int *bad)
{
    for (int w = threadIdx.x; w < words; w += blockDim.x)
        bits[w] = 0u;
    __syncthreads();
    for (int i = r0; i < r1; ++i)
    {
        const int n = En[i];
        if (n < 0 || n > ldE)
        {
            *bad = 1;
            continue;
        }
        for (int p = threadIdx.x; p < n; p += blockDim.x)
        {
            const int j = Ei[(size_t) i * ldE + p];
            if (j < 0 || j >= N)
            {
                *bad = 1;
                continue;
            }
            const int jb = colblk[j];
            atomicOr(&bits[jb >> 5], 1u << (jb & 31));
        }
    }
    __syncthreads();
}

template <typename Tin>
__global__ void __launch_bounds__(256) conv_count_kernel(const int *En, const int *Ei, int ldE, int N,
                                                         const int *colblk, const int *boff, int NB, int *maxcnt)
{
    extern __shared__ unsigned bits[];
    const int words = (NB + 31) >> 5;
    __shared__ int cnt;
    for (int ib = blockIdx.x; ib < NB; ib += gridDim.x)
    {
        conv_bitmap<Tin>(En, Ei, ldE, N, colblk, boff[ib], boff[ib + 1], bits, words, maxcnt + 1);
        if (threadIdx.x == 0)
            cnt = 0;
        __syncthreads();
        int c = 0;
        for (int w = threadIdx.x; w < words; w += blockDim.x)
            c += __popc(bits[w]);
        atomicAdd(&cnt, c);
        __syncthreads();
        if (threadIdx.x == 0)
            atomicMax(maxcnt, cnt);
        __syncthreads();
    }
}

// Slots in ascending block column (rank = popcount prefix of the bitmap),
// then every entry written into its block (the pool starts zeroed).
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) conv_fill_kernel(const Tin *Ev, const int *Ei, const int *En, int ldE, int N,
                                                        const int *colblk, EbView<Tout> B, int *bad)
{
    extern __shared__ unsigned bits[];
    const int words = (B.NB + 31) >> 5;
    int *pre = reinterpret_cast<int *>(bits + words); // prefix popcounts per word
    for (int ib = blockIdx.x; ib < B.NB; ib += gridDim.x)
    {
        const int r0 = B.boff[ib], r1 = B.boff[ib + 1];
        conv_bitmap<Tin>(En, Ei, ldE, N, colblk, r0, r1, bits, words, bad);
        if (threadIdx.x == 0)
        {
            int run = 0;
            for (int w = 0; w < words; ++w)
            {
                pre[w] = run;
                run += __popc(bits[w]);
            }
            B.nnzb[ib] = run;
        }
        __syncthreads();
        for (int w = threadIdx.x; w < words; w += blockDim.x)
        {
            unsigned m = bits[w];
            int r = pre[w];
            while (m)
            {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                B.indexb[(size_t) ib * B.MB + r++] = w * 32 + b;
            }
        }
        for (int i = r0; i < r1; ++i)
        {
            const int n = En[i];
            const int ii = i - r0;
            if (n < 0 || n > ldE)
                continue;
            for (int p = threadIdx.x; p < n; p += blockDim.x)
            {
                const int j = Ei[(size_t) i * ldE + p];
                if (j < 0 || j >= N)
                    continue;
                const int jb = colblk[j];
                const int w = jb >> 5;
                const int rank = pre[w] + __popc(bits[w] & ((1u << (jb & 31)) - 1u));
                Tout *blk = B.blk(ib, rank);
                blk[ii * B.bsize[jb] + (j - B.boff[jb])] = (Tout) Ev[(size_t) i * ldE + p];
            }
        }
        __syncthreads();
    }
}

// ELLBLOCK -> ELLPACK: row i takes the nonzero elements of its block row's
// row ii, blocks in list order; one warp per scalar row.  Counts only when
// `count` (the widest row into *maxw).
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(256) conv_back_kernel(EbView<Tin> A, const int *rowblk, Tout *Ev, int *Ei, int *En,
                                                        int ldE, int M, int N, int count, int *maxw)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int ib = rowblk[i];
        const int ii = i - A.boff[ib];
        int n = 0;
        for (int jp = 0; jp < A.nnzb[ib]; ++jp)
        {
            const int jb = A.indexb[(size_t) ib * A.MB + jp];
            const int bs = A.bsize[jb];
            const Tin *row = A.blk(ib, jp) + (size_t) ii * bs;
            for (int b = 0; b < bs; b += 32)
            {
                const int jj = b + lane;
                const Tin v = jj < bs ? row[jj] : Tin(0);
                const bool keep = jj < bs && v != Tin(0);
                const unsigned bal = __ballot_sync(FULL, keep);
                const int pos = n + __popc(bal & lanemask_lt());
                if (!count && keep && pos < M)
                {
                    Ei[(size_t) i * ldE + pos] = A.boff[jb] + jj;
                    Ev[(size_t) i * ldE + pos] = (Tout) v;
                }
                n += __popc(bal);
            }
        }
        if (lane == 0)
        {
            atomicMax(maxw, n);
            if (!count)
                En[i] = min(n, M);
        }
    }
}

template <typename Tin, typename Tout>
bool conv_fill(B200Context *c, bml_matrix_ellpack_t *E, const int *colblk, bml_matrix_ellblock_t *B, size_t smem)
{
    const int grid = max(1, min(B->NB, c->sm_count * 4));
    conv_fill_kernel<Tin, Tout><<<grid, 256, smem, c->stream>>>(static_cast<const Tin *>(E->d_value), E->d_index,
                                                                E->d_nnz, E->ld, E->N, colblk, view<Tout>(B),
                                                                eb_flags(c) + 1);
    return LAUNCH_OK("conv_fill_kernel");
}

} // namespace

bml_matrix_ellblock_t *eb_from_ellpack(bml_matrix_ellpack_t *E, bml_matrix_precision_t prec, int M,
                                       bml_distribution_mode_t mode)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(E))
        return nullptr;
    const int N = E->N;
    int *bsize = bml_get_block_sizes(N, M);
    const int NB = bml_get_nb();
    std::vector<int> colblk(N), boff(NB + 1, 0);
    for (int ib = 0; ib < NB; ++ib)
    {
        boff[ib + 1] = boff[ib] + bsize[ib];
        for (int r = boff[ib]; r < boff[ib + 1] && r < N; ++r)
            colblk[r] = ib;
    }
    if (boff[NB] != N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "convert: the block sizes sum to %d, N=%d", boff[NB], N);
        return nullptr;
    }
    const size_t words = (size_t) (NB + 31) / 32;
    const size_t smem = words * (sizeof(unsigned) + sizeof(int));
    if (smem > c->smem_optin)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "convert: NB=%d block columns", NB);
        return nullptr;
    }
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch((size_t) (N + NB + 1) * sizeof(int) + 256));
    int *f = eb_flags(c);
    if (!scr || !f)
        return nullptr;
    int *dcolblk = reinterpret_cast<int *>(scr);
    int *dboff = dcolblk + N;
    if (!CUDA_OK(cudaMemcpyAsync(dcolblk, colblk.data(), sizeof(int) * N, cudaMemcpyHostToDevice, c->stream)) ||
        !CUDA_OK(cudaMemcpyAsync(dboff, boff.data(), sizeof(int) * (NB + 1), cudaMemcpyHostToDevice, c->stream)))
        return nullptr;
    for (auto kern : {conv_count_kernel<double>})
        if (!CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return nullptr;
    conv_count_kernel<double><<<max(1, min(NB, c->sm_count * 4)), 256, smem, c->stream>>>(
        E->d_nnz, E->d_index, E->ld, N, dcolblk, dboff, NB, f);
    int hf[2] = {0, 0};
    if (!LAUNCH_OK("conv_count_kernel") || !eb_read_flags(c, f, hf, 2))
        return nullptr;
    if (hf[1])
    {
        b200_set_error(BML_B200_ERR_INVALID, "convert: a column index or row length out of range");
        return nullptr;
    }
    const int maxcnt = hf[0];
    int MB = maxcnt > 0 ? maxcnt : 1;
    const int mb_state = bml_get_mb();
    if (mb_state > MB)
        MB = mb_state < NB ? mb_state : NB;
    bml_matrix_ellblock_t *B = eb_alloc_blocks(prec, NB, MB, M, bsize, mode);
    if (!B)
        return nullptr;
    bool ok;
    const bool din = E->matrix_precision == double_real, dout = prec == double_real;
    auto set_smem = [&](auto kern) {
        return CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    };
    if (din && dout)
        ok = set_smem(conv_fill_kernel<double, double>) && conv_fill<double, double>(c, E, dcolblk, B, smem);
    else if (din)
        ok = set_smem(conv_fill_kernel<double, float>) && conv_fill<double, float>(c, E, dcolblk, B, smem);
    else if (dout)
        ok = set_smem(conv_fill_kernel<float, double>) && conv_fill<float, double>(c, E, dcolblk, B, smem);
    else
        ok = set_smem(conv_fill_kernel<float, float>) && conv_fill<float, float>(c, E, dcolblk, B, smem);
    if (!ok)
    {
        eb_free(B);
        return nullptr;
    }
    eb_mark_device(B);
    return B;
}

bml_matrix_ellpack_t *ell_from_ellblock(bml_matrix_ellblock_t *A, bml_matrix_precision_t prec, int M,
                                        bml_distribution_mode_t mode)
{
    B200Context *c = b200_ctx();
    if (!c || !eb_to_device(A))
        return nullptr;
    const int N = A->N;
    std::vector<int> rowblk(N);
    for (int ib = 0, r = 0; ib < A->NB; ++ib)
        for (int k = 0; k < A->bsize[ib]; ++k)
            rowblk[r++] = ib;
    int *drowblk = static_cast<int *>(b200_scratch(sizeof(int) * (size_t) N + 256));
    int *f = eb_flags(c);
    if (!drowblk || !f ||
        !CUDA_OK(cudaMemcpyAsync(drowblk, rowblk.data(), sizeof(int) * N, cudaMemcpyHostToDevice, c->stream)))
        return nullptr;
    bml_matrix_ellpack_t *E = ell_alloc(prec, N, M, mode, true);
    if (!E)
        return nullptr;
    const int grid = max(1, min(b200_ceil_div(N, 8), c->sm_count * 16));
    const bool din = A->matrix_precision == double_real, dout = prec == double_real;
    auto launch = [&](int count) {
        if (din && dout)
            conv_back_kernel<double, double><<<grid, 256, 0, c->stream>>>(
                view<double>(A), drowblk, static_cast<double *>(E->d_value), E->d_index, E->d_nnz, E->ld, E->M, N,
                count, f);
        else if (din)
            conv_back_kernel<double, float><<<grid, 256, 0, c->stream>>>(
                view<double>(A), drowblk, static_cast<float *>(E->d_value), E->d_index, E->d_nnz, E->ld, E->M, N,
                count, f);
        else if (dout)
            conv_back_kernel<float, double><<<grid, 256, 0, c->stream>>>(
                view<float>(A), drowblk, static_cast<double *>(E->d_value), E->d_index, E->d_nnz, E->ld, E->M, N,
                count, f);
        else
            conv_back_kernel<float, float><<<grid, 256, 0, c->stream>>>(
                view<float>(A), drowblk, static_cast<float *>(E->d_value), E->d_index, E->d_nnz, E->ld, E->M, N,
                count, f);
        return LAUNCH_OK("conv_back_kernel");
    };
    int maxw = 0;
    if (!launch(0) || !eb_read_flags(c, f, &maxw, 1))
    {
        ell_free(E);
        return nullptr;
    }
    ell_mark_device(E);
    if (maxw > M)
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "convert: a row holds %d nonzeros, M=%d", maxw, M);
    return E;
}

bml_matrix_ellblock_t *eb_import_dense(bml_matrix_precision_t prec, bml_dense_order_t order, int N, int M,
                                       void *D, double threshold, bml_distribution_mode_t mode)
{
    bml_matrix_ellblock_t *A = eb_constructor(0, prec, N, M, mode);
    B200Context *c = b200_ctx();
    if (!A || !c)
        return A;
    if (A->N != N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLBLOCK import: block sizes sum to %d, N=%d", A->N, N);
        eb_free(A);
        return nullptr;
    }
    const size_t sz = prec_size(prec);
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch((size_t) N * N * sz));
    int *f = eb_flags(c);
    if (!scr || !f || !CUDA_OK(cudaMemcpyAsync(scr, D, (size_t) N * N * sz, cudaMemcpyHostToDevice, c->stream)))
    {
        eb_free(A);
        return nullptr;
    }
    const int grid = eb_grid<double>(c, A->NB, 8);
    const int colmajor = order == dense_column_major;
    if (prec == double_real)
        eb_import_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), reinterpret_cast<double *>(scr), N,
                                                              colmajor, threshold, f);
    else
        eb_import_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), reinterpret_cast<float *>(scr), N,
                                                             colmajor, threshold, f);
    int hf = 0;
    if (!LAUNCH_OK("eb_import_kernel") || !eb_read_flags(c, f, &hf, 1))
    {
        eb_free(A);
        return nullptr;
    }
    eb_mark_device(A);
    if (hf)
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "ELLBLOCK import: more than MB blocks above threshold in a row");
    return A;
}

void *eb_export_dense(bml_matrix_ellblock_t *A, bml_dense_order_t order)
{
    B200Context *c = b200_ctx();
    if (!A || !c || !eb_to_device(A))
        return nullptr;
    const size_t sz = prec_size(A->matrix_precision);
    const size_t bytes = (size_t) A->N * A->N * sz;
    void *D = calloc((size_t) A->N * A->N, sz);
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(bytes));
    if (!D || !scr || !CUDA_OK(cudaMemsetAsync(scr, 0, bytes, c->stream)))
    {
        free(D);
        return nullptr;
    }
    const int grid = eb_grid<double>(c, A->NB, 8);
    const int colmajor = order == dense_column_major;
    if (A->matrix_precision == double_real)
        eb_export_kernel<double><<<grid, 256, 0, c->stream>>>(view<double>(A), reinterpret_cast<double *>(scr), A->N,
                                                              colmajor);
    else
        eb_export_kernel<float><<<grid, 256, 0, c->stream>>>(view<float>(A), reinterpret_cast<float *>(scr), A->N,
                                                             colmajor);
    if (!LAUNCH_OK("eb_export_kernel") ||
        !CUDA_OK(cudaMemcpyAsync(D, scr, bytes, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
    {
        free(D);
        return nullptr;
    }
    return D;
}

bool eb_multiply_x2(bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, double threshold, double *trace)
{
    if (!same_partition(X, X2, "multiply_x2") || X == X2)
        return false;
    if (!eb_to_device(X) || !eb_to_device(X2))
        return false;
    if (X2->mirror == MIRROR_HOST_NEWER)
        X2->mirror = MIRROR_SYNCED;
    double tr[2] = {0, 0};
    const bool ok = X->matrix_precision == double_real
                        ? eb_multiply_typed<double>(X, X, X2, threshold, true, tr)
                        : eb_multiply_typed<float>(X, X, X2, threshold, true, tr);
    if (trace)
    {
        trace[0] = tr[0];
        trace[1] = tr[1];
    }
    return ok;
}

bool eb_multiply_AB(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C, double threshold)
{
    if (!same_partition(A, B, "multiply_AB") || !same_partition(A, C, "multiply_AB") || C == A || C == B)
        return false;
    if (!eb_to_device(A) || !eb_to_device(B) || !eb_to_device(C))
        return false;
    return A->matrix_precision == double_real ? eb_multiply_typed<double>(A, B, C, threshold, false, nullptr)
                                              : eb_multiply_typed<float>(A, B, C, threshold, false, nullptr);
}

// C <- alpha*A*B + beta*C (ellblock/bml_multiply_ellblock_typed.c:183-231)
bool eb_multiply(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C, double alpha,
                 double beta, double threshold)
{
    if (A == B && alpha == 1.0 && beta == 0.0)
        return eb_multiply_x2(A, C, threshold, nullptr);
    bml_matrix_ellblock_t *T0 = eb_alloc_blocks(C->matrix_precision, C->NB, C->MB, C->M, C->bsize,
                                                C->distribution_mode);
    if (!T0)
        return false;
    bool ok = A == B ? eb_multiply_x2(A, T0, threshold, nullptr) : eb_multiply_AB(A, B, T0, threshold);
    if (ok)
        ok = eb_add(C, T0, beta, alpha, threshold);
    eb_free(T0);
    return ok;
}

// ---------------------------------------------------------------------------
// Synthetic ELLBLOCK Hamiltonian on a block lattice (no reference
// counterpart): L^3 block sites (x fastest), block (a, b) present when the
// sites are within `radius` (open boundaries), entries N(0,1) * exp(-d).
// Symmetric: the block of (a, b), a < b, is drawn once in row a (row-major)
// and transposed into row b; a diagonal block draws its upper triangle.
// splitmix64 + Box-Muller as the ELLPACK generators.  The block partition
// must already be L^3 blocks of bs (bml_set_block_sizes), MB at least the
// number of neighbours.
// ---------------------------------------------------------------------------
namespace {

struct Sm64
{
    uint64_t s;
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double) (next() >> 11) * 0x1.0p-53; }
    double normal()
    {
        const double u1 = 1.0 - uniform();
        const double u2 = uniform();
        return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925 * u2);
    }
};

template <typename T> void fill_block_lattice(bml_matrix_ellblock_t *A, int L, double radius, uint64_t seed)
{
    const int bs = A->bsize[0];
    const int R = (int) floor(radius);
    Sm64 rng{seed};
    T *pool = static_cast<T *>(A->h_pool);
    for (int a = 0; a < A->NB; ++a)
    {
        const int ax = a % L, ay = (a / L) % L, az = a / (L * L);
        int n = 0;
        // neighbours in ascending index order: z, then y, then x
        for (int dz = -R; dz <= R; ++dz)
            for (int dy = -R; dy <= R; ++dy)
                for (int dx = -R; dx <= R; ++dx)
                {
                    const int x = ax + dx, y = ay + dy, z = az + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= L || y >= L || z >= L)
                        continue;
                    const double d = sqrt((double) (dx * dx + dy * dy + dz * dz));
                    if (d > radius)
                        continue;
                    const int b = (z * L + y) * L + x;
                    T *blk = pool + ((size_t) a * A->MB + n) * A->slot_elems;
                    if (b > a)
                    {
                        const double s = exp(-d);
                        for (int e = 0; e < bs * bs; ++e)
                            blk[e] = (T) (rng.normal() * s);
                    }
                    else if (b == a)
                    {
                        for (int r = 0; r < bs; ++r)
                            for (int c = r; c < bs; ++c)
                                blk[r * bs + c] = blk[c * bs + r] = (T) rng.normal();
                    }
                    else
                    {
                        // (b, a) was drawn in row b: find it and transpose
                        int p = 0;
                        while (A->indexb[(size_t) b * A->MB + p] != a)
                            ++p;
                        const T *src = pool + ((size_t) b * A->MB + p) * A->slot_elems;
                        for (int r = 0; r < bs; ++r)
                            for (int c = 0; c < bs; ++c)
                                blk[r * bs + c] = src[c * bs + r];
                    }
                    A->indexb[(size_t) a * A->MB + n] = b;
                    ++n;
                }
        A->nnzb[a] = n;
    }
}

} // namespace

extern "C" BML_B200_API long long bml_b200_set_ellblock_slab_budget(long long bytes)
{
    const long long old = g_eb_slab_budget;
    g_eb_slab_budget = bytes > 0 ? bytes : EB_SLAB_BUDGET_DEFAULT;
    return old;
}

extern "C" bml_matrix_t *bml_b200_gen_block_lattice(int L, double radius, int bs, unsigned long long seed,
                                                    bml_matrix_precision_t prec)
{
    const int NB = L * L * L;
    const int R = (int) floor(radius);
    int span = 0;
    for (int dz = -R; dz <= R; ++dz)
        for (int dy = -R; dy <= R; ++dy)
            for (int dx = -R; dx <= R; ++dx)
                if (dx * dx + dy * dy + dz * dz <= radius * radius)
                    ++span;
    if (L <= 0 || bs <= 0 || bml_get_nb() != NB || bml_get_mb() < span)
    {
        b200_set_error(BML_B200_ERR_INVALID,
                       "gen_block_lattice: set a partition of L^3 = %d blocks of %d with MB >= %d first", NB, bs,
                       span);
        return nullptr;
    }
    int *bsize = bml_get_block_sizes(NB * bs, NB * bs);
    for (int ib = 0; ib < NB; ++ib)
        if (bsize[ib] != bs)
        {
            b200_set_error(BML_B200_ERR_INVALID, "gen_block_lattice: block %d has size %d, not %d", ib, bsize[ib], bs);
            return nullptr;
        }
    bml_matrix_ellblock_t *A = eb_alloc_blocks(prec, NB, bml_get_mb(), NB * bs, bsize, sequential);
    if (!A)
        return nullptr;
    if (prec == double_real)
        fill_block_lattice<double>(A, L, radius, seed);
    else
        fill_block_lattice<float>(A, L, radius, seed);
    host_pointers(A);
    eb_mark_host(A);
    if (!eb_to_device(A))
    {
        eb_free(A);
        return nullptr;
    }
    return A;
}
