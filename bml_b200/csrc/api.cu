// Public bml_* entry points: dispatch on the matrix type (the first int of the
// struct, as bml_introspection.c:21-32 reads it) and precision, argument
// checks, and the host-side conveniences (element access, printing, I/O).
#include "internal.h"
#include "ellblock.h"

#include <cmath>
#include <cstdlib>
#include <cstring>

bml_matrix_ellpack_t *ell_constructor(int kind, bml_matrix_precision_t prec, int N, int M,
                                      bml_distribution_mode_t mode);

namespace {

thread_local int g_required_M = 0;

bml_matrix_type_t type_of(const bml_matrix_t *A)
{
    return A ? *static_cast<const bml_matrix_type_t *>(A) : type_uninitialized;
}

bml_matrix_precision_t prec_of(const bml_matrix_t *A)
{
    return A ? static_cast<const bml_matrix_precision_t *>(A)[1] : precision_uninitialized;
}

bool real_prec(bml_matrix_precision_t p) { return p == single_real || p == double_real; }

bml_matrix_ellpack_t *as_ell(bml_matrix_t *A, const char *op)
{
    if (!A)
    {
        b200_set_error(BML_B200_ERR_INVALID, "%s: NULL matrix", op);
        return nullptr;
    }
    auto *E = static_cast<bml_matrix_ellpack_t *>(A);
    if (E->matrix_type != ellpack || !real_prec(E->matrix_precision))
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "%s: matrix type %d precision %d", op,
                       (int) E->matrix_type, (int) E->matrix_precision);
        return nullptr;
    }
    return E;
}

bool unsupported(const bml_matrix_t *A, const char *op)
{
    b200_set_error(BML_B200_ERR_UNSUPPORTED, "%s: matrix type %d precision %d", op,
                   (int) type_of(A), (int) prec_of(A));
    return false;
}

template <typename T> void print_value(T v) { printf(" % 1.5e", (double) v); }

} // namespace

extern "C" {

// ---------------------------------------------------------------------------
// memory helpers (bml_allocate.c:43-120)
// ---------------------------------------------------------------------------
void *bml_allocate_memory(size_t s)
{
    void *p = calloc(1, s ? s : 1);
    if (!p)
        b200_set_error(BML_B200_ERR_ALLOC, "host allocation of %zu bytes", s);
    return p;
}

void *bml_noinit_allocate_memory(size_t s)
{
    void *p = malloc(s ? s : 1);
    if (!p)
        b200_set_error(BML_B200_ERR_ALLOC, "host allocation of %zu bytes", s);
    return p;
}

void bml_free_memory(void *ptr) { free(ptr); }

void bml_free_ptr(void **ptr)
{
    if (ptr)
    {
        free(*ptr);
        *ptr = nullptr;
    }
}

int bml_allocated(bml_matrix_t *A) { return A != nullptr; }

bml_domain_t *bml_default_domain(int N, int M, bml_distribution_mode_t distrib_mode)
{
    return b200_default_domain(N, M, distrib_mode);
}

void bml_deallocate_domain(bml_domain_t *D) { b200_free_domain(D); }

void bml_deallocate(bml_matrix_t **A)
{
    if (!A || !*A)
        return;
    switch (type_of(*A))
    {
    case ellpack: ell_free(static_cast<bml_matrix_ellpack_t *>(*A)); break;
    case ellblock: eb_free(static_cast<bml_matrix_ellblock_t *>(*A)); break;
    default: unsupported(*A, "deallocate"); return;
    }
    *A = nullptr;
}

void bml_clear(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
    {
        eb_clear(static_cast<bml_matrix_ellblock_t *>(A));
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "clear");
    B200Context *c = b200_ctx();
    if (!E || !c)
        return;
    const size_t sz = prec_size(E->matrix_precision);
    if (E->mirror == MIRROR_HOST_NEWER)
        E->mirror = MIRROR_SYNCED;
    if (CUDA_OK(cudaMemsetAsync(E->d_nnz, 0, (size_t) E->N * sizeof(int), c->stream)) &&
        CUDA_OK(cudaMemsetAsync(E->d_value, 0, (size_t) E->N * E->ld * sz, c->stream)) &&
        CUDA_OK(cudaMemsetAsync(E->d_index, 0, (size_t) E->N * E->ld * sizeof(int), c->stream)))
        ell_mark_device(E);
}

static bml_matrix_t *make_matrix(int kind, bml_matrix_type_t type, bml_matrix_precision_t prec,
                                 int N, int M, bml_distribution_mode_t mode, const char *op)
{
    if (!real_prec(prec))
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "%s: precision %d", op, (int) prec);
        return nullptr;
    }
    if (type == ellpack)
    {
        if (kind == 0)
            return ell_alloc(prec, N, M, mode, true);
        if (kind == 4)
            return ell_alloc(prec, N, M, mode, false);
        return ell_constructor(kind, prec, N, M, mode);
    }
    if (type == ellblock)
        return eb_constructor(kind, prec, N, M, mode);
    b200_set_error(BML_B200_ERR_UNSUPPORTED, "%s: matrix type %d", op, (int) type);
    return nullptr;
}

bml_matrix_t *bml_zero_matrix(bml_matrix_type_t t, bml_matrix_precision_t p, int N, int M,
                              bml_distribution_mode_t d)
{
    return make_matrix(0, t, p, N, M, d, "zero_matrix");
}

bml_matrix_t *bml_noinit_matrix(bml_matrix_type_t t, bml_matrix_precision_t p, int N, int M,
                                bml_distribution_mode_t d)
{
    return make_matrix(4, t, p, N, M, d, "noinit_matrix");
}

bml_matrix_t *bml_random_matrix(bml_matrix_type_t t, bml_matrix_precision_t p, int N, int M,
                                bml_distribution_mode_t d)
{
    return make_matrix(1, t, p, N, M, d, "random_matrix");
}

bml_matrix_t *bml_banded_matrix(bml_matrix_type_t t, bml_matrix_precision_t p, int N, int M,
                                bml_distribution_mode_t d)
{
    return make_matrix(2, t, p, N, M, d, "banded_matrix");
}

bml_matrix_t *bml_identity_matrix(bml_matrix_type_t t, bml_matrix_precision_t p, int N, int M,
                                  bml_distribution_mode_t d)
{
    return make_matrix(3, t, p, N, M, d, "identity_matrix");
}

// ---------------------------------------------------------------------------
// introspection
// ---------------------------------------------------------------------------
bml_matrix_type_t bml_get_type(bml_matrix_t *A) { return type_of(A); }
bml_matrix_type_t bml_get_deep_type(bml_matrix_t *A) { return type_of(A); }
bml_matrix_precision_t bml_get_precision(bml_matrix_t *A) { return prec_of(A); }

int bml_get_N(bml_matrix_t *A)
{
    if (!A)
        return -1;
    return type_of(A) == ellblock ? static_cast<bml_matrix_ellblock_t *>(A)->N
                                  : static_cast<bml_matrix_ellpack_t *>(A)->N;
}

int bml_get_M(bml_matrix_t *A)
{
    if (!A)
        return -1;
    return type_of(A) == ellblock ? static_cast<bml_matrix_ellblock_t *>(A)->M
                                  : static_cast<bml_matrix_ellpack_t *>(A)->M;
}

int bml_get_NB(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
        return static_cast<bml_matrix_ellblock_t *>(A)->NB;
    return -1;
}

bml_distribution_mode_t bml_get_distribution_mode(bml_matrix_t *A)
{
    return A ? static_cast<const bml_distribution_mode_t *>(A)[2] : sequential;
}

int bml_get_row_bandwidth(bml_matrix_t *A, int i)
{
    if (type_of(A) == ellblock)
        return eb_row_bandwidth(static_cast<bml_matrix_ellblock_t *>(A), i);
    bml_matrix_ellpack_t *E = as_ell(A, "get_row_bandwidth");
    if (!E || i < 0 || i >= E->N || !ell_to_host(E))
        return -1;
    return E->nnz[i];
}

int bml_get_bandwidth(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
        return eb_bandwidth(static_cast<bml_matrix_ellblock_t *>(A));
    bml_matrix_ellpack_t *E = as_ell(A, "get_bandwidth");
    long long tot = 0;
    int maxrow = 0;
    if (!E || !ell_nnz_total(E, &tot, &maxrow))
        return -1;
    return maxrow;
}

double bml_get_sparsity(bml_matrix_t *A, double threshold)
{
    if (type_of(A) == ellblock)
        return eb_sparsity(static_cast<bml_matrix_ellblock_t *>(A), threshold);
    bml_matrix_ellpack_t *E = as_ell(A, "get_sparsity");
    if (!E || !ell_to_host(E))
        return -1.0;
    long long nnzs = 0;
    for (int i = 0; i < E->N; i++)
        for (int j = 0; j < E->nnz[i]; j++)
        {
            const double v = E->matrix_precision == double_real
                                 ? fabs(static_cast<double *>(E->value)[(size_t) i * E->M + j])
                                 : fabsf(static_cast<float *>(E->value)[(size_t) i * E->M + j]);
            if (v > threshold)
                nnzs++;
        }
    return 1.0 - (double) nnzs / ((double) E->N * E->N);
}

// ---------------------------------------------------------------------------
// copy / convert / import / export
// ---------------------------------------------------------------------------
bml_matrix_t *bml_copy_new(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
        return eb_copy_new(static_cast<bml_matrix_ellblock_t *>(A));
    bml_matrix_ellpack_t *E = as_ell(A, "copy_new");
    if (!E)
        return nullptr;
    bml_matrix_ellpack_t *B = ell_alloc(E->matrix_precision, E->N, E->M, E->distribution_mode, false);
    if (!B)
        return nullptr;
    if (!ell_copy(E, B))
    {
        ell_free(B);
        return nullptr;
    }
    return B;
}

void bml_copy(bml_matrix_t *A, bml_matrix_t *B)
{
    if (type_of(A) == ellblock && type_of(B) == ellblock)
    {
        eb_copy(static_cast<bml_matrix_ellblock_t *>(A), static_cast<bml_matrix_ellblock_t *>(B));
        return;
    }
    bml_matrix_ellpack_t *EA = as_ell(A, "copy"), *EB = as_ell(B, "copy");
    if (EA && EB)
        ell_copy(EA, EB);
}

bml_matrix_t *bml_import_from_dense(bml_matrix_type_t matrix_type,
                                    bml_matrix_precision_t matrix_precision,
                                    bml_dense_order_t order, int N, int M, void *A,
                                    double threshold, bml_distribution_mode_t distrib_mode)
{
    if (!A)
    {
        b200_set_error(BML_B200_ERR_INVALID, "import_from_dense: NULL array");
        return nullptr;
    }
    if (matrix_type == ellblock)
        return eb_import_dense(matrix_precision, order, N, M, A, threshold, distrib_mode);
    if (matrix_type != ellpack || !real_prec(matrix_precision))
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "import_from_dense: type %d precision %d",
                       (int) matrix_type, (int) matrix_precision);
        return nullptr;
    }
    bml_matrix_ellpack_t *E = ell_alloc(matrix_precision, N, M, distrib_mode, true);
    if (!E)
        return nullptr;
    ell_import_dense(E, A, order, threshold); // ROW_OVERFLOW keeps the first M per row
    return E;
}

void *bml_export_to_dense(bml_matrix_t *A, bml_dense_order_t order)
{
    if (type_of(A) == ellblock)
        return eb_export_dense(static_cast<bml_matrix_ellblock_t *>(A), order);
    bml_matrix_ellpack_t *E = as_ell(A, "export_to_dense");
    if (!E)
        return nullptr;
    void *D = calloc((size_t) E->N * E->N, prec_size(E->matrix_precision));
    if (!D)
    {
        b200_set_error(BML_B200_ERR_ALLOC, "export_to_dense: %d x %d", E->N, E->N);
        return nullptr;
    }
    if (!ell_export_dense(E, D, order))
    {
        free(D);
        return nullptr;
    }
    return D;
}

bml_matrix_t *bml_convert(bml_matrix_t *A, bml_matrix_type_t matrix_type,
                          bml_matrix_precision_t matrix_precision, int M,
                          bml_distribution_mode_t distrib_mode)
{
    if (!A)
        return nullptr;
    if (type_of(A) == ellpack && matrix_type == ellpack && real_prec(matrix_precision))
    {
        // ELLPACK to ELLPACK: the same entries, each rounded to the new
        // precision, on the device.  (The reference sets every one of the
        // N*N elements, zeros included, through bml_set_element,
        // ellpack/bml_convert_ellpack_typed.c:13-36, which needs M = N.)
        bml_matrix_ellpack_t *E = as_ell(A, "convert");
        if (!E)
            return nullptr;
        bml_matrix_t *B = bml_zero_matrix(ellpack, matrix_precision, E->N, M, distrib_mode);
        if (!B)
            return nullptr;
        if (!ell_convert(E, static_cast<bml_matrix_ellpack_t *>(B)))
        {
            bml_deallocate(&B);
            return nullptr;
        }
        return B;
    }
    // ELLPACK <-> ELLBLOCK on the device, without a dense copy
    if (type_of(A) == ellpack && matrix_type == ellblock && real_prec(matrix_precision))
    {
        bml_matrix_ellpack_t *E = as_ell(A, "convert");
        return E ? eb_from_ellpack(E, matrix_precision, M, distrib_mode) : nullptr;
    }
    if (type_of(A) == ellblock && matrix_type == ellpack && real_prec(matrix_precision))
        return ell_from_ellblock(static_cast<bml_matrix_ellblock_t *>(A), matrix_precision, M, distrib_mode);
    // Other types through a dense copy, as the reference does
    // (bml_convert.c:20-63).
    void *D = bml_export_to_dense(A, dense_row_major);
    if (!D)
        return nullptr;
    bml_matrix_t *B = nullptr;
    if (matrix_precision == prec_of(A))
        B = bml_import_from_dense(matrix_type, matrix_precision, dense_row_major, bml_get_N(A), M, D,
                                  0.0, distrib_mode);
    else
        unsupported(A, "convert between precisions");
    free(D);
    return B;
}

// ---------------------------------------------------------------------------
// norms (bml_norm.h): ELLPACK
// ---------------------------------------------------------------------------
double bml_sum_squares(bml_matrix_t *A)
{
    bml_matrix_ellpack_t *E = as_ell(A, "sum_squares");
    double s = 0.0;
    if (E)
        ell_sum_squares(E, &s);
    return s;
}

double bml_fnorm(bml_matrix_t *A)
{
    return sqrt(bml_sum_squares(A));
}

double bml_fnorm2(bml_matrix_t *A, bml_matrix_t *B)
{
    bml_matrix_ellpack_t *EA = as_ell(A, "fnorm2"), *EB = as_ell(B, "fnorm2");
    double f = 0.0;
    if (EA && EB)
        ell_fnorm2(EA, EB, &f);
    return f;
}

// ---------------------------------------------------------------------------
// elements (on the host mirror; a following device operation re-uploads)
// ---------------------------------------------------------------------------
void *bml_get_element(bml_matrix_t *A, int i, int j)
{
    static double minus_one_d = -1.0, zero_d = 0.0;
    static float minus_one_f = -1.0f, zero_f = 0.0f;
    if (type_of(A) == ellblock)
        return eb_get_element(static_cast<bml_matrix_ellblock_t *>(A), i, j);
    bml_matrix_ellpack_t *E = as_ell(A, "get_element");
    if (!E)
        return nullptr;
    const bool dbl = E->matrix_precision == double_real;
    if (i < 0 || i >= E->N || j < 0 || j >= E->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "get_element: index (%d, %d) out of bounds", i, j);
        return dbl ? (void *) &minus_one_d : (void *) &minus_one_f;
    }
    if (!ell_to_host(E))
        return nullptr;
    for (int p = 0; p < E->nnz[i]; p++)
        if (E->index[(size_t) i * E->M + p] == j)
            return static_cast<char *>(E->value) + ((size_t) i * E->M + p) * prec_size(E->matrix_precision);
    return dbl ? (void *) &zero_d : (void *) &zero_f;
}

void *bml_get_row(bml_matrix_t *A, int i)
{
    if (type_of(A) == ellblock)
        return eb_get_row(static_cast<bml_matrix_ellblock_t *>(A), i);
    bml_matrix_ellpack_t *E = as_ell(A, "get_row");
    if (!E || !ell_to_host(E))
        return nullptr;
    const size_t sz = prec_size(E->matrix_precision);
    char *row = static_cast<char *>(calloc(E->N, sz));
    if (!row || i < 0 || i >= E->N)
        return row;
    for (int p = 0; p < E->nnz[i]; p++)
    {
        const int col = E->index[(size_t) i * E->M + p];
        if (col >= 0 && col < E->N)
            memcpy(row + col * sz, static_cast<char *>(E->value) + ((size_t) i * E->M + p) * sz, sz);
    }
    return row;
}

void *bml_get_diagonal(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
        return eb_get_diagonal(static_cast<bml_matrix_ellblock_t *>(A));
    bml_matrix_ellpack_t *E = as_ell(A, "get_diagonal");
    if (!E || !ell_to_host(E))
        return nullptr;
    const size_t sz = prec_size(E->matrix_precision);
    char *d = static_cast<char *>(calloc(E->N, sz));
    if (!d)
        return nullptr;
    for (int i = 0; i < E->N; i++)
        for (int p = 0; p < E->nnz[i]; p++)
            if (E->index[(size_t) i * E->M + p] == i)
                memcpy(d + i * sz, static_cast<char *>(E->value) + ((size_t) i * E->M + p) * sz, sz);
    return d;
}

// Append (i, j, value) at the end of row i (ellpack/bml_setters_ellpack_typed.c:26-50).
void bml_set_element_new(bml_matrix_t *A, int i, int j, void *value)
{
    if (type_of(A) == ellblock)
    {
        eb_set_element(static_cast<bml_matrix_ellblock_t *>(A), i, j, value, true);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "set_element_new");
    if (!E || !value || !ell_to_host(E))
        return;
    if (i < 0 || i >= E->N || j < 0 || j >= E->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "set_element_new: index (%d, %d) out of bounds", i, j);
        return;
    }
    if (E->nnz[i] >= E->M)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "set_element_new: row %d already holds M=%d entries",
                       i, E->M);
        return;
    }
    const size_t sz = prec_size(E->matrix_precision);
    const size_t at = (size_t) i * E->M + E->nnz[i];
    memcpy(static_cast<char *>(E->value) + at * sz, value, sz);
    E->index[at] = j;
    E->nnz[i]++;
    ell_mark_host(E);
}

// Overwrite (i, j) if present, else append (ellpack/bml_setters_ellpack_typed.c:65-112,
// including its rule that rows with at most two entries are appended to).
void bml_set_element(bml_matrix_t *A, int i, int j, void *value)
{
    if (type_of(A) == ellblock)
    {
        eb_set_element(static_cast<bml_matrix_ellblock_t *>(A), i, j, value, false);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "set_element");
    if (!E || !value || !ell_to_host(E))
        return;
    if (i < 0 || i >= E->N || j < 0 || j >= E->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "set_element: index (%d, %d) out of bounds", i, j);
        return;
    }
    const size_t sz = prec_size(E->matrix_precision);
    if (E->nnz[i] > 2)
        for (int p = 0; p < E->nnz[i]; p++)
            if (E->index[(size_t) i * E->M + p] == j)
            {
                memcpy(static_cast<char *>(E->value) + ((size_t) i * E->M + p) * sz, value, sz);
                ell_mark_host(E);
                return;
            }
    bml_set_element_new(A, i, j, value);
}

// Row i <- the entries of the dense row above threshold
// (ellpack/bml_setters_ellpack_typed.c:126-160).
void bml_set_row(bml_matrix_t *A, int i, void *row, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_set_row(static_cast<bml_matrix_ellblock_t *>(A), i, row, threshold);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "set_row");
    if (!E || !row || !ell_to_host(E) || i < 0 || i >= E->N)
        return;
    const bool dbl = E->matrix_precision == double_real;
    int ll = 0;
    for (int j = 0; j < E->N; j++)
    {
        const double v = dbl ? static_cast<double *>(row)[j] : static_cast<float *>(row)[j];
        if (fabs(v) > threshold)
        {
            if (ll >= E->M)
            {
                b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "set_row: more than M entries");
                break;
            }
            if (dbl)
                static_cast<double *>(E->value)[(size_t) i * E->M + ll] = static_cast<double *>(row)[j];
            else
                static_cast<float *>(E->value)[(size_t) i * E->M + ll] = static_cast<float *>(row)[j];
            E->index[(size_t) i * E->M + ll] = j;
            ll++;
        }
    }
    E->nnz[i] = ll;
    ell_mark_host(E);
}

// Diagonal <- diagonal[i] where above threshold (else 0 if present, nothing
// if absent), as ellpack/bml_setters_ellpack_typed.c:175-225.
void bml_set_diagonal(bml_matrix_t *A, void *diagonal, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_set_diagonal(static_cast<bml_matrix_ellblock_t *>(A), diagonal, threshold);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "set_diagonal");
    if (!E || !diagonal || !ell_to_host(E))
        return;
    const bool dbl = E->matrix_precision == double_real;
    for (int i = 0; i < E->N; i++)
    {
        const double d = dbl ? static_cast<double *>(diagonal)[i] : static_cast<float *>(diagonal)[i];
        int found = 0;
        for (int p = 0; p < E->nnz[i]; p++)
            if (E->index[(size_t) i * E->M + p] == i)
            {
                const bool keep = fabs(d) > threshold;
                if (dbl)
                    static_cast<double *>(E->value)[(size_t) i * E->M + p] = keep ? d : 0.0;
                else
                    static_cast<float *>(E->value)[(size_t) i * E->M + p] =
                        keep ? static_cast<float *>(diagonal)[i] : 0.0f;
                found = 1;
            }
        if (!found && fabs(d) > threshold && E->nnz[i] < E->M)
        {
            const size_t at = (size_t) i * E->M + E->nnz[i];
            if (dbl)
                static_cast<double *>(E->value)[at] = d;
            else
                static_cast<float *>(E->value)[at] = static_cast<float *>(diagonal)[i];
            E->index[at] = i;
            E->nnz[i]++;
        }
    }
    ell_mark_host(E);
}

// ---------------------------------------------------------------------------
// the thresholded sparse path
// ---------------------------------------------------------------------------
int bml_b200_multiply_x2(bml_matrix_t *X, bml_matrix_t *X2, double threshold, double *trace)
{
    if (type_of(X) == ellblock && type_of(X2) == ellblock)
    {
        bool ok = eb_multiply_x2(static_cast<bml_matrix_ellblock_t *>(X),
                                 static_cast<bml_matrix_ellblock_t *>(X2), threshold, trace);
        return ok ? BML_B200_OK : b200_get_error();
    }
    bml_matrix_ellpack_t *EX = as_ell(X, "multiply_x2"), *E2 = as_ell(X2, "multiply_x2");
    if (!EX || !E2)
        return b200_get_error();
    double tr[2] = {0.0, 0.0};
    const bool ok = ell_multiply_AB(EX, EX, E2, threshold, tr, &g_required_M);
    if (trace)
    {
        trace[0] = tr[0];
        trace[1] = tr[1];
    }
    return ok ? BML_B200_OK : b200_get_error();
}

int bml_b200_last_required_M(void) { return g_required_M; }

// Rows [r0, r1) of X^2 (row-sharded SP2): the other rows of X2 are left as
// they are; the traces are those rows' partial sums.
int bml_b200_multiply_x2_rows(bml_matrix_t *X, bml_matrix_t *X2, double threshold, int r0, int r1,
                              double *trace)
{
    bml_matrix_ellpack_t *EX = as_ell(X, "multiply_x2_rows"), *E2 = as_ell(X2, "multiply_x2_rows");
    if (!EX || !E2)
        return b200_get_error();
    if (EX == E2 || EX->N != E2->N || r0 < 0 || r1 > EX->N || r0 >= r1)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply_x2_rows: rows [%d, %d) of N=%d", r0, r1, EX->N);
        return BML_B200_ERR_INVALID;
    }
    if (!ell_to_device(EX) || !ell_to_device(E2))
        return b200_get_error();
    bml_matrix_ellpack_t A = ell_row_view(EX, r0, r1), C = ell_row_view(E2, r0, r1);
    double tr[2] = {0.0, 0.0};
    const bool ok = ell_multiply_AB(&A, EX, &C, threshold, tr, &g_required_M, 1);
    ell_mark_device(E2);
    if (trace)
    {
        trace[0] = tr[0];
        trace[1] = tr[1];
    }
    return ok ? BML_B200_OK : b200_get_error();
}

// SP2 update of rows [r0, r1): X <- X2 (branch 0) or X <- 2X - X2 (branch 1,
// thresholded as bml_add).
int bml_b200_sp2_update_rows(bml_matrix_t *X, bml_matrix_t *X2, double threshold, int branch, int r0, int r1)
{
    bml_matrix_ellpack_t *EX = as_ell(X, "sp2_update_rows"), *E2 = as_ell(X2, "sp2_update_rows");
    if (!EX || !E2)
        return b200_get_error();
    if (EX == E2 || EX->N != E2->N || r0 < 0 || r1 > EX->N || r0 >= r1 || (branch != 0 && branch != 1))
    {
        b200_set_error(BML_B200_ERR_INVALID, "sp2_update_rows: rows [%d, %d) of N=%d, branch %d", r0, r1,
                       EX->N, branch);
        return BML_B200_ERR_INVALID;
    }
    if (!ell_to_device(EX) || !ell_to_device(E2))
        return b200_get_error();
    bml_b200_clear_error();
    bml_matrix_ellpack_t A = ell_row_view(EX, r0, r1), B = ell_row_view(E2, r0, r1);
    const bool ok = branch == 0 ? ell_copy(&B, &A) : ell_add(&A, &B, 2.0, -1.0, threshold);
    ell_mark_device(EX);
    return ok ? BML_B200_OK : b200_get_error();
}

void *bml_multiply_x2(bml_matrix_t *X, bml_matrix_t *X2, double threshold)
{
    double *trace = static_cast<double *>(bml_allocate_memory(2 * sizeof(double)));
    if (!trace)
        return nullptr;
    bml_b200_multiply_x2(X, X2, threshold, trace);
    return trace;
}

void bml_multiply_AB(bml_matrix_t *A, bml_matrix_t *B, bml_matrix_t *C, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_multiply_AB(static_cast<bml_matrix_ellblock_t *>(A), static_cast<bml_matrix_ellblock_t *>(B),
                       static_cast<bml_matrix_ellblock_t *>(C), threshold);
        return;
    }
    bml_matrix_ellpack_t *EA = as_ell(A, "multiply_AB"), *EB = as_ell(B, "multiply_AB"),
                         *EC = as_ell(C, "multiply_AB");
    if (EA && EB && EC)
        ell_multiply_AB(EA, EB, EC, threshold, nullptr, &g_required_M);
}

// The reference doubles the threshold while any pre-threshold row is wider
// than M, a condition the threshold cannot change (its loop then never ends,
// ellpack/bml_multiply_ellpack_typed.c:566-707); here the threshold doubles
// while a thresholded row is wider than M, at most 64 times.
void bml_multiply_adjust_AB(bml_matrix_t *A, bml_matrix_t *B, bml_matrix_t *C, double threshold)
{
    bml_matrix_ellpack_t *EA = as_ell(A, "multiply_adjust_AB"), *EB = as_ell(B, "multiply_adjust_AB"),
                         *EC = as_ell(C, "multiply_adjust_AB");
    if (!EA || !EB || !EC)
        return;
    double t = threshold;
    for (int it = 0; it < 64; ++it)
    {
        bml_b200_set_verbose(0);
        const bool ok = ell_multiply_AB(EA, EB, EC, t, nullptr, &g_required_M);
        bml_b200_set_verbose(1);
        if (ok || b200_get_error() != BML_B200_ERR_ROW_OVERFLOW)
            return;
        bml_b200_clear_error();
        t = t > 0.0 ? 2.0 * t : 1e-300;
    }
    b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "multiply_adjust_AB: no threshold fits M=%d", EC->M);
}

// C <- alpha*A*B + beta*C (bml_multiply.c:27-59 -> ellpack/bml_multiply_ellpack_typed.c:55-118):
// X^2 straight into C when A == B, alpha == 1, beta == 0; otherwise the
// product into a temporary with C's dimensions, then C <- beta*C + alpha*T.
void bml_multiply(bml_matrix_t *A, bml_matrix_t *B, bml_matrix_t *C, double alpha, double beta,
                  double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_multiply(static_cast<bml_matrix_ellblock_t *>(A), static_cast<bml_matrix_ellblock_t *>(B),
                    static_cast<bml_matrix_ellblock_t *>(C), alpha, beta, threshold);
        return;
    }
    bml_matrix_ellpack_t *EA = as_ell(A, "multiply"), *EB = as_ell(B, "multiply"),
                         *EC = as_ell(C, "multiply");
    if (!EA || !EB || !EC)
        return;
    double tr[2];
    if (A == B && alpha == 1.0 && beta == 0.0)
    {
        ell_multiply_AB(EA, EA, EC, threshold, tr, &g_required_M);
        return;
    }
    bml_matrix_ellpack_t *T = ell_alloc(EC->matrix_precision, EC->N, EC->M, EC->distribution_mode, false);
    if (!T)
        return;
    bool ok = A == B ? ell_multiply_AB(EA, EA, T, threshold, tr, &g_required_M)
                     : ell_multiply_AB(EA, EB, T, threshold, nullptr, &g_required_M);
    if (ok)
        ell_add(EC, T, beta, alpha, threshold);
    ell_free(T);
}

void bml_add(bml_matrix_t *A, bml_matrix_t *B, double alpha, double beta, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_add(static_cast<bml_matrix_ellblock_t *>(A), static_cast<bml_matrix_ellblock_t *>(B), alpha,
               beta, threshold);
        return;
    }
    bml_matrix_ellpack_t *EA = as_ell(A, "add"), *EB = as_ell(B, "add");
    if (EA && EB)
        ell_add(EA, EB, alpha, beta, threshold);
}

void bml_add_identity(bml_matrix_t *A, double beta, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_add_identity(static_cast<bml_matrix_ellblock_t *>(A), beta, threshold);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "add_identity");
    if (E)
        ell_add_identity(E, beta, threshold);
}

void bml_scale_inplace(void *scale_factor, bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
    {
        eb_scale(scale_factor, static_cast<bml_matrix_ellblock_t *>(A),
                 static_cast<bml_matrix_ellblock_t *>(A));
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "scale_inplace");
    if (E && scale_factor)
        ell_scale(scale_factor, E, E);
}

void bml_scale(void *scale_factor, bml_matrix_t *A, bml_matrix_t *B)
{
    if (type_of(A) == ellblock)
    {
        eb_scale(scale_factor, static_cast<bml_matrix_ellblock_t *>(A),
                 static_cast<bml_matrix_ellblock_t *>(B));
        return;
    }
    bml_matrix_ellpack_t *EA = as_ell(A, "scale"), *EB = as_ell(B, "scale");
    if (EA && EB && scale_factor)
        ell_scale(scale_factor, EA, EB);
}

bml_matrix_t *bml_scale_new(void *scale_factor, bml_matrix_t *A)
{
    bml_matrix_t *B = bml_copy_new(A);
    if (B)
        bml_scale_inplace(scale_factor, B);
    return B;
}

// A <- alpha*A + beta*I: scale then add_identity (bml_add_ellpack_typed.c:562-573).
// The scale factor is converted to the matrix precision, as the reference's
// bml_scale_inplace_ellpack receives &alpha reinterpreted by precision.
void bml_scale_add_identity(bml_matrix_t *A, double alpha, double beta, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_scale_add_identity(static_cast<bml_matrix_ellblock_t *>(A), alpha, beta, threshold);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "scale_add_identity");
    if (!E)
        return;
    float af = (float) alpha;
    if (!ell_scale(E->matrix_precision == double_real ? (void *) &alpha : (void *) &af, E, E))
        return;
    ell_add_identity(E, beta, threshold);
}

bml_matrix_t *bml_threshold_new(bml_matrix_t *A, double threshold)
{
    if (type_of(A) == ellblock)
        return eb_threshold_new(static_cast<bml_matrix_ellblock_t *>(A), threshold);
    bml_matrix_ellpack_t *E = as_ell(A, "threshold_new");
    if (!E)
        return nullptr;
    bml_matrix_ellpack_t *B = ell_alloc(E->matrix_precision, E->N, E->M, E->distribution_mode, true);
    if (!B)
        return nullptr;
    if (!ell_threshold_new(E, B, threshold))
    {
        ell_free(B);
        return nullptr;
    }
    return B;
}

void bml_threshold(bml_matrix_t *A, double threshold)
{
    if (type_of(A) == ellblock)
    {
        eb_threshold(static_cast<bml_matrix_ellblock_t *>(A), threshold);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "threshold");
    if (E)
        ell_threshold(E, threshold);
}

double bml_trace(bml_matrix_t *A)
{
    double t = 0.0;
    if (type_of(A) == ellblock)
    {
        eb_trace(static_cast<bml_matrix_ellblock_t *>(A), &t);
        return t;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "trace");
    if (E)
        ell_trace(E, &t);
    return t;
}

double bml_trace_mult(bml_matrix_t *A, bml_matrix_t *B)
{
    double t = 0.0;
    if (type_of(A) == ellblock)
    {
        eb_trace_mult(static_cast<bml_matrix_ellblock_t *>(A), static_cast<bml_matrix_ellblock_t *>(B),
                      &t);
        return t;
    }
    bml_matrix_ellpack_t *EA = as_ell(A, "trace_mult"), *EB = as_ell(B, "trace_mult");
    if (EA && EB)
    {
        if (EA->M != EB->M)
        {
            b200_set_error(BML_B200_ERR_INVALID,
                           "bml_trace_mult_ellpack: Matrices A and B have different sizes.");
            return 0.0;
        }
        ell_trace_mult(EA, EB, &t);
    }
    return t;
}

bml_matrix_t *bml_transpose_new(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
        return eb_transpose_new(static_cast<bml_matrix_ellblock_t *>(A));
    bml_matrix_ellpack_t *E = as_ell(A, "transpose_new");
    if (!E)
        return nullptr;
    bml_matrix_ellpack_t *B = ell_alloc(E->matrix_precision, E->N, E->M, E->distribution_mode, false);
    if (!B)
        return nullptr;
    if (!ell_transpose_new(E, B))
    {
        ell_free(B);
        return nullptr;
    }
    return B;
}

// In place through a device temporary.  The reference's sequential
// left-looking swap (ellpack/bml_transpose_ellpack_typed.c:172-284) leaves
// rows in a swap-determined order; here each row is in ascending source row.
void bml_transpose(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
    {
        eb_transpose(static_cast<bml_matrix_ellblock_t *>(A));
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "transpose");
    if (!E)
        return;
    bml_matrix_ellpack_t *B = ell_alloc(E->matrix_precision, E->N, E->M, E->distribution_mode, false);
    if (!B)
        return;
    if (ell_transpose_new(E, B))
        ell_copy(B, E);
    ell_free(B);
}

void *bml_gershgorin(bml_matrix_t *A)
{
    double *eval = static_cast<double *>(bml_allocate_memory(2 * sizeof(double)));
    if (!eval)
        return nullptr;
    if (type_of(A) == ellblock)
    {
        eb_gershgorin(static_cast<bml_matrix_ellblock_t *>(A), eval);
        return eval;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "gershgorin");
    if (E)
        ell_gershgorin(E, eval);
    return eval;
}

// (emax*I - A)/(emax - emin): scale by (precision)(-1/(emax-emin)), then add
// emax/(emax-emin) on the diagonal with threshold 0
// (ellpack/bml_normalize_ellpack_typed.c:32-45).
void bml_normalize(bml_matrix_t *A, double mineval, double maxeval)
{
    const double maxminusmin = maxeval - mineval;
    const double gershfact = maxeval / maxminusmin;
    if (type_of(A) == ellblock)
    {
        eb_normalize(static_cast<bml_matrix_ellblock_t *>(A), mineval, maxeval);
        return;
    }
    bml_matrix_ellpack_t *E = as_ell(A, "normalize");
    if (!E)
        return;
    double sd = -1.0 / maxminusmin;
    float sf = (float) (-1.0 / maxminusmin);
    if (!ell_scale(E->matrix_precision == double_real ? (void *) &sd : (void *) &sf, E, E))
        return;
    ell_add_identity(E, gershfact, 0.0);
}

// ---------------------------------------------------------------------------
// printing and Matrix Market I/O (host side)
// ---------------------------------------------------------------------------
void bml_print_dense_matrix(int N, bml_matrix_precision_t matrix_precision, bml_dense_order_t order,
                            void *A, int i_l, int i_u, int j_l, int j_u)
{
    if (!A)
        return;
    for (int i = i_l; i < i_u; i++)
    {
        for (int j = j_l; j < j_u; j++)
        {
            const size_t at = order == dense_row_major ? (size_t) i * N + j : (size_t) j * N + i;
            if (matrix_precision == double_real)
                print_value(static_cast<double *>(A)[at]);
            else if (matrix_precision == single_real)
                print_value(static_cast<float *>(A)[at]);
        }
        printf("\n");
    }
}

void bml_print_bml_matrix(bml_matrix_t *A, int i_l, int i_u, int j_l, int j_u)
{
    void *D = bml_export_to_dense(A, dense_row_major);
    if (!D)
        return;
    bml_print_dense_matrix(bml_get_N(A), prec_of(A), dense_row_major, D, i_l, i_u, j_l, j_u);
    free(D);
}

int bml_sqrtint(const int x)
{
    int r = (int) sqrt((double) x);
    while (r * r > x)
        r--;
    while ((r + 1) * (r + 1) <= x)
        r++;
    return r;
}

// Matrix Market coordinate files, 1-based, in the reference's formats
// (bml_utilities.c:496-540 dispatch; ellpack/bml_utilities_ellpack_typed.c:
// 22-203, ellblock/bml_utilities_ellblock_typed.c:25-256).  Both formats
// write the header "%%%MatrixMarket matrix coordinate real general" and
// "N N nnz"; ELLPACK writes each stored entry as "%d %d %20.15lg" (FP32:
// "%20.15g"), ELLBLOCK every element of every stored block as
// "%d %d %20.15e".  Reading appends to the matrix it is given (entries
// already there are kept); a "symmetric" header mirrors off-diagonal entries.
void bml_write_bml_matrix(bml_matrix_t *A, char *filename)
{
    if (!A || !filename)
    {
        b200_set_error(BML_B200_ERR_INVALID, "write_bml_matrix: NULL argument");
        return;
    }
    const bml_matrix_type_t t = type_of(A);
    if (t != ellpack && t != ellblock)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "write_bml_matrix: matrix type %d", (int) t);
        return;
    }
    if (t == ellpack && !ell_to_host(static_cast<bml_matrix_ellpack_t *>(A)))
        return;
    FILE *f = fopen(filename, "w");
    if (!f)
    {
        b200_set_error(BML_B200_ERR_INVALID, "write_bml_matrix: cannot open %s", filename);
        return;
    }
    if (t == ellblock)
    {
        eb_write_mm(static_cast<bml_matrix_ellblock_t *>(A), f);
        fclose(f);
        return;
    }
    bml_matrix_ellpack_t *E = static_cast<bml_matrix_ellpack_t *>(A);
    long long nnz = 0;
    for (int i = 0; i < E->N; i++)
        nnz += E->nnz[i];
    fprintf(f, "%%%%%%MatrixMarket matrix coordinate real general\n");
    fprintf(f, "%d %d %lld\n", E->N, E->N, nnz);
    for (int i = 0; i < E->N; i++)
        for (int p = 0; p < E->nnz[i]; p++)
        {
            const size_t at = (size_t) i * E->M + p;
            if (E->matrix_precision == double_real)
                fprintf(f, "%d %d %20.15lg\n", i + 1, E->index[at] + 1, static_cast<double *>(E->value)[at]);
            else
                fprintf(f, "%d %d %20.15g\n", i + 1, E->index[at] + 1, (double) static_cast<float *>(E->value)[at]);
        }
    fclose(f);
}

} // extern "C"

namespace {

// Header: five words, the fifth "symmetric" or not (the reference reads them
// with "%s %s %s %s %s"), then "rows cols entries" after any comment lines.
bool read_mm_header(FILE *f, const char *filename, int *n, long long *ne, bool *symmetric)
{
    char w[5][64];
    if (fscanf(f, "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) != 5)
    {
        b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: %s: read error on header", filename);
        return false;
    }
    *symmetric = strcmp(w[4], "symmetric") == 0;
    int c;
    while ((c = fgetc(f)) != EOF)
    {
        if (c == '%')
        {
            while ((c = fgetc(f)) != EOF && c != '\n')
                ;
            continue;
        }
        if (c != ' ' && c != '\t' && c != '\n' && c != '\r')
        {
            ungetc(c, f);
            break;
        }
    }
    int nc = 0;
    if (fscanf(f, "%d %d %lld", n, &nc, ne) != 3 || *ne < 0)
    {
        b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: %s: read error on the size line", filename);
        return false;
    }
    return true;
}

template <typename T> bool ell_read_mm(bml_matrix_ellpack_t *E, FILE *f, long long ne, bool symmetric)
{
    T *val = static_cast<T *>(E->value);
    auto put = [&](int i, int j, T v) {
        if (E->nnz[i] >= E->M)
        {
            b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "read_bml_matrix: row %d needs more than M=%d entries",
                           i + 1, E->M);
            return false;
        }
        const size_t at = (size_t) i * E->M + E->nnz[i];
        E->index[at] = j;
        val[at] = v;
        E->nnz[i]++;
        return true;
    };
    for (long long e = 0; e < ne; e++)
    {
        int i, j;
        T v;
        const int got = sizeof(T) == 8 ? fscanf(f, "%d %d %lf", &i, &j, reinterpret_cast<double *>(&v))
                                       : fscanf(f, "%d %d %f", &i, &j, reinterpret_cast<float *>(&v));
        if (got != 3)
        {
            b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: entry %lld of %lld unreadable", e + 1, ne);
            return false;
        }
        i--;
        j--;
        if (i < 0 || j < 0 || i >= E->N || j >= E->N)
        {
            b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: entry (%d, %d) outside N=%d", i + 1, j + 1, E->N);
            return false;
        }
        if (!put(i, j, v) || (symmetric && j != i && !put(j, i, v)))
            return false;
    }
    return true;
}

} // namespace

extern "C" {

void bml_read_bml_matrix(bml_matrix_t *A, char *filename)
{
    if (!A || !filename)
    {
        b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: NULL argument");
        return;
    }
    const bml_matrix_type_t t = type_of(A);
    if (t != ellpack && t != ellblock)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "read_bml_matrix: matrix type %d", (int) t);
        return;
    }
    FILE *f = fopen(filename, "r");
    if (!f)
    {
        b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: cannot open %s", filename);
        return;
    }
    int n = 0;
    long long ne = 0;
    bool symmetric = false;
    if (read_mm_header(f, filename, &n, &ne, &symmetric))
    {
        if (n != bml_get_N(A))
            b200_set_error(BML_B200_ERR_INVALID, "read_bml_matrix: %s holds N=%d, the matrix has N=%d", filename, n,
                           bml_get_N(A));
        else if (t == ellblock)
            eb_read_mm(static_cast<bml_matrix_ellblock_t *>(A), f, ne, symmetric);
        else
        {
            bml_matrix_ellpack_t *E = static_cast<bml_matrix_ellpack_t *>(A);
            if (ell_to_host(E))
            {
                if (E->matrix_precision == double_real)
                    ell_read_mm<double>(E, f, ne, symmetric);
                else
                    ell_read_mm<float>(E, f, ne, symmetric);
                ell_mark_host(E);
            }
        }
    }
    fclose(f);
}

// ---------------------------------------------------------------------------
// raw array transfer
// ---------------------------------------------------------------------------
int bml_b200_ellpack_upload(bml_matrix_t *A, const void *value, const int *index, const int *nnz)
{
    bml_matrix_ellpack_t *E = as_ell(A, "ellpack_upload");
    if (!E)
        return b200_get_error();
    if (!value || !index || !nnz)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ellpack_upload: NULL array");
        return BML_B200_ERR_INVALID;
    }
    const size_t sz = prec_size(E->matrix_precision);
    // Only the columns up to the widest row travel (entries past a row's nnz
    // are never read).
    int w = 0;
    for (int i = 0; i < E->N; ++i)
    {
        if (nnz[i] < 0 || nnz[i] > E->M)
        {
            b200_set_error(BML_B200_ERR_INVALID, "ellpack_upload: nnz[%d] = %d outside [0, M=%d]", i, nnz[i],
                           E->M);
            return BML_B200_ERR_INVALID;
        }
        w = nnz[i] > w ? nnz[i] : w;
    }
    // Write straight to the device; the host mirror becomes stale.
    B200Context *c = b200_ctx();
    if (!c)
        return b200_get_error();
    if ((w > 0 && (!CUDA_OK(cudaMemcpy2DAsync(E->d_value, E->ld * sz, value, E->M * sz, w * sz, E->N,
                                              cudaMemcpyHostToDevice, c->stream)) ||
                   !CUDA_OK(cudaMemcpy2DAsync(E->d_index, E->ld * sizeof(int), index, E->M * sizeof(int),
                                              w * sizeof(int), E->N, cudaMemcpyHostToDevice, c->stream)))) ||
        !CUDA_OK(cudaMemcpyAsync(E->d_nnz, nnz, (size_t) E->N * sizeof(int), cudaMemcpyHostToDevice,
                                 c->stream)) ||
        !b200_sync())
        return b200_get_error();
    ell_mark_device(E);
    return BML_B200_OK;
}

int bml_b200_ellpack_download(bml_matrix_t *A, void *value, int *index, int *nnz)
{
    bml_matrix_ellpack_t *E = as_ell(A, "ellpack_download");
    if (!E)
        return b200_get_error();
    if (!value || !index || !nnz)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ellpack_download: NULL array");
        return BML_B200_ERR_INVALID;
    }
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(E))
        return b200_get_error();
    const size_t sz = prec_size(E->matrix_precision);
    // Row lengths first; then only the columns up to the widest row travel
    // (entries past a row's nnz are left as the caller had them).
    if (!CUDA_OK(cudaMemcpyAsync(nnz, E->d_nnz, (size_t) E->N * sizeof(int), cudaMemcpyDeviceToHost,
                                 c->stream)) ||
        !b200_sync())
        return b200_get_error();
    int w = 0;
    for (int i = 0; i < E->N; ++i)
        w = nnz[i] > w ? nnz[i] : w;
    w = w < E->M ? w : E->M;
    if (w > 0 &&
        (!CUDA_OK(cudaMemcpy2DAsync(value, E->M * sz, E->d_value, E->ld * sz, w * sz, E->N,
                                    cudaMemcpyDeviceToHost, c->stream)) ||
         !CUDA_OK(cudaMemcpy2DAsync(index, E->M * sizeof(int), E->d_index, E->ld * sizeof(int),
                                    w * sizeof(int), E->N, cudaMemcpyDeviceToHost, c->stream)) ||
         !b200_sync()))
        return b200_get_error();
    return BML_B200_OK;
}

int bml_b200_ellpack_device_arrays(bml_matrix_t *A, void **d_value, int **d_index, int **d_nnz,
                                   int *ld)
{
    bml_matrix_ellpack_t *E = as_ell(A, "ellpack_device_arrays");
    if (!E || !ell_to_device(E))
        return b200_get_error();
    if (d_value)
        *d_value = E->d_value;
    if (d_index)
        *d_index = E->d_index;
    if (d_nnz)
        *d_nnz = E->d_nnz;
    if (ld)
        *ld = E->ld;
    // The caller may use these arrays on any stream: finish the library's
    // queued work on them (and their stream-ordered allocation) first.
    if (!b200_sync())
        return b200_get_error();
    // The caller may write through these pointers: treat the device as newer.
    ell_mark_device(E);
    return BML_B200_OK;
}

long long bml_b200_nnz(bml_matrix_t *A)
{
    if (type_of(A) == ellblock)
        return eb_nnz(static_cast<bml_matrix_ellblock_t *>(A));
    bml_matrix_ellpack_t *E = as_ell(A, "nnz");
    long long tot = -1;
    int maxrow = 0;
    if (!E || !ell_nnz_total(E, &tot, &maxrow))
        return -1;
    return tot;
}

} // extern "C"
