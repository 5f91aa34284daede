// Temporary ELLBLOCK entry points: every call reports UNSUPPORTED until the
// block kernels land.
#include "ellblock.h"

static bool eb_unsupported(const char *op)
{
    b200_set_error(BML_B200_ERR_UNSUPPORTED, "ELLBLOCK %s", op);
    return false;
}

bml_matrix_ellblock_t * eb_constructor(int kind, bml_matrix_precision_t prec, int N, int M,
                                      bml_distribution_mode_t mode)
{
    eb_unsupported("eb_constructor"); return nullptr;
}

bml_matrix_ellblock_t * eb_alloc_blocks(bml_matrix_precision_t prec, int NB, int MB, int M,
                                       const int *bsize, bml_distribution_mode_t mode)
{
    eb_unsupported("eb_alloc_blocks"); return nullptr;
}

void eb_free(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_free");
}

void eb_clear(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_clear");
}

bool eb_to_device(bml_matrix_ellblock_t *A)
{
    return eb_unsupported("eb_to_device");
}

bool eb_to_host(bml_matrix_ellblock_t *A)
{
    return eb_unsupported("eb_to_host");
}

int eb_row_bandwidth(bml_matrix_ellblock_t *A, int i)
{
    eb_unsupported("eb_row_bandwidth"); return -1;
}

int eb_bandwidth(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_bandwidth"); return -1;
}

double eb_sparsity(bml_matrix_ellblock_t *A, double threshold)
{
    eb_unsupported("eb_sparsity"); return -1.0;
}

long long eb_nnz(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_nnz"); return -1;
}

bml_matrix_ellblock_t * eb_copy_new(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_copy_new"); return nullptr;
}

bool eb_copy(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B)
{
    return eb_unsupported("eb_copy");
}

bml_matrix_ellblock_t * eb_import_dense(bml_matrix_precision_t prec, bml_dense_order_t order, int N,
                                       int M, void *A, double threshold,
                                       bml_distribution_mode_t mode)
{
    eb_unsupported("eb_import_dense"); return nullptr;
}

void * eb_export_dense(bml_matrix_ellblock_t *A, bml_dense_order_t order)
{
    eb_unsupported("eb_export_dense"); return nullptr;
}

void * eb_get_element(bml_matrix_ellblock_t *A, int i, int j)
{
    eb_unsupported("eb_get_element"); return nullptr;
}

void * eb_get_row(bml_matrix_ellblock_t *A, int i)
{
    eb_unsupported("eb_get_row"); return nullptr;
}

void * eb_get_diagonal(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_get_diagonal"); return nullptr;
}

void eb_set_element(bml_matrix_ellblock_t *A, int i, int j, const void *value, bool append_new)
{
    eb_unsupported("eb_set_element");
}

bool eb_multiply_x2(bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, double threshold,
                    double *trace)
{
    return eb_unsupported("eb_multiply_x2");
}

bool eb_multiply_AB(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C,
                    double threshold)
{
    return eb_unsupported("eb_multiply_AB");
}

bool eb_multiply(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C,
                 double alpha, double beta, double threshold)
{
    return eb_unsupported("eb_multiply");
}

bool eb_add(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, double alpha, double beta,
            double threshold)
{
    return eb_unsupported("eb_add");
}

bool eb_add_identity(bml_matrix_ellblock_t *A, double beta, double threshold)
{
    return eb_unsupported("eb_add_identity");
}

bool eb_scale_add_identity(bml_matrix_ellblock_t *A, double alpha, double beta, double threshold)
{
    return eb_unsupported("eb_scale_add_identity");
}

bool eb_scale(const void *scale, bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B)
{
    return eb_unsupported("eb_scale");
}

bml_matrix_ellblock_t * eb_threshold_new(bml_matrix_ellblock_t *A, double threshold)
{
    eb_unsupported("eb_threshold_new"); return nullptr;
}

bool eb_threshold(bml_matrix_ellblock_t *A, double threshold)
{
    return eb_unsupported("eb_threshold");
}

bool eb_trace(bml_matrix_ellblock_t *A, double *trace)
{
    return eb_unsupported("eb_trace");
}

bool eb_trace_mult(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, double *trace)
{
    return eb_unsupported("eb_trace_mult");
}

bml_matrix_ellblock_t * eb_transpose_new(bml_matrix_ellblock_t *A)
{
    eb_unsupported("eb_transpose_new"); return nullptr;
}

bool eb_transpose(bml_matrix_ellblock_t *A)
{
    return eb_unsupported("eb_transpose");
}

bool eb_gershgorin(bml_matrix_ellblock_t *A, double *bounds)
{
    return eb_unsupported("eb_gershgorin");
}

bool eb_normalize(bml_matrix_ellblock_t *A, double mineval, double maxeval)
{
    return eb_unsupported("eb_normalize");
}

