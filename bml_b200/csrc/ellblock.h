// ELLBLOCK operations (ellblock.cu / ellblock_mma.cu).
#pragma once

#include "internal.h"

bml_matrix_ellblock_t *eb_constructor(int kind, bml_matrix_precision_t prec, int N, int M,
                                      bml_distribution_mode_t mode);
bml_matrix_ellblock_t *eb_alloc_blocks(bml_matrix_precision_t prec, int NB, int MB, int M,
                                       const int *bsize, bml_distribution_mode_t mode);
void eb_free(bml_matrix_ellblock_t *A);
void eb_clear(bml_matrix_ellblock_t *A);
bool eb_to_device(bml_matrix_ellblock_t *A);
bool eb_to_host(bml_matrix_ellblock_t *A);
int eb_row_bandwidth(bml_matrix_ellblock_t *A, int i);
int eb_bandwidth(bml_matrix_ellblock_t *A);
double eb_sparsity(bml_matrix_ellblock_t *A, double threshold);
long long eb_nnz(bml_matrix_ellblock_t *A);
bml_matrix_ellblock_t *eb_copy_new(bml_matrix_ellblock_t *A);
bool eb_copy(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B);
bml_matrix_ellblock_t *eb_import_dense(bml_matrix_precision_t prec, bml_dense_order_t order, int N,
                                       int M, void *A, double threshold,
                                       bml_distribution_mode_t mode);
void *eb_export_dense(bml_matrix_ellblock_t *A, bml_dense_order_t order);
void *eb_get_element(bml_matrix_ellblock_t *A, int i, int j);
void *eb_get_row(bml_matrix_ellblock_t *A, int i);
void *eb_get_diagonal(bml_matrix_ellblock_t *A);
void eb_set_element(bml_matrix_ellblock_t *A, int i, int j, const void *value, bool append_new);
// Conversions between the formats on the device (values rounded to `prec`).
bml_matrix_ellblock_t *eb_from_ellpack(bml_matrix_ellpack_t *E, bml_matrix_precision_t prec, int M,
                                       bml_distribution_mode_t mode);
bml_matrix_ellpack_t *ell_from_ellblock(bml_matrix_ellblock_t *A, bml_matrix_precision_t prec, int M,
                                        bml_distribution_mode_t mode);
void eb_set_row(bml_matrix_ellblock_t *A, int i, const void *row, double threshold);
void eb_set_diagonal(bml_matrix_ellblock_t *A, const void *diagonal, double threshold);
// Matrix Market coordinate I/O on the host mirror (the header is handled by the caller).
bool eb_write_mm(bml_matrix_ellblock_t *A, FILE *f);
bool eb_read_mm(bml_matrix_ellblock_t *A, FILE *f, long long ne, bool symmetric);
// X2 = X*X on the tensor cores: FP16 hi/lo split, FP32 accumulation; blocks of 32.
bool eb_multiply_x2_tc(bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, double threshold, double *trace);
bool eb_multiply_x2(bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, double threshold,
                    double *trace);
bool eb_multiply_AB(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C,
                    double threshold);
bool eb_multiply(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, bml_matrix_ellblock_t *C,
                 double alpha, double beta, double threshold);
bool eb_add(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, double alpha, double beta,
            double threshold);
bool eb_add_identity(bml_matrix_ellblock_t *A, double beta, double threshold);
bool eb_scale_add_identity(bml_matrix_ellblock_t *A, double alpha, double beta, double threshold);
bool eb_scale(const void *scale, bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B);
bml_matrix_ellblock_t *eb_threshold_new(bml_matrix_ellblock_t *A, double threshold);
bool eb_threshold(bml_matrix_ellblock_t *A, double threshold);
bool eb_trace(bml_matrix_ellblock_t *A, double *trace);
bool eb_trace_mult(bml_matrix_ellblock_t *A, bml_matrix_ellblock_t *B, double *trace);
bml_matrix_ellblock_t *eb_transpose_new(bml_matrix_ellblock_t *A);
bool eb_transpose(bml_matrix_ellblock_t *A);
bool eb_gershgorin(bml_matrix_ellblock_t *A, double *bounds);
bool eb_normalize(bml_matrix_ellblock_t *A, double mineval, double maxeval);
