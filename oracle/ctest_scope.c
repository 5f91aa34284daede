/*
 * Test functions of the reference's C test driver (tests/C-tests/bml_test.c)
 * whose bml operations lie outside libbml_b200's path: dense
 * diagonalisation, inverse, submatrices, adjacency, the internal GEMM,
 * element-wise products and norms of sums.  The driver's table names every
 * test, so these stand in for them: each reports that the test is out of
 * scope and fails.  TEST INFRASTRUCTURE ONLY: linked into the reference's
 * test driver, which is built against libbml_b200.so by oracle/Makefile
 * (target ctest) to show that the reference's own tests pass on this library.
 */
#include <stdio.h>

#define OUT_OF_SCOPE(name)                                                          \
    int name(const int N, const int type, const int precision, const int M)         \
    {                                                                               \
        (void) N;                                                                   \
        (void) type;                                                                \
        (void) precision;                                                           \
        (void) M;                                                                   \
        fprintf(stderr, #name ": outside libbml_b200's path\n");                    \
        return 2;                                                                   \
    }

OUT_OF_SCOPE(test_adjacency)
OUT_OF_SCOPE(test_adjungate_triangle)
OUT_OF_SCOPE(test_bml_gemm)
OUT_OF_SCOPE(test_diagonalize)
OUT_OF_SCOPE(test_inverse)
OUT_OF_SCOPE(test_submatrix)
OUT_OF_SCOPE(test_element_multiply)
OUT_OF_SCOPE(test_norm)
