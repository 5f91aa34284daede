// Process-wide ELLBLOCK block partition, with the reference's semantics
// (ellblock/bml_allocate_ellblock.c:15-95): set once by bml_set_block_sizes,
// or on first use from a default block dimension of 4.
#include "internal.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace {
int *s_bsize = nullptr;
int s_block_dim = 4;
int s_nb = 0;
int s_mb = 0;
} // namespace

extern "C" {

void bml_set_block_sizes(int *bsize, int nb, int mb)
{
    printf("bml_set_block_sizes %d %d\n", nb, mb);
    if (nb <= 0 || mb <= 0 || !bsize)
    {
        b200_set_error(BML_B200_ERR_INVALID, "bml_set_block_sizes: nb=%d mb=%d", nb, mb);
        return;
    }
    free(s_bsize);
    s_nb = nb;
    s_mb = mb;
    s_bsize = static_cast<int *>(malloc(sizeof(int) * nb));
    memcpy(s_bsize, bsize, sizeof(int) * nb);
}

int *bml_get_block_sizes(int N, int M)
{
    if (!s_bsize)
    {
        if (M <= 0)
            M = N;
        s_nb = N / s_block_dim;
        if (s_nb * s_block_dim < N)
            s_nb++;
        printf("s_nb = %d\n", s_nb);
        s_mb = M / s_block_dim;
        if (s_mb * s_block_dim < M)
            s_mb++;
        if (s_mb < 4)
            s_mb = 4;
        if (s_mb > s_nb)
            s_mb = s_nb;
        printf("s_mb = %d\n", s_mb);
        s_bsize = static_cast<int *>(malloc(sizeof(int) * s_nb));
        for (int ib = 0; ib < s_nb - 1; ib++)
            s_bsize[ib] = s_block_dim;
        s_bsize[s_nb - 1] = N - s_block_dim * (s_nb - 1);
    }
    return s_bsize;
}

int bml_get_mb(void) { return s_mb; }

int bml_get_nb(void) { return s_nb; }

// Forget the partition so that a new one can be set (the reference allows one
// per process; a test harness running many cases in one process needs more).
BML_B200_API void bml_b200_reset_block_sizes(void)
{
    free(s_bsize);
    s_bsize = nullptr;
    s_nb = 0;
    s_mb = 0;
}

} // extern "C"
