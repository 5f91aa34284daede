/*
 * Seeded synthetic Hamiltonians for the CPU side of the checks and of the
 * reference arm of bench.py.  TEST INFRASTRUCTURE ONLY.
 *
 * These are the same generators as the library's own (splitmix64 ->
 * U[0,1) from the top 53 bits, N(0,1) by the cosine branch of Box-Muller,
 * symmetric matrices drawn once per pair while row min(i, j) is generated,
 * rows in ascending column order), restated here so that a process that runs
 * only the reference library never has to load libbml_b200.so to build its
 * inputs.  tests/test_oracle.py pins both generators to the sha256 digests in
 * tests/golden/generators.json, which the library's generators also match.
 *
 * Layout: the reference ELLPACK host layout, row-major value[N*M],
 * index[N*M], nnz[N].  Return value: N, or -1 on bad arguments or when a row
 * needs more than M entries.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct
{
    uint64_t s;
} sm64_t;

static uint64_t sm64_next(sm64_t *r)
{
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double sm64_uniform(sm64_t *r)
{
    return (double) (sm64_next(r) >> 11) * 0x1.0p-53;
}

static double sm64_normal(sm64_t *r)
{
    const double u1 = 1.0 - sm64_uniform(r); /* (0, 1] */
    const double u2 = sm64_uniform(r);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925 * u2);
}

static int put(int M, double *value, int *index, int *nnz, int i, int j, double v)
{
    if (nnz[i] >= M)
        return 0;
    value[(size_t) i * M + nnz[i]] = v;
    index[(size_t) i * M + nnz[i]] = j;
    nnz[i]++;
    return 1;
}

/* 1-D chain: H_ii ~ U[-1,1); H_ij = u exp(-|i-j|/4), u ~ U[-1,1), 0<|i-j|<=16. */
int oracle_gen_chain(int N, int M, unsigned long long seed, double *value, int *index, int *nnz)
{
    if (N <= 0 || M <= 0 || !value || !index || !nnz)
        return -1;
    sm64_t r = {seed};
    int ok = 1;
    for (int i = 0; i < N; i++)
        nnz[i] = 0;
    for (int i = 0; i < N; i++)
    {
        ok &= put(M, value, index, nnz, i, i, 2.0 * sm64_uniform(&r) - 1.0);
        for (int d = 1; d <= 16 && i + d < N; d++)
        {
            const double v = (2.0 * sm64_uniform(&r) - 1.0) * exp(-d / 4.0);
            ok &= put(M, value, index, nnz, i, i + d, v);
            ok &= put(M, value, index, nnz, i + d, i, v);
        }
    }
    return ok ? N : -1;
}

/* L^3 cubic lattice, site x + L*y + L*L*z, open boundaries, neighbours within
 * Euclidean distance radius: H_ij = -exp(-d) (1 + 0.1 g), g ~ N(0,1);
 * H_ii ~ N(0,1).  Only the first N sites are kept. */
int oracle_gen_lattice(int L, int radius, int N, int M, unsigned long long seed, double *value,
                       int *index, int *nnz)
{
    if (L <= 2 * radius || N <= 0 || (long long) N > (long long) L * L * L || M <= 0 || !value ||
        !index || !nnz)
        return -1;
    /* offsets towards a larger site index, in ascending index order */
    const int side = 2 * radius + 1;
    int *odx = malloc(sizeof(int) * side * side * side);
    int *ody = malloc(sizeof(int) * side * side * side);
    int *odz = malloc(sizeof(int) * side * side * side);
    double *od = malloc(sizeof(double) * side * side * side);
    if (!odx || !ody || !odz || !od)
    {
        free(odx);
        free(ody);
        free(odz);
        free(od);
        return -1;
    }
    int nup = 0;
    for (int dz = -radius; dz <= radius; dz++)
        for (int dy = -radius; dy <= radius; dy++)
            for (int dx = -radius; dx <= radius; dx++)
            {
                const int r2 = dx * dx + dy * dy + dz * dz;
                if (r2 == 0 || r2 > radius * radius)
                    continue;
                if (dx + L * dy + L * L * dz > 0)
                {
                    odx[nup] = dx;
                    ody[nup] = dy;
                    odz[nup] = dz;
                    od[nup] = sqrt((double) r2);
                    nup++;
                }
            }
    sm64_t r = {seed};
    int ok = 1;
    for (int i = 0; i < N; i++)
        nnz[i] = 0;
    for (int i = 0; i < N; i++)
    {
        const int x = i % L, y = (i / L) % L, z = i / (L * L);
        ok &= put(M, value, index, nnz, i, i, sm64_normal(&r));
        for (int u = 0; u < nup; u++)
        {
            const int X = x + odx[u], Y = y + ody[u], Z = z + odz[u];
            if (X < 0 || X >= L || Y < 0 || Y >= L || Z < 0 || Z >= L)
                continue;
            const int j = X + L * Y + L * L * Z;
            if (j >= N)
                continue;
            const double v = -exp(-od[u]) * (1.0 + 0.1 * sm64_normal(&r));
            ok &= put(M, value, index, nnz, i, j, v);
            ok &= put(M, value, index, nnz, j, i, v);
        }
    }
    free(odx);
    free(ody);
    free(odz);
    free(od);
    return ok ? N : -1;
}
