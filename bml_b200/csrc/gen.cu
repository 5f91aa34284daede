// Synthetic Hamiltonians in the reference ELLPACK host layout (row-major
// value[N*M], index[N*M], nnz[N]), shared by the tests, the benchmark and
// the oracle so that both libraries see byte-identical inputs.
//
// Random numbers: splitmix64 (Steele, Lea, Flood, OOPSLA 2014) -> U[0,1) from
// the top 53 bits; N(0,1) by Box-Muller (cosine branch, one normal per two
// uniforms).  Matrices are symmetric: the value of (i, j) and (j, i) is drawn
// once, while row min(i, j) is generated.  Rows come out in ascending column
// order.
#include "internal.h"

#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct SplitMix64
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
    double sym_uniform() { return 2.0 * uniform() - 1.0; } // U[-1, 1)
    double normal()
    {
        const double u1 = 1.0 - uniform(); // (0, 1]
        const double u2 = uniform();
        return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925 * u2);
    }
};

struct RowWriter
{
    int M;
    double *value;
    int *index;
    int *nnz;
    bool overflow = false;
    void put(int i, int j, double v)
    {
        if (nnz[i] >= M)
        {
            overflow = true;
            return;
        }
        value[(size_t) i * M + nnz[i]] = v;
        index[(size_t) i * M + nnz[i]] = j;
        nnz[i]++;
    }
};

} // namespace

extern "C" {

// 1-D chain: H_ii ~ U[-1,1]; H_ij = u exp(-|i-j|/4), u ~ U[-1,1], 0<|i-j|<=16.
int bml_b200_gen_chain(int N, int M, unsigned long long seed, double *value, int *index, int *nnz)
{
    if (N <= 0 || M <= 0 || !value || !index || !nnz)
        return -1;
    SplitMix64 rng{seed};
    RowWriter w{M, value, index, nnz};
    for (int i = 0; i < N; i++)
        nnz[i] = 0;
    for (int i = 0; i < N; i++)
    {
        w.put(i, i, rng.sym_uniform());
        for (int d = 1; d <= 16 && i + d < N; d++)
        {
            const double v = rng.sym_uniform() * exp(-d / 4.0);
            w.put(i, i + d, v);
            w.put(i + d, i, v);
        }
    }
    return w.overflow ? -1 : N;
}

// L^3 cubic lattice, site s = x + L*y + L*L*z, open boundaries, neighbours at
// Euclidean distance d <= radius; H_ij = -exp(-d) (1 + 0.1 g), g ~ N(0,1);
// H_ii ~ N(0,1).  Only the first N sites (N <= L^3) are kept.
int bml_b200_gen_lattice(int L, int radius, int N, int M, unsigned long long seed, double *value,
                         int *index, int *nnz)
{
    if (L <= 2 * radius || N <= 0 || (long long) N > (long long) L * L * L || M <= 0 || !value ||
        !index || !nnz)
        return -1;
    struct Off
    {
        int dx, dy, dz;
        double d;
    };
    // Offsets pointing to a larger site index, in ascending index order.
    std::vector<Off> up;
    for (int dz = -radius; dz <= radius; dz++)
        for (int dy = -radius; dy <= radius; dy++)
            for (int dx = -radius; dx <= radius; dx++)
            {
                const int r2 = dx * dx + dy * dy + dz * dz;
                if (r2 == 0 || r2 > radius * radius)
                    continue;
                if (dx + L * dy + L * L * dz > 0)
                    up.push_back({dx, dy, dz, sqrt((double) r2)});
            }
    SplitMix64 rng{seed};
    RowWriter w{M, value, index, nnz};
    for (int i = 0; i < N; i++)
        nnz[i] = 0;
    for (int i = 0; i < N; i++)
    {
        const int x = i % L, y = (i / L) % L, z = i / (L * L);
        w.put(i, i, rng.normal());
        for (const Off &o : up)
        {
            const int X = x + o.dx, Y = y + o.dy, Z = z + o.dz;
            if (X < 0 || X >= L || Y < 0 || Y >= L || Z < 0 || Z >= L)
                continue;
            const int j = X + L * Y + L * L * Z;
            if (j >= N)
                continue;
            const double v = -exp(-o.d) * (1.0 + 0.1 * rng.normal());
            w.put(i, j, v);
            w.put(j, i, v);
        }
    }
    return w.overflow ? -1 : N;
}

} // extern "C"
