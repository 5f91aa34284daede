// Device helpers shared by the kernel translation units.
#pragma once

#include "internal.h"

namespace b200 {

constexpr unsigned FULL = 0xffffffffu;

// Correctly rounded multiply / add that the compiler may not contract into an
// FMA.  The reference is built -std=c99 without -mfma, so every product and
// sum it forms is a separately rounded IEEE operation; these reproduce that.
template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }

// x + s*y where s is a double scalar and x, y are of the matrix precision,
// evaluated the way C evaluates `x + alpha * y` with a double alpha: in double,
// then rounded once to the matrix precision.
template <typename T> __device__ __forceinline__ T axpy_d(T x, double s, T y)
{
    return (T) __dadd_rn((double) x, __dmul_rn(s, (double) y));
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Barrier over the W warps of one team; team t uses named barrier t+1.
template <int W> __device__ __forceinline__ void team_sync(int team)
{
    if (W == 1)
        __syncwarp();
    else
        asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(W * 32) : "memory");
}

__device__ __forceinline__ unsigned hash_slot(int k, unsigned mask)
{
    return ((unsigned) k * 2654435761u) & mask;
}

// Open-addressing insert of key k with payload v into (keys, pay) of size
// mask+1; returns the slot, or -1 when the table is full.  Concurrent inserts
// of distinct keys are safe.
__device__ __forceinline__ int hash_put(int *keys, int *pay, unsigned mask, int k, int v)
{
    unsigned h = hash_slot(k, mask);
    volatile int *vk = keys;
#pragma unroll 1
    for (unsigned p = 0; p <= mask; ++p)
    {
        const int cur = vk[h];
        if (cur == B200_EMPTY_KEY)
        {
            const int old = atomicCAS(&keys[h], B200_EMPTY_KEY, k);
            if (old == B200_EMPTY_KEY || old == k)
            {
                pay[h] = v;
                return (int) h;
            }
        }
        else if (cur == k)
        {
            pay[h] = v;
            return (int) h;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

// Lookup of key k; returns its payload or -1.
__device__ __forceinline__ int hash_get(const int *keys, const int *pay, unsigned mask, int k)
{
    unsigned h = hash_slot(k, mask);
#pragma unroll 1
    for (unsigned p = 0; p <= mask; ++p)
    {
        const int cur = keys[h];
        if (cur == k)
            return pay[h];
        if (cur == B200_EMPTY_KEY)
            return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

} // namespace b200

// Sum of one or two per-row arrays in FP64 with a fixed order (each thread a
// contiguous stripe, then a tree), written to out[0..1].  Launch <<<1, 1024>>>.
__global__ void b200_sum_rows_kernel(const double *a, const double *b, int n, double *out);
// Max and min of per-row arrays (hi, lo) into out[0] = max(init_max, hi[i]),
// out[1] = min(init_min, lo[i]).  Launch <<<1, 1024>>>.
__global__ void b200_maxmin_rows_kernel(const double *hi, const double *lo, int n,
                                        double init_max, double init_min, double *out);
