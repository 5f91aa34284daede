// Trace of an ELLPACK matrix that allocates no memory.
//
// bml_trace (and every other entry point of this library) may allocate: the
// library creates its stream, pinned buffers and a scratch arena on first use
// and grows the arena on demand.  Some callers cannot accept that: programs
// that own all device memory through their own fixed pool and forbid a
// library from calling cudaMalloc, and latency-critical loops in which a
// cudaMalloc/cudaFree (cudaFree synchronises the device) is not acceptable.
// For them this entry point computes tr A from device arrays they pass in,
// writing the result to device memory they pass in, and keeps its per-row
// partial sums in a fixed array in device global memory that is part of the
// library image.
//
// That array holds up to B200_NOALLOC_MAX_ROWS doubles (4 MiB) on every GPU
// that loads the library, until the process exits.  All calls share it and
// it keeps the last call's contents, so two calls whose kernels overlap on
// the GPU (on different streams, or from different host threads) race on it
// and give wrong results; calls on one stream run one after the other.
#include "device_util.cuh"

#include <atomic>
#include <mutex>

#define B200_NOALLOC_MAX_ROWS (1 << 19)

namespace {

static __device__ __align__(256) double g_noalloc_rows[B200_NOALLOC_MAX_ROWS];

// Device address of g_noalloc_rows per device ordinal, found once per device.
constexpr int kMaxDevices = 64;
// published with release order under the mutex, read with acquire order
std::atomic<double *> g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

// Value of the first diagonal entry of each row (the reference's
// bml_trace_ellpack, ellpack/bml_trace_ellpack_typed.c:74-88), one warp per
// row, into rows[i].
template <typename T>
__global__ void noalloc_diag_kernel(const T *__restrict__ V, const int *__restrict__ I,
                                    const int *__restrict__ Nz, int ld, int N, double *rows)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = Nz[i];
        int first = n;
        for (int c0 = 0; c0 < n && first == n; c0 += 32)
        {
            const int q = c0 + lane;
            const unsigned bal = __ballot_sync(b200::FULL, q < n && I[(size_t) i * ld + q] == i);
            if (bal)
                first = c0 + __ffs(bal) - 1;
        }
        if (lane == 0)
            rows[i] = first < n ? (double) V[(size_t) i * ld + first] : 0.0;
    }
}

// Fixed-order FP64 sum of rows[0..N) into *out (one block).
__global__ void __launch_bounds__(1024) noalloc_sum_kernel(const double *rows, int N, double *out)
{
    __shared__ double s[1024];
    const int t = threadIdx.x;
    const int per = b200_ceil_div(N, 1024);
    double x = 0.0;
    for (int r = t * per; r < min(N, (t + 1) * per); ++r)
        x += rows[r];
    s[t] = x;
    __syncthreads();
    for (int k = 512; k; k >>= 1)
    {
        if (t < k)
            s[t] += s[t + k];
        __syncthreads();
    }
    if (t == 0)
        *out = s[0];
}

} // namespace

extern "C" int bml_b200_ellpack_trace_noalloc(const void *d_value, const int *d_index,
                                              const int *d_nnz, int N, int ld, int precision,
                                              double *d_trace, void *stream)
{
    if (!d_value || !d_index || !d_nnz || !d_trace || ld < 1 || N < 0 ||
        (precision != single_real && precision != double_real))
    {
        b200_set_error(BML_B200_ERR_INVALID, "ellpack_trace_noalloc: bad argument");
        return BML_B200_ERR_INVALID;
    }
    if (N > B200_NOALLOC_MAX_ROWS)
    {
        b200_set_error(BML_B200_ERR_INVALID,
                       "ellpack_trace_noalloc: N=%d exceeds the fixed scratch of %d rows", N,
                       B200_NOALLOC_MAX_ROWS);
        return BML_B200_ERR_INVALID;
    }
    int dev = 0;
    if (!CUDA_OK(cudaGetDevice(&dev)))
        return BML_B200_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ellpack_trace_noalloc: device %d", dev);
        return BML_B200_ERR_INVALID;
    }
    double *rows = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!rows)
    {
        // First call on this device (with it current): host code cannot use
        // the array's name as a device address, so look the address up.
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev].load(std::memory_order_relaxed))
        {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_rows);
            if (e != cudaSuccess)
            {
                b200_set_error(BML_B200_ERR_CUDA, "ellpack_trace_noalloc: cudaGetSymbolAddress: %s",
                               cudaGetErrorString(e));
                return BML_B200_ERR_CUDA;
            }
            g_noalloc_ptr[dev].store(static_cast<double *>(p), std::memory_order_release);
        }
        rows = g_noalloc_ptr[dev].load(std::memory_order_relaxed);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (N > 0)
    {
        const int grid = b200_ceil_div(N, 8) < 4096 ? b200_ceil_div(N, 8) : 4096;
        if (precision == double_real)
            noalloc_diag_kernel<double><<<grid, 256, 0, s>>>(static_cast<const double *>(d_value), d_index,
                                                             d_nnz, ld, N, rows);
        else
            noalloc_diag_kernel<float><<<grid, 256, 0, s>>>(static_cast<const float *>(d_value), d_index,
                                                            d_nnz, ld, N, rows);
        if (!LAUNCH_OK("noalloc_diag_kernel"))
            return BML_B200_ERR_CUDA;
    }
    noalloc_sum_kernel<<<1, 1024, 0, s>>>(rows, N, d_trace);
    if (!LAUNCH_OK("noalloc_sum_kernel"))
        return BML_B200_ERR_CUDA;
    return BML_B200_OK;
}
