// ELLPACK matrix storage: allocation, the host mirror, uploads/downloads,
// dense import/export kernels, and the reference's matrix constructors.
#include "internal.h"

#include <cstdlib>
#include <cstring>
#include <cmath>

size_t prec_size(bml_matrix_precision_t p)
{
    switch (p)
    {
    case single_real: return sizeof(float);
    case double_real: return sizeof(double);
    default: return 0;
    }
}

bool ell_is_supported(const bml_matrix_ellpack_t *A)
{
    return A && A->matrix_type == ellpack &&
           (A->matrix_precision == single_real || A->matrix_precision == double_real);
}

// Single-rank form of the reference's bml_default_domain (bml_allocate.c:599-716):
// one rank owning rows [0, N).
bml_domain_t *b200_default_domain(int N, int M, bml_distribution_mode_t mode)
{
    (void) mode;
    bml_domain_t *d = static_cast<bml_domain_t *>(calloc(1, sizeof(bml_domain_t)));
    if (!d)
        return nullptr;
    d->localRowMin = static_cast<int *>(calloc(1, sizeof(int)));
    d->localRowMax = static_cast<int *>(calloc(1, sizeof(int)));
    d->localRowExtent = static_cast<int *>(calloc(1, sizeof(int)));
    d->localElements = static_cast<int *>(calloc(1, sizeof(int)));
    d->localDispl = static_cast<int *>(calloc(1, sizeof(int)));
    d->totalProcs = 1;
    d->totalRows = N;
    d->totalCols = M;
    d->globalRowMin = 0;
    d->globalRowMax = N;
    d->globalRowExtent = N;
    d->maxLocalExtent = N;
    d->minLocalExtent = N;
    d->localRowMin[0] = 0;
    d->localRowMax[0] = N;
    d->localRowExtent[0] = N;
    d->localElements[0] = N * M;
    d->localDispl[0] = 0;
    return d;
}

void b200_free_domain(bml_domain_t *d)
{
    if (!d)
        return;
    free(d->localRowMin);
    free(d->localRowMax);
    free(d->localRowExtent);
    free(d->localElements);
    free(d->localDispl);
    free(d);
}

bml_matrix_ellpack_t *ell_alloc(bml_matrix_precision_t prec, int N, int M,
                                bml_distribution_mode_t mode, bool zero)
{
    const size_t sz = prec_size(prec);
    if (sz == 0)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "ELLPACK precision %d", (int) prec);
        return nullptr;
    }
    if (N <= 0 || M <= 0)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ELLPACK dimensions N=%d M=%d", N, M);
        return nullptr;
    }
    B200Context *c = b200_ctx();
    if (!c)
        return nullptr;
    auto *A = static_cast<bml_matrix_ellpack_t *>(calloc(1, sizeof(bml_matrix_ellpack_t)));
    if (!A)
    {
        b200_set_error(BML_B200_ERR_ALLOC, "host struct");
        return nullptr;
    }
    A->matrix_type = ellpack;
    A->matrix_precision = prec;
    A->distribution_mode = mode;
    A->N = N;
    A->M = M;
    A->ld = b200_round_up(M, 32);
    // Host mirror: calloc pages are mapped on first touch, so an unused
    // mirror of a large matrix costs no host memory traffic.
    A->value = calloc((size_t) N * M, sz);
    A->index = static_cast<int *>(calloc((size_t) N * M, sizeof(int)));
    A->nnz = static_cast<int *>(calloc((size_t) N, sizeof(int)));
    A->domain = b200_default_domain(N, M, mode);
    A->domain2 = b200_default_domain(N, M, mode);
    bool ok = A->value && A->index && A->nnz && A->domain && A->domain2;
    if (!ok)
        b200_set_error(BML_B200_ERR_ALLOC, "host arrays for N=%d M=%d", N, M);
    if (ok)
    {
        const size_t elems = (size_t) N * A->ld;
        cudaError_t e1 = cudaMallocAsync(&A->d_value, elems * sz, c->stream);
        cudaError_t e2 = cudaMallocAsync(reinterpret_cast<void **>(&A->d_index), elems * sizeof(int), c->stream);
        cudaError_t e3 = cudaMallocAsync(reinterpret_cast<void **>(&A->d_nnz), (size_t) N * sizeof(int), c->stream);
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
        {
            cudaGetLastError();
            b200_set_error(BML_B200_ERR_ALLOC, "device arrays for N=%d M=%d (%.1f MB)", N, M,
                           (elems * (sz + 4) + N * 4.0) / 1e6);
            ok = false;
        }
    }
    if (ok)
    {
        ok = CUDA_OK(cudaMemsetAsync(A->d_nnz, 0, (size_t) N * sizeof(int), c->stream));
        if (ok && zero)
            ok = CUDA_OK(cudaMemsetAsync(A->d_value, 0, (size_t) N * A->ld * sz, c->stream)) &&
                 CUDA_OK(cudaMemsetAsync(A->d_index, 0, (size_t) N * A->ld * sizeof(int),
                                         c->stream));
    }
    if (!ok)
    {
        ell_free(A);
        return nullptr;
    }
    A->mirror = MIRROR_SYNCED;
    return A;
}

void ell_free(bml_matrix_ellpack_t *A)
{
    if (!A)
        return;
    if (A->d_value || A->d_index || A->d_nnz)
    {
        // Freed in stream order, after the kernels queued on these arrays.
        B200Context *c = b200_ctx();
        if (c)
        {
            if (A->d_value)
                cudaFreeAsync(A->d_value, c->stream);
            if (A->d_index)
                cudaFreeAsync(A->d_index, c->stream);
            if (A->d_nnz)
                cudaFreeAsync(A->d_nnz, c->stream);
        }
    }
    free(A->value);
    free(A->index);
    free(A->nnz);
    b200_free_domain(A->domain);
    b200_free_domain(A->domain2);
    free(A);
}

bool ell_to_device(bml_matrix_ellpack_t *A)
{
    if (A->mirror != MIRROR_HOST_NEWER)
        return true;
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const size_t sz = prec_size(A->matrix_precision);
    if (!CUDA_OK(cudaMemcpy2DAsync(A->d_value, A->ld * sz, A->value, A->M * sz, A->M * sz, A->N,
                                   cudaMemcpyHostToDevice, c->stream)) ||
        !CUDA_OK(cudaMemcpy2DAsync(A->d_index, A->ld * sizeof(int), A->index, A->M * sizeof(int),
                                   A->M * sizeof(int), A->N, cudaMemcpyHostToDevice, c->stream)) ||
        !CUDA_OK(cudaMemcpyAsync(A->d_nnz, A->nnz, (size_t) A->N * sizeof(int),
                                 cudaMemcpyHostToDevice, c->stream)))
        return false;
    // Pageable sources: the copies are staged before the calls return, but
    // synchronise so that the caller may reuse the host arrays at once.
    if (!b200_sync())
        return false;
    A->mirror = MIRROR_SYNCED;
    return true;
}

bool ell_to_host(bml_matrix_ellpack_t *A)
{
    if (A->mirror != MIRROR_DEVICE_NEWER)
        return true;
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const size_t sz = prec_size(A->matrix_precision);
    if (!CUDA_OK(cudaMemcpy2DAsync(A->value, A->M * sz, A->d_value, A->ld * sz, A->M * sz, A->N,
                                   cudaMemcpyDeviceToHost, c->stream)) ||
        !CUDA_OK(cudaMemcpy2DAsync(A->index, A->M * sizeof(int), A->d_index, A->ld * sizeof(int),
                                   A->M * sizeof(int), A->N, cudaMemcpyDeviceToHost, c->stream)) ||
        !CUDA_OK(cudaMemcpyAsync(A->nnz, A->d_nnz, (size_t) A->N * sizeof(int),
                                 cudaMemcpyDeviceToHost, c->stream)))
        return false;
    if (!b200_sync())
        return false;
    A->mirror = MIRROR_SYNCED;
    return true;
}

// ---------------------------------------------------------------------------
// Dense import/export kernels (one warp per row).
// Import follows ellpack/bml_import_ellpack_typed.c:30-75: columns in
// ascending order, kept when |a_ij| > threshold.  Export follows
// ellpack/bml_export_ellpack_typed.c:26-73.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void import_dense_kernel(const T *__restrict__ D, int N, int colmajor, T thr,
                                    T *__restrict__ V, int *__restrict__ I, int *__restrict__ Nz,
                                    int ld, int M, int *overflow)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        int cnt = 0;
        for (int j0 = 0; j0 < N; j0 += 32)
        {
            const int j = j0 + lane;
            T a = T(0);
            if (j < N)
                a = colmajor ? D[(size_t) j * N + i] : D[(size_t) i * N + j];
            const bool keep = j < N && fabs(a) > thr;
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            const int p = cnt + __popc(bal & ((1u << lane) - 1u));
            if (keep && p < M)
            {
                V[(size_t) i * ld + p] = a;
                I[(size_t) i * ld + p] = j;
            }
            cnt += __popc(bal);
        }
        if (lane == 0)
        {
            Nz[i] = min(cnt, M);
            if (cnt > M)
                atomicExch(overflow, 1);
        }
    }
}

template <typename T>
__global__ void export_dense_kernel(const T *__restrict__ V, const int *__restrict__ I,
                                    const int *__restrict__ Nz, int ld, int N, int colmajor,
                                    T *__restrict__ D)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = Nz[i];
        for (int p = lane; p < n; p += 32)
        {
            const int j = I[(size_t) i * ld + p];
            if (j >= 0 && j < N)
                D[colmajor ? (size_t) j * N + i : (size_t) i * N + j] = V[(size_t) i * ld + p];
        }
    }
}

__global__ void nnz_stats_kernel(const int *Nz, int N, unsigned long long *total, int *maxrow)
{
    unsigned long long s = 0;
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    {
        s += (unsigned long long) Nz[i];
        m = max(m, Nz[i]);
    }
    for (int o = 16; o; o >>= 1)
    {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if ((threadIdx.x & 31) == 0)
    {
        atomicAdd(total, s);
        atomicMax(maxrow, m);
    }
}

} // namespace

bool ell_import_dense(bml_matrix_ellpack_t *A, const void *dense, bml_dense_order_t order,
                      double threshold)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const size_t sz = prec_size(A->matrix_precision);
    const size_t bytes = (size_t) A->N * A->N * sz;
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(bytes + 256));
    if (!scr)
        return false;
    int *overflow = reinterpret_cast<int *>(scr + bytes);
    if (!CUDA_OK(cudaMemcpyAsync(scr, dense, bytes, cudaMemcpyHostToDevice, c->stream)) ||
        !CUDA_OK(cudaMemsetAsync(overflow, 0, sizeof(int), c->stream)))
        return false;
    const int grid = min(b200_ceil_div(A->N, 8), c->sm_count * 16);
    const int colmajor = order == dense_column_major;
    if (A->matrix_precision == double_real)
        import_dense_kernel<double><<<grid, 256, 0, c->stream>>>(
            reinterpret_cast<double *>(scr), A->N, colmajor, (double) threshold,
            static_cast<double *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->M, overflow);
    else
        import_dense_kernel<float><<<grid, 256, 0, c->stream>>>(
            reinterpret_cast<float *>(scr), A->N, colmajor, (float) threshold,
            static_cast<float *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->M, overflow);
    if (!LAUNCH_OK("import_dense_kernel"))
        return false;
    int hov = 0;
    if (!CUDA_OK(cudaMemcpyAsync(&hov, overflow, sizeof(int), cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    ell_mark_device(A);
    if (hov)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW,
                       "import_from_dense: a row has more than M=%d entries above threshold", A->M);
        return false;
    }
    return true;
}

bool ell_export_dense(bml_matrix_ellpack_t *A, void *dense, bml_dense_order_t order)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    const size_t sz = prec_size(A->matrix_precision);
    const size_t bytes = (size_t) A->N * A->N * sz;
    void *scr = b200_scratch(bytes);
    if (!scr)
        return false;
    if (!CUDA_OK(cudaMemsetAsync(scr, 0, bytes, c->stream)))
        return false;
    const int grid = min(b200_ceil_div(A->N, 8), c->sm_count * 16);
    const int colmajor = order == dense_column_major;
    if (A->matrix_precision == double_real)
        export_dense_kernel<double><<<grid, 256, 0, c->stream>>>(
            static_cast<double *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->N, colmajor,
            static_cast<double *>(scr));
    else
        export_dense_kernel<float><<<grid, 256, 0, c->stream>>>(
            static_cast<float *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->N, colmajor,
            static_cast<float *>(scr));
    if (!LAUNCH_OK("export_dense_kernel"))
        return false;
    return CUDA_OK(cudaMemcpyAsync(dense, scr, bytes, cudaMemcpyDeviceToHost, c->stream)) &&
           b200_sync();
}

bool ell_nnz_total(bml_matrix_ellpack_t *A, long long *total, int *maxrow)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    unsigned char *small = static_cast<unsigned char *>(c->d_small) + 1024;
    if (!CUDA_OK(cudaMemsetAsync(small, 0, 16, c->stream)))
        return false;
    nnz_stats_kernel<<<min(b200_ceil_div(A->N, 256), c->sm_count * 4), 256, 0, c->stream>>>(
        A->d_nnz, A->N, reinterpret_cast<unsigned long long *>(small),
        reinterpret_cast<int *>(small + 8));
    if (!LAUNCH_OK("nnz_stats_kernel"))
        return false;
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 1024;
    if (!CUDA_OK(cudaMemcpyAsync(pin, small, 16, cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    if (total)
        *total = (long long) *reinterpret_cast<unsigned long long *>(pin);
    if (maxrow)
        *maxrow = *reinterpret_cast<int *>(pin + 8);
    return true;
}

// ---------------------------------------------------------------------------
// The reference's random / banded / identity constructors.  They are filled
// on the host with the C library rand() in exactly the reference's call order
// (ellpack/bml_allocate_ellpack_typed.c:300-443), so a caller that seeds with
// srand() gets the same matrix from either library, then uploaded once.
// ---------------------------------------------------------------------------
template <typename T> static void fill_random(bml_matrix_ellpack_t *A)
{
    const int N = A->N, M = A->M;
    T *V = static_cast<T *>(A->value);
    int *I = A->index, *Z = A->nnz;
    int *col_marker = static_cast<int *>(malloc(sizeof(int) * N));
    int *col_marker_pos = static_cast<int *>(malloc(sizeof(int) * M));
    const T inv = (T) 1.0 / (T) RAND_MAX;
    for (int j = 0; j < N; j++)
        col_marker[j] = -1;
    for (int i = 0; i < N; i++)
    {
        int col = i, nnz_row = 0;
        for (int j = 0; j < M; j++)
        {
            if (col_marker[col] == -1)
            {
                V[(size_t) i * M + nnz_row] = rand() * inv;
                I[(size_t) i * M + nnz_row] = col;
                col_marker_pos[nnz_row] = col;
                col_marker[col] = 1;
                nnz_row++;
            }
            col = rand() % N;
        }
        Z[i] = nnz_row;
        for (int j = 0; j < nnz_row; j++)
            col_marker[col_marker_pos[j]] = -1;
    }
    free(col_marker);
    free(col_marker_pos);
}

template <typename T> static void fill_banded(bml_matrix_ellpack_t *A)
{
    const int N = A->N, M = A->M;
    T *V = static_cast<T *>(A->value);
    const T inv = (T) 1.0 / (T) RAND_MAX;
    for (int i = 0; i < N; i++)
    {
        int jind = 0;
        for (int j = (i - M / 2 >= 0 ? i - M / 2 : 0); j < (i - M / 2 + M <= N ? i - M / 2 + M : N);
             j++)
        {
            V[(size_t) i * M + jind] = rand() * inv;
            A->index[(size_t) i * M + jind] = j;
            jind++;
        }
        A->nnz[i] = jind;
    }
}

template <typename T> static void fill_identity(bml_matrix_ellpack_t *A)
{
    T *V = static_cast<T *>(A->value);
    for (int i = 0; i < A->N; i++)
    {
        V[(size_t) i * A->M] = (T) 1.0;
        A->index[(size_t) i * A->M] = i;
        A->nnz[i] = 1;
    }
}

bml_matrix_ellpack_t *ell_constructor(int kind, bml_matrix_precision_t prec, int N, int M,
                                      bml_distribution_mode_t mode)
{
    bml_matrix_ellpack_t *A = ell_alloc(prec, N, M, mode, true);
    if (!A)
        return nullptr;
    if (!b200_sync())
    {
        ell_free(A);
        return nullptr;
    }
    const bool dbl = prec == double_real;
    switch (kind)
    {
    case 1: dbl ? fill_random<double>(A) : fill_random<float>(A); break;
    case 2: dbl ? fill_banded<double>(A) : fill_banded<float>(A); break;
    case 3: dbl ? fill_identity<double>(A) : fill_identity<float>(A); break;
    default: break;
    }
    ell_mark_host(A);
    if (!ell_to_device(A))
    {
        ell_free(A);
        return nullptr;
    }
    return A;
}

bml_matrix_ellpack_t ell_row_view(const bml_matrix_ellpack_t *A, int r0, int r1)
{
    bml_matrix_ellpack_t V = *A;
    const size_t sz = prec_size(A->matrix_precision);
    V.N = r1 - r0;
    V.d_value = static_cast<unsigned char *>(A->d_value) + (size_t) r0 * A->ld * sz;
    V.d_index = A->d_index + (size_t) r0 * A->ld;
    V.d_nnz = A->d_nnz + r0;
    V.value = static_cast<unsigned char *>(A->value) + (size_t) r0 * A->M * sz;
    V.index = A->index + (size_t) r0 * A->M;
    V.nnz = A->nnz + r0;
    return V;
}
