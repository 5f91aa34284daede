// Dense tier of the unordered ELLPACK product C = A*B, for operands whose
// rows are a large share of N wide (the SP2 iterates of a metallic
// Hamiltonian fill in to dense rows within a few iterations).
//
// Same result set as the sparse products (ellpack/bml_multiply_ellpack_typed.c:
// 252-333 for X^2, :468-542 for A*B): A and B are scattered into zero-filled
// dense images, C = A B is formed by a register-tiled GEMM (each product a
// single rounded multiply-add; the products of one entry are summed in no
// fixed order, within the same bound as the unordered sparse kernel), and a
// compaction kernel applies the reference's keep rule row by row, in
// ascending column order: the diagonal when it is touched, another column
// when |c| > threshold (compared in the matrix precision).  A column that no
// structural product touches holds an exact zero in the image and is
// dropped by the rule, as the sparse kernels drop it, so only the diagonal
// needs the structure: it is touched when some j has A[i,j] and B[j,i]
// stored, found through a byte image of B's pattern.  The traces are those of
// the sparse kernels: tr A from A's diagonal entries, tr C from the
// pre-threshold diagonal where touched.
//
// The GEMM: 128 x 128 tiles of C per CTA of 256 threads, each thread 8 x 8
// outputs (rows ty + 16 m, columns tx + 16 n) in registers; K in steps of 16
// staged through shared memory, the next step's operands loaded into
// registers while the current one is multiplied.  A's tile is stored
// transposed (k-major), so every inner step reads 8 values of A (two
// addresses per warp, broadcast) and 8 of B (16 consecutive per half warp).
// The images are padded to multiples of 128 with zeros, so the kernel has no
// edge cases.
#include "device_util.cuh"

#include <cstring>

using namespace b200;

namespace {

constexpr int DT = 128;   // tile edge of C
constexpr int DK = 16;    // k step
constexpr int DTHREADS = 256;

struct DenseFlags
{
    int overflow;
    int max_width;
    int bad_input;
    int pad;
};

// image[i * ld + col] += value for every stored entry (duplicates add up, as
// they do in the sparse products); rows padded with zeros.  One warp per row.
template <typename T>
__global__ void __launch_bounds__(256) dense_scatter_kernel(const T *v, const int *ix, const int *nz, int ldE, int nrows,
                                                            int ncols, T *img, size_t ld, unsigned char *pat,
                                                            DenseFlags *flags)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nrows; i += warps)
    {
        const int n = nz[i];
        if (n < 0 || n > ldE)
        {
            if (lane == 0)
                atomicExch(&flags->bad_input, 1);
            continue;
        }
        for (int p = lane; p < n; p += 32)
        {
            const int c = ix[(size_t) i * ldE + p];
            if (c < 0 || c >= ncols)
            {
                atomicExch(&flags->bad_input, 1);
                continue;
            }
            atomicAdd(&img[(size_t) i * ld + c], v[(size_t) i * ldE + p]);
            if (pat)
                pat[(size_t) c * ld + i] = 1; // pattern of B, transposed: pat[col * ld + row]
        }
    }
}

// touched[i] = 1 when some stored A[i,j] meets a stored B[j,i]; dA[i] = sum of
// A's diagonal entries.  One warp per row of A.
template <typename T>
__global__ void __launch_bounds__(256) dense_diag_kernel(const T *v, const int *ix, const int *nz, int ldE, int nrows,
                                                         int ncols, const unsigned char *patBt, size_t ld,
                                                         int *touched, double *dA)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nrows; i += warps)
    {
        const int n = nz[i];
        int hit = 0;
        double d = 0.0;
        if (n >= 0 && n <= ldE)
            for (int p = lane; p < n; p += 32)
            {
                const int j = ix[(size_t) i * ldE + p];
                if (j < 0 || j >= ncols)
                    continue;
                // B[j,i] stored <=> patBt[i * ld + j]
                if (i < ncols && patBt[(size_t) i * ld + j])
                    hit = 1;
                if (j == i)
                    d += (double) v[(size_t) i * ldE + p];
            }
        hit = __any_sync(FULL, hit);
        for (int o = 16; o; o >>= 1)
            d += __shfl_xor_sync(FULL, d, o);
        if (lane == 0)
        {
            touched[i] = hit;
            if (dA)
                dA[i] = d;
        }
    }
}

template <typename T> __device__ __forceinline__ T fma_t(T a, T b, T c);
template <> __device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return fma(a, b, c); }
template <> __device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return fmaf(a, b, c); }

// C[Mp x Np] = A[Mp x Kp] B[Kp x Np], all row-major with leading dimension ld,
// every dimension a multiple of 128.  Dynamic shared memory: two stages of
// A^T (16 x 128) and B (16 x 128).
template <typename T>
__global__ void __launch_bounds__(DTHREADS, 1) dense_gemm_kernel(const T *__restrict__ A, const T *__restrict__ B,
                                                                 T *__restrict__ Cm, size_t ld, int Kp)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    T(*As)[DK][DT] = reinterpret_cast<T(*)[DK][DT]>(dsm);
    T(*Bs)[DK][DT] = reinterpret_cast<T(*)[DK][DT]>(dsm + 2 * sizeof(T) * DK * DT);
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const size_t i0 = (size_t) blockIdx.y * DT, j0 = (size_t) blockIdx.x * DT;
    // loads: A tile 128 rows x 16 k, thread t takes row t >> 1 and the 8 k
    // from (t & 1) * 8; B tile 16 rows x 128, thread t takes row t >> 4 and
    // columns (t & 15) + 16 q, q < 8 (a half warp reads 16 consecutive)
    const int ar = tid >> 1, ak = (tid & 1) * 8;
    const int br = tid >> 4, bc = tid & 15;
    T ra[8], rb[8];
    auto load = [&](int k0) {
        const T *pa = A + (i0 + ar) * ld + k0 + ak;
        const T *pb = B + (size_t) (k0 + br) * ld + j0 + bc;
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            ra[q] = __ldg(pa + q);
            rb[q] = __ldg(pb + 16 * q);
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            As[buf][ak + q][ar] = ra[q];
            Bs[buf][br][bc + 16 * q] = rb[q];
        }
    };
    T acc[8][8];
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
        for (int n = 0; n < 8; ++n)
            acc[m][n] = T(0);
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < Kp; k0 += DK)
    {
        const bool more = k0 + DK < Kp;
        if (more)
            load(k0 + DK);
#pragma unroll
        for (int k = 0; k < DK; ++k)
        {
            T a[8], b[8];
#pragma unroll
            for (int m = 0; m < 8; ++m)
                a[m] = As[buf][k][ty + 16 * m];
#pragma unroll
            for (int n = 0; n < 8; ++n)
                b[n] = Bs[buf][k][tx + 16 * n];
#pragma unroll
            for (int m = 0; m < 8; ++m)
#pragma unroll
                for (int n = 0; n < 8; ++n)
                    acc[m][n] = fma_t(a[m], b[n], acc[m][n]);
        }
        if (more)
        {
            store(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
        for (int n = 0; n < 8; ++n)
            Cm[(i0 + ty + 16 * m) * ld + j0 + tx + 16 * n] = acc[m][n];
}

template <typename T> __device__ __forceinline__ bool above_d(T x, double thr);
template <> __device__ __forceinline__ bool above_d<double>(double x, double thr) { return fabs(x) > thr; }
template <> __device__ __forceinline__ bool above_d<float>(float x, double thr) { return fabsf(x) > (float) thr; }

// Row i of C from the image: the diagonal when touched, other columns when
// above the threshold, ascending; one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) dense_compact_kernel(const T *img, size_t ld, int nrows, int ncols,
                                                            const int *touched, double thr, T *Cv, int *Ci, int *Cn,
                                                            int ldc, int Mc, double *dC, DenseFlags *flags)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nrows; i += warps)
    {
        const T *row = img + (size_t) i * ld;
        const bool dt = touched[i] != 0;
        int n = 0;
        for (int b = 0; b < ncols; b += 32)
        {
            const int k = b + lane;
            bool keep = false;
            T x = T(0);
            if (k < ncols)
            {
                x = row[k];
                keep = k == i ? dt : above_d<T>(x, thr);
            }
            const unsigned bal = __ballot_sync(FULL, keep);
            const int pos = n + __popc(bal & lanemask_lt());
            if (keep && pos < Mc)
            {
                Ci[(size_t) i * ldc + pos] = k;
                Cv[(size_t) i * ldc + pos] = x;
            }
            n += __popc(bal);
        }
        if (lane == 0)
        {
            Cn[i] = min(n, Mc);
            atomicMax(&flags->max_width, n);
            if (n > Mc)
                atomicExch(&flags->overflow, 1);
            if (dC)
                dC[i] = (dt && i < ncols) ? (double) row[i] : 0.0;
        }
    }
}

bool g_dense_tier = true;

template <typename T>
bool dense_typed(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C, double thr,
                 double *trace, int *required_M)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const int NA = A->N, ncols = B->N > C->N ? B->N : C->N;
    const int dim = NA > ncols ? NA : ncols;
    const size_t ld = (size_t) b200_round_up(dim > B->N ? dim : B->N, DT);
    const size_t img = ld * ld * sizeof(T);
    const bool same = A == B;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t off_b = al(img);
    const size_t off_c = al(off_b + (same ? 0 : img));
    const size_t off_p = al(off_c + img);
    const size_t off_t = al(off_p + ld * ld);
    const size_t off_d = al(off_t + (size_t) NA * sizeof(int));
    const size_t total = al(off_d + (size_t) 2 * NA * sizeof(double));
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(total));
    if (!scr)
        return false;
    T *DA = reinterpret_cast<T *>(scr);
    T *DB = same ? DA : reinterpret_cast<T *>(scr + off_b);
    T *DC = reinterpret_cast<T *>(scr + off_c);
    unsigned char *pat = scr + off_p;
    int *touched = reinterpret_cast<int *>(scr + off_t);
    double *dA = reinterpret_cast<double *>(scr + off_d);
    double *dC = dA + NA;
    unsigned char *small = static_cast<unsigned char *>(c->d_small) + 20480;
    DenseFlags *flags = reinterpret_cast<DenseFlags *>(small);
    double *dtrace = reinterpret_cast<double *>(small + 64);
    if (!CUDA_OK(cudaMemsetAsync(small, 0, 128, c->stream)) ||
        !CUDA_OK(cudaMemsetAsync(DA, 0, img, c->stream)) ||
        (!same && !CUDA_OK(cudaMemsetAsync(DB, 0, img, c->stream))) ||
        !CUDA_OK(cudaMemsetAsync(pat, 0, ld * ld, c->stream)))
        return false;
    const int wgrid = max(1, min(b200_ceil_div(dim, 8), c->sm_count * 16));
    if (!same)
    {
        dense_scatter_kernel<T><<<wgrid, 256, 0, c->stream>>>(static_cast<const T *>(A->d_value), A->d_index, A->d_nnz,
                                                              A->ld, NA, B->N, DA, ld, nullptr, flags);
        if (!LAUNCH_OK("dense_scatter_kernel"))
            return false;
    }
    dense_scatter_kernel<T><<<wgrid, 256, 0, c->stream>>>(static_cast<const T *>(B->d_value), B->d_index, B->d_nnz,
                                                          B->ld, B->N, ncols, DB, ld, pat, flags);
    if (!LAUNCH_OK("dense_scatter_kernel"))
        return false;
    dense_diag_kernel<T><<<wgrid, 256, 0, c->stream>>>(static_cast<const T *>(A->d_value), A->d_index, A->d_nnz,
                                                       A->ld, NA, B->N, pat, ld, touched, trace ? dA : nullptr);
    if (!LAUNCH_OK("dense_diag_kernel"))
        return false;
    const dim3 grid((unsigned) (ld / DT), (unsigned) (ld / DT));
    const size_t smemG = 4 * sizeof(T) * DK * DT;
    if (!CUDA_OK(cudaFuncSetAttribute(dense_gemm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemG)))
        return false;
    dense_gemm_kernel<T><<<grid, DTHREADS, smemG, c->stream>>>(DA, DB, DC, ld, (int) ld);
    if (!LAUNCH_OK("dense_gemm_kernel"))
        return false;
    dense_compact_kernel<T><<<wgrid, 256, 0, c->stream>>>(DC, ld, NA, ncols, touched, thr, static_cast<T *>(C->d_value),
                                                          C->d_index, C->d_nnz, C->ld, C->M, trace ? dC : nullptr,
                                                          flags);
    if (!LAUNCH_OK("dense_compact_kernel"))
        return false;
    if (trace)
    {
        b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(dA, dC, NA, dtrace);
        if (!LAUNCH_OK("b200_sum_rows_kernel"))
            return false;
    }
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 20480;
    if (!CUDA_OK(cudaMemcpyAsync(pin, small, 128, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    const DenseFlags *hf = reinterpret_cast<const DenseFlags *>(pin);
    if (required_M)
        *required_M = hf->max_width;
    if (hf->bad_input)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply: a column index or row length of an input is out of range");
        return false;
    }
    if (trace)
        memcpy(trace, pin + 64, 2 * sizeof(double));
    if (hf->overflow)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "Number of non-zeroes per row > M, Increase M (need %d, M = %d)",
                       hf->max_width, C->M);
        return false;
    }
    return true;
}

} // namespace

// The dense tier applies when both operands' rows fill at least 40 % of
// their columns on average (there the GEMM beats the sparse kernels), the
// threshold is >= 0, and the three images (and B's pattern) take at most
// 64 GiB.  The row totals cost one small reduction and a synchronisation,
// and are only looked at when M allows rows that wide.
bool ell_dense_fits(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C, double thr)
{
    if (!g_dense_tier || !(thr >= 0.0) || A->N < 1024)
        return false;
    const int ncols = B->N > C->N ? B->N : C->N;
    if ((double) A->M < 0.4 * ncols || (double) B->M < 0.4 * ncols)
        return false;
    const size_t ld = (size_t) b200_round_up(A->N > ncols ? A->N : ncols, DT);
    const size_t bytes = ld * ld * (3 * prec_size(A->matrix_precision) + 1);
    if (bytes > ((size_t) 64 << 30))
        return false;
    long long ta = 0, tb = 0;
    int wa = 0, wb = 0;
    if (!ell_nnz_total(A, &ta, &wa) || (B != A && !ell_nnz_total(B, &tb, &wb)))
        return false;
    if (B == A)
        tb = ta;
    return (double) ta >= 0.4 * (double) A->N * ncols && (double) tb >= 0.4 * (double) B->N * ncols;
}

bool ell_multiply_dense(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C, double thr,
                        double *trace, int *required_M)
{
    return A->matrix_precision == double_real ? dense_typed<double>(A, B, C, thr, trace, required_M)
                                              : dense_typed<float>(A, B, C, thr, trace, required_M);
}

// Allows (1, the default) or forbids (0) the dense tier; returns the previous setting.
extern "C" BML_B200_API int bml_b200_set_dense_tier(int allow)
{
    const int old = g_dense_tier ? 1 : 0;
    g_dense_tier = allow != 0;
    return old;
}
