// ELLPACK operations on rows too wide for the shared-memory hash kernels of
// ellpack_ops.cu (rows of many thousand entries: SP2 iterates that have
// filled in).  Each works through a dense image of one operand's rows in
// device memory (N x N values, zeros where nothing is stored), so a column's
// entry is found by one load instead of a hash lookup:
//   add           A <- alpha A + beta B (ellpack/bml_add_ellpack_typed.c:50-216):
//                 the image takes x = alpha a for A's entries, then
//                 x = x + beta b for B's, each rounded to the matrix precision
//                 exactly as the reference rounds it, and the row is rebuilt
//                 from the image keeping |x| > threshold, in ascending column
//                 order (the reference lists A's columns, then B's new ones);
//   trace_mult    sum_ij A_ij B_ij (ellpack/bml_trace_ellpack_typed.c:103-162);
//   fnorm2        ||A - B||_F by the reference's rule (ellpack/bml_norm_ellpack_typed.c);
//   restrict      S's values on P's pattern, in P's order.
// The sums run in another order than the hash kernels' (rows summed in FP64).
#include "device_util.cuh"

using namespace b200;

namespace {

struct WideFlags
{
    int overflow;
    int bad_input;
};

// mode 0: img = v; mode 1: img = (T)(alpha v); mode 2: img = (T)(img + alpha v)
// (C evaluation of `x = alpha * a` and `x = x + beta * b` with a double
// scalar).  One warp per row; entries outside [0, ncols) raise bad_input.
template <typename T>
__global__ void __launch_bounds__(256) wide_image_kernel(const T *v, const int *ix, const int *nz, int ld, int N,
                                                         int ncols, T *img, size_t ldi, int mode, double alpha,
                                                         WideFlags *flags)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = nz[i];
        if (n < 0 || n > ld)
        {
            if (lane == 0)
                atomicExch(&flags->bad_input, 1);
            continue;
        }
        for (int p = lane; p < n; p += 32)
        {
            const int k = ix[(size_t) i * ld + p];
            if (k < 0 || k >= ncols)
            {
                atomicExch(&flags->bad_input, 1);
                continue;
            }
            T *x = img + (size_t) i * ldi + k;
            const T a = v[(size_t) i * ld + p];
            if (mode == 0)
                *x = a;
            else if (mode == 1)
                *x = axpy_d(T(0), alpha, a);
            else
                *x = axpy_d(*x, alpha, a);
        }
    }
}

// Rows of A rebuilt from the image: |x| > threshold, ascending; one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) wide_add_compact_kernel(const T *img, size_t ldi, int N, int ncols, double thr,
                                                               T *Av, int *Ai, int *An, int lda, int Ma,
                                                               WideFlags *flags)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const T thr_t = (T) thr;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        int n = 0;
        for (int b = 0; b < ncols; b += 32)
        {
            const int k = b + lane;
            const T x = k < ncols ? img[(size_t) i * ldi + k] : T(0);
            const bool keep = k < ncols && fabs(x) > thr_t;
            const unsigned bal = __ballot_sync(FULL, keep);
            const int pos = n + __popc(bal & lanemask_lt());
            if (keep && pos < Ma)
            {
                Ai[(size_t) i * lda + pos] = k;
                Av[(size_t) i * lda + pos] = x;
            }
            n += __popc(bal);
        }
        if (lane == 0)
        {
            An[i] = min(n, Ma);
            if (n > Ma)
                atomicExch(&flags->overflow, 1);
        }
    }
}

// kind 0: rows[i] = sum over A's entries of a * b (b from the image of B);
// kind 1: rows[i] = sum over A's entries of (a - b)^2;
// kind 2: rows[i] += sum over B's entries (here `A`) whose image value (of
//         the other matrix) is 0 of b^2.  One warp per row.
template <typename T>
__global__ void __launch_bounds__(256) wide_sum_kernel(const T *Av, const int *Ai, const int *An, int lda, int N,
                                                       int ncols, const T *img, size_t ldi, int kind, double *rows)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        double s = 0.0;
        if (n >= 0 && n <= lda)
            for (int p = lane; p < n; p += 32)
            {
                const int k = Ai[(size_t) i * lda + p];
                if (k < 0 || k >= ncols)
                    continue;
                const T a = Av[(size_t) i * lda + p];
                const T r = img[(size_t) i * ldi + k];
                if (kind == 0)
                    s += (double) mul_rn(a, r);
                else if (kind == 1)
                {
                    const T d = a - r;
                    s += (double) (d * d);
                }
                else if (r == T(0))
                    s += (double) (a * a);
            }
        for (int o = 16; o; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0)
            rows[i] = kind == 2 ? rows[i] + s : s;
    }
}

// O <- S's values (image) on P's pattern, in P's order; one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) wide_restrict_kernel(const T *img, size_t ldi, int ncols, const int *Pi,
                                                            const int *Pn, int ldp, T *Ov, int *Oi, int *On, int ldo,
                                                            int N)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int np = Pn[i];
        for (int p = lane; p < np; p += 32)
        {
            const int k = Pi[(size_t) i * ldp + p];
            Oi[(size_t) i * ldo + p] = k;
            Ov[(size_t) i * ldo + p] = (k >= 0 && k < ncols) ? img[(size_t) i * ldi + k] : T(0);
        }
        if (lane == 0)
            On[i] = np;
    }
}

struct Image
{
    unsigned char *base = nullptr;
    size_t ldi = 0;
    WideFlags *flags = nullptr;
    double *rows = nullptr;
};

// A zeroed N x ncols image of the given precision, a row-sum array and the
// flags, in the scratch arena; false (error recorded) when it exceeds 64 GiB.
bool get_image(B200Context *c, int N, int ncols, size_t sz, Image *im)
{
    im->ldi = (size_t) b200_round_up(ncols, 32);
    const size_t bytes = (size_t) N * im->ldi * sz;
    if (bytes > ((size_t) 64 << 30))
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "rows too wide: a dense image of %d x %d", N, ncols);
        return false;
    }
    const size_t off_rows = (bytes + 255) & ~size_t(255);
    im->base = static_cast<unsigned char *>(b200_scratch(off_rows + (size_t) N * sizeof(double)));
    if (!im->base)
        return false;
    im->rows = reinterpret_cast<double *>(im->base + off_rows);
    im->flags = reinterpret_cast<WideFlags *>(static_cast<unsigned char *>(c->d_small) + 24576);
    return CUDA_OK(cudaMemsetAsync(im->base, 0, bytes, c->stream)) &&
           CUDA_OK(cudaMemsetAsync(im->flags, 0, sizeof(WideFlags), c->stream));
}

bool read_flags(B200Context *c, WideFlags *out)
{
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 24576;
    if (!CUDA_OK(cudaMemcpyAsync(pin, static_cast<unsigned char *>(c->d_small) + 24576, sizeof(WideFlags),
                                 cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    memcpy(out, pin, sizeof(WideFlags));
    if (out->bad_input)
    {
        b200_set_error(BML_B200_ERR_INVALID, "a column index or row length of an input is out of range");
        return false;
    }
    return true;
}

int wgrid(B200Context *c, int N)
{
    return max(1, min(b200_ceil_div(N, 8), c->sm_count * 16));
}

template <typename T>
bool add_typed(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double alpha, double beta, double thr)
{
    B200Context *c = b200_ctx();
    Image im;
    const int ncols = A->N > B->N ? A->N : B->N;
    if (!c || !get_image(c, A->N, ncols, sizeof(T), &im))
        return false;
    T *img = reinterpret_cast<T *>(im.base);
    const int g = wgrid(c, A->N);
    if (alpha > 0.0 || alpha < 0.0)
    {
        wide_image_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(A->d_value), A->d_index, A->d_nnz,
                                                       A->ld, A->N, ncols, img, im.ldi, 1, alpha, im.flags);
        if (!LAUNCH_OK("wide_image_kernel"))
            return false;
    }
    if (beta > 0.0 || beta < 0.0)
    {
        wide_image_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(B->d_value), B->d_index, B->d_nnz,
                                                       B->ld, B->N, ncols, img, im.ldi, 2, beta, im.flags);
        if (!LAUNCH_OK("wide_image_kernel"))
            return false;
    }
    wide_add_compact_kernel<T><<<g, 256, 0, c->stream>>>(img, im.ldi, A->N, ncols, thr, static_cast<T *>(A->d_value),
                                                         A->d_index, A->d_nnz, A->ld, A->M, im.flags);
    if (!LAUNCH_OK("wide_add_compact_kernel"))
        return false;
    WideFlags f;
    if (!read_flags(c, &f))
        return false;
    if (f.overflow)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "add: a row of the sum needs more than M=%d entries", A->M);
        return false;
    }
    return true;
}

template <typename T>
bool sum_typed(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, int kind, double *result)
{
    B200Context *c = b200_ctx();
    Image im;
    const int ncols = A->N > B->N ? A->N : B->N;
    if (!c || !get_image(c, A->N, ncols, sizeof(T), &im))
        return false;
    T *img = reinterpret_cast<T *>(im.base);
    const int g = wgrid(c, A->N);
    // image of B; A's entries read it (trace_mult: kind 0; fnorm2: kind 1)
    wide_image_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(B->d_value), B->d_index, B->d_nnz, B->ld,
                                                   B->N, ncols, img, im.ldi, 0, 0.0, im.flags);
    wide_sum_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(A->d_value), A->d_index, A->d_nnz, A->ld,
                                                 A->N, ncols, img, im.ldi, kind, im.rows);
    if (!LAUNCH_OK("wide_sum_kernel"))
        return false;
    if (kind == 1)
    {
        // fnorm2: B's entries where A holds 0, through an image of A
        if (!CUDA_OK(cudaMemsetAsync(img, 0, (size_t) A->N * im.ldi * sizeof(T), c->stream)))
            return false;
        wide_image_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(A->d_value), A->d_index, A->d_nnz,
                                                       A->ld, A->N, ncols, img, im.ldi, 0, 0.0, im.flags);
        wide_sum_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(B->d_value), B->d_index, B->d_nnz, B->ld,
                                                     B->N, ncols, img, im.ldi, 2, im.rows);
        if (!LAUNCH_OK("wide_sum_kernel"))
            return false;
    }
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 24576 + 64);
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(im.rows, nullptr, A->N, out);
    if (!LAUNCH_OK("b200_sum_rows_kernel"))
        return false;
    WideFlags f;
    if (!read_flags(c, &f))
        return false;
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 24576 + 64;
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, sizeof(double), cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    memcpy(result, pin, sizeof(double));
    return true;
}

template <typename T>
bool restrict_typed(bml_matrix_ellpack_t *S, bml_matrix_ellpack_t *P, bml_matrix_ellpack_t *O)
{
    B200Context *c = b200_ctx();
    Image im;
    const int ncols = S->N;
    if (!c || !get_image(c, S->N, ncols, sizeof(T), &im))
        return false;
    T *img = reinterpret_cast<T *>(im.base);
    const int g = wgrid(c, S->N);
    wide_image_kernel<T><<<g, 256, 0, c->stream>>>(static_cast<const T *>(S->d_value), S->d_index, S->d_nnz, S->ld,
                                                   S->N, ncols, img, im.ldi, 0, 0.0, im.flags);
    wide_restrict_kernel<T><<<g, 256, 0, c->stream>>>(img, im.ldi, ncols, P->d_index, P->d_nnz, P->ld,
                                                      static_cast<T *>(O->d_value), O->d_index, O->d_nnz, O->ld,
                                                      S->N);
    if (!LAUNCH_OK("wide_restrict_kernel"))
        return false;
    WideFlags f;
    return read_flags(c, &f);
}

} // namespace

bool ell_add_wide(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double alpha, double beta, double threshold)
{
    return A->matrix_precision == double_real ? add_typed<double>(A, B, alpha, beta, threshold)
                                              : add_typed<float>(A, B, alpha, beta, threshold);
}

bool ell_trace_mult_wide(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *trace)
{
    return A->matrix_precision == double_real ? sum_typed<double>(A, B, 0, trace) : sum_typed<float>(A, B, 0, trace);
}

bool ell_fnorm2_wide(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *result)
{
    double ss = 0.0;
    const bool ok = A->matrix_precision == double_real ? sum_typed<double>(A, B, 1, &ss) : sum_typed<float>(A, B, 1, &ss);
    if (ok)
        *result = sqrt(ss);
    return ok;
}

bool ell_restrict_wide(bml_matrix_ellpack_t *S, bml_matrix_ellpack_t *P, bml_matrix_ellpack_t *O)
{
    return S->matrix_precision == double_real ? restrict_typed<double>(S, P, O) : restrict_typed<float>(S, P, O);
}
