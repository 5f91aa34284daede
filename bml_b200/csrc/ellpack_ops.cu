// ELLPACK-R bandwidth-bound operations around the product: add, add_identity,
// scale, threshold, trace, trace_mult, transpose, copy, Gershgorin bounds.
// Each kernel reproduces the reference loop's arithmetic and output order.
#include "device_util.cuh"

#include <cfloat>
#include <cstring>

using namespace b200;

// ---------------------------------------------------------------------------
// Reductions shared by several operations.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) b200_sum_rows_kernel(const double *a, const double *b,
                                                            int n, double *out)
{
    __shared__ double sa[1024], sb[1024];
    const int t = threadIdx.x;
    const int per = b200_ceil_div(n, 1024);
    double xa = 0.0, xb = 0.0;
    for (int r = t * per; r < min(n, (t + 1) * per); ++r)
    {
        if (a)
            xa += a[r];
        if (b)
            xb += b[r];
    }
    sa[t] = xa;
    sb[t] = xb;
    __syncthreads();
    for (int s = 512; s; s >>= 1)
    {
        if (t < s)
        {
            sa[t] += sa[t + s];
            sb[t] += sb[t + s];
        }
        __syncthreads();
    }
    if (t == 0)
    {
        out[0] = sa[0];
        out[1] = sb[0];
    }
}

__global__ void __launch_bounds__(1024) b200_maxmin_rows_kernel(const double *hi, const double *lo,
                                                               int n, double init_max,
                                                               double init_min, double *out)
{
    __shared__ double smax[1024], smin[1024];
    const int t = threadIdx.x;
    double mx = init_max, mn = init_min;
    for (int r = t; r < n; r += 1024)
    {
        mx = fmax(mx, hi[r]);
        mn = fmin(mn, lo[r]);
    }
    smax[t] = mx;
    smin[t] = mn;
    __syncthreads();
    for (int s = 512; s; s >>= 1)
    {
        if (t < s)
        {
            smax[t] = fmax(smax[t], smax[t + s]);
            smin[t] = fmin(smin[t], smin[t + s]);
        }
        __syncthreads();
    }
    if (t == 0)
    {
        out[0] = smax[0];
        out[1] = smin[0];
    }
}

namespace {

inline int rows_grid(B200Context *c, int N, int rows_per_block)
{
    return max(1, min(b200_ceil_div(N, rows_per_block), c->sm_count * 16));
}

// ---------------------------------------------------------------------------
// add: A <- alpha*A + beta*B, threshold without diagonal exemption.
// Reference: ellpack/bml_add_ellpack_typed.c:50-216.  Per row: A's columns in
// A's order (x = 0 + alpha*a), then B's (x += beta*b; new columns appended in
// B's order); kept when |x| > threshold.  A term is skipped entirely when its
// scalar is 0.  One team of W warps per row; A's row is staged in shared
// memory with a hash from column to position, so the row is rewritten in
// place only after it has been read.
// Shared memory per team: keys[TS] pos[TS] xa[ldA](T) ka[ldA] newpos[ldB] cnt.
// ---------------------------------------------------------------------------
constexpr int ADD_U = 8; // entries per thread in flight in the add's loads

template <typename T, int W>
__global__ void __launch_bounds__(W * 32) add_kernel(T *Av, int *Ai, int *An, int lda, int Ma,
                                                   const T *Bv, const int *Bi, const int *Bn,
                                                   int ldb, int N, double alpha, double beta,
                                                   double thr, int logts, int *overflow)
{
    constexpr int NT = W * 32;
    extern __shared__ __align__(128) unsigned char smem[];
    const int TS = 1 << logts;
    const unsigned mask = TS - 1;
    T *xa = reinterpret_cast<T *>(smem);    // A's entries, then x = alpha*a (+ beta*b)
    T *newx = xa + lda;                      // B's new entries: x = beta*b, by warp segment
    int *ka = reinterpret_cast<int *>(newx + ldb);
    int *keys = ka + lda;
    int *pos = keys + TS;
    int *newk = pos + TS;
    int *cnt = newk + ldb; // [W]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    const T thr_t = (T) thr;
    const bool use_a = alpha > 0.0 || alpha < 0.0;
    const bool use_b = beta > 0.0 || beta < 0.0;

    for (int i = blockIdx.x; i < N; i += gridDim.x)
    {
        for (int s = tid; s < TS; s += NT)
            keys[s] = B200_EMPTY_KEY;
        __syncthreads();
        const int na = use_a ? An[i] : 0;
        const int nb = use_b ? Bn[i] : 0;
        // A's row into shared memory: x = 0 + alpha*a, column -> position
        // (ADD_U entries per thread loaded before any is stored)
        for (int p0 = 0; p0 < na; p0 += NT * ADD_U)
        {
            int kk[ADD_U];
            T aa[ADD_U];
#pragma unroll
            for (int u = 0; u < ADD_U; ++u)
            {
                const int p = p0 + u * NT + tid;
                kk[u] = p < na ? Ai[(size_t) i * lda + p] : 0;
                aa[u] = p < na ? Av[(size_t) i * lda + p] : T(0);
            }
#pragma unroll
            for (int u = 0; u < ADD_U; ++u)
            {
                const int p = p0 + u * NT + tid;
                if (p < na)
                {
                    ka[p] = kk[u];
                    xa[p] = axpy_d(T(0), alpha, aa[u]);
                    hash_put(keys, pos, mask, kk[u], p);
                }
            }
        }
        __syncthreads();
        // B's row, one contiguous segment per warp: a column of A's row takes
        // x + beta*b (one writer: B's columns are distinct); a new column is
        // listed at its segment's start, in B order
        const int seg = b200_round_up(b200_ceil_div(max(nb, 1), W), 32);
        const int s0 = min(warp * seg, nb), s1 = min(s0 + seg, nb);
        int local = 0;
        for (int q0 = s0; q0 < s1; q0 += 32 * ADD_U)
        {
            int kk[ADD_U];
            T bb[ADD_U];
#pragma unroll
            for (int u = 0; u < ADD_U; ++u)
            {
                const int q = q0 + u * 32 + lane;
                kk[u] = q < s1 ? Bi[(size_t) i * ldb + q] : 0;
                bb[u] = q < s1 ? Bv[(size_t) i * ldb + q] : T(0);
            }
#pragma unroll
            for (int u = 0; u < ADD_U; ++u)
            {
                const int q = q0 + u * 32 + lane;
                bool isnew = false;
                if (q < s1)
                {
                    const int p = hash_get(keys, pos, mask, kk[u]);
                    if (p >= 0)
                        xa[p] = axpy_d(xa[p], beta, bb[u]);
                    else
                        isnew = true;
                }
                const unsigned bal = __ballot_sync(FULL, isnew);
                if (isnew)
                {
                    const int at = s0 + local + __popc(bal & lanemask_lt());
                    newk[at] = kk[u];
                    newx[at] = axpy_d(T(0), beta, bb[u]);
                }
                local += __popc(bal);
            }
        }
        if (lane == 0)
            cnt[warp] = local;
        __syncthreads();
        int npre[W];
        int nnew = 0;
#pragma unroll
        for (int w = 0; w < W; ++w)
        {
            npre[w] = nnew;
            nnew += cnt[w];
        }
        // the sum's entries: A's, then the new ones; e -> (column, value)
        auto entry = [&](int e, int &k, T &x) {
            if (e < na)
            {
                k = ka[e];
                x = xa[e];
                return;
            }
            const int r = e - na;
            int w = 0, base = 0;
#pragma unroll
            for (int v = 1; v < W; ++v)
                if (r >= npre[v])
                {
                    w = v;
                    base = npre[v];
                }
            const int at = w * seg + (r - base);
            k = newk[at];
            x = newx[at];
        };
        const int total = na + nnew;
        const int seg3 = b200_round_up(b200_ceil_div(max(total, 1), W), 32);
        const int e0 = min(warp * seg3, total), e1 = min(e0 + seg3, total);
        int kept = 0;
        for (int c0 = e0; c0 < e1; c0 += 32)
        {
            const int e = c0 + lane;
            int k = 0;
            T x = T(0);
            if (e < e1)
                entry(e, k, x);
            kept += __popc(__ballot_sync(FULL, e < e1 && fabs(x) > thr_t));
        }
        __syncthreads(); // every thread has read cnt
        if (lane == 0)
            cnt[warp] = kept;
        __syncthreads();
        int ll = 0, total_kept = 0;
#pragma unroll
        for (int w = 0; w < W; ++w)
        {
            ll += w < warp ? cnt[w] : 0;
            total_kept += cnt[w];
        }
        for (int c0 = e0; c0 < e1; c0 += 32)
        {
            const int e = c0 + lane;
            int k = 0;
            T x = T(0);
            if (e < e1)
                entry(e, k, x);
            const bool keep = e < e1 && fabs(x) > thr_t;
            const unsigned bal = __ballot_sync(FULL, keep);
            const int p = ll + __popc(bal & lanemask_lt());
            if (keep && p < Ma)
            {
                Av[(size_t) i * lda + p] = x;
                Ai[(size_t) i * lda + p] = k;
            }
            ll += __popc(bal);
        }
        if (tid == 0)
        {
            An[i] = min(total_kept, Ma);
            if (total_kept > Ma)
                atomicExch(overflow, 1);
        }
        __syncthreads(); // before the next row reuses the shared arrays
    }
}

// ---------------------------------------------------------------------------
// add_identity: A <- A + beta*I, then threshold.  Reference:
// ellpack/bml_add_ellpack_typed.c:420-549.  The last diagonal entry of the row
// gets x + beta (or (beta, i) is appended when the row has none); entries are
// kept when |x| > threshold, in row order.  One warp per row, in place.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void add_identity_kernel(T *Av, int *Ai, int *An, int ld, int M, int N, double beta,
                                    double thr, int *overflow)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const T thr_t = (T) thr;
    const bool use_b = beta > 0.0 || beta < 0.0;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        T *v = Av + (size_t) i * ld;
        int *ix = Ai + (size_t) i * ld;
        int diag = -1;
        for (int p = lane; p < n; p += 32)
            if (ix[p] == i)
                diag = p;
        for (int o = 16; o; o >>= 1)
            diag = max(diag, __shfl_xor_sync(FULL, diag, o));
        const int total = n + ((use_b && diag < 0) ? 1 : 0);
        int ll = 0;
        for (int c0 = 0; c0 < total; c0 += 32)
        {
            const int q = c0 + lane;
            T x = T(0);
            int k = 0;
            if (q < n)
            {
                x = v[q];
                k = ix[q];
                if (use_b && q == diag)
                    x = (T) __dadd_rn((double) x, beta);
            }
            else if (q < total)
            {
                x = (T) beta;
                k = i;
            }
            const bool keep = q < total && fabs(x) > thr_t;
            const unsigned bal = __ballot_sync(FULL, keep);
            const int p = ll + __popc(bal & lanemask_lt());
            if (keep && p < M)
            {
                v[p] = x;
                ix[p] = k;
            }
            ll += __popc(bal);
        }
        if (lane == 0)
        {
            An[i] = min(ll, M);
            if (ll > M)
                atomicExch(overflow, 1);
        }
    }
}

// ---------------------------------------------------------------------------
// threshold: stable in-place compaction keeping |v| > threshold (no diagonal
// exemption).  Reference: ellpack/bml_threshold_ellpack_typed.c:88-133 (in
// place) and :28-78 (into a new matrix).  One warp per row.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void threshold_kernel(const T *Av, const int *Ai, const int *An, int lda, T *Bv,
                                 int *Bi, int *Bn, int ldb, int N, double thr)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const T thr_t = (T) thr;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        const T *av = Av + (size_t) i * lda;
        const int *ai = Ai + (size_t) i * lda;
        // the next 32 entries are loaded before this chunk's are written
        // (in place, writes land below the chunk being read)
        T xn = T(0);
        int kn = 0;
        if (lane < n)
        {
            xn = av[lane];
            kn = ai[lane];
        }
        int ll = 0;
        for (int c0 = 0; c0 < n; c0 += 32)
        {
            const int q = c0 + lane;
            const T x = xn;
            const int k = kn;
            if (q + 32 < n)
            {
                xn = av[q + 32];
                kn = ai[q + 32];
            }
            const bool keep = q < n && fabs(x) > thr_t;
            const unsigned bal = __ballot_sync(FULL, keep);
            const int p = ll + __popc(bal & lanemask_lt());
            if (keep)
            {
                Bv[(size_t) i * ldb + p] = x;
                Bi[(size_t) i * ldb + p] = k;
            }
            ll += __popc(bal);
        }
        if (lane == 0)
            Bn[i] = ll;
    }
}

// One warp moves n 4-byte words from src to dst (both 16-byte aligned; rows
// start on 32-entry boundaries): 16-byte vectors, four in flight per lane,
// then the words past the last whole vector.
__device__ __forceinline__ void warp_copy_words(unsigned *dst, const unsigned *src, int n, int lane)
{
    const int nv = n >> 2;
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    int v = lane;
    for (; v + 96 < nv; v += 128)
    {
        const uint4 a = s4[v], b = s4[v + 32], c = s4[v + 64], d = s4[v + 96];
        d4[v] = a;
        d4[v + 32] = b;
        d4[v + 64] = c;
        d4[v + 96] = d;
    }
    for (; v < nv; v += 32)
        d4[v] = s4[v];
    for (int w = (nv << 2) + lane; w < n; w += 32)
        dst[w] = src[w];
}

// scale: B = s*A over the stored entries (the reference scales the padded
// N*M array with BLAS ?scal, bml_scale_ellpack_typed.c:85,119; entries past
// nnz are never read).  One warp per row.
template <typename T>
__global__ void scale_kernel(const T *Av, const int *Ai, const int *An, int lda, T *Bv, int *Bi,
                             int *Bn, int ldb, int N, T s, int copy_structure)
{
    constexpr int E = 16 / sizeof(T); // entries per 16-byte vector
    struct alignas(16) Vec
    {
        T v[E];
    };
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        const Vec *a = reinterpret_cast<const Vec *>(Av + (size_t) i * lda);
        Vec *b = reinterpret_cast<Vec *>(Bv + (size_t) i * ldb);
        const int nv = n / E;
        int v = lane;
        for (; v + 32 < nv; v += 64)
        {
            Vec x = a[v], y = a[v + 32];
#pragma unroll
            for (int e = 0; e < E; ++e)
            {
                x.v[e] = mul_rn(s, x.v[e]);
                y.v[e] = mul_rn(s, y.v[e]);
            }
            b[v] = x;
            b[v + 32] = y;
        }
        for (; v < nv; v += 32)
        {
            Vec x = a[v];
#pragma unroll
            for (int e = 0; e < E; ++e)
                x.v[e] = mul_rn(s, x.v[e]);
            b[v] = x;
        }
        for (int p = nv * E + lane; p < n; p += 32)
            Bv[(size_t) i * ldb + p] = mul_rn(s, Av[(size_t) i * lda + p]);
        if (copy_structure)
        {
            warp_copy_words(reinterpret_cast<unsigned *>(Bi + (size_t) i * ldb),
                            reinterpret_cast<const unsigned *>(Ai + (size_t) i * lda), n, lane);
            if (lane == 0)
                Bn[i] = n;
        }
    }
}

// copy: B <- A row by row (reference ellpack/bml_copy_ellpack_typed.c:86-148).
template <typename T>
__global__ void copy_kernel(const T *Av, const int *Ai, const int *An, int lda, T *Bv, int *Bi,
                            int *Bn, int ldb, int Mb, int N, int *overflow)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        const int m = min(n, Mb);
        warp_copy_words(reinterpret_cast<unsigned *>(Bv + (size_t) i * ldb),
                        reinterpret_cast<const unsigned *>(Av + (size_t) i * lda),
                        m * (int) (sizeof(T) / 4), lane);
        warp_copy_words(reinterpret_cast<unsigned *>(Bi + (size_t) i * ldb),
                        reinterpret_cast<const unsigned *>(Ai + (size_t) i * lda), m, lane);
        if (lane == 0)
        {
            Bn[i] = m;
            if (n > Mb)
                atomicExch(overflow, 1);
        }
    }
}

// trace: value of the first diagonal entry of each row (reference
// ellpack/bml_trace_ellpack_typed.c:74-88, `break` at the first match).
template <typename T>
__global__ void diag_kernel(const T *Av, const int *Ai, const int *An, int ld, int N, double *d)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        int first = n;
        for (int c0 = 0; c0 < n && first == n; c0 += 32)
        {
            const int q = c0 + lane;
            const unsigned bal = __ballot_sync(FULL, q < n && Ai[(size_t) i * ld + q] == i);
            if (bal)
                first = c0 + __ffs(bal) - 1;
        }
        if (lane == 0)
            d[i] = first < n ? (double) Av[(size_t) i * ld + first] : 0.0;
    }
}

// trace_mult: sum over row i and the columns c of A's row of A[i,c]*B[i,c]
// (the reference's bml_getVector_ellpack reads B's row i at A's columns,
// ellpack/bml_trace_ellpack_typed.c:145-158 with
// ellpack/bml_submatrix_ellpack_typed.c:380-406; a column absent from B's row
// contributes 0).  Per-row partial sums in FP64.  One warp per row, B's row in
// a shared-memory hash of 2^logts slots per warp.
template <typename T>
__global__ void trace_mult_kernel(const T *Av, const int *Ai, const int *An, int lda,
                                  const T *Bv, const int *Bi, const int *Bn, int ldb, int N,
                                  int logts, double *part)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int TS = 1 << logts;
    const unsigned mask = TS - 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *keys = reinterpret_cast<int *>(smem) + (size_t) warp * 2 * TS;
    int *pos = keys + TS;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        for (int s = lane; s < TS; s += 32)
            keys[s] = B200_EMPTY_KEY;
        __syncwarp();
        const int nb = Bn[i];
        for (int c0 = 0; c0 < nb; c0 += 32)
        {
            const int p = c0 + lane;
            if (p < nb)
                hash_put(keys, pos, mask, Bi[(size_t) i * ldb + p], p);
            __syncwarp();
        }
        __syncwarp();
        double s = 0.0;
        const int na = An[i];
        for (int p = lane; p < na; p += 32)
        {
            const int q = hash_get(keys, pos, mask, Ai[(size_t) i * lda + p]);
            if (q >= 0)
                s += (double) mul_rn(Av[(size_t) i * lda + p], Bv[(size_t) i * ldb + q]);
        }
        for (int o = 16; o; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0)
            part[i] = s;
        __syncwarp();
    }
}

// Gershgorin per row (reference ellpack/bml_normalize_ellpack_typed.c:82-175):
// radius = sum of |a| over off-diagonal entries, accumulated as
// `radius += (double) |a|` into a variable of the matrix precision; dvalue =
// the last diagonal entry; hi = dvalue + radius, lo = dvalue - radius in the
// matrix precision.
// One lane per row, so each row's sum runs in row order in one thread; the
// warp stages its 32 rows through shared memory 32 entries at a time, each
// row's entries read by one coalesced load.
constexpr int GER_WARPS = 4;

template <typename T>
__global__ void __launch_bounds__(GER_WARPS * 32) gershgorin_kernel(const T *Av, const int *Ai,
                                                                    const int *An, int ld, int N,
                                                                    double *hi, double *lo)
{
    __shared__ T tv[GER_WARPS][32][33];
    __shared__ unsigned char tdg[GER_WARPS][32][33]; // entry is on the diagonal
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int groups = (N + 31) / 32;
    for (int gi = blockIdx.x * GER_WARPS + w; gi < groups; gi += gridDim.x * GER_WARPS)
    {
        const int i = gi * 32 + lane; // this lane's row
        const int n = i < N ? An[i] : 0;
        int nmax = n;
#pragma unroll
        for (int o = 16; o; o >>= 1)
            nmax = max(nmax, __shfl_xor_sync(FULL, nmax, o));
        T radius = T(0), dvalue = T(0);
        for (int c0 = 0; c0 < nmax; c0 += 32)
        {
            // row r of the group: its entries c0 .. c0 + 31, lane = entry;
            // 16 rows' loads are issued before any is stored
            for (int r0 = 0; r0 < 32; r0 += 16)
            {
                T v[16];
                int k[16];
#pragma unroll
                for (int r = 0; r < 16; ++r)
                {
                    const int row = gi * 32 + r0 + r;
                    const int nr = __shfl_sync(FULL, n, r0 + r);
                    const int q = c0 + lane;
                    v[r] = T(0);
                    k[r] = -1;
                    if (row < N && q < nr)
                    {
                        v[r] = Av[(size_t) row * ld + q];
                        k[r] = Ai[(size_t) row * ld + q];
                    }
                }
#pragma unroll
                for (int r = 0; r < 16; ++r)
                {
                    tv[w][r0 + r][lane] = v[r];
                    tdg[w][r0 + r][lane] = k[r] == gi * 32 + r0 + r;
                }
            }
            __syncwarp();
            const int m = min(32, n - c0);
            for (int t = 0; t < m; ++t)
            {
                const T vt = tv[w][lane][t];
                if (tdg[w][lane][t])
                    dvalue = vt;
                else
                    radius = (T) __dadd_rn((double) radius, (double) fabs(vt));
            }
            __syncwarp();
        }
        if (i < N)
        {
            hi[i] = (double) add_rn(dvalue, radius);
            lo[i] = (double) add_rn(dvalue, (T) -radius);
        }
    }
}

// transpose, step 1: count entries per column and scatter (row, value) into
// the column's output row at an atomically reserved position.
template <typename T>
__global__ void transpose_scatter_kernel(const T *Av, const int *Ai, const int *An, int lda,
                                         int N, T *Bv, int *Bi, int *Bn, int ldb, int Mb,
                                         int *overflow)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        for (int p = lane; p < n; p += 32)
        {
            const int j = Ai[(size_t) i * lda + p];
            const int slot = atomicAdd(&Bn[j], 1);
            if (slot < Mb)
            {
                Bi[(size_t) j * ldb + slot] = i;
                Bv[(size_t) j * ldb + slot] = Av[(size_t) i * lda + p];
            }
            else
                atomicExch(overflow, 1);
        }
    }
}

// transpose, step 2: sort every output row by source row (the serial order of
// the reference's bml_transpose_new_ellpack, bml_transpose_ellpack_typed.c:
// 76-96, whose OpenMP version is otherwise nondeterministic).  One block per
// row, bitonic sort of (row, value) pairs in shared memory.
template <typename T>
__global__ void row_sort_kernel(T *Bv, int *Bi, int *Bn, int ldb, int Mb, int N, int pow2)
{
    extern __shared__ __align__(128) unsigned char smem[];
    T *sv = reinterpret_cast<T *>(smem);
    int *sk = reinterpret_cast<int *>(sv + pow2);
    for (int j = blockIdx.x; j < N; j += gridDim.x)
    {
        const int n = min(Bn[j], Mb);
        if (n <= 1)
        {
            if (threadIdx.x == 0)
                Bn[j] = n;
            continue;
        }
        int p2 = 1;
        while (p2 < n)
            p2 <<= 1;
        for (int t = threadIdx.x; t < p2; t += blockDim.x)
        {
            sk[t] = t < n ? Bi[(size_t) j * ldb + t] : 0x7fffffff;
            sv[t] = t < n ? Bv[(size_t) j * ldb + t] : T(0);
        }
        __syncthreads();
        for (int k = 2; k <= p2; k <<= 1)
            for (int s = k >> 1; s > 0; s >>= 1)
            {
                for (int t = threadIdx.x; t < p2; t += blockDim.x)
                {
                    const int u = t ^ s;
                    if (u > t)
                    {
                        const bool up = (t & k) == 0;
                        const int a = sk[t], b = sk[u];
                        if ((a > b) == up)
                        {
                            sk[t] = b;
                            sk[u] = a;
                            const T tv = sv[t];
                            sv[t] = sv[u];
                            sv[u] = tv;
                        }
                    }
                }
                __syncthreads();
            }
        for (int t = threadIdx.x; t < n; t += blockDim.x)
        {
            Bi[(size_t) j * ldb + t] = sk[t];
            Bv[(size_t) j * ldb + t] = sv[t];
        }
        if (threadIdx.x == 0)
            Bn[j] = n;
        __syncthreads();
    }
}

bool read_flag(B200Context *c, int *dflag, int *out)
{
    int *pin = reinterpret_cast<int *>(static_cast<unsigned char *>(c->pinned) + 2048);
    if (!CUDA_OK(cudaMemcpyAsync(pin, dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    *out = *pin;
    return true;
}

int *zeroed_flag(B200Context *c)
{
    int *f = reinterpret_cast<int *>(static_cast<unsigned char *>(c->d_small) + 2048);
    if (!CUDA_OK(cudaMemsetAsync(f, 0, sizeof(int), c->stream)))
        return nullptr;
    return f;
}

bool check_pair(const bml_matrix_ellpack_t *A, const bml_matrix_ellpack_t *B, const char *op)
{
    if (!A || !B)
    {
        b200_set_error(BML_B200_ERR_INVALID, "%s: NULL matrix", op);
        return false;
    }
    if (A->N != B->N || A->matrix_precision != B->matrix_precision)
    {
        b200_set_error(BML_B200_ERR_INVALID, "%s: matrices differ in size or precision", op);
        return false;
    }
    return true;
}

} // namespace

bool ell_add(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double alpha, double beta,
             double threshold)
{
    if (!check_pair(A, B, "add"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A) || !ell_to_device(B))
        return false;
    if (A == B)
    {
        // x = 0 + alpha*a, then x + beta*a: same arithmetic through a copy.
        bml_matrix_ellpack_t *T0 = ell_alloc(A->matrix_precision, A->N, A->M, A->distribution_mode, false);
        if (!T0)
            return false;
        bool ok = ell_copy(A, T0) && ell_add(A, T0, alpha, beta, threshold);
        ell_free(T0);
        return ok;
    }
    int *ovf = zeroed_flag(c);
    if (!ovf)
        return false;
    // the hash holds A's row at most half full
    const int need = 2 * A->M;
    int logts = 5;
    while ((1 << logts) < need)
        ++logts;
    const size_t sz = prec_size(A->matrix_precision);
    // xa[lda] newx[ldb] (matrix precision) | ka[lda] keys[TS] pos[TS] newk[ldb] cnt[8]
    const size_t smem = (size_t) (A->ld + B->ld) * (sz + 4) + ((size_t) 2 << logts) * 4 + 8 * 4 + 64;
    if (smem > c->smem_optin)
    {
        // rows too wide for the hash: through a dense image of the row sums
        // (unordered form; rows come out in ascending column order)
        if (!ell_x2_exact() && threshold >= 0.0)
        {
            const bool ok = ell_add_wide(A, B, alpha, beta, threshold);
            ell_mark_device(A);
            return ok;
        }
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "add: rows of width %d/%d exceed shared memory",
                       A->M, B->M);
        return false;
    }
    if (A->matrix_precision == double_real)
    {
        auto k = add_kernel<double, 8>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem);
        const int grid = min(A->N, c->sm_count * (occ > 0 ? occ : 1));
        k<<<grid, 256, smem, c->stream>>>(static_cast<double *>(A->d_value), A->d_index, A->d_nnz,
                                          A->ld, A->M, static_cast<const double *>(B->d_value),
                                          B->d_index, B->d_nnz, B->ld, A->N, alpha, beta,
                                          threshold, logts, ovf);
    }
    else
    {
        auto k = add_kernel<float, 8>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 256, smem);
        const int grid = min(A->N, c->sm_count * (occ > 0 ? occ : 1));
        k<<<grid, 256, smem, c->stream>>>(static_cast<float *>(A->d_value), A->d_index, A->d_nnz,
                                          A->ld, A->M, static_cast<const float *>(B->d_value),
                                          B->d_index, B->d_nnz, B->ld, A->N, alpha, beta,
                                          threshold, logts, ovf);
    }
    if (!LAUNCH_OK("add_kernel"))
        return false;
    ell_mark_device(A);
    int hov = 0;
    if (!read_flag(c, ovf, &hov))
        return false;
    if (hov)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "add: a row of the sum has more than M=%d entries",
                       A->M);
        return false;
    }
    return true;
}

bool ell_add_identity(bml_matrix_ellpack_t *A, double beta, double threshold)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    int *ovf = zeroed_flag(c);
    if (!ovf)
        return false;
    const int grid = rows_grid(c, A->N, 8);
    if (A->matrix_precision == double_real)
        add_identity_kernel<double><<<grid, 256, 0, c->stream>>>(
            static_cast<double *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->M, A->N, beta,
            threshold, ovf);
    else
        add_identity_kernel<float><<<grid, 256, 0, c->stream>>>(
            static_cast<float *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->M, A->N, beta,
            threshold, ovf);
    if (!LAUNCH_OK("add_identity_kernel"))
        return false;
    ell_mark_device(A);
    int hov = 0;
    if (!read_flag(c, ovf, &hov))
        return false;
    if (hov)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "add_identity: a row needs more than M=%d entries",
                       A->M);
        return false;
    }
    return true;
}

bool ell_scale(const void *scale, bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B)
{
    if (!check_pair(A, B, "scale"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A) || (B != A && !ell_to_device(B)))
        return false;
    if (B != A && B->M < A->M)
    {
        long long tot;
        int maxrow = 0;
        if (!ell_nnz_total(A, &tot, &maxrow))
            return false;
        if (maxrow > B->M)
        {
            b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "scale: output M=%d < row width %d", B->M,
                           maxrow);
            return false;
        }
    }
    const int grid = rows_grid(c, A->N, 8);
    const int copy = B != A;
    if (A->matrix_precision == double_real)
        scale_kernel<double><<<grid, 256, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<double *>(B->d_value), B->d_index, B->d_nnz, B->ld, A->N,
            *static_cast<const double *>(scale), copy);
    else
        scale_kernel<float><<<grid, 256, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<float *>(B->d_value), B->d_index, B->d_nnz, B->ld, A->N,
            *static_cast<const float *>(scale), copy);
    if (!LAUNCH_OK("scale_kernel"))
        return false;
    ell_mark_device(B);
    return true;
}

bool ell_threshold_new(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double threshold)
{
    if (!check_pair(A, B, "threshold"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A) || !ell_to_device(B))
        return false;
    const int grid = rows_grid(c, A->N, 8);
    if (A->matrix_precision == double_real)
        threshold_kernel<double><<<grid, 256, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<double *>(B->d_value), B->d_index, B->d_nnz, B->ld, A->N, threshold);
    else
        threshold_kernel<float><<<grid, 256, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<float *>(B->d_value), B->d_index, B->d_nnz, B->ld, A->N, threshold);
    if (!LAUNCH_OK("threshold_kernel"))
        return false;
    ell_mark_device(B);
    return true;
}

bool ell_threshold(bml_matrix_ellpack_t *A, double threshold)
{
    // Stable in-place compaction: every write lands at or before the position
    // being read within the same warp chunk, so aliasing A with B is safe.
    return ell_threshold_new(A, A, threshold);
}

bool ell_copy(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B)
{
    if (!check_pair(A, B, "copy"))
        return false;
    if (A == B)
        return true;
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    if (B->mirror == MIRROR_HOST_NEWER)
        B->mirror = MIRROR_SYNCED; // overwritten entirely below
    int *ovf = zeroed_flag(c);
    if (!ovf)
        return false;
    const int grid = rows_grid(c, A->N, 8);
    if (A->matrix_precision == double_real)
        copy_kernel<double><<<grid, 256, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<double *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, A->N, ovf);
    else
        copy_kernel<float><<<grid, 256, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<float *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, A->N, ovf);
    if (!LAUNCH_OK("copy_kernel"))
        return false;
    ell_mark_device(B);
    if (B->M >= A->M)
        return true;
    int hov = 0;
    if (!read_flag(c, ovf, &hov))
        return false;
    if (hov)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "copy: a row of A is wider than B's M=%d", B->M);
        return false;
    }
    return true;
}

bool ell_trace(bml_matrix_ellpack_t *A, double *trace)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    double *d = static_cast<double *>(b200_scratch((size_t) A->N * sizeof(double)));
    if (!d)
        return false;
    const int grid = rows_grid(c, A->N, 8);
    if (A->matrix_precision == double_real)
        diag_kernel<double><<<grid, 256, 0, c->stream>>>(static_cast<const double *>(A->d_value),
                                                         A->d_index, A->d_nnz, A->ld, A->N, d);
    else
        diag_kernel<float><<<grid, 256, 0, c->stream>>>(static_cast<const float *>(A->d_value),
                                                        A->d_index, A->d_nnz, A->ld, A->N, d);
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 3072);
    b200_count_launch(); // diag_kernel
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(d, nullptr, A->N, out);
    if (!LAUNCH_OK("trace kernels"))
        return false;
    double *pin = reinterpret_cast<double *>(static_cast<unsigned char *>(c->pinned) + 3072);
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    *trace = pin[0];
    return true;
}

bool ell_trace_mult(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *trace)
{
    if (!check_pair(A, B, "trace_mult"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A) || !ell_to_device(B))
        return false;
    double *part = static_cast<double *>(b200_scratch((size_t) A->N * sizeof(double)));
    if (!part)
        return false;
    int logts = 5;
    while ((1 << logts) < 2 * B->M)
        ++logts;
    int warps_per_block = 4;
    size_t smem = (size_t) warps_per_block * 2 * (1 << logts) * sizeof(int);
    while (smem > c->smem_optin && warps_per_block > 1)
    {
        warps_per_block >>= 1;
        smem >>= 1;
    }
    if (smem > c->smem_optin)
        return ell_trace_mult_wide(A, B, trace);
    const int grid = min(b200_ceil_div(A->N, warps_per_block), c->sm_count * 16);
    if (A->matrix_precision == double_real)
    {
        auto k = trace_mult_kernel<double>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<grid, 32 * warps_per_block, smem, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<const double *>(B->d_value), B->d_index, B->d_nnz, B->ld, A->N, logts, part);
    }
    else
    {
        auto k = trace_mult_kernel<float>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<grid, 32 * warps_per_block, smem, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<const float *>(B->d_value), B->d_index, B->d_nnz, B->ld, A->N, logts, part);
    }
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 3072);
    b200_count_launch(); // trace_mult_kernel
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(part, nullptr, A->N, out);
    if (!LAUNCH_OK("trace_mult kernels"))
        return false;
    double *pin = reinterpret_cast<double *>(static_cast<unsigned char *>(c->pinned) + 3072);
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    *trace = pin[0];
    return true;
}

bool ell_transpose_new(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B)
{
    if (!check_pair(A, B, "transpose"))
        return false;
    if (A == B)
    {
        b200_set_error(BML_B200_ERR_INVALID, "transpose: output aliases input");
        return false;
    }
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    if (B->mirror == MIRROR_HOST_NEWER)
        B->mirror = MIRROR_SYNCED;
    int *ovf = zeroed_flag(c);
    if (!ovf || !CUDA_OK(cudaMemsetAsync(B->d_nnz, 0, (size_t) B->N * sizeof(int), c->stream)))
        return false;
    const int grid = rows_grid(c, A->N, 8);
    int pow2 = 1;
    while (pow2 < B->M)
        pow2 <<= 1;
    const size_t sz = prec_size(A->matrix_precision);
    const size_t smem = (size_t) pow2 * (sz + 4);
    if (smem > c->smem_optin)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "transpose: M=%d too wide for the row sort", B->M);
        return false;
    }
    const int sgrid = min(B->N, c->sm_count * 8);
    if (A->matrix_precision == double_real)
    {
        transpose_scatter_kernel<double><<<grid, 256, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->N,
            static_cast<double *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, ovf);
        auto k = row_sort_kernel<double>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<sgrid, 256, smem, c->stream>>>(static_cast<double *>(B->d_value), B->d_index, B->d_nnz,
                                           B->ld, B->M, B->N, pow2);
    }
    else
    {
        transpose_scatter_kernel<float><<<grid, 256, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->N,
            static_cast<float *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, ovf);
        auto k = row_sort_kernel<float>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<sgrid, 256, smem, c->stream>>>(static_cast<float *>(B->d_value), B->d_index, B->d_nnz,
                                           B->ld, B->M, B->N, pow2);
    }
    b200_count_launch(); // transpose_scatter_kernel
    if (!LAUNCH_OK("transpose kernels"))
        return false;
    ell_mark_device(B);
    int hov = 0;
    if (!read_flag(c, ovf, &hov))
        return false;
    if (hov)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "transpose: a column of A has more than M=%d entries",
                       B->M);
        return false;
    }
    return true;
}

bool ell_gershgorin(bml_matrix_ellpack_t *A, double *bounds)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    double *hi = static_cast<double *>(b200_scratch((size_t) 2 * A->N * sizeof(double)));
    if (!hi)
        return false;
    double *lo = hi + A->N;
    const int grid = max(1, min(b200_ceil_div(A->N, 32 * GER_WARPS), c->sm_count * 8));
    if (A->matrix_precision == double_real)
        gershgorin_kernel<double><<<grid, GER_WARPS * 32, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->N, hi, lo);
    else
        gershgorin_kernel<float><<<grid, GER_WARPS * 32, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld, A->N, hi, lo);
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 3072);
    // emax starts at DBL_MIN and emin at DBL_MAX, as in the reference (:88-89).
    b200_count_launch(); // gershgorin_kernel
    b200_maxmin_rows_kernel<<<1, 1024, 0, c->stream>>>(hi, lo, A->N, DBL_MIN, DBL_MAX, out);
    if (!LAUNCH_OK("gershgorin kernels"))
        return false;
    double *pin = reinterpret_cast<double *>(static_cast<unsigned char *>(c->pinned) + 3072);
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    bounds[0] = pin[1]; // emin
    bounds[1] = pin[0]; // emax
    return true;
}

// ---------------------------------------------------------------------------
// Norms.  sum_squares: sum of a*a over the stored entries
// (ellpack/bml_norm_ellpack_typed.c:31-60); fnorm2: ||A - B||_F over A's
// entries, with B's entry of the same column or 0, plus B's entries whose
// column A lacks or holds as exactly 0 (:371-440).  Each product is formed in
// the matrix precision as in the reference; the sums are FP64, one per row,
// then added in a fixed order.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void sumsq_kernel(const T *V, const int *Nz, int ld, int N, double *rows)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        double s = 0.0;
        for (int p = lane; p < Nz[i]; p += 32)
        {
            const T x = V[(size_t) i * ld + p];
            s += (double) (x * x);
        }
        for (int o = 16; o; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0)
            rows[i] = s;
    }
}

// One block per row; tables map each row's columns to positions.
template <typename T>
__global__ void __launch_bounds__(256) fnorm2_kernel(const T *Av, const int *Ai, const int *An, int lda,
                                                     const T *Bv, const int *Bi, const int *Bn, int ldb,
                                                     int N, int logts, double *rows)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int TS = 1 << logts;
    const unsigned mask = TS - 1;
    int *ka = reinterpret_cast<int *>(smem);
    int *pa = ka + TS;
    int *kb = pa + TS;
    int *pb = kb + TS;
    __shared__ double part[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = blockIdx.x; i < N; i += gridDim.x)
    {
        for (int s = tid; s < TS; s += 256)
        {
            ka[s] = B200_EMPTY_KEY;
            kb[s] = B200_EMPTY_KEY;
        }
        __syncthreads();
        const int na = An[i], nb = Bn[i];
        // columns are distinct within a row, so each key is put once
        for (int p = tid; p < na; p += 256)
            hash_put(ka, pa, mask, Ai[(size_t) i * lda + p], p);
        for (int p = tid; p < nb; p += 256)
            hash_put(kb, pb, mask, Bi[(size_t) i * ldb + p], p);
        __syncthreads();
        double s = 0.0;
        for (int p = tid; p < na; p += 256)
        {
            const int q = hash_get(kb, pb, mask, Ai[(size_t) i * lda + p]);
            const T r = q >= 0 ? Bv[(size_t) i * ldb + q] : T(0);
            const T d = Av[(size_t) i * lda + p] - r;
            s += (double) (d * d);
        }
        for (int p = tid; p < nb; p += 256)
        {
            const int q = hash_get(ka, pa, mask, Bi[(size_t) i * ldb + p]);
            const T r = q >= 0 ? Av[(size_t) i * lda + q] : T(0);
            if (r == T(0))
            {
                const T x = Bv[(size_t) i * ldb + p];
                s += (double) (x * x);
            }
        }
        for (int o = 16; o; o >>= 1)
            s += __shfl_xor_sync(FULL, s, o);
        if (lane == 0)
            part[warp] = s;
        __syncthreads();
        if (tid == 0)
        {
            double t = 0.0;
            for (int w = 0; w < 8; ++w)
                t += part[w];
            rows[i] = t;
        }
        __syncthreads();
    }
}

// Entry-for-entry copy between precisions (round to nearest).
template <typename S, typename D>
__global__ void convert_kernel(const S *Av, const int *Ai, const int *An, int lda, D *Bv, int *Bi,
                               int *Bn, int ldb, int Mb, int N, int *overflow)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < N; i += warps)
    {
        const int n = An[i];
        const int m = min(n, Mb);
        for (int p = lane; p < m; p += 32)
        {
            Bv[(size_t) i * ldb + p] = (D) Av[(size_t) i * lda + p];
            Bi[(size_t) i * ldb + p] = Ai[(size_t) i * lda + p];
        }
        if (lane == 0)
        {
            Bn[i] = m;
            if (n > Mb)
                atomicExch(overflow, 1);
        }
    }
}

bool sum_rows_to_host(B200Context *c, double *rows, int N, double *result)
{
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 3072);
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(rows, nullptr, N, out);
    if (!LAUNCH_OK("b200_sum_rows_kernel"))
        return false;
    double *pin = reinterpret_cast<double *>(static_cast<unsigned char *>(c->pinned) + 3072);
    if (!CUDA_OK(cudaMemcpyAsync(pin, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream)) ||
        !b200_sync())
        return false;
    *result = pin[0];
    return true;
}

} // namespace

bool ell_sum_squares(bml_matrix_ellpack_t *A, double *result)
{
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    double *rows = static_cast<double *>(b200_scratch((size_t) A->N * sizeof(double)));
    if (!rows)
        return false;
    const int grid = rows_grid(c, A->N, 8);
    if (A->matrix_precision == double_real)
        sumsq_kernel<double><<<grid, 256, 0, c->stream>>>(static_cast<const double *>(A->d_value),
                                                          A->d_nnz, A->ld, A->N, rows);
    else
        sumsq_kernel<float><<<grid, 256, 0, c->stream>>>(static_cast<const float *>(A->d_value),
                                                         A->d_nnz, A->ld, A->N, rows);
    if (!LAUNCH_OK("sumsq_kernel"))
        return false;
    return sum_rows_to_host(c, rows, A->N, result);
}

bool ell_fnorm2(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, double *result)
{
    if (!check_pair(A, B, "fnorm2"))
        return false;
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A) || !ell_to_device(B))
        return false;
    int logts = 5;
    while ((1 << logts) < 2 * (A->M > B->M ? A->M : B->M))
        ++logts;
    const size_t smem = (size_t) 4 * (1 << logts) * sizeof(int);
    if (smem > c->smem_optin)
        return ell_fnorm2_wide(A, B, result);
    double *rows = static_cast<double *>(b200_scratch((size_t) A->N * sizeof(double)));
    if (!rows)
        return false;
    const int grid = max(1, min(A->N, c->sm_count * 8));
    if (A->matrix_precision == double_real)
    {
        auto k = fnorm2_kernel<double>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<grid, 256, smem, c->stream>>>(static_cast<const double *>(A->d_value), A->d_index, A->d_nnz,
                                          A->ld, static_cast<const double *>(B->d_value), B->d_index,
                                          B->d_nnz, B->ld, A->N, logts, rows);
    }
    else
    {
        auto k = fnorm2_kernel<float>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<grid, 256, smem, c->stream>>>(static_cast<const float *>(A->d_value), A->d_index, A->d_nnz,
                                          A->ld, static_cast<const float *>(B->d_value), B->d_index,
                                          B->d_nnz, B->ld, A->N, logts, rows);
    }
    if (!LAUNCH_OK("fnorm2_kernel"))
        return false;
    double ss = 0.0;
    if (!sum_rows_to_host(c, rows, A->N, &ss))
        return false;
    *result = sqrt(ss);
    return true;
}

bool ell_convert(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B)
{
    if (!A || !B || A->N != B->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "convert: matrices differ in size");
        return false;
    }
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(A))
        return false;
    if (B->mirror == MIRROR_HOST_NEWER)
        B->mirror = MIRROR_SYNCED; // overwritten entirely below
    int *ovf = zeroed_flag(c);
    if (!ovf)
        return false;
    const int grid = rows_grid(c, A->N, 8);
    const bool ad = A->matrix_precision == double_real, bd = B->matrix_precision == double_real;
    if (ad && bd)
        convert_kernel<double, double><<<grid, 256, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<double *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, A->N, ovf);
    else if (ad)
        convert_kernel<double, float><<<grid, 256, 0, c->stream>>>(
            static_cast<const double *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<float *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, A->N, ovf);
    else if (bd)
        convert_kernel<float, double><<<grid, 256, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<double *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, A->N, ovf);
    else
        convert_kernel<float, float><<<grid, 256, 0, c->stream>>>(
            static_cast<const float *>(A->d_value), A->d_index, A->d_nnz, A->ld,
            static_cast<float *>(B->d_value), B->d_index, B->d_nnz, B->ld, B->M, A->N, ovf);
    if (!LAUNCH_OK("convert_kernel"))
        return false;
    ell_mark_device(B);
    int hov = 0;
    if (!read_flag(c, ovf, &hov))
        return false;
    if (hov)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "convert: a row of A is wider than B's M=%d", B->M);
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// restrict: out takes P's pattern (P's columns, in P's order) with S's value
// at each of those columns, 0 where S has none.  Used by the SP2 adjoint to
// keep a gradient on the entries a thresholded product retained.  One block
// per row; P's row is hashed (column -> position) and S's row streams past.
// ---------------------------------------------------------------------------
namespace {

template <typename T>
__global__ void __launch_bounds__(256) restrict_kernel(const T *Sv, const int *Si, const int *Sn, int lds,
                                                       const int *Pi, const int *Pn, int ldp, T *Ov,
                                                       int *Oi, int *On, int ldo, int N, int logts)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int TS = 1 << logts;
    const unsigned mask = TS - 1;
    int *keys = reinterpret_cast<int *>(smem);
    int *pos = keys + TS;
    const int tid = threadIdx.x;
    for (int i = blockIdx.x; i < N; i += gridDim.x)
    {
        for (int s = tid; s < TS; s += 256)
            keys[s] = B200_EMPTY_KEY;
        __syncthreads();
        const int np = Pn[i];
        for (int p = tid; p < np; p += 256)
        {
            const int k = Pi[(size_t) i * ldp + p];
            Oi[(size_t) i * ldo + p] = k;
            Ov[(size_t) i * ldo + p] = T(0);
            hash_put(keys, pos, mask, k, p);
        }
        __syncthreads();
        const int ns = Sn[i];
        for (int p = tid; p < ns; p += 256)
        {
            const int q = hash_get(keys, pos, mask, Si[(size_t) i * lds + p]);
            if (q >= 0)
                Ov[(size_t) i * ldo + q] = Sv[(size_t) i * lds + p];
        }
        if (tid == 0)
            On[i] = np;
        __syncthreads();
    }
}

} // namespace

bool ell_restrict(bml_matrix_ellpack_t *S, bml_matrix_ellpack_t *P, bml_matrix_ellpack_t *O)
{
    if (!S || !P || !O || S->N != P->N || S->N != O->N || S->matrix_precision != O->matrix_precision)
    {
        b200_set_error(BML_B200_ERR_INVALID, "restrict: matrices differ in size or precision");
        return false;
    }
    if (O == S)
    {
        b200_set_error(BML_B200_ERR_INVALID, "restrict: output aliases the source");
        return false;
    }
    long long tot = 0;
    int maxrow = 0;
    if (!ell_nnz_total(P, &tot, &maxrow))
        return false;
    if (maxrow > O->M)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "restrict: a row of the pattern has %d entries, M=%d",
                       maxrow, O->M);
        return false;
    }
    B200Context *c = b200_ctx();
    if (!c || !ell_to_device(S) || !ell_to_device(P))
        return false;
    if (O != P && O->mirror == MIRROR_HOST_NEWER)
        O->mirror = MIRROR_SYNCED; // overwritten entirely below
    int logts = 5;
    while ((1 << logts) < 2 * (maxrow > 16 ? maxrow : 16))
        ++logts;
    const size_t smem = (size_t) 2 * (1 << logts) * sizeof(int);
    if (smem > c->smem_optin)
    {
        const bool ok = ell_restrict_wide(S, P, O);
        ell_mark_device(O);
        return ok;
    }
    const int grid = max(1, min(S->N, c->sm_count * 8));
    if (S->matrix_precision == double_real)
    {
        auto k = restrict_kernel<double>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<grid, 256, smem, c->stream>>>(static_cast<const double *>(S->d_value), S->d_index, S->d_nnz, S->ld,
                                          P->d_index, P->d_nnz, P->ld, static_cast<double *>(O->d_value),
                                          O->d_index, O->d_nnz, O->ld, S->N, logts);
    }
    else
    {
        auto k = restrict_kernel<float>;
        if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
            return false;
        k<<<grid, 256, smem, c->stream>>>(static_cast<const float *>(S->d_value), S->d_index, S->d_nnz, S->ld,
                                          P->d_index, P->d_nnz, P->ld, static_cast<float *>(O->d_value),
                                          O->d_index, O->d_nnz, O->ld, S->N, logts);
    }
    if (!LAUNCH_OK("restrict_kernel"))
        return false;
    ell_mark_device(O);
    return true;
}
