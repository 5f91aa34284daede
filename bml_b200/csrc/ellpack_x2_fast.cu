// ELLPACK-R thresholded sparse product C = A*B (X^2 when A == B), unordered
// form, on sm_100a.
//
// Same result set as the reference row-Gustavson loop
// (ellpack/bml_multiply_ellpack_typed.c:252-333 for X^2, :468-542 for A*B):
// C[i,k] = sum_j A[i,j] B[j,k] over the structural products, kept when
// k == i (if touched) or |C[i,k]| > threshold (typed.h:36,73, strict, compared
// in the matrix precision); tr A is the sum of A's diagonal entries and
// tr C the sum of the pre-threshold diagonal values of C.  Unlike the ordered
// tiers (ellpack_multiply.cu), the products of one C[i,k] are added in no
// fixed order and a row's kept columns come out in ascending column order.
// Every product a*b is still a separately rounded multiply followed by one
// rounded add, so |C - C_ref| <= (n-1) u sum_j |A_ij B_jk| for a column summed
// from n products: 1e-12 of that sum for any n below 4500 in FP64.
//
// B200 design.  One CTA per output row at a time (persistent CTAs claim rows
// from a counter, so rows in flight are neighbours and share the rows of B
// they read in L2).  The row's columns accumulate in a dense window of
// shared memory, TILE entries wide, by shared-memory atomic adds: no hash,
// no probe, no barrier between products, and lanes of a warp that read
// consecutive columns of a row of B hit consecutive banks.  The window spans
// [min, max] of the columns the row can touch (first and last columns of the
// referenced rows of B, which are kept sorted); a wider span is covered in
// tiles, each row of B resuming from a per-jp cursor where the last tile
// stopped, so every product is read once.  After each tile the block scans
// the window in column order, keeps by the threshold rule, writes the kept
// entries with a warp-ballot prefix and zeroes the window for the next tile.
//
// Rows of B that are not in ascending column order are sorted once per call
// into a scratch copy by the prep kernel (bitonic sort in shared memory),
// which also validates B; the product kernel reads each row of B through a
// per-row offset that points into B or into that copy.
//
// Symmetric X^2.  When A == B and X is exactly symmetric (every entry has its
// mirror with the same bits, checked on the device each call), X^2 is
// symmetric and C[k,i] is formed from the same products as C[i,k].  The
// product kernel then forms only columns k >= i of each row (about half the
// products, and half the window), into a scratch matrix U; three small
// kernels mirror U's strictly upper entries into the rows below (count per
// row, scatter, then per row a sort of the mirrored part and a copy of the
// upper part), so every row of C again lists its kept entries in ascending
// column order.  The mirrored value is the same number as the upper one, so
// C is exactly symmetric, and the keep rule, applied to each pair once, keeps
// both or neither.  The SP2 iterates of a symmetric Hamiltonian stay exactly
// symmetric (X0 = (emax I - H)/(emax - emin), 2X - X^2 and X^2 all map
// mirrored pairs to equal values).  A matrix that is not symmetric takes the
// full product; the decision is read on the device, so no host round trip.
#include "device_util.cuh"

#include <climits>
#include <type_traits>
#include <cstring>

using namespace b200;

namespace {

struct FastFlags
{
    int overflow;   // some row needed more than Mc entries
    int max_width;  // largest pre-truncation output width
    int bad_input;  // a column index or row length out of range
    int unsorted;   // rows of B that were sorted into the scratch copy
    int next_row;   // row counter of the product kernel
    int asym;       // the symmetry check found an entry without an equal mirror
};

struct FastArgs
{
    const void *Av; const int *Ai; const int *An; int lda; int NA;
    const void *Bv; const int *Bi; const int *Bn; int ldb; int NB;
    const void *Sv; const int *Si;   // sorted copies of the unsorted rows of B
    const long long *roff;           // row j of B starts at B + roff[j], or at S + (-roff[j] - 1)
    void *Cv; int *Ci; int *Cn; int ldc; int Mc;
    double thr;
    double *dA;                      // per-row sum of A's diagonal entries (nullable)
    double *dC;                      // per-row pre-threshold diagonal of C (nullable)
    FastFlags *flags;
    int ncols;
    int tile;                        // accumulator entries per tile
    int check_pre;                   // also report rows whose touched width > Mc (A*B)
    int sym_try;                     // X^2 of a square matrix: use the symmetric form if X is symmetric
    void *Uv; int *Ui; int *Un; int ldu; // upper parts of the rows (symmetric form)
    int *lcnt; int *lfill;           // mirrored entries per row: count, and placement cursor
    const int *Pi; const int *Pn; int ldp; // masked form: row i of C takes exactly P's row i pattern
    int masked;
};

// Row j of B through its offset: B itself, or its sorted copy.
template <typename T> struct RowView
{
    const int *k;
    const T *v;
};
template <typename T> __device__ __forceinline__ RowView<T> row_of(const FastArgs &g, int j)
{
    const long long o = g.roff[j];
    return o >= 0 ? RowView<T>{g.Bi + o, static_cast<const T *>(g.Bv) + o}
                  : RowView<T>{g.Si + (-o - 1), static_cast<const T *>(g.Sv) + (-o - 1)};
}

// First position in the ascending k[0..n) holding a column >= c.
__device__ __forceinline__ int lower_bound(const int *k, int n, int c)
{
    int lo = 0, hi = n;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (__ldg(k + mid) < c)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// -------------------------------------------------------------------------
// Prep: validate B, find its unsorted rows and sort them into the copy S.
// One CTA of PREP_T threads per row (grid-stride).
// -------------------------------------------------------------------------
constexpr int PREP_T = 256;

template <typename T>
__global__ void __launch_bounds__(PREP_T) fast_prep_kernel(FastArgs g, int p2, T *Sv, int *Si,
                                                           long long *roff)
{
    extern __shared__ __align__(16) unsigned char smem[];
    T *sv = reinterpret_cast<T *>(smem);
    int *sk = reinterpret_cast<int *>(smem + (size_t) p2 * sizeof(T));
    const T *Bv = static_cast<const T *>(g.Bv);
    for (int j = blockIdx.x; j < g.NB; j += gridDim.x)
    {
        const int nj = g.Bn[j];
        const size_t base = (size_t) j * g.ldb;
        int bad = (nj < 0 || nj > g.ldb) ? 1 : 0;
        int uns = 0;
        if (!bad)
            for (int p = threadIdx.x; p < nj; p += PREP_T)
            {
                const int k = g.Bi[base + p];
                if (k < 0 || k >= g.ncols)
                    bad = 1;
                if (p + 1 < nj && g.Bi[base + p + 1] < k)
                    uns = 1;
            }
        bad = __syncthreads_or(bad);
        uns = __syncthreads_or(uns);
        if (bad)
        {
            if (threadIdx.x == 0)
            {
                atomicExch(&g.flags->bad_input, 1);
                roff[j] = (long long) base;
            }
            continue;
        }
        if (!uns)
        {
            if (threadIdx.x == 0)
                roff[j] = (long long) base;
            continue;
        }
        // bitonic sort of the row's (column, value) pairs, padded to a power
        // of two with INT_MAX keys
        int n2 = 1;
        while (n2 < nj)
            n2 <<= 1;
        for (int p = threadIdx.x; p < n2; p += PREP_T)
        {
            sk[p] = p < nj ? g.Bi[base + p] : INT_MAX;
            sv[p] = p < nj ? Bv[base + p] : T(0);
        }
        __syncthreads();
        for (int size = 2; size <= n2; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1)
            {
                for (int t = threadIdx.x; t < (n2 >> 1); t += PREP_T)
                {
                    const int lo = 2 * t - (t & (stride - 1));
                    const int hi = lo + stride;
                    const bool up = (lo & size) == 0;
                    const int klo = sk[lo], khi = sk[hi];
                    if ((klo > khi) == up)
                    {
                        sk[lo] = khi;
                        sk[hi] = klo;
                        const T v = sv[lo];
                        sv[lo] = sv[hi];
                        sv[hi] = v;
                    }
                }
                __syncthreads();
            }
        for (int p = threadIdx.x; p < nj; p += PREP_T)
        {
            Si[base + p] = sk[p];
            Sv[base + p] = sv[p];
        }
        if (threadIdx.x == 0)
        {
            roff[j] = -(long long) base - 1;
            atomicAdd(&g.flags->unsorted, 1);
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------------------
// Symmetry check of X (A == B): every entry (i, j, v) must have a mirror
// (j, i) holding the same bits.  One warp per row, a binary search in the
// (sorted view of the) mirror row per entry.
// -------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) sym_check_kernel(FastArgs g)
{
    using Bits = typename std::conditional<sizeof(T) == 8, unsigned long long, unsigned>::type;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    if (g.flags->bad_input)
        return;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < g.NB; i += warps)
    {
        if (*(volatile int *) &g.flags->asym)
            return;
        const int ni = g.Bn[i];
        const RowView<T> r = row_of<T>(g, i);
        int bad = 0;
        for (int p = lane; p < ni; p += 32)
        {
            const int j = __ldg(r.k + p);
            const RowView<T> m = row_of<T>(g, j);
            const int nj = g.Bn[j];
            const int q = lower_bound(m.k, nj, i);
            const T a = __ldg(r.v + p);
            if (q >= nj || __ldg(m.k + q) != i)
                bad = 1;
            else
            {
                const T b = __ldg(m.v + q);
                Bits ba, bb;
                memcpy(&ba, &a, sizeof(T));
                memcpy(&bb, &b, sizeof(T));
                if (ba != bb)
                    bad = 1;
            }
        }
        if (__any_sync(FULL, bad) && lane == 0)
            atomicExch(&g.flags->asym, 1);
    }
}

// -------------------------------------------------------------------------
// Product kernel.
// Shared memory: acc[tile] (T) | touched bits[tile/32] (TOUCH) | cur[lda] (int)
// -------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ bool above(T x, double thr);
template <> __device__ __forceinline__ bool above<double>(double x, double thr) { return fabs(x) > thr; }
template <> __device__ __forceinline__ bool above<float>(float x, double thr) { return fabsf(x) > (float) thr; }

struct FastMisc
{
    double dA;        // sum of A's diagonal entries in the row
    double dC;        // pre-threshold diagonal of C (when touched)
    int lo, hi;       // column span of the row
    int plo, phi;     // masked form: column span of P's row
    int count;        // kept entries written so far
    int touched;      // touched columns so far (TOUCH)
    int diag_touched;
    int row;
    int bad;
    int wcnt[32];
};

// Keep rule of one scanned column c0 + c: the diagonal when touched, other
// columns when touched and above the threshold (every touched column for a
// negative threshold).  Without the bitmap, an untouched column holds 0,
// which the rule drops for thresholds >= 0, the only ones that run without it.
template <typename T, bool TOUCH>
__device__ __forceinline__ bool keep_col(T x, bool touched, bool is_diag, bool diag_touched, double thr)
{
    if (is_diag)
        return TOUCH ? touched : diag_touched;
    if (TOUCH)
        return touched && (thr < 0.0 || above<T>(x, thr));
    return above<T>(x, thr);
}

// W warps per CTA; U chunks of 32 entries of a row of B in flight per lane;
// TOUCH: keep a touched-column bitmap (negative thresholds, A*B's
// pre-threshold width check).
template <typename T, int W, int U, int MINB, bool TOUCH>
__global__ void __launch_bounds__(W * 32, MINB) fast_x2_kernel(FastArgs g)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int tile = g.tile;
    T *acc = reinterpret_cast<T *>(smem);
    unsigned *tbits = reinterpret_cast<unsigned *>(smem + (size_t) tile * sizeof(T));
    int *cur = reinterpret_cast<int *>(smem + (size_t) tile * sizeof(T) + (TOUCH ? (size_t) tile / 8 : 0));
    __shared__ FastMisc ms;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const T *Av = static_cast<const T *>(g.Av);
    const T *Bv = static_cast<const T *>(g.Bv);
    const T *Sv = static_cast<const T *>(g.Sv);

    // the prep kernel found an input out of range: touch nothing
    if (g.flags->bad_input)
        return;
    // symmetric form: columns k >= i only, rows written to U (the check
    // kernel has finished; every thread reads the same flag)
    const bool sym = g.sym_try && !g.flags->asym;
    T *outv = static_cast<T *>(sym ? g.Uv : g.Cv);
    int *outi = sym ? g.Ui : g.Ci;
    const size_t ldo = sym ? (size_t) g.ldu : (size_t) g.ldc;
    for (int c = threadIdx.x; c < tile; c += W * 32)
        acc[c] = T(0);
    if (TOUCH)
        for (int c = threadIdx.x; c < tile / 32; c += W * 32)
            tbits[c] = 0u;
    const bool masked = g.masked != 0;

    for (;;)
    {
        if (threadIdx.x == 0)
        {
            ms.row = atomicAdd(&g.flags->next_row, 1);
            ms.dA = 0.0;
            ms.dC = 0.0;
            ms.lo = INT_MAX;
            ms.hi = -1;
            ms.count = 0;
            ms.touched = 0;
            ms.diag_touched = 0;
            ms.bad = 0;
            ms.plo = INT_MAX;
            ms.phi = -1;
        }
        __syncthreads();
        const int i = ms.row;
        if (i >= g.NA)
            break;
        const int ni = g.An[i];
        const size_t arow = (size_t) i * g.lda;
        // masked form: P's row, written with zero values (the tiles below
        // overwrite the columns they form), and its column span
        const int np = masked ? g.Pn[i] : 0;
        if (masked)
        {
            int plo = INT_MAX, phi = -1, bad = (np < 0 || np > g.ldp || np > g.Mc) ? 1 : 0;
            if (!bad)
                for (int q = threadIdx.x; q < np; q += W * 32)
                {
                    const int col = g.Pi[(size_t) i * g.ldp + q];
                    if (col < 0 || col >= g.ncols)
                        bad = 1;
                    plo = min(plo, col);
                    phi = max(phi, col);
                    outi[(size_t) i * ldo + q] = col;
                    outv[(size_t) i * ldo + q] = T(0);
                }
            for (int o = 16; o; o >>= 1)
            {
                plo = min(plo, __shfl_xor_sync(FULL, plo, o));
                phi = max(phi, __shfl_xor_sync(FULL, phi, o));
                bad |= __shfl_xor_sync(FULL, bad, o);
            }
            if (lane == 0)
            {
                if (bad)
                    ms.bad = 1;
                if (phi >= 0)
                {
                    atomicMin(&ms.plo, plo);
                    atomicMax(&ms.phi, phi);
                }
            }
            __syncthreads();
        }
        const int plo = masked ? ms.plo : 0;
        // span of the row, A's diagonal, validation of A's row
        {
            int lo = INT_MAX, hi = -1, bad = (ni < 0 || ni > g.lda) ? 1 : 0;
            if (!bad)
                for (int jp = threadIdx.x; jp < ni; jp += W * 32)
                {
                    cur[jp] = 0;
                    const int j = g.Ai[arow + jp];
                    if (j < 0 || j >= g.NB)
                    {
                        bad = 1;
                        continue;
                    }
                    if (j == i)
                        atomicAdd(&ms.dA, (double) Av[arow + jp]);
                    const int nj = g.Bn[j];
                    if (nj <= 0)
                        continue;
                    const int *ki = row_of<T>(g, j).k;
                    if (masked)
                    {
                        // the part of row j at columns >= the start of P's row
                        const int q = lower_bound(ki, nj, plo);
                        cur[jp] = q;
                        if (q < nj)
                        {
                            lo = min(lo, ki[q]);
                            hi = max(hi, ki[nj - 1]);
                        }
                        continue;
                    }
                    if (sym)
                    {
                        // the part of row j at columns >= i
                        const int q = lower_bound(ki, nj, i);
                        cur[jp] = q;
                        if (q < nj)
                        {
                            lo = i;
                            hi = max(hi, ki[nj - 1]);
                        }
                        continue;
                    }
                    lo = min(lo, ki[0]);
                    hi = max(hi, ki[nj - 1]);
                }
            if (bad)
                ms.bad = 1;
            for (int o = 16; o; o >>= 1)
            {
                lo = min(lo, __shfl_xor_sync(FULL, lo, o));
                hi = max(hi, __shfl_xor_sync(FULL, hi, o));
            }
            if (lane == 0 && hi >= 0)
            {
                atomicMin(&ms.lo, lo);
                atomicMax(&ms.hi, hi);
            }
        }
        __syncthreads();
        if (ms.bad)
        {
            if (threadIdx.x == 0)
            {
                atomicExch(&g.flags->bad_input, 1);
                g.Cn[i] = 0;
            }
            __syncthreads();
            continue;
        }
        const int lo = ms.lo, hi = masked ? min(ms.hi, ms.phi) : ms.hi;
        const bool multi = hi - lo + 1 > tile;
        for (int c0 = lo; c0 <= hi; c0 += tile)
        {
            const int len = min(tile, hi - c0 + 1);
            const int cend = c0 + len; // every column of this tile is below cend
            // Products.  Warp w takes jp = w, w + W, ...; the metadata of 32
            // of its jps is loaded at once, one jp per lane, and broadcast.
            for (int jb = warp; jb < ni; jb += 32 * W)
            {
                const int myjp = jb + lane * W;
                int mn = 0;
                long long mo = 0;
                T ma = T(0);
                if (myjp < ni)
                {
                    const int mj = g.Ai[arow + myjp];
                    ma = Av[arow + myjp];
                    mn = g.Bn[mj];
                    mo = g.roff[mj];
                }
                const int nb = min(32, (ni - jb + W - 1) / W);
                for (int t = 0; t < nb; ++t)
                {
                    const int jp = jb + t * W;
                    const T a = __shfl_sync(FULL, ma, t);
                    const int nj = __shfl_sync(FULL, mn, t);
                    const long long o = __shfl_sync(FULL, mo, t);
                    const int *ki = o >= 0 ? g.Bi + o : g.Si + (-o - 1);
                    const T *kv = o >= 0 ? Bv + o : Sv + (-o - 1);
                    int pos = (multi || sym || masked) ? cur[jp] : 0;
                    while (pos < nj)
                    {
                        int k[U];
                        T v[U];
#pragma unroll
                        for (int u = 0; u < U; ++u)
                        {
                            const int p = pos + u * 32 + lane;
                            k[u] = p < nj ? __ldg(ki + p) : INT_MAX;
                            v[u] = p < nj ? __ldg(kv + p) : T(0);
                        }
                        // rows of B are sorted: the columns below cend are a
                        // prefix of what is left of the row
                        int stop = -1;
#pragma unroll
                        for (int u = 0; u < U; ++u)
                        {
                            if (stop < 0)
                            {
                                if (k[u] < cend)
                                {
                                    const int c = k[u] - c0;
                                    atomicAdd(&acc[c], a * v[u]);
                                    if (TOUCH)
                                        atomicOr(&tbits[c >> 5], 1u << (c & 31));
                                    if (k[u] == i)
                                        ms.diag_touched = 1;
                                }
                                const unsigned out = __ballot_sync(FULL, k[u] >= cend);
                                if (out)
                                    stop = pos + u * 32 + __ffs(out) - 1;
                            }
                        }
                        if (stop >= 0)
                        {
                            pos = stop;
                            break;
                        }
                        pos += U * 32;
                    }
                    if (multi && lane == 0)
                        cur[jp] = min(pos, nj);
                }
            }
            __syncthreads();
            if (masked)
            {
                // P's columns in this tile take their sums (0 where nothing
                // was added); then the window is zeroed
                for (int q = threadIdx.x; q < np; q += W * 32)
                {
                    const int col = g.Pi[(size_t) i * g.ldp + q];
                    if (col >= c0 && col < cend)
                    {
                        const T x = acc[col - c0];
                        outv[(size_t) i * ldo + q] = x;
                        if (col == i)
                            ms.dC = (double) x;
                    }
                }
                __syncthreads();
                for (int c = threadIdx.x; c < len; c += W * 32)
                    acc[c] = T(0);
                __syncthreads();
                continue;
            }
            // Scan of the window in column order: count per warp, prefix over
            // warps, then write the kept entries and zero the window.
            const int per = (((len + W - 1) / W) + 31) & ~31;
            const int cb = warp * per;
            const int ce = min(len, cb + per);
            const bool dtouch = ms.diag_touched != 0;
            int cnt = 0, tcnt = 0;
            for (int b = cb; b < ce; b += 32)
            {
                const int c = b + lane;
                bool keep = false;
                if (c < ce)
                {
                    const bool tt = TOUCH ? ((tbits[c >> 5] >> (c & 31)) & 1u) != 0 : true;
                    keep = keep_col<T, TOUCH>(acc[c], tt, c0 + c == i, dtouch, g.thr);
                    if (TOUCH)
                        tcnt += tt ? 1 : 0;
                }
                cnt += __popc(__ballot_sync(FULL, keep));
            }
            if (TOUCH)
                for (int o = 16; o; o >>= 1)
                    tcnt += __shfl_xor_sync(FULL, tcnt, o);
            if (lane == 0)
            {
                ms.wcnt[warp] = cnt;
                if (TOUCH)
                    atomicAdd(&ms.touched, tcnt);
            }
            __syncthreads();
            int off = ms.count;
            for (int w = 0; w < warp; ++w)
                off += ms.wcnt[w];
            for (int b = cb; b < ce; b += 32)
            {
                const int c = b + lane;
                bool keep = false;
                T x = T(0);
                if (c < ce)
                {
                    x = acc[c];
                    const bool tt = TOUCH ? ((tbits[c >> 5] >> (c & 31)) & 1u) != 0 : true;
                    keep = keep_col<T, TOUCH>(x, tt, c0 + c == i, dtouch, g.thr);
                    if (c0 + c == i && (TOUCH ? tt : dtouch))
                        ms.dC = (double) x;
                    acc[c] = T(0);
                }
                const unsigned bal = __ballot_sync(FULL, keep);
                const int pos = off + __popc(bal & lanemask_lt());
                if (keep && pos < g.Mc)
                {
                    outi[(size_t) i * ldo + pos] = c0 + c;
                    outv[(size_t) i * ldo + pos] = x;
                }
                off += __popc(bal);
            }
            if (TOUCH)
                for (int c = cb / 32 + lane; c < (ce + 31) / 32; c += 32)
                    tbits[c] = 0u;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                int tot = 0;
                for (int w = 0; w < W; ++w)
                    tot += ms.wcnt[w];
                ms.count += tot;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            const int ll = masked ? np : ms.count;
            if (sym)
                g.Un[i] = ll; // the mirror kernels complete the row
            else
            {
                g.Cn[i] = min(ll, g.Mc);
                atomicMax(&g.flags->max_width, ll);
                if (ll > g.Mc || (g.check_pre && ms.touched > g.Mc))
                    atomicExch(&g.flags->overflow, 1);
            }
            if (g.dA)
                g.dA[i] = ms.dA;
            if (g.dC)
                g.dC[i] = ms.dC;
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------------------
// Symmetric form, after the product kernel: mirror U's strictly upper kept
// entries (k, i > k) into row i.  Each kernel returns at once when the
// product kernel took the full form.
// -------------------------------------------------------------------------
__device__ __forceinline__ bool sym_on(const FastArgs &g)
{
    return !g.flags->bad_input && g.sym_try && !g.flags->asym;
}

// lcnt[i] = number of kept entries (k, i) with k < i; one warp per row k.
__global__ void __launch_bounds__(256) sym_count_kernel(FastArgs g)
{
    if (!sym_on(g))
        return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < g.NA; k += warps)
    {
        const int n = min(g.Un[k], g.Mc);
        for (int p = lane; p < n; p += 32)
        {
            const int i = g.Ui[(size_t) k * g.ldu + p];
            if (i > k)
                atomicAdd(&g.lcnt[i], 1);
        }
    }
}

// Scatter of the mirrored entries into the first lcnt[i] slots of row i of C
// (in arrival order; the finish kernel sorts them).
template <typename T>
__global__ void __launch_bounds__(256) sym_place_kernel(FastArgs g)
{
    if (!sym_on(g))
        return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const T *Uv = static_cast<const T *>(g.Uv);
    T *Cv = static_cast<T *>(g.Cv);
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < g.NA; k += warps)
    {
        const int n = min(g.Un[k], g.Mc);
        for (int p = lane; p < n; p += 32)
        {
            const size_t at = (size_t) k * g.ldu + p;
            const int i = g.Ui[at];
            if (i <= k)
                continue;
            const int q = atomicAdd(&g.lfill[i], 1);
            if (q < g.Mc)
            {
                g.Ci[(size_t) i * g.ldc + q] = k;
                Cv[(size_t) i * g.ldc + q] = Uv[at];
            }
        }
    }
}

// Row i of C: its mirrored part sorted by column (bitonic sort in shared
// memory, padded with INT_MAX keys), then its upper part copied from U; the
// row's width, overflow and the widest row are recorded.  One CTA of 256
// threads per row (grid-stride); shared memory: vals[p2] | keys[p2], p2 the
// power of two >= Mc.
template <typename T>
__global__ void __launch_bounds__(256) sym_finish_kernel(FastArgs g, int p2)
{
    if (!sym_on(g))
        return;
    extern __shared__ __align__(16) unsigned char smem[];
    T *sv = reinterpret_cast<T *>(smem);
    int *sk = reinterpret_cast<int *>(smem + (size_t) p2 * sizeof(T));
    const T *Uv = static_cast<const T *>(g.Uv);
    T *Cv = static_cast<T *>(g.Cv);
    for (int i = blockIdx.x; i < g.NA; i += gridDim.x)
    {
        const int L = g.lcnt[i];
        const int Lk = min(L, g.Mc);
        const int total = L + g.Un[i];
        const size_t crow = (size_t) i * g.ldc;
        int n2 = 1;
        while (n2 < Lk)
            n2 <<= 1;
        for (int p = threadIdx.x; p < n2; p += 256)
        {
            sk[p] = p < Lk ? g.Ci[crow + p] : INT_MAX;
            sv[p] = p < Lk ? Cv[crow + p] : T(0);
        }
        __syncthreads();
        for (int size = 2; size <= n2; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1)
            {
                for (int t = threadIdx.x; t < (n2 >> 1); t += 256)
                {
                    const int lo = 2 * t - (t & (stride - 1));
                    const int hi = lo + stride;
                    const bool up = (lo & size) == 0;
                    const int klo = sk[lo], khi = sk[hi];
                    if ((klo > khi) == up)
                    {
                        sk[lo] = khi;
                        sk[hi] = klo;
                        const T v = sv[lo];
                        sv[lo] = sv[hi];
                        sv[hi] = v;
                    }
                }
                __syncthreads();
            }
        for (int p = threadIdx.x; p < Lk; p += 256)
        {
            g.Ci[crow + p] = sk[p];
            Cv[crow + p] = sv[p];
        }
        const int nu = min(g.Un[i], g.Mc);
        for (int p = threadIdx.x; p < nu && L + p < g.Mc; p += 256)
        {
            g.Ci[crow + L + p] = g.Ui[(size_t) i * g.ldu + p];
            Cv[crow + L + p] = Uv[(size_t) i * g.ldu + p];
        }
        if (threadIdx.x == 0)
        {
            g.Cn[i] = min(total, g.Mc);
            atomicMax(&g.flags->max_width, total);
            if (total > g.Mc)
                atomicExch(&g.flags->overflow, 1);
        }
        __syncthreads();
    }
}

} // namespace

namespace {

// Warps per CTA, chunks in flight per lane and CTAs per SM of the product
// kernel.  Two CTAs of 16 warps with 8 chunks per lane were the fastest of
// the shapes measured on the 30^3 lattice iterate (X^2 in 60.8 ms FP64,
// 43.4 ms FP32; one CTA of 32 warps with 4 chunks: 63.4 and 52.1 ms).
#ifndef B200_FX_W
#define B200_FX_W 16
#endif
#ifndef B200_FX_U
#define B200_FX_U 8
#endif
#ifndef B200_FX_MINB
#define B200_FX_MINB 2
#endif
constexpr int FX_W = B200_FX_W, FX_U = B200_FX_U, FX_MINB = B200_FX_MINB;
// Offsets in the context's small device/pinned buffers.
constexpr size_t FX_SMALL = 16384;

bool g_x2_exact = false;
// The symmetric form of X^2 (on by default; off only to measure the full form).
bool g_x2_symmetric = true;
bool g_last_symmetric = false;
bool g_last_dense = false;
// CUDA events around the product kernel (when timing is on), on the library
// stream; the last duration in ms, or -1.
bool g_time_kernel = false;
cudaEvent_t g_kev[2] = {nullptr, nullptr};
float g_last_kernel_ms = -1.0f;

// Dynamic shared memory a product CTA may take: its share of the SM's
// 228 KiB (less the 1 KiB the SM reserves per CTA), within the per-block
// opt-in limit, less the static FastMisc.
size_t fast_smem_budget(const B200Context *c)
{
    size_t b = (size_t) 228 * 1024 / FX_MINB - 1024;
    if (b > c->smem_optin)
        b = c->smem_optin;
    return b - sizeof(FastMisc) - 64;
}

template <typename T, bool TOUCH> auto fast_kernel()
{
    return fast_x2_kernel<T, FX_W, FX_U, FX_MINB, TOUCH>;
}

template <typename T>
bool fast_multiply_typed(FastArgs g, double *trace, int *required_M, bool touch)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const int N = g.NA;
    // the symmetric form's row sort holds a row of C in shared memory
    int p2c = 1;
    while (p2c < g.Mc)
        p2c <<= 1;
    const size_t smemF = (size_t) p2c * (sizeof(T) + sizeof(int));
    if (touch || smemF > c->smem_optin)
        g.sym_try = 0;
    // scratch: roff[NB] | sorted copy of B (values, columns) | diag arrays |
    // (symmetric form) U values, U columns, U widths, lcnt, lfill
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t nbe = (size_t) g.NB * g.ldb;
    const size_t nue = g.sym_try ? (size_t) N * g.ldc : 0;
    const size_t off_sv = al((size_t) g.NB * sizeof(long long));
    const size_t off_si = al(off_sv + nbe * sizeof(T));
    const size_t off_diag = al(off_si + nbe * sizeof(int));
    const size_t off_uv = al(off_diag + (size_t) 2 * N * sizeof(double));
    const size_t off_ui = al(off_uv + nue * sizeof(T));
    const size_t off_un = al(off_ui + nue * sizeof(int));
    const size_t total = al(off_un + (g.sym_try ? (size_t) 3 * N * sizeof(int) : 0));
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(total));
    if (!scr)
        return false;
    long long *roff = reinterpret_cast<long long *>(scr);
    T *Sv = reinterpret_cast<T *>(scr + off_sv);
    int *Si = reinterpret_cast<int *>(scr + off_si);
    double *diagA = reinterpret_cast<double *>(scr + off_diag);
    double *diagC = diagA + N;
    g.Sv = Sv;
    g.Si = Si;
    g.roff = roff;
    if (g.sym_try)
    {
        g.Uv = scr + off_uv;
        g.Ui = reinterpret_cast<int *>(scr + off_ui);
        g.Un = reinterpret_cast<int *>(scr + off_un);
        g.lcnt = g.Un + N;
        g.lfill = g.lcnt + N;
        g.ldu = g.ldc;
        if (!CUDA_OK(cudaMemsetAsync(g.lcnt, 0, (size_t) 2 * N * sizeof(int), c->stream)))
            return false;
    }

    unsigned char *small = static_cast<unsigned char *>(c->d_small) + FX_SMALL;
    FastFlags *flags = reinterpret_cast<FastFlags *>(small);
    double *dtrace = reinterpret_cast<double *>(small + 64);
    if (!CUDA_OK(cudaMemsetAsync(small, 0, 128, c->stream)))
        return false;
    g.flags = flags;
    g.dA = trace ? diagA : nullptr;
    g.dC = trace ? diagC : nullptr;
    if (trace && !CUDA_OK(cudaMemsetAsync(diagA, 0, (size_t) 2 * N * sizeof(double), c->stream)))
        return false;

    // prep: validation and sorted copies of unsorted rows of B
    int p2 = 1;
    while (p2 < g.ldb)
        p2 <<= 1;
    const size_t smemP = (size_t) p2 * (sizeof(T) + sizeof(int));
    if (!CUDA_OK(cudaFuncSetAttribute(fast_prep_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) smemP)))
        return false;
    int occP = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occP, fast_prep_kernel<T>, PREP_T, smemP);
    const int pgrid = max(1, min(g.NB, c->sm_count * max(occP, 1)));
    fast_prep_kernel<T><<<pgrid, PREP_T, smemP, c->stream>>>(g, p2, Sv, Si, roff);
    if (!LAUNCH_OK("fast_prep_kernel"))
        return false;
    const int wgrid = max(1, min(b200_ceil_div(N, 8), c->sm_count * 16));
    if (g.sym_try)
    {
        sym_check_kernel<T><<<wgrid, 256, 0, c->stream>>>(g);
        if (!LAUNCH_OK("sym_check_kernel"))
            return false;
    }

    // product kernel: the accumulator window takes the shared memory left
    // after the cursors (and the touched bitmap)
    auto kern = touch ? fast_kernel<T, true>() : fast_kernel<T, false>();
    const size_t budget = fast_smem_budget(c);
    const size_t cur_bytes = (size_t) b200_round_up(g.lda, 32) * sizeof(int);
    if (cur_bytes + 4096 * (sizeof(T) + 1) > budget)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply: row width %d too large for the unordered kernel",
                       g.lda);
        return false;
    }
    const double per_col = (double) sizeof(T) + (touch ? 0.125 : 0.0);
    int tile = (int) ((double) (budget - cur_bytes) / per_col);
    tile &= ~1023;
    g.tile = tile;
    const size_t smemK = (size_t) tile * sizeof(T) + (touch ? (size_t) tile / 8 : 0) + cur_bytes;
    if (!CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemK)))
        return false;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, FX_W * 32, smemK);
    if (occ < 1)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply: the unordered kernel does not fit the device");
        return false;
    }
    const bool timed = g_time_kernel && (g_kev[0] || (CUDA_OK(cudaEventCreate(&g_kev[0])) &&
                                                        CUDA_OK(cudaEventCreate(&g_kev[1]))));
    if (timed && !CUDA_OK(cudaEventRecord(g_kev[0], c->stream)))
        return false;
    kern<<<c->sm_count * occ, FX_W * 32, smemK, c->stream>>>(g);
    if (!LAUNCH_OK("fast_x2_kernel"))
        return false;
    if (timed && !CUDA_OK(cudaEventRecord(g_kev[1], c->stream)))
        return false;
    if (g.sym_try)
    {
        sym_count_kernel<<<wgrid, 256, 0, c->stream>>>(g);
        if (!LAUNCH_OK("sym_count_kernel"))
            return false;
        sym_place_kernel<T><<<wgrid, 256, 0, c->stream>>>(g);
        if (!LAUNCH_OK("sym_place_kernel"))
            return false;
        if (!CUDA_OK(cudaFuncSetAttribute(sym_finish_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) smemF)))
            return false;
        int occF = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occF, sym_finish_kernel<T>, 256, smemF);
        sym_finish_kernel<T><<<max(1, min(N, c->sm_count * max(occF, 1))), 256, smemF, c->stream>>>(g, p2c);
        if (!LAUNCH_OK("sym_finish_kernel"))
            return false;
    }
    if (trace)
    {
        b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(diagA, diagC, N, dtrace);
        if (!LAUNCH_OK("b200_sum_rows_kernel"))
            return false;
    }
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + FX_SMALL;
    if (!CUDA_OK(cudaMemcpyAsync(pin, small, 128, cudaMemcpyDeviceToHost, c->stream)))
        return false;
    if (!b200_sync())
        return false;
    const FastFlags *hf = reinterpret_cast<const FastFlags *>(pin);
    const double *ht = reinterpret_cast<const double *>(pin + 64);
    g_last_symmetric = g.sym_try && !hf->asym && !hf->bad_input;
    g_last_kernel_ms = -1.0f;
    if (timed && !CUDA_OK(cudaEventElapsedTime(&g_last_kernel_ms, g_kev[0], g_kev[1])))
        return false;
    if (required_M)
        *required_M = hf->max_width;
    if (hf->bad_input)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply: a column index or row length of an input is out of range");
        return false;
    }
    if (trace)
    {
        trace[0] = ht[0];
        trace[1] = ht[1];
    }
    if (hf->overflow)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW, "Number of non-zeroes per row > M, Increase M (need %d, M = %d)",
                       hf->max_width, g.Mc);
        return false;
    }
    return true;
}

} // namespace

bool ell_x2_exact()
{
    return g_x2_exact;
}

// The dense tier, when the operands' rows fill in (its A*B width check counts
// the nonzero entries of the product, which are the touched ones unless
// products cancel to an exact zero).
bool ell_multiply_dense_tier(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C,
                             double threshold, double *trace, int *required_M, bool *taken)
{
    *taken = false;
    if (!ell_dense_fits(A, B, C, threshold))
        return false;
    *taken = true;
    g_last_symmetric = false;
    g_last_dense = true;
    return ell_multiply_dense(A, B, C, threshold, trace, required_M);
}

bool ell_unordered_fits(const bml_matrix_ellpack_t *A)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const size_t cur_bytes = (size_t) b200_round_up(A->ld, 32) * sizeof(int);
    return cur_bytes + 4096 * (prec_size(A->matrix_precision) + 1) <= fast_smem_budget(c) &&
           (size_t) 1 << (32 - __builtin_clz((unsigned) (A->ld | 1))) <= 16384;
}

bool ell_multiply_unordered(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C,
                            double threshold, double *trace, int *required_M, bool check_pre)
{
    g_last_dense = false;
    FastArgs g{};
    g.Av = A->d_value; g.Ai = A->d_index; g.An = A->d_nnz; g.lda = A->ld; g.NA = A->N;
    g.Bv = B->d_value; g.Bi = B->d_index; g.Bn = B->d_nnz; g.ldb = B->ld; g.NB = B->N;
    g.Cv = C->d_value; g.Ci = C->d_index; g.Cn = C->d_nnz; g.ldc = C->ld; g.Mc = C->M;
    g.thr = threshold;
    g.check_pre = check_pre ? 1 : 0;
    g.ncols = B->N > C->N ? B->N : C->N;
    // X^2 of a square matrix: the symmetric form runs if X proves symmetric
    g.sym_try = (A == B && A->N == C->N && g_x2_symmetric) ? 1 : 0;
    // a touched-column bitmap is needed where untouched zeros could pass the
    // keep rule (threshold < 0 or NaN) or the pre-threshold width is checked
    const bool touch = check_pre || !(threshold >= 0.0);
    return A->matrix_precision == double_real ? fast_multiply_typed<double>(g, trace, required_M, touch)
                                              : fast_multiply_typed<float>(g, trace, required_M, touch);
}

bool ell_multiply_masked(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *P,
                         bml_matrix_ellpack_t *C, bool *taken)
{
    *taken = false;
    if (!A || !B || !P || !C || C == A || C == B || C == P || A->matrix_precision != B->matrix_precision ||
        A->matrix_precision != C->matrix_precision || A->N != C->N || P->N != C->N || P->M > C->M)
    {
        b200_set_error(BML_B200_ERR_INVALID, "masked multiply: operands of one precision, C distinct, "
                                             "P and C with A's rows, C at least as wide as P");
        return false;
    }
    if (g_x2_exact || !ell_unordered_fits(A) || !ell_unordered_fits(B) || ell_dense_fits(A, B, C, 0.0))
        return false;
    if (!ell_to_device(A) || (B != A && !ell_to_device(B)) || (P != A && P != B && !ell_to_device(P)) ||
        !ell_to_device(C))
        return false;
    if (C->mirror == MIRROR_HOST_NEWER)
        C->mirror = MIRROR_SYNCED;
    *taken = true;
    g_last_dense = false;
    FastArgs g{};
    g.Av = A->d_value; g.Ai = A->d_index; g.An = A->d_nnz; g.lda = A->ld; g.NA = A->N;
    g.Bv = B->d_value; g.Bi = B->d_index; g.Bn = B->d_nnz; g.ldb = B->ld; g.NB = B->N;
    g.Cv = C->d_value; g.Ci = C->d_index; g.Cn = C->d_nnz; g.ldc = C->ld; g.Mc = C->M;
    g.Pi = P->d_index; g.Pn = P->d_nnz; g.ldp = P->ld; g.masked = 1;
    g.thr = 0.0;
    g.ncols = B->N > C->N ? B->N : C->N;
    const bool ok = A->matrix_precision == double_real ? fast_multiply_typed<double>(g, nullptr, nullptr, false)
                                                       : fast_multiply_typed<float>(g, nullptr, nullptr, false);
    ell_mark_device(C);
    return ok;
}

// Allows (1, the default) or forbids (0) the symmetric form of the unordered
// X^2; returns the previous setting.
extern "C" BML_B200_API int bml_b200_set_x2_symmetric(int allow)
{
    const int old = g_x2_symmetric ? 1 : 0;
    g_x2_symmetric = allow != 0;
    return old;
}

// Times the product kernel of later unordered products with CUDA events on
// the library stream (on = 1); returns the previous setting.
extern "C" BML_B200_API int bml_b200_set_kernel_timing(int on)
{
    const int old = g_time_kernel ? 1 : 0;
    g_time_kernel = on != 0;
    return old;
}

// Device time of the last unordered product's product kernel in ms (-1 when
// it was not timed).
extern "C" BML_B200_API double bml_b200_last_x2_kernel_ms(void)
{
    return (double) g_last_kernel_ms;
}

// 1 when the last unordered product ran on the dense tier.
extern "C" BML_B200_API int bml_b200_last_x2_dense(void)
{
    return g_last_dense ? 1 : 0;
}

// 1 when the last unordered product took the symmetric form.
extern "C" BML_B200_API int bml_b200_last_x2_symmetric(void)
{
    return g_last_symmetric ? 1 : 0;
}

// Selects the ordered (bit-identical to the reference) or the unordered
// multiply for later ELLPACK products; returns the previous choice.
extern "C" BML_B200_API int bml_b200_set_x2_exact(int exact)
{
    const int old = g_x2_exact ? 1 : 0;
    g_x2_exact = exact != 0;
    return old;
}
