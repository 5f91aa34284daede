// ELLPACK-R thresholded sparse product C = A*B (X^2 when A == B) on sm_100a.
//
// Follows the reference row-Gustavson loop
// (ellpack/bml_multiply_ellpack_typed.c:252-333 for X^2, :468-542 for A*B):
// for every row i, for jp in row order, for kp in the order of row j = col(i,jp),
//   x[k] = x[k] + a_ij * b_jk    (k = col(j,kp)); first touch starts at 0.0
// then the touched columns are visited in first-touch order and kept when
// k == i or |x| > threshold (typed.h:73, strict), and tr A / tr C are summed.
//
// B200 design.  A team of W warps owns one output row.  The team walks jp in
// order; within one jp every k is distinct, so the lanes update their
// accumulator slots without races, and a team barrier between consecutive
// jp keeps every x[k] summed in exactly the reference order.  Products and
// sums use __dmul_rn/__dadd_rn (no FMA contraction), matching the reference
// build (-std=c99, no -mfma), so each call is bit-identical to the reference
// on the same input.  New keys of a jp are appended to an order list with a
// warp ballot + popcount prefix (and a cross-warp prefix for W > 1), which
// rebuilds the reference's first-touch output order without sorting.
//
// Three tiers, chosen per row by a planning kernel:
//   tier A  one warp per row, 1024-slot shared-memory hash (rows whose
//           product count already bounds their width by 640);
//   tier B  8 warps per row, 8192-slot shared-memory hash (optimistic: a row
//           whose distinct columns exceed 5/8 of the table is handed on);
//   tier C  8 warps per row, dense accumulator over all N columns in global
//           memory (any width; the reference's own x[N]/ix[N]/jx[N] scheme).
// All tiers are persistent grids that pull rows from device-side lists, so a
// multiply needs no host round trip until the traces are read back.
#include "internal.h"

namespace {

constexpr unsigned FULL = 0xffffffffu;

template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Barrier over the W warps of one team.  Team t uses named barrier t+1.
template <int W> __device__ __forceinline__ void team_sync(int team)
{
    if (W == 1)
        __syncwarp();
    else
        asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(W * 32) : "memory");
}

// Flags shared by all tiers of one multiply call (device memory).
struct MulFlags
{
    int overflow;     // some row needed more than Mc entries
    int max_width;    // largest pre-truncation output width
    int bad_input;    // an input column index or nnz out of range
    int pad;
};

struct MulArgs
{
    const void *Av; const int *Ai; const int *An; int lda; int NA;
    const void *Bv; const int *Bi; const int *Bn; int ldb; int NB;
    void *Cv; int *Ci; int *Cn; int ldc; int Mc;
    double thr;
    double *dA;       // per-row sum of A's diagonal entries (nullable)
    double *dC;       // per-row C diagonal value (nullable)
    MulFlags *flags;
    int check_pre;    // A*B: also report rows whose pre-threshold width > Mc
};

// Row lists and cursors for the three tiers.
struct TierLists
{
    int count[3];
    int cursor[3];
};

// -------------------------------------------------------------------------
// Planning: product-count bound per row, input validation, tier assignment.
// One warp per row.
// -------------------------------------------------------------------------
__global__ void plan_kernel(MulArgs g, int capA, TierLists *tl, int *listA, int *listB)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < g.NA; i += warps)
    {
        const int ni = g.An[i];
        long long P = 0;
        int bad = (ni < 0 || ni > g.lda) ? 1 : 0;
        if (!bad)
        {
            for (int jp = lane; jp < ni; jp += 32)
            {
                const int j = g.Ai[(size_t) i * g.lda + jp];
                if (j < 0 || j >= g.NB)
                {
                    bad = 1;
                    continue;
                }
                const int nj = g.Bn[j];
                if (nj < 0 || nj > g.ldb)
                    bad = 1;
                else
                    P += nj;
            }
        }
        for (int o = 16; o; o >>= 1)
            P += __shfl_xor_sync(FULL, P, o);
        bad = __any_sync(FULL, bad);
        if (lane == 0)
        {
            if (bad)
                atomicExch(&g.flags->bad_input, 1);
            else if (P <= capA)
                listA[atomicAdd(&tl->count[0], 1)] = i;
            else
                listB[atomicAdd(&tl->count[1], 1)] = i;
        }
    }
}

// Column indices of B inside the kernels are validated by the plan kernel
// (which checks every index of A and the nnz of every referenced B row); B's
// own column indices are checked here when they are used.
__global__ void validate_cols_kernel(const int *Bi, const int *Bn, int ldb, int NB, int ncols,
                                     MulFlags *flags)
{
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < NB; j += warps)
    {
        const int nj = Bn[j];
        int bad = (nj < 0 || nj > ldb) ? 1 : 0;
        if (!bad)
            for (int kp = lane; kp < nj; kp += 32)
            {
                const int k = Bi[(size_t) j * ldb + kp];
                if (k < 0 || k >= ncols)
                    bad = 1;
            }
        if (__any_sync(FULL, bad) && lane == 0)
            atomicExch(&flags->bad_input, 1);
    }
}

// -------------------------------------------------------------------------
// Shared-memory hash tiers (A and B).
// Per-team shared memory: vals[TS] | keys[TS] | order[TS] | stage[W][smax] |
//                         cnt[2][W] | misc
// -------------------------------------------------------------------------
template <typename T> struct TeamMisc
{
    T diag;
    int row;
    int pad;
};

template <typename T, int W, int LOGTS>
__host__ __device__ constexpr size_t team_smem_bytes(int smax)
{
    return (size_t(1) << LOGTS) * (sizeof(T) + 2 * sizeof(int)) +
           (W > 1 ? size_t(W) * smax * sizeof(int) : 0) + 2 * W * sizeof(int) + 32;
}

template <int LOGTS>
__device__ __forceinline__ int probe_insert(int *keys, int k, bool &inserted)
{
    constexpr int TS = 1 << LOGTS;
    unsigned h = ((unsigned) k * 2654435761u) >> (32 - LOGTS);
    volatile int *vk = keys;
#pragma unroll 1
    for (int p = 0; p < TS; ++p)
    {
        const int cur = vk[h];
        if (cur == k)
        {
            inserted = false;
            return (int) h;
        }
        if (cur == B200_EMPTY_KEY)
        {
            const int old = atomicCAS(&keys[h], B200_EMPTY_KEY, k);
            if (old == B200_EMPTY_KEY)
            {
                inserted = true;
                return (int) h;
            }
            if (old == k)
            {
                inserted = false;
                return (int) h;
            }
        }
        h = (h + 1) & (TS - 1);
    }
    inserted = false;
    return -1;
}

template <typename T, int W, int LOGTS>
__global__ void __launch_bounds__(W == 1 ? 128 : W * 32) hash_tier_kernel(MulArgs g, int smax,
                                                       const int *rows, TierLists *tl, int tier,
                                                       int *next_rows)
{
    constexpr int TS = 1 << LOGTS;
    constexpr int CAP = TS * 5 / 8;
    extern __shared__ __align__(16) unsigned char smem[];

    if (g.flags->bad_input)
        return;
    const int nrows = tl->count[tier];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = warp / W, wt = warp % W, tid = wt * 32 + lane;
    unsigned char *base = smem + (size_t) team * team_smem_bytes<T, W, LOGTS>(smax);
    T *vals = reinterpret_cast<T *>(base);
    int *keys = reinterpret_cast<int *>(vals + TS);
    int *order = keys + TS;
    int *stage = order + TS + (W > 1 ? wt * smax : 0);
    int *cnt = order + TS + (W > 1 ? W * smax : 0);
    TeamMisc<T> *misc = reinterpret_cast<TeamMisc<T> *>(cnt + 2 * W);

    const T *Av = static_cast<const T *>(g.Av);
    const T *Bv = static_cast<const T *>(g.Bv);
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;

    for (;;)
    {
        int pos;
        if (W == 1)
        {
            if (lane == 0)
                pos = atomicAdd(&tl->cursor[tier], 1);
            pos = __shfl_sync(FULL, pos, 0);
        }
        else
        {
            if (tid == 0)
                misc->row = atomicAdd(&tl->cursor[tier], 1);
            team_sync<W>(team);
            pos = misc->row;
        }
        if (pos >= nrows)
            break;
        const int i = rows[pos];

        for (int s = tid; s < TS; s += W * 32)
        {
            keys[s] = B200_EMPTY_KEY;
            vals[s] = T(0);
        }
        if (tid == 0)
            misc->diag = T(0);
        team_sync<W>(team);

        const int ni = g.An[i];
        const T *arow = Av + (size_t) i * g.lda;
        const int *airow = g.Ai + (size_t) i * g.lda;
        int distinct = 0;
        T dA = T(0);
        bool aborted = false;

        for (int jp0 = 0; jp0 < ni && !aborted; jp0 += 32)
        {
            const int q = jp0 + lane;
            T av = T(0);
            int aj = 0, nj_l = 0;
            if (q < ni)
            {
                av = arow[q];
                aj = airow[q];
                nj_l = g.Bn[aj];
            }
            const int cnt_here = min(32, ni - jp0);
            for (int t = 0; t < cnt_here; ++t)
            {
                const int jp = jp0 + t;
                const T a = __shfl_sync(FULL, av, t);
                const int j = __shfl_sync(FULL, aj, t);
                const int nj = __shfl_sync(FULL, nj_l, t);
                if (j == i)
                    dA = add_rn(dA, a);
                const T *brow = Bv + (size_t) j * g.ldb;
                const int *birow = g.Bi + (size_t) j * g.ldb;
                int k0 = 0, k1 = nj;
                if (W > 1)
                {
                    const int S = b200_round_up(b200_ceil_div(nj, W), 32);
                    k0 = min(wt * S, nj);
                    k1 = min(k0 + S, nj);
                }
                int local = 0;
                bool fail = false;
                for (int kb = k0; kb < k1; kb += 32)
                {
                    const int kp = kb + lane;
                    bool ins = false;
                    int slot = -1;
                    if (kp < k1)
                    {
                        const int k = birow[kp];
                        const T p = mul_rn(a, brow[kp]);
                        slot = probe_insert<LOGTS>(keys, k, ins);
                        if (slot >= 0)
                            vals[slot] = add_rn(vals[slot], p);
                        else
                            fail = true;
                    }
                    const unsigned bal = __ballot_sync(FULL, ins);
                    if (W == 1)
                    {
                        if (ins)
                            order[distinct + local + __popc(bal & lanemask_lt())] = slot;
                    }
                    else if (ins)
                    {
                        stage[local + __popc(bal & lanemask_lt())] = slot;
                    }
                    local += __popc(bal);
                    fail = __any_sync(FULL, fail);
                    if (fail || (W == 1 && distinct + local > CAP))
                    {
                        fail = true;
                        break;
                    }
                }
                if (W == 1)
                {
                    __syncwarp();
                    distinct += local;
                    if (fail)
                        aborted = true;
                }
                else
                {
                    // A failed probe is signalled as a negative count, so that
                    // every warp of the team reads the same decision after the
                    // barrier (the counts are double-buffered by jp parity).
                    if (lane == 0)
                        cnt[(jp & 1) * W + wt] = fail ? -1 : local;
                    team_sync<W>(team);
                    int pre = 0, tot = 0;
                    bool any_fail = false;
#pragma unroll
                    for (int w = 0; w < W; ++w)
                    {
                        const int c = cnt[(jp & 1) * W + w];
                        any_fail |= c < 0;
                        pre += (w < wt) ? c : 0;
                        tot += c;
                    }
                    if (!any_fail && distinct + tot <= TS)
                        for (int s = lane; s < local; s += 32)
                            order[distinct + pre + s] = stage[s];
                    __syncwarp();
                    distinct += tot;
                    if (any_fail || distinct > CAP)
                        aborted = true;
                }
                if (aborted)
                    break;
            }
        }

        if (aborted)
        {
            if (tid == 0)
                next_rows[atomicAdd(&tl->count[tier + 1], 1)] = i;
            team_sync<W>(team);
            continue;
        }

        // Compaction in first-touch order: keep k == i or |x| > threshold.
        // The barrier separates the last jp's reads of cnt from the rounds'.
        team_sync<W>(team);
        if (g.check_pre && distinct > g.Mc && tid == 0)
            atomicExch(&g.flags->overflow, 1);
        int ll = 0;
        int round = 0;
        for (int c0 = 0; c0 < distinct; c0 += W * 32, ++round)
        {
            const int q = c0 + wt * 32 + lane;
            bool keep = false;
            int k = 0;
            T x = T(0);
            if (q < distinct)
            {
                const int s = order[q];
                k = keys[s];
                x = vals[s];
                if (k == i)
                {
                    keep = true;
                    misc->diag = x;
                }
                else
                    keep = fabs(x) > thr;
            }
            const unsigned bal = __ballot_sync(FULL, keep);
            int pre = 0, tot = __popc(bal);
            if (W > 1)
            {
                if (lane == 0)
                    cnt[(round & 1) * W + wt] = tot;
                team_sync<W>(team);
                tot = 0;
#pragma unroll
                for (int w = 0; w < W; ++w)
                {
                    const int c = cnt[(round & 1) * W + w];
                    pre += (w < wt) ? c : 0;
                    tot += c;
                }
            }
            const int p = ll + pre + __popc(bal & lanemask_lt());
            if (keep && p < g.Mc)
            {
                Cv[(size_t) i * g.ldc + p] = x;
                g.Ci[(size_t) i * g.ldc + p] = k;
            }
            ll += tot;
        }
        team_sync<W>(team);
        if (tid == 0)
        {
            g.Cn[i] = min(ll, g.Mc);
            atomicMax(&g.flags->max_width, ll);
            if (ll > g.Mc)
                atomicExch(&g.flags->overflow, 1);
            if (g.dA)
                g.dA[i] = (double) dA;
            if (g.dC)
                g.dC[i] = (double) misc->diag;
        }
        team_sync<W>(team);
    }
}

// -------------------------------------------------------------------------
// Tier C: dense accumulator over all columns, in global memory, one slab per
// CTA: acc[ncols] (T), mark[ncols] (int, row+1 while the column is live),
// order[ncols] (int, column ids in first-touch order).  Marks are cleared
// column by column at the end of each row, as the reference clears ix[].
// -------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) dense_tier_kernel(MulArgs g, int smax, int ncols,
                                                        const int *rows, TierLists *tl,
                                                        unsigned char *slabs)
{
    constexpr int W = 8;
    extern __shared__ __align__(16) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int nrows = tl->count[2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wt = warp;
    const int tid = threadIdx.x;
    int *stage = reinterpret_cast<int *>(smem) + wt * smax;
    int *cnt = reinterpret_cast<int *>(smem) + W * smax;
    TeamMisc<T> *misc = reinterpret_cast<TeamMisc<T> *>(cnt + 2 * W);

    const size_t slab_bytes = (size_t) ncols * (sizeof(T) + 2 * sizeof(int));
    unsigned char *slab = slabs + (size_t) blockIdx.x * slab_bytes;
    T *acc = reinterpret_cast<T *>(slab);
    int *mark = reinterpret_cast<int *>(acc + ncols);
    int *order = mark + ncols;

    const T *Av = static_cast<const T *>(g.Av);
    const T *Bv = static_cast<const T *>(g.Bv);
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;

    bool marks_clear = false;
    for (;;)
    {
        if (tid == 0)
            misc->row = atomicAdd(&tl->cursor[2], 1);
        __syncthreads();
        const int pos = misc->row;
        if (pos >= nrows)
            break;
        const int i = rows[pos];
        if (!marks_clear)
        {
            // The slab is shared scratch: clear this CTA's marks once.
            for (int s = tid; s < ncols; s += 256)
                __stcg(&mark[s], 0);
            __syncthreads();
            marks_clear = true;
        }
        if (tid == 0)
            misc->diag = T(0);
        const int ni = g.An[i];
        const T *arow = Av + (size_t) i * g.lda;
        const int *airow = g.Ai + (size_t) i * g.lda;
        int distinct = 0;
        T dA = T(0);
        for (int jp0 = 0; jp0 < ni; jp0 += 32)
        {
            const int q = jp0 + lane;
            T av = T(0);
            int aj = 0, nj_l = 0;
            if (q < ni)
            {
                av = arow[q];
                aj = airow[q];
                nj_l = g.Bn[aj];
            }
            const int cnt_here = min(32, ni - jp0);
            for (int t = 0; t < cnt_here; ++t)
            {
                const int jp = jp0 + t;
                const T a = __shfl_sync(FULL, av, t);
                const int j = __shfl_sync(FULL, aj, t);
                const int nj = __shfl_sync(FULL, nj_l, t);
                if (j == i)
                    dA = add_rn(dA, a);
                const T *brow = Bv + (size_t) j * g.ldb;
                const int *birow = g.Bi + (size_t) j * g.ldb;
                const int S = b200_round_up(b200_ceil_div(nj, W), 32);
                const int k0 = min(wt * S, nj), k1 = min(k0 + S, nj);
                int local = 0;
                for (int kb = k0; kb < k1; kb += 32)
                {
                    const int kp = kb + lane;
                    bool ins = false;
                    int k = 0;
                    if (kp < k1)
                    {
                        k = birow[kp];
                        const T p = mul_rn(a, brow[kp]);
                        if (__ldcg(&mark[k]) != i + 1)
                        {
                            __stcg(&mark[k], i + 1);
                            __stcg(&acc[k], add_rn(T(0), p));
                            ins = true;
                        }
                        else
                            __stcg(&acc[k], add_rn(__ldcg(&acc[k]), p));
                    }
                    const unsigned bal = __ballot_sync(FULL, ins);
                    if (ins)
                        stage[local + __popc(bal & lanemask_lt())] = k;
                    local += __popc(bal);
                }
                if (lane == 0)
                    cnt[(jp & 1) * W + wt] = local;
                __syncthreads();
                int pre = 0, tot = 0;
#pragma unroll
                for (int w = 0; w < W; ++w)
                {
                    const int c = cnt[(jp & 1) * W + w];
                    pre += (w < wt) ? c : 0;
                    tot += c;
                }
                for (int s = lane; s < local; s += 32)
                    __stcg(&order[distinct + pre + s], stage[s]);
                __syncwarp();
                distinct += tot;
            }
        }
        __syncthreads();
        if (g.check_pre && distinct > g.Mc && tid == 0)
            atomicExch(&g.flags->overflow, 1);
        int ll = 0, round = 0;
        for (int c0 = 0; c0 < distinct; c0 += W * 32, ++round)
        {
            const int q = c0 + wt * 32 + lane;
            bool keep = false;
            int k = 0;
            T x = T(0);
            if (q < distinct)
            {
                k = __ldcg(&order[q]);
                x = __ldcg(&acc[k]);
                __stcg(&mark[k], 0);
                if (k == i)
                {
                    keep = true;
                    misc->diag = x;
                }
                else
                    keep = fabs(x) > thr;
            }
            const unsigned bal = __ballot_sync(FULL, keep);
            if (lane == 0)
                cnt[(round & 1) * W + wt] = __popc(bal);
            __syncthreads();
            int pre = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < W; ++w)
            {
                const int c = cnt[(round & 1) * W + w];
                pre += (w < wt) ? c : 0;
                tot += c;
            }
            const int p = ll + pre + __popc(bal & lanemask_lt());
            if (keep && p < g.Mc)
            {
                Cv[(size_t) i * g.ldc + p] = x;
                g.Ci[(size_t) i * g.ldc + p] = k;
            }
            ll += tot;
        }
        __syncthreads();
        if (tid == 0)
        {
            g.Cn[i] = min(ll, g.Mc);
            atomicMax(&g.flags->max_width, ll);
            if (ll > g.Mc)
                atomicExch(&g.flags->overflow, 1);
            if (g.dA)
                g.dA[i] = (double) dA;
            if (g.dC)
                g.dC[i] = (double) misc->diag;
        }
        __syncthreads();
    }
}

// Sum of per-row diagonal values (two arrays) in FP64, fixed order: each
// thread sums a contiguous stripe, then a tree over threads.  One block.
__global__ void __launch_bounds__(1024) trace_pair_kernel(const double *a, const double *b, int n,
                                                         double *out)
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

constexpr int TIER_A_LOGTS = 10; // 1024 slots, capacity 640
constexpr int TIER_B_LOGTS = 13; // 8192 slots, capacity 5120
constexpr int TIER_A_TEAMS = 4;  // one-warp teams per 128-thread block

template <typename T>
bool multiply_typed(MulArgs g, int ncols, double *trace, int *required_M)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const int N = g.NA;
    const int smaxB = b200_round_up(b200_ceil_div(g.ldb, 8), 32);
    const size_t smemA = team_smem_bytes<T, 1, TIER_A_LOGTS>(0) * TIER_A_TEAMS;
    const size_t smemB = team_smem_bytes<T, 8, TIER_B_LOGTS>(smaxB);
    const size_t smemC = (size_t) 8 * smaxB * sizeof(int) + 2 * 8 * sizeof(int) + 32;
    const bool tierB_ok = smemB <= c->smem_optin;
    if (smemC > c->smem_optin)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "row width %d too large for the multiply kernels", g.ldb);
        return false;
    }
    const int gridC = c->sm_count;
    const size_t slab_bytes = (size_t) ncols * (sizeof(T) + 2 * sizeof(int));

    // scratch: lists A/B/C (N ints each), diag arrays (2N doubles), slabs
    size_t off_lists = 0;
    size_t off_diag = (size_t) 3 * N * sizeof(int);
    off_diag = (off_diag + 255) & ~size_t(255);
    size_t off_slabs = off_diag + (size_t) 2 * N * sizeof(double);
    off_slabs = (off_slabs + 255) & ~size_t(255);
    size_t total = off_slabs + (size_t) gridC * slab_bytes;
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(total));
    if (!scr)
        return false;
    int *listA = reinterpret_cast<int *>(scr + off_lists);
    int *listB = listA + N;
    int *listC = listB + N;
    double *diagA = reinterpret_cast<double *>(scr + off_diag);
    double *diagC = diagA + N;
    unsigned char *slabs = scr + off_slabs;

    // small device block: TierLists | MulFlags | trace[2]
    unsigned char *small = static_cast<unsigned char *>(c->d_small);
    TierLists *tl = reinterpret_cast<TierLists *>(small);
    MulFlags *flags = reinterpret_cast<MulFlags *>(small + 64);
    double *dtrace = reinterpret_cast<double *>(small + 128);
    if (!CUDA_OK(cudaMemsetAsync(small, 0, 256, c->stream)))
        return false;
    g.flags = flags;
    if (trace)
    {
        g.dA = diagA;
        g.dC = diagC;
        if (!CUDA_OK(cudaMemsetAsync(diagA, 0, (size_t) 2 * N * sizeof(double), c->stream)))
            return false;
    }
    else
    {
        g.dA = nullptr;
        g.dC = nullptr;
    }

    const int plan_blocks = min(b200_ceil_div(N, 8), c->sm_count * 16);
    validate_cols_kernel<<<min(b200_ceil_div(g.NB, 8), c->sm_count * 16), 256, 0, c->stream>>>(
        g.Bi, g.Bn, g.ldb, g.NB, ncols, flags);
    // When tier B cannot hold its staging area (very wide rows), the rows past
    // tier A go straight to the dense tier: they are listed in listC under
    // count[1], and count[1] is copied to count[2] after tier A.
    int *listBC = tierB_ok ? listB : listC;
    plan_kernel<<<max(plan_blocks, 1), 256, 0, c->stream>>>(g, 640, tl, listA, listBC);
    if (!LAUNCH_OK("plan_kernel"))
        return false;

    if (!CUDA_OK(cudaFuncSetAttribute(hash_tier_kernel<T, 1, TIER_A_LOGTS>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemA)))
        return false;
    int occA = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occA, hash_tier_kernel<T, 1, TIER_A_LOGTS>,
                                                  32 * TIER_A_TEAMS, smemA);
    const int gridA = c->sm_count * max(occA, 1);
    hash_tier_kernel<T, 1, TIER_A_LOGTS><<<gridA, 32 * TIER_A_TEAMS, smemA, c->stream>>>(
        g, 0, listA, tl, 0, listBC);
    if (!LAUNCH_OK("hash_tier_kernel<A>"))
        return false;

    if (tierB_ok)
    {
        if (!CUDA_OK(cudaFuncSetAttribute(hash_tier_kernel<T, 8, TIER_B_LOGTS>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemB)))
            return false;
        int occB = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occB, hash_tier_kernel<T, 8, TIER_B_LOGTS>,
                                                      256, smemB);
        const int gridB = c->sm_count * max(occB, 1);
        hash_tier_kernel<T, 8, TIER_B_LOGTS><<<gridB, 256, smemB, c->stream>>>(g, smaxB, listB, tl,
                                                                               1, listC);
        if (!LAUNCH_OK("hash_tier_kernel<B>"))
            return false;
    }
    else
    {
        if (!CUDA_OK(cudaMemcpyAsync(&tl->count[2], &tl->count[1], sizeof(int),
                                     cudaMemcpyDeviceToDevice, c->stream)))
            return false;
    }

    if (!CUDA_OK(cudaFuncSetAttribute(dense_tier_kernel<T>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemC)))
        return false;
    dense_tier_kernel<T><<<gridC, 256, smemC, c->stream>>>(g, smaxB, ncols, listC, tl, slabs);
    if (!LAUNCH_OK("dense_tier_kernel"))
        return false;

    if (trace)
    {
        trace_pair_kernel<<<1, 1024, 0, c->stream>>>(diagA, diagC, N, dtrace);
        if (!LAUNCH_OK("trace_pair_kernel"))
            return false;
    }
    // bring back flags (+ traces)
    unsigned char *pin = static_cast<unsigned char *>(c->pinned);
    if (!CUDA_OK(cudaMemcpyAsync(pin, small, 256, cudaMemcpyDeviceToHost, c->stream)))
        return false;
    if (!b200_sync())
        return false;
    const MulFlags *hf = reinterpret_cast<const MulFlags *>(pin + 64);
    const double *ht = reinterpret_cast<const double *>(pin + 128);
    if (required_M)
        *required_M = hf->max_width;
    if (hf->bad_input)
    {
        b200_set_error(BML_B200_ERR_INVALID,
                       "multiply: a column index or row length of an input is out of range");
        return false;
    }
    if (trace)
    {
        trace[0] = ht[0];
        trace[1] = ht[1];
    }
    if (hf->overflow)
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW,
                       "Number of non-zeroes per row > M, Increase M (need %d, M = %d)",
                       hf->max_width, g.Mc);
        return false;
    }
    return true;
}

} // namespace

bool ell_multiply_AB(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C,
                     double threshold, double *trace, int *required_M)
{
    if (!A || !B || !C)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply: NULL matrix");
        return false;
    }
    if (A->matrix_precision != B->matrix_precision || A->matrix_precision != C->matrix_precision)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply: precision mismatch");
        return false;
    }
    if (A->N != C->N)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply: A has %d rows, C has %d", A->N, C->N);
        return false;
    }
    if (C == A || C == B)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply: output aliases an input");
        return false;
    }
    if (!ell_to_device(A) || (B != A && !ell_to_device(B)) || !ell_to_device(C))
        return false;
    MulArgs g{};
    g.Av = A->d_value; g.Ai = A->d_index; g.An = A->d_nnz; g.lda = A->ld; g.NA = A->N;
    g.Bv = B->d_value; g.Bi = B->d_index; g.Bn = B->d_nnz; g.ldb = B->ld; g.NB = B->N;
    g.Cv = C->d_value; g.Ci = C->d_index; g.Cn = C->d_nnz; g.ldc = C->ld; g.Mc = C->M;
    g.thr = threshold;
    // Column indices of B address columns of the product: at most max(B->N, C->N).
    const int ncols = B->N > C->N ? B->N : C->N;
    bool ok = A->matrix_precision == double_real
                  ? multiply_typed<double>(g, ncols, trace, required_M)
                  : multiply_typed<float>(g, ncols, trace, required_M);
    // C's device arrays now hold the product (also on ROW_OVERFLOW, truncated).
    ell_mark_device(C);
    return ok;
}
