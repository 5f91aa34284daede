// ELLPACK-R thresholded sparse product C = A*B (X^2 when A == B) on sm_100a.
//
// Follows the reference row-Gustavson loop
// (ellpack/bml_multiply_ellpack_typed.c:252-333 for X^2, :468-542 for A*B):
// for every row i, for jp in row order, for kp in the order of row j = col(i,jp),
//   x[k] = x[k] + a_ij * b_jk    (k = col(j,kp)); first touch starts at 0.0
// then the touched columns are visited in first-touch order and kept when
// k == i or |x| > threshold (typed.h:73, strict), and tr A / tr C are summed.
//
// B200 design.  A team of warps owns one output row and walks jp in order.
// Within one jp every k is distinct, so the lanes update their accumulator
// slots without races; a barrier between consecutive units of work keeps every
// x[k] summed in exactly the reference order.  Products and sums use
// __dmul_rn/__dadd_rn (no FMA contraction), matching the reference build
// (-std=c99, no -mfma), so each call is bit-identical to the reference on the
// same input.  New keys are appended to an order list with a warp ballot +
// popcount prefix (plus a cross-warp prefix), which rebuilds the reference's
// first-touch output order without sorting.
//
// Rows of B are staged into shared memory by TMA bulk copies
// (cp.async.bulk, completion on an mbarrier), STAGES units ahead of the team,
// so the gather latency overlaps the hash work of the preceding units.
//
// Tiers, chosen per row by a planning kernel from a bound or an estimate of
// the row's distinct columns (the previous call's counts, when the matrix
// size matches), each handing rows that outgrow it to the next:
//   A   1 warp per row, 1024-slot hash, direct loads (4 rows per block);
//   B1  4 warps, 2048-slot hash, TMA staging;
//   B2  4 warps, 4096-slot hash, TMA staging;
//   B3  16 warps, 8192-slot hash, TMA staging;
//   C   8 warps, dense accumulator over all columns in global memory (the
//       reference's own x[N]/ix[N]/jx[N] scheme; any width).
// All tiers are persistent grids pulling rows from device-side lists, so a
// multiply needs no host round trip until the traces are read back.
#include "device_util.cuh"

#include <cstring>

using namespace b200;

namespace {

// Flags shared by all tiers of one multiply call (device memory).
struct MulFlags
{
    int overflow;     // some row needed more than Mc entries
    int max_width;    // largest pre-truncation output width
    int bad_input;    // an input column index or nnz out of range
    int timeout;      // a bounded wait on a bulk copy ran out
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
    const int *hint;  // previous distinct-column counts per row (nullable)
    int *hint_out;    // distinct-column counts of this call
};

// Tiers: A (warp, 1024 slots), B1 (2048), B2 (4096), B3 (8192), C (dense).
// B200_X2_TIERS: bit t set = tier t in use (rows skip unused tiers);
// B200_C_BLOCKS: blocks per SM of the dense tier.
// Measured on B200 (SP2 on the 40^3 lattice): past ~1280 distinct columns a
// row runs faster in the dense tier at full occupancy than in the 4096- and
// 8192-slot shared-memory tables, so those two tiers are off by default.
#ifndef B200_X2_TIERS
#define B200_X2_TIERS 0x13
#endif
#ifndef B200_C_BLOCKS
#define B200_C_BLOCKS 8
#endif
constexpr int NTIERS = 5;
__constant__ int TIER_CAP[NTIERS] = {640, 1280, 2560, 5120, 0x7fffffff};

struct TierLists
{
    int count[NTIERS];
    int cursor[NTIERS];
};

struct TeamMisc
{
    double diag;
    int row;
    int pad;
};

// -------------------------------------------------------------------------
// Planning: product-count bound per row, input validation, tier choice.
// One warp per row.
// -------------------------------------------------------------------------
__global__ void plan_kernel(MulArgs g, int ncols, int skip_mid, TierLists *tl, int *lists)
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
            {
                atomicExch(&g.flags->bad_input, 1);
                continue;
            }
            long long est = P < ncols ? P : ncols;
            if (g.hint)
            {
                const long long h = (long long) g.hint[i] + g.hint[i] / 4 + 16;
                if (h < est)
                    est = h;
            }
            int t = 0;
            while (t < NTIERS - 1 && (est > TIER_CAP[t] || !((B200_X2_TIERS >> t) & 1)))
                ++t;
            if (skip_mid && t > 0)
                t = NTIERS - 1;
            lists[(size_t) t * g.NA + atomicAdd(&tl->count[t], 1)] = i;
        }
    }
}

// B's own column indices are checked where they are used (plan checks A's).
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

// Common row epilogue: write the row's results and bookkeeping.
template <typename T>
__device__ __forceinline__ void finish_row(const MulArgs &g, int i, int ll, int distinct, T dA,
                                           double diag)
{
    g.Cn[i] = min(ll, g.Mc);
    atomicMax(&g.flags->max_width, ll);
    if (ll > g.Mc || (g.check_pre && distinct > g.Mc))
        atomicExch(&g.flags->overflow, 1);
    if (g.dA)
        g.dA[i] = (double) dA;
    if (g.dC)
        g.dC[i] = diag;
    if (g.hint_out)
        g.hint_out[i] = distinct;
}

// -------------------------------------------------------------------------
// Tier A: one warp per row, 1024-slot table, direct (L1-cached) loads.
// Shared memory per warp: vals[TS] | keys[TS] | order[TS] (ushort)
// -------------------------------------------------------------------------
constexpr int A_LOGTS = 10;
constexpr int A_WARPS = 4;

template <typename T> constexpr size_t tierA_warp_bytes()
{
    return (size_t(1) << A_LOGTS) * (sizeof(T) + sizeof(int) + sizeof(unsigned short));
}

template <typename T>
__global__ void __launch_bounds__(32 * A_WARPS, 4) tierA_kernel(MulArgs g, const int *rows,
                                                            TierLists *tl, int next_tier,
                                                            int *next_rows)
{
    constexpr int TS = 1 << A_LOGTS;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int CAP = TIER_CAP[0];
    const int nrows = tl->count[0];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *base = smem + (size_t) warp * tierA_warp_bytes<T>();
    T *vals = reinterpret_cast<T *>(base);
    int *keys = reinterpret_cast<int *>(vals + TS);
    unsigned short *order = reinterpret_cast<unsigned short *>(keys + TS);
    const T *Av = static_cast<const T *>(g.Av);
    const T *Bv = static_cast<const T *>(g.Bv);
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;

    for (;;)
    {
        int pos = 0;
        if (lane == 0)
            pos = atomicAdd(&tl->cursor[0], 1);
        pos = __shfl_sync(FULL, pos, 0);
        if (pos >= nrows)
            break;
        const int i = rows[pos];
        for (int s = lane; s < TS; s += 32)
        {
            keys[s] = B200_EMPTY_KEY;
            vals[s] = T(0);
        }
        __syncwarp();
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
            for (int t = 0; t < cnt_here && !aborted; ++t)
            {
                const T a = __shfl_sync(FULL, av, t);
                const int j = __shfl_sync(FULL, aj, t);
                const int nj = __shfl_sync(FULL, nj_l, t);
                if (j == i)
                    dA = add_rn(dA, a);
                const T *brow = Bv + (size_t) j * g.ldb;
                const int *birow = g.Bi + (size_t) j * g.ldb;
                for (int kb = 0; kb < nj; kb += 32)
                {
                    const int kp = kb + lane;
                    bool ins = false;
                    int slot = -1;
                    if (kp < nj)
                    {
                        const int k = birow[kp];
                        const T p = mul_rn(a, brow[kp]);
                        slot = probe_insert<A_LOGTS>(keys, k, ins);
                        if (slot >= 0)
                            vals[slot] = add_rn(vals[slot], p);
                    }
                    const unsigned bal = __ballot_sync(FULL, ins);
                    if (ins)
                        order[distinct + __popc(bal & lanemask_lt())] = (unsigned short) slot;
                    distinct += __popc(bal);
                    if (__any_sync(FULL, kp < nj && slot < 0) || distinct > CAP)
                    {
                        aborted = true;
                        break;
                    }
                }
                __syncwarp();
            }
        }
        if (aborted)
        {
            if (lane == 0)
                next_rows[atomicAdd(&tl->count[next_tier], 1)] = i;
            __syncwarp();
            continue;
        }
        int ll = 0;
        double diag = 0.0;
        for (int c0 = 0; c0 < distinct; c0 += 32)
        {
            const int q = c0 + lane;
            bool keep = false;
            int k = 0;
            T x = T(0);
            if (q < distinct)
            {
                const int s = order[q];
                k = keys[s];
                x = vals[s];
                keep = (k == i) || fabs(x) > thr;
            }
            const unsigned dbal = __ballot_sync(FULL, q < distinct && k == i);
            if (dbal)
                diag = (double) __shfl_sync(FULL, x, __ffs(dbal) - 1);
            const unsigned bal = __ballot_sync(FULL, keep);
            const int p = ll + __popc(bal & lanemask_lt());
            if (keep && p < g.Mc)
            {
                Cv[(size_t) i * g.ldc + p] = x;
                g.Ci[(size_t) i * g.ldc + p] = k;
            }
            ll += __popc(bal);
        }
        if (lane == 0)
            finish_row<T>(g, i, ll, distinct, dA, diag);
        __syncwarp();
    }
}

// -------------------------------------------------------------------------
// Tiers B1-B3: a team of W warps per row (one team per block), rows of B
// staged by TMA bulk copies in units of at most CHUNK entries.
// Shared memory: mbar[STAGES] | sv[STAGES][CHUNK] | sk[STAGES][CHUNK] |
//                vals[TS] | keys[TS] | order[TS] (ushort) |
//                stg[W][SPW] (ushort) | cnt[2][W] | misc
// -------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of `bar`, giving up after ~2 s (a bulk copy that
// never lands); on timeout the caller's flag is raised and false returned.
__device__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *timeout_flag)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const unsigned long long t0 = global_ns();
    for (;;)
    {
        if (mbar_try_wait(bar, parity))
            return true;
        if (global_ns() - t0 > 2000000000ull)
        {
            atomicExch(timeout_flag, 1);
            return false;
        }
    }
}

template <typename T, int W, int LOGTS, int STAGES, int CHUNK> struct TeamCfg
{
    static constexpr int TS = 1 << LOGTS;
    static constexpr int NT = W * 32;
    static constexpr int SPW = ((CHUNK + W - 1) / W + 31) / 32 * 32; // staging per warp
    static constexpr size_t off_sv = 128;
    static constexpr size_t off_sk = off_sv + size_t(STAGES) * CHUNK * sizeof(T);
    static constexpr size_t off_vals = off_sk + size_t(STAGES) * CHUNK * sizeof(int);
    static constexpr size_t off_keys = off_vals + size_t(TS) * sizeof(T);
    static constexpr size_t off_order = off_keys + size_t(TS) * sizeof(int);
    static constexpr size_t off_stg = off_order + size_t(TS) * sizeof(unsigned short);
    static constexpr size_t off_cnt =
        (off_stg + size_t(W) * SPW * sizeof(unsigned short) + 15) / 16 * 16;
    static constexpr size_t off_misc = off_cnt + 2 * W * sizeof(int);
    static constexpr size_t bytes = off_misc + sizeof(TeamMisc) + 16;
};

template <typename T, int W, int LOGTS, int STAGES, int CHUNK, int MINB>
__global__ void __launch_bounds__(W * 32, MINB) team_kernel(MulArgs g, const int *rows, TierLists *tl,
                                                           int tier, int next_tier, int *next_rows)
{
    using Cfg = TeamCfg<T, W, LOGTS, STAGES, CHUNK>;
    constexpr int TS = Cfg::TS, NT = Cfg::NT, SPW = Cfg::SPW;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int CAP = TIER_CAP[tier];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);
    T *sv = reinterpret_cast<T *>(smem + Cfg::off_sv);
    int *sk = reinterpret_cast<int *>(smem + Cfg::off_sk);
    T *vals = reinterpret_cast<T *>(smem + Cfg::off_vals);
    int *keys = reinterpret_cast<int *>(smem + Cfg::off_keys);
    unsigned short *order = reinterpret_cast<unsigned short *>(smem + Cfg::off_order);
    int *cnt = reinterpret_cast<int *>(smem + Cfg::off_cnt);
    TeamMisc *misc = reinterpret_cast<TeamMisc *>(smem + Cfg::off_misc);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned short *stg = reinterpret_cast<unsigned short *>(smem + Cfg::off_stg) + warp * SPW;

    const int nrows = tl->count[tier];
    const T *Av = static_cast<const T *>(g.Av);
    const T *Bv = static_cast<const T *>(g.Bv);
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;
    int *tflag = &g.flags->timeout;

    if (tid == 0)
    {
        for (int s = 0; s < STAGES; ++s)
            mbar_init(&mbar[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    unsigned ucount = 0; // units consumed by this block (uniform)
    for (;;)
    {
        if (tid == 0)
            misc->row = atomicAdd(&tl->cursor[tier], 1);
        __syncthreads();
        const int pos = misc->row;
        if (pos >= nrows || *reinterpret_cast<volatile int *>(tflag))
            break;
        const int i = rows[pos];
        for (int s = tid; s < TS; s += NT)
        {
            keys[s] = B200_EMPTY_KEY;
            vals[s] = T(0);
        }
        if (tid == 0)
            misc->diag = 0.0;
        __syncthreads();

        const int ni = g.An[i];
        const T *arow = Av + (size_t) i * g.lda;
        const int *airow = g.Ai + (size_t) i * g.lda;

        // Producer position (tracked by every thread, issued by thread 0):
        // the next unit to copy is chunk pc of the B row named at position pj.
        int pj = 0, pc = 0, pnj = 0;
        auto prod_skip = [&]() {
            while (pj < ni)
            {
                pnj = g.Bn[airow[pj]];
                if (pc * CHUNK < pnj)
                    return;
                ++pj;
                pc = 0;
            }
        };
        auto issue = [&](unsigned slot_u) {
            const int s = slot_u % STAGES;
            const int j = airow[pj];
            const int off = pc * CHUNK;
            const int n = min(CHUNK, pnj - off);
            const unsigned bv = (unsigned) ((n * sizeof(T) + 15) & ~size_t(15));
            const unsigned bk = (unsigned) ((n * sizeof(int) + 15) & ~size_t(15));
            if (tid == 0)
            {
                mbar_expect_tx(&mbar[s], bv + bk);
                bulk_g2s(sv + (size_t) s * CHUNK, Bv + (size_t) j * g.ldb + off, bv, &mbar[s]);
                bulk_g2s(sk + (size_t) s * CHUNK, g.Bi + (size_t) j * g.ldb + off, bk, &mbar[s]);
            }
            ++pc;
        };
        prod_skip();
        unsigned issued = 0;
        while (issued < STAGES && pj < ni)
        {
            issue(ucount + issued);
            ++issued;
            prod_skip();
        }

        int distinct = 0;
        T dA = T(0);
        bool aborted = false;
        unsigned consumed = 0;
        for (int jp = 0; jp < ni && !aborted; ++jp)
        {
            const T a = arow[jp];
            const int j = airow[jp];
            const int nj = g.Bn[j];
            if (j == i)
                dA = add_rn(dA, a);
            for (int off = 0; off < nj; off += CHUNK)
            {
                const unsigned u = ucount + consumed;
                const int s = u % STAGES;
                const int n = min(CHUNK, nj - off);
                mbar_wait_bounded(&mbar[s], (u / STAGES) & 1, tflag);
                const T *uv = sv + (size_t) s * CHUNK;
                const int *uk = sk + (size_t) s * CHUNK;
                const int S = b200_round_up(b200_ceil_div(n, W), 32);
                const int k0 = min(warp * S, n), k1 = min(k0 + S, n);
                int local = 0;
                bool fail = false;
                for (int kb = k0; kb < k1; kb += 32)
                {
                    const int kp = kb + lane;
                    bool ins = false;
                    int slot = -1;
                    if (kp < k1)
                    {
                        const int k = uk[kp];
                        const T p = mul_rn(a, uv[kp]);
                        slot = probe_insert<LOGTS>(keys, k, ins);
                        if (slot >= 0)
                            vals[slot] = add_rn(vals[slot], p);
                        else
                            fail = true;
                    }
                    const unsigned bal = __ballot_sync(FULL, ins);
                    if (ins)
                        stg[local + __popc(bal & lanemask_lt())] = (unsigned short) slot;
                    local += __popc(bal);
                }
                fail = __any_sync(FULL, fail);
                if (lane == 0)
                    cnt[(u & 1) * W + warp] = fail ? -1 : local;
                __syncthreads();
                ++consumed;
                int pre = 0, tot = 0;
                bool any_fail = false;
#pragma unroll
                for (int w = 0; w < W; ++w)
                {
                    const int cw = cnt[(u & 1) * W + w];
                    any_fail |= cw < 0;
                    pre += (w < warp) ? cw : 0;
                    tot += cw;
                }
                if (!any_fail && distinct + tot <= TS)
                    for (int q = lane; q < local; q += 32)
                        order[distinct + pre + q] = stg[q];
                __syncwarp();
                distinct += tot;
                if (any_fail || distinct > CAP)
                {
                    aborted = true;
                    break;
                }
                // the stage just consumed is free: refill it
                if (pj < ni)
                {
                    issue(ucount + issued);
                    ++issued;
                    prod_skip();
                }
            }
        }
        // Drain copies still in flight for this row (only after an abort).
        while (consumed < issued)
        {
            const unsigned u = ucount + consumed;
            mbar_wait_bounded(&mbar[u % STAGES], (u / STAGES) & 1, tflag);
            ++consumed;
        }
        ucount += consumed;
        __syncthreads();
        if (aborted)
        {
            if (tid == 0)
                next_rows[atomicAdd(&tl->count[next_tier], 1)] = i;
            continue;
        }

        // Compaction in first-touch order: keep k == i or |x| > threshold.
        int ll = 0, round = 0;
        for (int c0 = 0; c0 < distinct; c0 += NT, ++round)
        {
            const int q = c0 + warp * 32 + lane;
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
                    misc->diag = (double) x;
                }
                else
                    keep = fabs(x) > thr;
            }
            const unsigned bal = __ballot_sync(FULL, keep);
            if (lane == 0)
                cnt[(round & 1) * W + warp] = __popc(bal);
            __syncthreads();
            int pre = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < W; ++w)
            {
                const int cw = cnt[(round & 1) * W + w];
                pre += (w < warp) ? cw : 0;
                tot += cw;
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
            finish_row<T>(g, i, ll, distinct, dA, misc->diag);
    }
}

// -------------------------------------------------------------------------
// Tier C: dense accumulator over all columns, in global memory, one slab per
// block: acc[ncols] (T), mark[ncols] (int, row+1 while the column is live),
// order[ncols] (int, column ids in first-touch order).  Marks are cleared
// column by column at the end of each row, as the reference clears ix[].
// -------------------------------------------------------------------------
constexpr int C_W = 8;

template <typename T>
__global__ void __launch_bounds__(256, B200_C_BLOCKS) dense_tier_kernel(MulArgs g, int smax, int ncols,
                                                        const int *rows, TierLists *tl,
                                                        unsigned char *slabs)
{
    constexpr int W = C_W;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int nrows = tl->count[NTIERS - 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wt = warp;
    const int tid = threadIdx.x;
    int *stage = reinterpret_cast<int *>(smem) + wt * smax;
    int *cnt = reinterpret_cast<int *>(smem) + W * smax;
    TeamMisc *misc = reinterpret_cast<TeamMisc *>(cnt + 2 * W);

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
            misc->row = atomicAdd(&tl->cursor[NTIERS - 1], 1);
        __syncthreads();
        const int pos = misc->row;
        if (pos >= nrows)
            break;
        const int i = rows[pos];
        if (!marks_clear)
        {
            // The slab is shared scratch: clear this block's marks once.
            for (int s = tid; s < ncols; s += 256)
                mark[s] = 0;
            __syncthreads();
            marks_clear = true;
        }
        if (tid == 0)
            misc->diag = 0.0;
        const int ni = g.An[i];
        const T *arow = Av + (size_t) i * g.lda;
        const int *airow = g.Ai + (size_t) i * g.lda;
        int distinct = 0;
        T dA = T(0);
        int step = 0;
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
            for (int t = 0; t < cnt_here; ++t, ++step)
            {
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
                        if (mark[k] != i + 1)
                        {
                            mark[k] = i + 1;
                            acc[k] = add_rn(T(0), p);
                            ins = true;
                        }
                        else
                            acc[k] = add_rn(acc[k], p);
                    }
                    const unsigned bal = __ballot_sync(FULL, ins);
                    if (ins)
                        stage[local + __popc(bal & lanemask_lt())] = k;
                    local += __popc(bal);
                }
                if (lane == 0)
                    cnt[(step & 1) * W + wt] = local;
                __syncthreads();
                int pre = 0, tot = 0;
#pragma unroll
                for (int w = 0; w < W; ++w)
                {
                    const int c = cnt[(step & 1) * W + w];
                    pre += (w < wt) ? c : 0;
                    tot += c;
                }
                for (int s = lane; s < local; s += 32)
                    order[distinct + pre + s] = stage[s];
                __syncwarp();
                distinct += tot;
            }
        }
        __syncthreads();
        int ll = 0, round = 0;
        for (int c0 = 0; c0 < distinct; c0 += W * 32, ++round)
        {
            const int q = c0 + wt * 32 + lane;
            bool keep = false;
            int k = 0;
            T x = T(0);
            if (q < distinct)
            {
                k = order[q];
                x = acc[k];
                mark[k] = 0;
                if (k == i)
                {
                    keep = true;
                    misc->diag = (double) x;
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
            finish_row<T>(g, i, ll, distinct, dA, misc->diag);
        __syncthreads();
    }
}

// Team tier configurations: (W, LOGTS, STAGES, CHUNK, min blocks per SM)
#define B1_CFG 4, 11, 3, 256, 4
#define B2_CFG 4, 12, 3, 256, 3
#define B3_CFG 16, 13, 3, 512, 1

template <typename T, int W, int LOGTS, int STAGES, int CHUNK, int MINB>
bool launch_team(B200Context *c, const MulArgs &g, const int *rows, TierLists *tl, int tier,
                 int next_tier, int *next_rows)
{
    using Cfg = TeamCfg<T, W, LOGTS, STAGES, CHUNK>;
    auto k = team_kernel<T, W, LOGTS, STAGES, CHUNK, MINB>;
    if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Cfg::bytes)))
        return false;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, W * 32, Cfg::bytes);
    const int grid = c->sm_count * (occ > 0 ? occ : 1);
    k<<<grid, W * 32, Cfg::bytes, c->stream>>>(g, rows, tl, tier, next_tier, next_rows);
    return LAUNCH_OK("team_kernel");
}

constexpr int C_BLOCKS_PER_SM = B200_C_BLOCKS;

// Distinct-column counts of the last multiply, reused as the next call's
// tier estimate when the row count matches (SP2 multiplies the same-size
// matrix over and over; a stale estimate only costs a retry in a larger tier).
int *g_hint = nullptr;
int g_hint_n = 0;
bool g_hint_valid = false;
int g_last_tiers[NTIERS] = {0};

template <typename T>
bool multiply_typed(MulArgs g, int ncols, double *trace, int *required_M)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const int N = g.NA;
    const int smaxC = b200_round_up(b200_ceil_div(g.ldb, C_W), 32);
    const size_t smemA = tierA_warp_bytes<T>() * A_WARPS;
    const size_t smemC = (size_t) C_W * smaxC * sizeof(int) + 2 * C_W * sizeof(int) + 32;
    if (smemC > c->smem_optin)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "row width %d too large for the multiply kernels", g.ldb);
        return false;
    }
    const int gridC = c->sm_count * C_BLOCKS_PER_SM;
    const size_t slab_bytes = (size_t) ncols * (sizeof(T) + 2 * sizeof(int));

    if (g_hint_n != N)
    {
        if (g_hint)
            cudaFree(g_hint);
        g_hint = nullptr;
        g_hint_valid = false;
        g_hint_n = 0;
        if (!CUDA_OK(cudaMalloc(&g_hint, (size_t) N * sizeof(int))))
            return false;
        g_hint_n = N;
    }
    g.hint = g_hint_valid ? g_hint : nullptr;
    g.hint_out = g_hint;

    // scratch: NTIERS lists of N ints, diag arrays (2N doubles), dense slabs
    size_t off_diag = ((size_t) NTIERS * N * sizeof(int) + 255) & ~size_t(255);
    size_t off_slabs = (off_diag + (size_t) 2 * N * sizeof(double) + 255) & ~size_t(255);
    size_t total = off_slabs + (size_t) gridC * slab_bytes;
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(total));
    if (!scr)
        return false;
    int *lists = reinterpret_cast<int *>(scr);
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

    const int vgrid = max(1, min(b200_ceil_div(g.NB, 8), c->sm_count * 16));
    validate_cols_kernel<<<vgrid, 256, 0, c->stream>>>(g.Bi, g.Bn, g.ldb, g.NB, ncols, flags);
    if (!LAUNCH_OK("validate_cols_kernel"))
        return false;
    const int pgrid = max(1, min(b200_ceil_div(N, 8), c->sm_count * 16));
    // The team tiers keep order positions in 16 bits: tables of at most 8192.
    plan_kernel<<<pgrid, 256, 0, c->stream>>>(g, ncols, 0, tl, lists);
    if (!LAUNCH_OK("plan_kernel"))
        return false;

    auto list = [&](int t) { return lists + (size_t) t * N; };
    if (!CUDA_OK(cudaFuncSetAttribute(tierA_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) smemA)))
        return false;
    int occA = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occA, tierA_kernel<T>, 32 * A_WARPS, smemA);
    int nextA = 1;
    while (nextA < NTIERS - 1 && !((B200_X2_TIERS >> nextA) & 1))
        ++nextA;
    tierA_kernel<T><<<c->sm_count * max(occA, 1), 32 * A_WARPS, smemA, c->stream>>>(
        g, list(0), tl, nextA, list(nextA));
    if (!LAUNCH_OK("tierA_kernel"))
        return false;
    // Rows a tier cannot hold go to the next tier in use (the dense tier
    // always is); tiers switched off are not launched.
    {
        auto next_on = [](int t) {
            int n = t + 1;
            while (n < NTIERS - 1 && !((B200_X2_TIERS >> n) & 1))
                ++n;
            return n;
        };
        if ((B200_X2_TIERS >> 1) & 1)
            if (!launch_team<T, B1_CFG>(c, g, list(1), tl, 1, next_on(1), list(next_on(1))))
                return false;
        if ((B200_X2_TIERS >> 2) & 1)
            if (!launch_team<T, B2_CFG>(c, g, list(2), tl, 2, next_on(2), list(next_on(2))))
                return false;
        if ((B200_X2_TIERS >> 3) & 1)
            if (!launch_team<T, B3_CFG>(c, g, list(3), tl, 3, next_on(3), list(next_on(3))))
                return false;
    }
    if (!CUDA_OK(cudaFuncSetAttribute(dense_tier_kernel<T>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemC)))
        return false;
    dense_tier_kernel<T><<<gridC, 256, smemC, c->stream>>>(g, smaxC, ncols, list(NTIERS - 1), tl, slabs);
    if (!LAUNCH_OK("dense_tier_kernel"))
        return false;

    if (trace)
    {
        b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(diagA, diagC, N, dtrace);
        if (!LAUNCH_OK("b200_sum_rows_kernel"))
            return false;
    }
    unsigned char *pin = static_cast<unsigned char *>(c->pinned);
    if (!CUDA_OK(cudaMemcpyAsync(pin, small, 256, cudaMemcpyDeviceToHost, c->stream)))
        return false;
    if (!b200_sync())
        return false;
    const MulFlags *hf = reinterpret_cast<const MulFlags *>(pin + 64);
    const double *ht = reinterpret_cast<const double *>(pin + 128);
    memcpy(g_last_tiers, reinterpret_cast<const TierLists *>(pin)->count, sizeof(g_last_tiers));
    if (required_M)
        *required_M = hf->max_width;
    if (hf->bad_input)
    {
        g_hint_valid = false;
        b200_set_error(BML_B200_ERR_INVALID,
                       "multiply: a column index or row length of an input is out of range");
        return false;
    }
    if (hf->timeout)
    {
        g_hint_valid = false;
        b200_set_error(BML_B200_ERR_TIMEOUT, "multiply: a shared-memory bulk copy did not complete");
        return false;
    }
    g_hint_valid = true;
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
    if (C->mirror == MIRROR_HOST_NEWER)
        C->mirror = MIRROR_SYNCED;
    MulArgs g{};
    g.Av = A->d_value; g.Ai = A->d_index; g.An = A->d_nnz; g.lda = A->ld; g.NA = A->N;
    g.Bv = B->d_value; g.Bi = B->d_index; g.Bn = B->d_nnz; g.ldb = B->ld; g.NB = B->N;
    g.Cv = C->d_value; g.Ci = C->d_index; g.Cn = C->d_nnz; g.ldc = C->ld; g.Mc = C->M;
    g.thr = threshold;
    g.check_pre = (A != B) ? 1 : 0;
    // Column indices of B address columns of the product: at most max(B->N, C->N).
    const int ncols = B->N > C->N ? B->N : C->N;
    bool ok = A->matrix_precision == double_real
                  ? multiply_typed<double>(g, ncols, trace, required_M)
                  : multiply_typed<float>(g, ncols, trace, required_M);
    // C's device arrays now hold the product (also on ROW_OVERFLOW, truncated).
    ell_mark_device(C);
    return ok;
}

// Rows handled by each multiply tier in the last call on this process
// (A, O1, O2, O3, C; a row handed on is counted in every tier it entered).
extern "C" BML_B200_API int bml_b200_last_tier_counts(int *counts, int n)
{
    for (int t = 0; t < n && t < NTIERS; ++t)
        counts[t] = g_last_tiers[t];
    return NTIERS;
}
