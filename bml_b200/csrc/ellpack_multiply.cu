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
// size matches), each handing rows that outgrow it to the next tier in use:
//   A   1 warp per row, 1024-slot hash, direct loads (4 rows per block);
//   W8  8 warps per row, each owning 4 of the 32 column classes k % 32,
//       256-slot private hash per warp, no barrier between jps;
//   B1  4 warps sharing a 2048-slot hash, rows of B staged by TMA;
//   W16 16 warps (2 classes each), 256 slots per warp;
//   K4  8 warps, two passes: a bitmap of the row's column window ranks the
//       columns into a compact accumulator of up to 4096 entries;
//   K8  as K4 with up to 8192 entries in shared memory, more in a compact
//       per-block slab in device memory (any width up to a 65536-column
//       window and 2048 kept columns);
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

// Tiers in routing order: A, W8, B1, W16, K4, K8, C (dense).
// B200_X2_TIERS: bit t set = tier t in use (rows skip unused tiers; the dense
// tier is always in use).
// Measured on B200 over 4 FP64 SP2 iterations on the 40^3 lattice (N=64000,
// radius 3), with the dense tier's first form: A + B1 + C 776 ms, A + K8
// 791 ms, A + B1 + K4 + K8 927 ms, A + W8 + W16 + K4 + K8 994 ms.  The dense
// tier's later forms (below) took A + B1 + C to 358 ms and A + C to 348 ms:
// the staged dense tier is now faster than B1 on B1's rows too.  The rows
// there reach 8000+ distinct columns before thresholding, where the dense
// tier's device-memory accumulator wins; the other tiers stay selectable at
// run time.
#ifndef B200_X2_TIERS
#define B200_X2_TIERS 0x01
#endif
#ifndef B200_C_BLOCKS
#define B200_C_BLOCKS 6
#endif
#ifndef B200_DENSE_BITS
#define B200_DENSE_BITS 1
#endif
constexpr int NTIERS = 7;
constexpr int TIER_W8 = 1, TIER_B1 = 2, TIER_W16 = 3, TIER_K4 = 4, TIER_K8 = 5, TIER_C = NTIERS - 1;
constexpr int BUCKET_TIERS_MASK = (1 << TIER_W8) | (1 << TIER_W16) | (1 << TIER_K4) | (1 << TIER_K8);
constexpr int WINDOW_TIERS_MASK = (1 << TIER_K4) | (1 << TIER_K8);
__constant__ int TIER_CAP[NTIERS] = {640, 1100, 1280, 2200, 4096, 0x7fffffff, 0x7fffffff};

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
__global__ void plan_kernel(MulArgs g, int ncols, int tmask, TierLists *tl, int *lists)
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
                const long long h = 2 * (long long) g.hint[i] + 16;
                if (h < est)
                    est = h;
            }
            int t = 0;
            while (t < NTIERS - 1 && (est > TIER_CAP[t] || !((tmask >> t) & 1)))
                ++t;
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
        // one thread decides (a flag read by every thread could change
        // between their reads and split the block at the barrier)
        if (tid == 0)
            misc->row = *reinterpret_cast<volatile int *>(tflag) ? nrows : atomicAdd(&tl->cursor[tier], 1);
        __syncthreads();
        const int pos = misc->row;
        if (pos >= nrows)
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
// Wide tiers W8, W16: a team of W warps per row (one team per
// block).  Columns fall in 32 classes, k % 32, and warp w owns the classes
// [w*32/W, (w+1)*32/W).  Each warp keeps a private hash of its own columns and
// walks every jp of the row in order over its share of row j of B, so each
// x[k] is summed by one warp in the reference order and the warps never wait
// for one another inside a row.
// B's rows are first regrouped by class into a bucketed copy (stable, so each
// bucket keeps the row's order, with every entry's original position): a
// warp's share of row j is one contiguous range, read with coalesced loads,
// PF jps ahead of the one it is summing.
// A warp's inserts carry the key (jp << 16 | original position); sorted by
// that key (already sorted when a warp owns one class) a list is the
// reference's first-touch order restricted to the warp's columns, and a kept
// entry's output slot is the number of kept entries with a smaller key in all
// W lists.
// Shared memory per warp: vals[TS] | keys[TS] | okey[LP] (u32) |
//                         oslot[LP] (u16) | kcnt[CAP+1] (u16, kept prefix)
// -------------------------------------------------------------------------
constexpr int NCLS = 32; // column classes
constexpr int PF = 4;    // jps of prefetch

struct BucketArgs
{
    void *v;           // values [NB][ldb], matrix precision
    int *c;            // columns [NB][ldb]
    unsigned short *p; // original position of each entry within its row [NB][ldb]
    int *off;          // [NB][NCLS + 1]: start of bucket b; off[NCLS] = row length
    int *cmin, *cmax;  // [NB]: smallest / largest column of each row (empty: INT_MAX / -1)
};

// Stable regrouping of every row of B by column class.  One warp per row;
// eight warps per block.
template <typename T>
__global__ void __launch_bounds__(256) bucket_kernel(const T *__restrict__ Bv, const int *__restrict__ Bi,
                                                     const int *__restrict__ Bn, int ldb, int NB,
                                                     BucketArgs ba)
{
    __shared__ int run_s[8][NCLS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int *run = run_s[wib];
    const int warps = (gridDim.x * blockDim.x) >> 5;
    T *Pv = static_cast<T *>(ba.v);
    for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < NB; j += warps)
    {
        int nj = Bn[j];
        if (nj < 0 || nj > ldb) // rejected by the plan; keep the copy in bounds
            nj = 0;
        const size_t rb = (size_t) j * ldb;
        run[lane] = 0;
        __syncwarp();
        for (int c0 = 0; c0 < nj; c0 += 32)
        {
            const int q = c0 + lane;
            const int b = q < nj ? (Bi[rb + q] & (NCLS - 1)) : -1;
            const unsigned same = __match_any_sync(FULL, b);
            if (b >= 0 && (same & lanemask_lt()) == 0)
                run[b] += __popc(same);
            __syncwarp();
        }
        const int cnt = run[lane];
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1)
        {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o)
                incl += y;
        }
        int *off = ba.off + (size_t) j * (NCLS + 1);
        off[lane] = incl - cnt;
        if (lane == 31)
            off[NCLS] = incl;
        int mn = 0x7fffffff, mx = -1;
        for (int q = lane; q < nj; q += 32)
        {
            const int k = Bi[rb + q];
            mn = min(mn, k);
            mx = max(mx, k);
        }
        mn = __reduce_min_sync(FULL, mn);
        mx = __reduce_max_sync(FULL, mx);
        if (lane == 0)
        {
            ba.cmin[j] = mn;
            ba.cmax[j] = mx;
        }
        __syncwarp();
        run[lane] = incl - cnt;
        __syncwarp();
        for (int c0 = 0; c0 < nj; c0 += 32)
        {
            const int q = c0 + lane;
            int k = 0, b = -1;
            T v = T(0);
            if (q < nj)
            {
                k = Bi[rb + q];
                v = Bv[rb + q];
                b = k & (NCLS - 1);
            }
            const unsigned same = __match_any_sync(FULL, b);
            if (b >= 0)
            {
                const size_t dst = rb + run[b] + __popc(same & lanemask_lt());
                Pv[dst] = v;
                ba.c[dst] = k;
                ba.p[dst] = (unsigned short) q;
            }
            __syncwarp();
            if (b >= 0 && (same & lanemask_lt()) == 0)
                run[b] += __popc(same);
            __syncwarp();
        }
    }
}

struct WideMisc
{
    double diag;
    int row;
    int abort;
    int dw[32];   // list length per warp
    int kept[32]; // kept entries per warp
};

constexpr int pow2_ceil(int x)
{
    int p = 1;
    while (p < x)
        p <<= 1;
    return p;
}

constexpr int ilog2(int x)
{
    int l = 0;
    while ((1 << (l + 1)) <= x)
        ++l;
    return l;
}

template <typename T, int W, int TS> struct WideCfg
{
    static constexpr int R = NCLS / W;        // buckets per warp
    static constexpr int CAP = TS * 11 / 16;  // distinct columns per warp before handing on
    static constexpr int LP = R > 1 ? pow2_ceil(CAP) : CAP; // list length (sort padding)
    static constexpr size_t off_keys = size_t(TS) * sizeof(T);
    static constexpr size_t off_okey = off_keys + size_t(TS) * sizeof(int);
    static constexpr size_t off_oslot = off_okey + size_t(LP) * sizeof(unsigned);
    static constexpr size_t off_kcnt = off_oslot + size_t(LP) * sizeof(unsigned short);
    static constexpr size_t warp_bytes =
        (off_kcnt + size_t(CAP + 1) * sizeof(unsigned short) + 15) / 16 * 16;
    static constexpr size_t off_misc = W * warp_bytes;
    static constexpr size_t bytes = off_misc + sizeof(WideMisc);
};

// Open-addressing slot of column k in a table of TS slots (any TS): the
// column rotated right by 5 (class bits on top), Fibonacci-hashed, scaled.
template <int TS> __device__ __forceinline__ unsigned wide_hash(int k)
{
    const unsigned x = (((unsigned) k >> 5) | ((unsigned) k << 27)) * 2654435761u;
    if ((TS & (TS - 1)) == 0)
        return x >> (32 - ilog2(TS));
    return __umulhi(x, (unsigned) TS);
}

template <int TS>
__device__ __forceinline__ int wide_probe(int *keys, int k, bool &inserted)
{
    unsigned h = wide_hash<TS>(k);
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
        h = (h + 1 == TS) ? 0 : h + 1;
    }
    inserted = false;
    return -1;
}

// Row meta of one block of 32 jps, one jp per lane: A's value, the B row, and
// the warp's bucket range in that row.
template <typename T> struct JpMeta
{
    T a;
    int j, lo, hi;
};

template <typename T, int W, int TS, int MINB>
__global__ void __launch_bounds__(W * 32, MINB)
    wide_kernel(MulArgs g, BucketArgs ba, const int *rows, TierLists *tl, int tier, int next_tier,
                int *next_rows)
{
    using Cfg = WideCfg<T, W, TS>;
    constexpr int R = Cfg::R, CAP = Cfg::CAP, LP = Cfg::LP;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *mine = smem + (size_t) warp * Cfg::warp_bytes;
    T *vals = reinterpret_cast<T *>(mine);
    int *keys = reinterpret_cast<int *>(mine + Cfg::off_keys);
    unsigned *okey = reinterpret_cast<unsigned *>(mine + Cfg::off_okey);
    unsigned short *oslot = reinterpret_cast<unsigned short *>(mine + Cfg::off_oslot);
    unsigned short *kcnt = reinterpret_cast<unsigned short *>(mine + Cfg::off_kcnt);
    WideMisc *misc = reinterpret_cast<WideMisc *>(smem + Cfg::off_misc);
    volatile int *vabort = &misc->abort;

    const int nrows = tl->count[tier];
    const T *Av = static_cast<const T *>(g.Av);
    const T *Pv = static_cast<const T *>(ba.v);
    const int *Pc = ba.c;
    const unsigned short *Pp = ba.p;
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;
    const int blo = warp * R; // this warp's buckets: [blo, blo + R)

    for (;;)
    {
        __syncthreads(); // every warp is done with the previous row's lists
        if (tid == 0)
        {
            misc->row = atomicAdd(&tl->cursor[tier], 1);
            misc->abort = 0;
            misc->diag = 0.0;
        }
        __syncthreads();
        const int pos = misc->row;
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

        // meta of jp block b into m (lanes past the row hold an empty range)
        auto load_aj = [&](int b, JpMeta<T> &m) {
            const int q = b * 32 + lane;
            m.a = T(0);
            m.j = 0;
            m.lo = m.hi = 0;
            if (q < ni)
            {
                m.a = arow[q];
                m.j = airow[q];
            }
        };
        auto load_off = [&](int b, JpMeta<T> &m) {
            if (b * 32 + lane < ni)
            {
                const int *o = ba.off + (size_t) m.j * (NCLS + 1) + blo;
                m.lo = o[0];
                m.hi = o[R];
            }
        };
        JpMeta<T> m0, m1; // blocks cb and cb + 1
        int cb = 0;
        load_aj(0, m0);
        load_aj(1, m1);
        load_off(0, m0);
        load_off(1, m1);
        bool m1_off = true; // m1's ranges are loaded

        // prefetch ring: the first 32 entries of the warp's share of the B
        // row of jp t sit in slot t % PF
        int cq[PF];
        T bq[PF];
        auto meta_of = [&](int t, T &a, int &j, int &k0, int &k1) {
            const bool first = (t >> 5) == cb;
            const int src = t & 31;
            a = __shfl_sync(FULL, first ? m0.a : m1.a, src);
            j = __shfl_sync(FULL, first ? m0.j : m1.j, src);
            k0 = __shfl_sync(FULL, first ? m0.lo : m1.lo, src);
            k1 = __shfl_sync(FULL, first ? m0.hi : m1.hi, src);
        };
#pragma unroll
        for (int s = 0; s < PF; ++s)
        {
            cq[s] = 0;
            bq[s] = T(0);
            if (s < ni)
            {
                T a;
                int j, k0, k1;
                meta_of(s, a, j, k0, k1);
                const int kp = k0 + lane;
                if (kp < k1)
                {
                    cq[s] = Pc[(size_t) j * g.ldb + kp];
                    bq[s] = Pv[(size_t) j * g.ldb + kp];
                }
            }
        }

        int d = 0;
        T dA = T(0);
        bool ab = false;
        // one (c, b) entry of jp t: accumulate and record a first touch
        auto take = [&](bool valid, int c, T b, T a, size_t rb, int kp, unsigned jkey) {
            bool ins = false;
            int slot = -1;
            if (valid)
            {
                const T p = mul_rn(a, b);
                slot = wide_probe<TS>(keys, c, ins);
                if (slot >= 0)
                    vals[slot] = add_rn(vals[slot], p);
            }
            const unsigned bal = __ballot_sync(FULL, ins);
            if (ins)
            {
                const int r = d + __popc(bal & lanemask_lt());
                if (r < CAP)
                {
                    oslot[r] = (unsigned short) slot;
                    okey[r] = jkey | Pp[rb + kp];
                }
            }
            d += __popc(bal);
            if (__any_sync(FULL, valid && slot < 0))
                d = CAP + 1; // table full: cannot happen below CAP
        };

        for (int t0 = 0; t0 < ni && !ab; t0 += PF)
        {
#pragma unroll
            for (int s = 0; s < PF; ++s)
            {
                const int t = t0 + s;
                if (t >= ni || ab)
                    break;
                if ((t & 31) == 0 && t > 0)
                {
                    // entering block cb + 1: shift, start loading the next one
                    m0 = m1;
                    ++cb;
                    load_aj(cb + 1, m1);
                    m1_off = false;
                    if (*vabort)
                    {
                        ab = true;
                        break;
                    }
                }
                if (!m1_off && (t & 31) == 8)
                {
                    load_off(cb + 1, m1);
                    m1_off = true;
                }
                T a;
                int j, k0, k1;
                meta_of(t, a, j, k0, k1);
                if (j == i)
                    dA = add_rn(dA, a);
                const size_t rb = (size_t) j * g.ldb;
                const unsigned jkey = (unsigned) t << 16;
                take(k0 + lane < k1, cq[s], bq[s], a, rb, k0 + lane, jkey);
                for (int kb = k0 + 32; kb < k1; kb += 32)
                {
                    const int kp = kb + lane;
                    int c = 0;
                    T b = T(0);
                    if (kp < k1)
                    {
                        c = Pc[rb + kp];
                        b = Pv[rb + kp];
                    }
                    take(kp < k1, c, b, a, rb, kp, jkey);
                }
                if (d > CAP)
                {
                    ab = true;
                    break;
                }
                // refill this slot with jp t + PF
                const int u = t + PF;
                if (u < ni)
                {
                    T au;
                    int ju, u0, u1;
                    meta_of(u, au, ju, u0, u1);
                    const int kp = u0 + lane;
                    if (kp < u1)
                    {
                        cq[s] = Pc[(size_t) ju * g.ldb + kp];
                        bq[s] = Pv[(size_t) ju * g.ldb + kp];
                    }
                }
                __syncwarp();
            }
        }
        if (ab)
            *vabort = 1;
        __syncthreads();
        if (*vabort)
        {
            if (tid == 0)
                next_rows[atomicAdd(&tl->count[next_tier], 1)] = i;
            continue;
        }

        if (R > 1)
        {
            // A warp with several classes took each jp's entries class by
            // class: bitonic-sort its list by key (padded to a power of two).
            int n = 1;
            while (n < d)
                n <<= 1;
            for (int p = d + lane; p < n; p += 32)
                okey[p] = 0xffffffffu;
            __syncwarp();
            for (int size = 2; size <= n; size <<= 1)
                for (int stride = size >> 1; stride > 0; stride >>= 1)
                {
                    for (int x = lane; x < (n >> 1); x += 32)
                    {
                        const int lo = 2 * stride * (x / stride) + (x % stride), hi = lo + stride;
                        const bool up = (lo & size) == 0;
                        const unsigned ka = okey[lo], kb = okey[hi];
                        if ((ka > kb) == up)
                        {
                            okey[lo] = kb;
                            okey[hi] = ka;
                            const unsigned short sa = oslot[lo];
                            oslot[lo] = oslot[hi];
                            oslot[hi] = sa;
                        }
                    }
                    __syncwarp();
                }
        }
        static_assert(LP >= CAP, "list shorter than its capacity");

        // Keep flags and the exclusive count of kept entries along this list.
        int kept = 0;
        for (int c0 = 0; c0 < d; c0 += 32)
        {
            const int p = c0 + lane;
            bool keep = false;
            if (p < d)
            {
                const int s = oslot[p];
                const int k = keys[s];
                const T x = vals[s];
                if (k == i)
                {
                    keep = true;
                    misc->diag = (double) x;
                }
                else
                    keep = fabs(x) > thr;
            }
            const unsigned bal = __ballot_sync(FULL, keep);
            if (p < d)
                kcnt[p] = (unsigned short) (kept + __popc(bal & lanemask_lt()));
            kept += __popc(bal);
        }
        if (lane == 0)
        {
            kcnt[d] = (unsigned short) kept;
            misc->dw[warp] = d;
            misc->kept[warp] = kept;
        }
        __syncthreads();
        // Output slot of a kept entry: kept entries before it in its own list
        // plus, in every other list, the kept entries with a smaller key.
        for (int c0 = 0; c0 < d; c0 += 32)
        {
            const int p = c0 + lane;
            if (p >= d)
                continue;
            const int s = oslot[p];
            const int k = keys[s];
            const T x = vals[s];
            if (!(k == i || fabs(x) > thr))
                continue;
            const unsigned key = okey[p];
            int out = kcnt[p];
            for (int w2 = 0; w2 < W; ++w2)
            {
                if (w2 == warp)
                    continue;
                const unsigned char *ob = smem + (size_t) w2 * Cfg::warp_bytes;
                const unsigned *ok2 = reinterpret_cast<const unsigned *>(ob + Cfg::off_okey);
                const unsigned short *kc2 = reinterpret_cast<const unsigned short *>(ob + Cfg::off_kcnt);
                int lo2 = 0, hi2 = misc->dw[w2];
                while (lo2 < hi2)
                {
                    const int mid = (lo2 + hi2) >> 1;
                    if (ok2[mid] < key)
                        lo2 = mid + 1;
                    else
                        hi2 = mid;
                }
                out += kc2[lo2];
            }
            if (out < g.Mc)
            {
                Cv[(size_t) i * g.ldc + out] = x;
                g.Ci[(size_t) i * g.ldc + out] = k;
            }
        }
        if (tid == 0)
        {
            int ll = 0, distinct = 0;
            for (int w = 0; w < W; ++w)
            {
                ll += misc->kept[w];
                distinct += misc->dw[w];
            }
            finish_row<T>(g, i, ll, distinct, dA, misc->diag);
        }
    }
}

// -------------------------------------------------------------------------
// Window tiers K4, K8: two passes over the row with a bitmap of its columns.
// A team of KW = 8 warps per row, warp w owning the column classes
// [4w, 4w+4) of the bucketed copy of B, as in the wide tiers.
//   pass 1: every product column sets its bit in a bitmap over the row's
//           column window [min, max] of the B rows it references; the owner
//           warp, walking jp in order, records the first touch of each
//           column (key jp << 16 | position) in global scratch.
//   rank:   a prefix of the bitmap's popcounts gives every column a compact
//           slot: vals needs only one entry per distinct column.
//   pass 2: the owner warps walk the jps again and sum each product into its
//           column's slot, in jp order.
//   output: the kept columns (k == i or |x| > threshold) are sorted by their
//           first-touch keys, which is the reference's output order.
// Shared memory: vals[DCAP] | bitmap {bits, prefix}[NWCAP] | kept keys[KCAP]
// -------------------------------------------------------------------------
constexpr int KW = 8;
constexpr int KR = NCLS / KW;
constexpr int K_NWCAP = 2048; // bitmap words: windows of up to 65536 columns
constexpr int K_KCAP = 2048;  // kept columns per row
constexpr int KU = 4;         // 32-entry steps per share held in registers
constexpr int KPF = 2;        // jps of prefetch

struct KMisc
{
    double diag;
    int row, base, nw, D, kept, pad;
    int red[2 * KW];
};

template <typename T, int DCAP> struct KCfg
{
    static constexpr size_t off_bmp = (size_t(DCAP) * sizeof(T) + 15) / 16 * 16;
    static constexpr size_t off_kbuf = off_bmp + size_t(K_NWCAP) * sizeof(uint2);
    static constexpr size_t off_misc = off_kbuf + size_t(K_KCAP) * sizeof(unsigned long long);
    static constexpr size_t bytes = off_misc + sizeof(KMisc);
};

// Sum of A's entries on the diagonal of row i, in row order (one warp).
template <typename T>
__device__ __forceinline__ T row_diag_sum(const T *arow, const int *airow, int ni, int i, int lane)
{
    T dA = T(0);
    for (int jp0 = 0; jp0 < ni; jp0 += 32)
    {
        const int q = jp0 + lane;
        const bool hit = q < ni && airow[q] == i;
        const T av = hit ? arow[q] : T(0);
        unsigned bal = __ballot_sync(FULL, hit);
        while (bal)
        {
            const int src = __ffs(bal) - 1;
            bal &= bal - 1;
            dA = add_rn(dA, __shfl_sync(FULL, av, src));
        }
    }
    return dA;
}

// Walks the jps of row i in order over this warp's buckets [blo, blo + KR)
// of each B row, calling op(valid, c, b, a, rb, kp, t) once per 32-entry step
// (every lane; `valid` says whether the lane holds an entry).  The first
// KU*32 entries of each share are loaded KPF jps ahead.
template <typename T, bool NEED_B, typename Op>
__device__ __forceinline__ void walk_shares(const MulArgs &g, const BucketArgs &ba, const T *arow,
                                            const int *airow, int ni, int blo, int lane, Op &op)
{
    const T *Pv = static_cast<const T *>(ba.v);
    const int *Pc = ba.c;
    auto load_aj = [&](int b, JpMeta<T> &m) {
        const int q = b * 32 + lane;
        m.a = T(0);
        m.j = 0;
        m.lo = m.hi = 0;
        if (q < ni)
        {
            m.a = arow[q];
            m.j = airow[q];
        }
    };
    auto load_off = [&](int b, JpMeta<T> &m) {
        if (b * 32 + lane < ni)
        {
            const int *o = ba.off + (size_t) m.j * (NCLS + 1) + blo;
            m.lo = o[0];
            m.hi = o[KR];
        }
    };
    JpMeta<T> m0, m1;
    int cb = 0;
    load_aj(0, m0);
    load_aj(1, m1);
    load_off(0, m0);
    load_off(1, m1);
    bool m1_off = true;
    auto meta_of = [&](int t, T &a, int &j, int &k0, int &k1) {
        const bool first = (t >> 5) == cb;
        const int src = t & 31;
        a = __shfl_sync(FULL, first ? m0.a : m1.a, src);
        j = __shfl_sync(FULL, first ? m0.j : m1.j, src);
        k0 = __shfl_sync(FULL, first ? m0.lo : m1.lo, src);
        k1 = __shfl_sync(FULL, first ? m0.hi : m1.hi, src);
    };
    int cq[KPF][KU];
    T bq[KPF][KU];
    auto fill = [&](int u, int s) {
        T a;
        int j, k0, k1;
        meta_of(u, a, j, k0, k1);
        const size_t rb = (size_t) j * g.ldb;
#pragma unroll
        for (int x = 0; x < KU; ++x)
        {
            const int kp = k0 + x * 32 + lane;
            cq[s][x] = 0;
            bq[s][x] = T(0);
            if (kp < k1)
            {
                cq[s][x] = Pc[rb + kp];
                if (NEED_B)
                    bq[s][x] = Pv[rb + kp];
            }
        }
    };
#pragma unroll
    for (int s = 0; s < KPF; ++s)
        if (s < ni)
            fill(s, s);
    for (int t0 = 0; t0 < ni; t0 += KPF)
    {
#pragma unroll
        for (int s = 0; s < KPF; ++s)
        {
            const int t = t0 + s;
            if (t >= ni)
                break;
            if ((t & 31) == 0 && t > 0)
            {
                m0 = m1;
                ++cb;
                load_aj(cb + 1, m1);
                m1_off = false;
            }
            if (!m1_off && (t & 31) == 8)
            {
                load_off(cb + 1, m1);
                m1_off = true;
            }
            T a;
            int j, k0, k1;
            meta_of(t, a, j, k0, k1);
            const size_t rb = (size_t) j * g.ldb;
#pragma unroll
            for (int x = 0; x < KU; ++x)
                if (k0 + x * 32 < k1)
                    op(k0 + x * 32 + lane < k1, cq[s][x], bq[s][x], a, rb, k0 + x * 32 + lane, t);
            for (int kb = k0 + KU * 32; kb < k1; kb += 32)
            {
                const int kp = kb + lane;
                int c = 0;
                T b = T(0);
                if (kp < k1)
                {
                    c = Pc[rb + kp];
                    if (NEED_B)
                        b = Pv[rb + kp];
                }
                op(kp < k1, c, b, a, rb, kp, t);
            }
            if (t + KPF < ni)
                fill(t + KPF, s);
            __syncwarp();
        }
    }
}

template <typename T, int DCAP, int MINB>
__global__ void __launch_bounds__(KW * 32, MINB)
    window_kernel(MulArgs g, BucketArgs ba, const int *rows, TierLists *tl, int tier, int next_tier,
                  int *next_rows, unsigned *keyg, void *gvals)
{
    using Cfg = KCfg<T, DCAP>;
    constexpr int NT = KW * 32;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    T *vals = reinterpret_cast<T *>(smem);
    uint2 *bmp = reinterpret_cast<uint2 *>(smem + Cfg::off_bmp);
    unsigned long long *kbuf = reinterpret_cast<unsigned long long *>(smem + Cfg::off_kbuf);
    KMisc *misc = reinterpret_cast<KMisc *>(smem + Cfg::off_misc);
    unsigned *mykey = keyg + (size_t) blockIdx.x * (K_NWCAP * 32);
    // accumulator of rows wider than DCAP: a compact slab of this block in
    // device memory (one entry per distinct column, so it stays in L2)
    T *myvals = static_cast<T *>(gvals) + (size_t) blockIdx.x * (K_NWCAP * 32);
    const unsigned short *Pp = ba.p;
    const int nrows = tl->count[tier];
    const T *Av = static_cast<const T *>(g.Av);
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;
    const int blo = warp * KR;

    for (;;)
    {
        __syncthreads(); // the previous row is written out
        if (tid == 0)
        {
            misc->row = atomicAdd(&tl->cursor[tier], 1);
            misc->diag = 0.0;
            misc->kept = 0;
        }
        __syncthreads();
        const int pos = misc->row;
        if (pos >= nrows)
            break;
        const int i = rows[pos];
        const int ni = g.An[i];
        const T *arow = Av + (size_t) i * g.lda;
        const int *airow = g.Ai + (size_t) i * g.lda;

        // column window of the row: the B rows' column ranges
        int mn = 0x7fffffff, mx = -1;
        for (int q = tid; q < ni; q += NT)
        {
            const int j = airow[q];
            mn = min(mn, ba.cmin[j]);
            mx = max(mx, ba.cmax[j]);
        }
        mn = __reduce_min_sync(FULL, mn);
        mx = __reduce_max_sync(FULL, mx);
        if (lane == 0)
        {
            misc->red[warp] = mn;
            misc->red[KW + warp] = mx;
        }
        __syncthreads();
        if (tid == 0)
        {
            for (int w = 1; w < KW; ++w)
            {
                mn = min(mn, misc->red[w]);
                mx = max(mx, misc->red[KW + w]);
            }
            misc->base = mx < 0 ? 0 : (mn & ~31);
            misc->nw = mx < 0 ? 0 : (mx >> 5) - (mn >> 5) + 1;
        }
        __syncthreads();
        const int base = misc->base, nw = misc->nw;
        if (nw > K_NWCAP)
        {
            if (tid == 0)
                next_rows[atomicAdd(&tl->count[next_tier], 1)] = i;
            continue;
        }
        for (int w = tid; w < nw; w += NT)
            bmp[w] = make_uint2(0u, 0u);
        __syncthreads();

        // pass 1: bitmap of the row's columns, first-touch keys
        auto mark = [&](bool valid, int c, T, T, size_t rb, int kp, int t) {
            if (valid)
            {
                const int bit = c - base;
                const unsigned m = 1u << (bit & 31);
                // most products land on a column already marked: test first
                if (!(bmp[bit >> 5].x & m))
                {
                    const unsigned old = atomicOr(&bmp[bit >> 5].x, m);
                    if (!(old & m))
                        mykey[bit] = ((unsigned) t << 16) | Pp[rb + kp];
                }
            }
        };
        walk_shares<T, false>(g, ba, arow, airow, ni, blo, lane, mark);
        __syncthreads();

        // rank: exclusive prefix of the popcounts, words split into NT runs
        {
            const int per = (nw + NT - 1) / NT;
            const int w0 = min(tid * per, nw), w1 = min(w0 + per, nw);
            int sum = 0;
            for (int w = w0; w < w1; ++w)
                sum += __popc(bmp[w].x);
            int incl = sum;
            for (int o = 1; o < 32; o <<= 1)
            {
                const int y = __shfl_up_sync(FULL, incl, o);
                if (lane >= o)
                    incl += y;
            }
            if (lane == 31)
                misc->red[warp] = incl;
            __syncthreads();
            int before = 0;
            for (int w = 0; w < warp; ++w)
                before += misc->red[w];
            int run = before + incl - sum;
            for (int w = w0; w < w1; ++w)
            {
                bmp[w].y = (unsigned) run;
                run += __popc(bmp[w].x);
            }
            if (tid == NT - 1)
                misc->D = before + incl;
        }
        __syncthreads();
        const int D = misc->D;
        T *acc_v = D <= DCAP ? vals : myvals;
        for (int s = tid; s < D; s += NT)
            acc_v[s] = T(0);
        __syncthreads();

        // pass 2: sums in jp order, one owner warp per column
        if (D <= DCAP)
        {
            auto acc = [&](bool valid, int c, T b, T a, size_t, int, int) {
                if (valid)
                {
                    const int bit = c - base;
                    const uint2 pr = bmp[bit >> 5];
                    const int slot = (int) pr.y + __popc(pr.x & ((1u << (bit & 31)) - 1u));
                    vals[slot] = add_rn(vals[slot], mul_rn(a, b));
                }
            };
            walk_shares<T, true>(g, ba, arow, airow, ni, blo, lane, acc);
        }
        else
        {
            auto acc = [&](bool valid, int c, T b, T a, size_t, int, int) {
                if (valid)
                {
                    const int bit = c - base;
                    const uint2 pr = bmp[bit >> 5];
                    const int slot = (int) pr.y + __popc(pr.x & ((1u << (bit & 31)) - 1u));
                    myvals[slot] = add_rn(myvals[slot], mul_rn(a, b));
                }
            };
            walk_shares<T, true>(g, ba, arow, airow, ni, blo, lane, acc);
        }
        T dA = T(0);
        if (warp == 0)
            dA = row_diag_sum<T>(arow, airow, ni, i, lane);
        __syncthreads();

        // kept columns with their first-touch keys
        for (int w = tid; w < nw; w += NT)
        {
            const uint2 pr = bmp[w];
            unsigned bits = pr.x;
            int slot = (int) pr.y;
            while (bits)
            {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1;
                const int c = base + 32 * w + b;
                const T x = acc_v[slot++];
                bool keep;
                if (c == i)
                {
                    keep = true;
                    misc->diag = (double) x;
                }
                else
                    keep = fabs(x) > thr;
                if (keep)
                {
                    const int p = atomicAdd(&misc->kept, 1);
                    if (p < K_KCAP)
                        kbuf[p] = ((unsigned long long) mykey[c - base] << 32) | (unsigned) c;
                }
            }
        }
        __syncthreads();
        const int kept = misc->kept;
        if (kept > K_KCAP)
        {
            if (tid == 0)
                next_rows[atomicAdd(&tl->count[next_tier], 1)] = i;
            continue;
        }
        // first-touch order: bitonic sort of the kept keys
        int n = 1;
        while (n < kept)
            n <<= 1;
        for (int p = kept + tid; p < n; p += NT)
            kbuf[p] = ~0ull;
        __syncthreads();
        for (int size = 2; size <= n; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1)
            {
                for (int x = tid; x < (n >> 1); x += NT)
                {
                    const int lo = 2 * stride * (x / stride) + (x % stride), hi = lo + stride;
                    const bool up = (lo & size) == 0;
                    const unsigned long long ka = kbuf[lo], kb = kbuf[hi];
                    if ((ka > kb) == up)
                    {
                        kbuf[lo] = kb;
                        kbuf[hi] = ka;
                    }
                }
                __syncthreads();
            }
        const int nout = min(kept, g.Mc);
        for (int p = tid; p < nout; p += NT)
        {
            const int c = (int) (unsigned) kbuf[p];
            const int bit = c - base;
            const uint2 pr = bmp[bit >> 5];
            const int slot = (int) pr.y + __popc(pr.x & ((1u << (bit & 31)) - 1u));
            Cv[(size_t) i * g.ldc + p] = acc_v[slot];
            g.Ci[(size_t) i * g.ldc + p] = c;
        }
        if (tid == 0)
            finish_row<T>(g, i, kept, D, dA, misc->diag);
    }
}

// -------------------------------------------------------------------------
// Tier C: dense accumulator over all columns, in global memory, one slab per
// block: acc[ncols] (T), mark[ncols] (int, row+1 while the column is live),
// order[ncols] (int, column ids in first-touch order).  Marks are cleared
// column by column at the end of each row, as the reference clears ix[].
// -------------------------------------------------------------------------
// Two forms of the accumulation, chosen per call:
//  - RED: acc[k] += p for a column already touched in this row is a
//    reduction at L2 (red.global.add), so the lane does not wait for the old
//    value.  Within one jp a column has one writer, and the block barrier
//    between jp's orders the reductions of successive jp's, so each column
//    is still summed in jp order.  The f64 reduction rounds to nearest even
//    and keeps subnormals, so FP64 always takes this form; the f32 one
//    flushes subnormals to zero, so FP32 takes it only when the caller allows
//    that (mixed-precision SP2's FP32 iterations).
//  - load/add/store (exact FP32).
// Warps per row, blocks per SM and chunks of 32 products in flight per lane
// of each form, measured on B200 over 4 FP64 SP2 iterations on the 40^3
// lattice: RED 4 warps x 10 blocks x 3 chunks 377 ms (x 8-12 blocks, 2-4
// chunks: 377-398 ms; 8 warps x 8 blocks 407 ms; 16 warps x 4 blocks
// 655 ms); load/store 8 warps x 6 blocks x 3 chunks 576 ms (5 blocks 580 ms,
// 8 blocks 689 ms with register spills).
#ifndef B200_C_W_RED
#define B200_C_W_RED 4
#endif
#ifndef B200_C_BLOCKS_RED
#define B200_C_BLOCKS_RED 10
#endif
#ifndef B200_C_U_RED
#define B200_C_U_RED 3
#endif
#ifndef B200_C_W
#define B200_C_W 8
#endif
#ifndef B200_C_U
#define B200_C_U 3
#endif
template <bool RED> struct DenseCfg
{
    static constexpr int warps = RED ? B200_C_W_RED : B200_C_W;
    static constexpr int blocks = RED ? B200_C_BLOCKS_RED : B200_C_BLOCKS;
    static constexpr int chunks = RED ? B200_C_U_RED : B200_C_U;
};

template <typename T, bool RED>
__global__ void __launch_bounds__(DenseCfg<RED>::warps * 32, DenseCfg<RED>::blocks) dense_tier_kernel(MulArgs g, int smax, int ncols,
                                                        const int *rows, TierLists *tl,
                                                        unsigned char *slabs, int use_bits)
{
    constexpr int W = DenseCfg<RED>::warps;
    constexpr int C_U = DenseCfg<RED>::chunks;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    const int nrows = tl->count[NTIERS - 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wt = warp;
    const int tid = threadIdx.x;
    int *stage = reinterpret_cast<int *>(smem) + wt * smax;
    int *cnt = reinterpret_cast<int *>(smem) + W * smax;
    TeamMisc *misc = reinterpret_cast<TeamMisc *>(cnt + 2 * W);
    unsigned *bits = reinterpret_cast<unsigned *>(reinterpret_cast<unsigned char *>(misc) + 32);

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
            if (use_bits)
                for (int s = tid; s < (ncols + 31) / 32; s += W * 32)
                    bits[s] = 0u;
            else
                for (int s = tid; s < ncols; s += W * 32)
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
                if (use_bits)
                {
                    // C_U chunks of 32 at once: all loads of B's entries, then
                    // the accumulators of columns already touched, then the
                    // sums (the columns of one jp are distinct, so the
                    // reordering changes no result)
                    for (int kb = k0; kb < k1; kb += 32 * C_U)
                    {
                        int kk[C_U];
                        T bb[C_U], old[C_U];
                        bool have[C_U], fresh[C_U];
#pragma unroll
                        for (int u = 0; u < C_U; ++u)
                        {
                            const int kp = kb + u * 32 + lane;
                            have[u] = kp < k1;
                            kk[u] = have[u] ? birow[kp] : 0;
                            bb[u] = have[u] ? brow[kp] : T(0);
                        }
#pragma unroll
                        for (int u = 0; u < C_U; ++u)
                        {
                            fresh[u] = false;
                            old[u] = T(0);
                            if (have[u])
                            {
                                // only this lane sets this bit within the jp
                                const unsigned m = 1u << (kk[u] & 31);
                                fresh[u] = !(bits[kk[u] >> 5] & m);
                                if (fresh[u])
                                    atomicOr(&bits[kk[u] >> 5], m);
                                else if (!RED)
                                    old[u] = acc[kk[u]];
                            }
                        }
#pragma unroll
                        for (int u = 0; u < C_U; ++u)
                            if (have[u])
                            {
                                const T p = mul_rn(a, bb[u]);
                                if (fresh[u])
                                    acc[kk[u]] = add_rn(T(0), p);
                                else if (RED)
                                    atomicAdd(acc + kk[u], p);
                                else
                                    acc[kk[u]] = add_rn(old[u], p);
                            }
#pragma unroll
                        for (int u = 0; u < C_U; ++u)
                        {
                            const bool ins = have[u] && fresh[u];
                            const unsigned bal = __ballot_sync(FULL, ins);
                            if (ins)
                                stage[local + __popc(bal & lanemask_lt())] = kk[u];
                            local += __popc(bal);
                        }
                    }
                }
                else
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
                            else if (RED)
                                atomicAdd(acc + k, p);
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
                if (use_bits)
                    atomicAnd(&bits[k >> 5], ~(1u << (k & 31)));
                else
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

// -------------------------------------------------------------------------
// Tier C, staged form (dense_tier_kernel with B's rows in shared memory):
// B's rows stream through a ring of STAGES units of at most CHUNK entries,
// copied by TMA bulk copies (cp.async.bulk) up to STAGES - 1 units ahead, as
// in the team tiers; the accumulator is the per-block slab with the
// shared-memory touched bitmap, summed by L2 reductions (RED) or by load,
// add and store.  The product loop then reads B from shared memory, so no
// lane waits on a global load of B.  The first-touch list is built per unit
// (units follow B's row order).
// Shared memory: mbar[STAGES] | sv[STAGES][CHUNK] | sk[STAGES][CHUNK] |
//                stg[W][SPW] (int) | cnt[2][W] | misc | bits[ncols/32]
// -------------------------------------------------------------------------
template <typename T, int W, int STAGES, int CHUNK> struct StagedCfg
{
    static constexpr int NT = W * 32;
    static constexpr int SPW = ((CHUNK + W - 1) / W + 31) / 32 * 32;
    static constexpr size_t off_sv = 128;
    static constexpr size_t off_sk = off_sv + size_t(STAGES) * CHUNK * sizeof(T);
    static constexpr size_t off_stg = off_sk + size_t(STAGES) * CHUNK * sizeof(int);
    static constexpr size_t off_cnt = off_stg + size_t(W) * SPW * sizeof(int);
    static constexpr size_t off_misc = off_cnt + 2 * W * sizeof(int);
    static constexpr size_t off_bits = (off_misc + sizeof(TeamMisc) + 15) / 16 * 16;
    static size_t bytes(int ncols) { return off_bits + (size_t) (ncols + 31) / 32 * sizeof(unsigned); }
};

// RED: touched columns summed by L2 reductions; otherwise loaded, added and
// stored (exact FP32, whose global add flushes subnormals).
template <typename T, int W, int STAGES, int CHUNK, int MINB, bool RED>
__global__ void __launch_bounds__(W * 32, MINB) dense_staged_kernel(MulArgs g, int ncols, const int *rows,
                                                                   TierLists *tl, unsigned char *slabs)
{
    using Cfg = StagedCfg<T, W, STAGES, CHUNK>;
    constexpr int NT = Cfg::NT, SPW = Cfg::SPW;
    extern __shared__ __align__(128) unsigned char smem[];
    if (g.flags->bad_input)
        return;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem);
    T *sv = reinterpret_cast<T *>(smem + Cfg::off_sv);
    int *sk = reinterpret_cast<int *>(smem + Cfg::off_sk);
    int *cnt = reinterpret_cast<int *>(smem + Cfg::off_cnt);
    TeamMisc *misc = reinterpret_cast<TeamMisc *>(smem + Cfg::off_misc);
    unsigned *bits = reinterpret_cast<unsigned *>(smem + Cfg::off_bits);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int *stg = reinterpret_cast<int *>(smem + Cfg::off_stg) + warp * SPW;

    const size_t slab_bytes = (size_t) ncols * (sizeof(T) + 2 * sizeof(int));
    T *acc = reinterpret_cast<T *>(slabs + (size_t) blockIdx.x * slab_bytes);
    int *order = reinterpret_cast<int *>(acc + ncols) + ncols;

    const int nrows = tl->count[NTIERS - 1];
    const T *Av = static_cast<const T *>(g.Av);
    const T *Bv = static_cast<const T *>(g.Bv);
    T *Cv = static_cast<T *>(g.Cv);
    const T thr = (T) g.thr;
    int *tflag = &g.flags->timeout;

    // Column ids in the ring start as 0, so a unit whose copy never landed
    // (a timed-out wait, reported to the host) still names a valid column.
    for (int s = tid; s < STAGES * CHUNK; s += NT)
        sk[s] = 0;
    for (int s = tid; s < (ncols + 31) / 32; s += NT)
        bits[s] = 0u;
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
        // one thread decides (a flag read by every thread could change
        // between their reads and split the block at the barrier)
        if (tid == 0)
            misc->row = *reinterpret_cast<volatile int *>(tflag) ? nrows : atomicAdd(&tl->cursor[NTIERS - 1], 1);
        __syncthreads();
        const int pos = misc->row;
        if (pos >= nrows)
            break;
        const int i = rows[pos];
        if (tid == 0)
            misc->diag = 0.0;
        const int ni = g.An[i];
        const T *arow = Av + (size_t) i * g.lda;
        const int *airow = g.Ai + (size_t) i * g.lda;

        // Producer (thread 0): the next unit to copy is chunk pc of the B row
        // named at position pj.  Every thread counts the units it consumes.
        int pj = 0, pc = 0, pnj = 0;
        unsigned issued = 0;
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
        auto issue = [&]() {
            const int s = (ucount + issued) % STAGES;
            const int j = airow[pj];
            const int off = pc * CHUNK;
            const int n = min(CHUNK, pnj - off);
            const unsigned bv = (unsigned) ((n * sizeof(T) + 15) & ~size_t(15));
            const unsigned bk = (unsigned) ((n * sizeof(int) + 15) & ~size_t(15));
            mbar_expect_tx(&mbar[s], bv + bk);
            bulk_g2s(sv + (size_t) s * CHUNK, Bv + (size_t) j * g.ldb + off, bv, &mbar[s]);
            bulk_g2s(sk + (size_t) s * CHUNK, g.Bi + (size_t) j * g.ldb + off, bk, &mbar[s]);
            ++pc;
            ++issued;
            prod_skip();
        };
        if (tid == 0)
        {
            prod_skip();
            while (issued < STAGES && pj < ni)
                issue();
        }

        int distinct = 0;
        T dA = T(0);
        unsigned consumed = 0;
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
                const T a = __shfl_sync(FULL, av, t);
                const int j = __shfl_sync(FULL, aj, t);
                const int nj = __shfl_sync(FULL, nj_l, t);
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
                    for (int kb = k0; kb < k1; kb += 32)
                    {
                        const int kp = kb + lane;
                        bool ins = false;
                        int k = 0;
                        if (kp < k1)
                        {
                            k = uk[kp];
                            const T p = mul_rn(a, uv[kp]);
                            // only this lane sets this bit within the unit
                            const unsigned m = 1u << (k & 31);
                            if (!(bits[k >> 5] & m))
                            {
                                atomicOr(&bits[k >> 5], m);
                                acc[k] = add_rn(T(0), p);
                                ins = true;
                            }
                            else if (RED)
                                atomicAdd(acc + k, p);
                            else
                                acc[k] = add_rn(acc[k], p);
                        }
                        const unsigned bal = __ballot_sync(FULL, ins);
                        if (ins)
                            stg[local + __popc(bal & lanemask_lt())] = k;
                        local += __popc(bal);
                    }
                    if (lane == 0)
                        cnt[(u & 1) * W + warp] = local;
                    __syncthreads();
                    ++consumed;
                    int pre = 0, tot = 0;
#pragma unroll
                    for (int w = 0; w < W; ++w)
                    {
                        const int cw = cnt[(u & 1) * W + w];
                        pre += (w < warp) ? cw : 0;
                        tot += cw;
                    }
                    for (int r = lane; r < local; r += 32)
                        order[distinct + pre + r] = stg[r];
                    __syncwarp();
                    distinct += tot;
                    // the stage just consumed is free: refill it
                    if (tid == 0 && pj < ni)
                        issue();
                }
            }
        }
        ucount += consumed;
        __syncthreads();

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
                k = order[q];
                x = acc[k];
                atomicAnd(&bits[k >> 5], ~(1u << (k & 31)));
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

// Staged dense tier: warps per row, ring stages, entries per unit, min
// blocks/SM.  Measured on B200 over 4 FP64 SP2 iterations on the 40^3
// lattice (A + dense tier): 4 warps x 2 stages x 1024 entries 360 ms;
// 3 stages 368 ms; 512 entries 369 ms; 8 warps 382 ms; 2 warps x 512 entries
// 355 ms, x 256 entries 386 ms (the unstaged reduction form: 377 ms).
#ifndef B200_C_STAGED
#define B200_C_STAGED 1
#endif
#ifndef B200_CS_W
#define B200_CS_W 4
#endif
#ifndef B200_CS_STAGES
#define B200_CS_STAGES 2
#endif
#ifndef B200_CS_CHUNK
#define B200_CS_CHUNK 1024
#endif
#ifndef B200_CS_MINB
#define B200_CS_MINB 6
#endif
constexpr int CS_W = B200_CS_W, CS_STAGES = B200_CS_STAGES, CS_CHUNK = B200_CS_CHUNK, CS_MINB = B200_CS_MINB;

// Team tier B1: (W, LOGTS, STAGES, CHUNK, min blocks per SM)
#define B1_CFG 4, 11, 3, 256, 4

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

// Wide tiers: (warps, slots per warp, min blocks per SM)
#define W8_CFG 8, 256, 4
#define W16_CFG 16, 256, 2
// Window tiers: (distinct columns held, min blocks per SM)
#define K4_CFG 4096, 3
#define K8_CFG 8192, 2

template <typename T, int DCAP, int MINB> constexpr size_t window_bytes()
{
    return KCfg<T, DCAP>::bytes;
}

template <typename T, int DCAP, int MINB> int window_grid(B200Context *c)
{
    auto k = window_kernel<T, DCAP, MINB>;
    if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) KCfg<T, DCAP>::bytes)))
        return 0;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, KW * 32, KCfg<T, DCAP>::bytes);
    return c->sm_count * (occ > 0 ? occ : 1);
}

template <typename T, int DCAP, int MINB>
bool launch_window(B200Context *c, int grid, const MulArgs &g, const BucketArgs &ba, const int *rows,
                   TierLists *tl, int tier, int next_tier, int *next_rows, unsigned *keyg, void *gvals)
{
    window_kernel<T, DCAP, MINB><<<grid, KW * 32, KCfg<T, DCAP>::bytes, c->stream>>>(
        g, ba, rows, tl, tier, next_tier, next_rows, keyg, gvals);
    return LAUNCH_OK("window_kernel");
}

template <typename T, int W, int TS, int MINB> constexpr size_t wide_bytes()
{
    return WideCfg<T, W, TS>::bytes;
}

template <typename T, int W, int TS, int MINB>
bool launch_wide(B200Context *c, const MulArgs &g, const BucketArgs &ba, const int *rows,
                 TierLists *tl, int tier, int next_tier, int *next_rows)
{
    using Cfg = WideCfg<T, W, TS>;
    auto k = wide_kernel<T, W, TS, MINB>;
    if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) Cfg::bytes)))
        return false;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, W * 32, Cfg::bytes);
    const int grid = c->sm_count * (occ > 0 ? occ : 1);
    k<<<grid, W * 32, Cfg::bytes, c->stream>>>(g, ba, rows, tl, tier, next_tier, next_rows);
    return LAUNCH_OK("wide_kernel");
}

// FP32 multiplies may use the flushing f32 reduction in the dense tier
// (set by mixed-precision SP2 around its FP32 iterations; off by default,
// which keeps FP32 products bit-exact).
bool g_f32_reduce = false;

// Distinct-column counts of the last multiply, reused as the next call's
// tier estimate when the row count matches (SP2 multiplies the same-size
// matrix over and over; a stale estimate only costs a retry in a larger tier).
int *g_hint = nullptr;
int g_hint_n = 0;
bool g_hint_valid = false;
int g_last_tiers[NTIERS] = {0};
int g_tier_mask = B200_X2_TIERS;

template <typename T>
bool multiply_typed(MulArgs g, int ncols, double *trace, int *required_M)
{
    B200Context *c = b200_ctx();
    if (!c)
        return false;
    const int N = g.NA;

    const size_t smemA = tierA_warp_bytes<T>() * A_WARPS;
    const bool red = sizeof(T) == 8 || g_f32_reduce;
    const int warps_c = red ? DenseCfg<true>::warps : DenseCfg<false>::warps;
    const int blocks_c = red ? DenseCfg<true>::blocks : DenseCfg<false>::blocks;
    const int smaxC = b200_round_up(b200_ceil_div(g.ldb, warps_c), 32);
    const size_t smemC0 = (size_t) warps_c * smaxC * sizeof(int) + 2 * warps_c * sizeof(int) + 32;
    // the touched-column bitmap, while it leaves each block its share
    const size_t bits_bytes = (size_t) (ncols + 31) / 32 * sizeof(unsigned);
    const int use_bits = B200_DENSE_BITS && (smemC0 + bits_bytes) * blocks_c <= 200 * 1024 ? 1 : 0;
    const size_t smemC = smemC0 + (use_bits ? bits_bytes : 0);
    if (smemC > c->smem_optin)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "row width %d too large for the multiply kernels", g.ldb);
        return false;
    }
    int gridC = c->sm_count * blocks_c;
    const size_t slab_bytes = (size_t) ncols * (sizeof(T) + 2 * sizeof(int));
    // the staged form of the dense tier, while its shared memory fits
    using SCfg = StagedCfg<T, CS_W, CS_STAGES, CS_CHUNK>;
    auto staged_k = red ? dense_staged_kernel<T, CS_W, CS_STAGES, CS_CHUNK, CS_MINB, true>
                        : dense_staged_kernel<T, CS_W, CS_STAGES, CS_CHUNK, CS_MINB, false>;
    const size_t smemS = SCfg::bytes(ncols);
    bool staged = B200_C_STAGED && smemS <= c->smem_optin;
    if (staged)
    {
        if (!CUDA_OK(cudaFuncSetAttribute(staged_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemS)))
            return false;
        int occS = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occS, staged_k, CS_W * 32, smemS);
        if (occS > 0)
            gridC = c->sm_count * occS;
        else
            staged = false;
    }

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

    // Tiers in use for this call.  The P tiers key order entries by
    // (jp << 16 | position), so both row lengths must stay below 2^16, and
    // their shared memory must fit the device.
    int tmask = g_tier_mask | (1 << TIER_C);
    if (g.lda >= 65536 || g.ldb >= 65536)
        tmask &= ~BUCKET_TIERS_MASK;
    if (wide_bytes<T, W8_CFG>() > c->smem_optin)
        tmask &= ~(1 << TIER_W8);
    if (wide_bytes<T, W16_CFG>() > c->smem_optin)
        tmask &= ~(1 << TIER_W16);
    if (window_bytes<T, K4_CFG>() > c->smem_optin)
        tmask &= ~(1 << TIER_K4);
    if (window_bytes<T, K8_CFG>() > c->smem_optin)
        tmask &= ~(1 << TIER_K8);
    const int gridK4 = ((tmask >> TIER_K4) & 1) ? window_grid<T, K4_CFG>(c) : 0;
    const int gridK8 = ((tmask >> TIER_K8) & 1) ? window_grid<T, K8_CFG>(c) : 0;
    if (((tmask >> TIER_K4) & 1) && !gridK4)
        return false;
    if (((tmask >> TIER_K8) & 1) && !gridK8)
        return false;
    const int gridK = gridK4 > gridK8 ? gridK4 : gridK8;
    const bool use_p = (tmask & BUCKET_TIERS_MASK) != 0;

    // scratch: NTIERS lists of N ints, diag arrays (2N doubles), dense slabs,
    // and (P tiers) the bucketed copy of B: values, columns, positions, offsets
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t nbe = (size_t) g.NB * g.ldb;
    const size_t off_diag = al((size_t) NTIERS * N * sizeof(int));
    const size_t off_slabs = al(off_diag + (size_t) 2 * N * sizeof(double));
    const size_t off_pv = al(off_slabs + (size_t) gridC * slab_bytes);
    const size_t off_pc = al(off_pv + (use_p ? nbe * sizeof(T) : 0));
    const size_t off_pp = al(off_pc + (use_p ? nbe * sizeof(int) : 0));
    const size_t off_po = al(off_pp + (use_p ? nbe * sizeof(unsigned short) : 0));
    const size_t off_mm = al(off_po + (use_p ? (size_t) g.NB * (NCLS + 1) * sizeof(int) : 0));
    const size_t off_keyg = al(off_mm + (use_p ? (size_t) 2 * g.NB * sizeof(int) : 0));
    const size_t off_gvals = al(off_keyg + (size_t) gridK * K_NWCAP * 32 * sizeof(unsigned));
    const size_t total = al(off_gvals + (size_t) gridK * K_NWCAP * 32 * sizeof(T));
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(total));
    if (!scr)
        return false;
    int *lists = reinterpret_cast<int *>(scr);
    double *diagA = reinterpret_cast<double *>(scr + off_diag);
    double *diagC = diagA + N;
    unsigned char *slabs = scr + off_slabs;
    BucketArgs ba{scr + off_pv, reinterpret_cast<int *>(scr + off_pc),
                  reinterpret_cast<unsigned short *>(scr + off_pp), reinterpret_cast<int *>(scr + off_po),
                  reinterpret_cast<int *>(scr + off_mm), reinterpret_cast<int *>(scr + off_mm) + g.NB};
    unsigned *keyg = reinterpret_cast<unsigned *>(scr + off_keyg);
    void *gvals = scr + off_gvals;

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
    plan_kernel<<<pgrid, 256, 0, c->stream>>>(g, ncols, tmask, tl, lists);
    if (!LAUNCH_OK("plan_kernel"))
        return false;
    if (use_p)
    {
        bucket_kernel<T><<<vgrid, 256, 0, c->stream>>>(static_cast<const T *>(g.Bv), g.Bi, g.Bn, g.ldb,
                                                       g.NB, ba);
        if (!LAUNCH_OK("bucket_kernel"))
            return false;
    }

    auto list = [&](int t) { return lists + (size_t) t * N; };
    if (!CUDA_OK(cudaFuncSetAttribute(tierA_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) smemA)))
        return false;
    int occA = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occA, tierA_kernel<T>, 32 * A_WARPS, smemA);
    // Rows a tier cannot hold go to the next tier in use (the dense tier
    // always is); tiers switched off are not launched.
    auto next_on = [tmask](int t) {
        int n = t + 1;
        while (n < NTIERS - 1 && !((tmask >> n) & 1))
            ++n;
        return n;
    };
    if (tmask & 1)
    {
        tierA_kernel<T><<<c->sm_count * max(occA, 1), 32 * A_WARPS, smemA, c->stream>>>(
            g, list(0), tl, next_on(0), list(next_on(0)));
        if (!LAUNCH_OK("tierA_kernel"))
            return false;
    }
    if ((tmask >> TIER_W8) & 1)
        if (!launch_wide<T, W8_CFG>(c, g, ba, list(TIER_W8), tl, TIER_W8, next_on(TIER_W8),
                                    list(next_on(TIER_W8))))
            return false;
    if ((tmask >> TIER_B1) & 1)
        if (!launch_team<T, B1_CFG>(c, g, list(TIER_B1), tl, TIER_B1, next_on(TIER_B1),
                                    list(next_on(TIER_B1))))
            return false;
    if ((tmask >> TIER_W16) & 1)
        if (!launch_wide<T, W16_CFG>(c, g, ba, list(TIER_W16), tl, TIER_W16, next_on(TIER_W16),
                                     list(next_on(TIER_W16))))
            return false;
    if ((tmask >> TIER_K4) & 1)
        if (!launch_window<T, K4_CFG>(c, gridK4, g, ba, list(TIER_K4), tl, TIER_K4, next_on(TIER_K4),
                                      list(next_on(TIER_K4)), keyg, gvals))
            return false;
    if ((tmask >> TIER_K8) & 1)
        if (!launch_window<T, K8_CFG>(c, gridK8, g, ba, list(TIER_K8), tl, TIER_K8, next_on(TIER_K8),
                                      list(next_on(TIER_K8)), keyg, gvals))
            return false;
    if (staged)
    {
        staged_k<<<gridC, CS_W * 32, smemS, c->stream>>>(g, ncols, list(TIER_C), tl, slabs);
        if (!LAUNCH_OK("dense_staged_kernel"))
            return false;
    }
    else
    {
        auto dense = red ? dense_tier_kernel<T, true> : dense_tier_kernel<T, false>;
        if (!CUDA_OK(cudaFuncSetAttribute(dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smemC)))
            return false;
        dense<<<gridC, warps_c * 32, smemC, c->stream>>>(g, smaxC, ncols, list(TIER_C), tl, slabs, use_bits);
        if (!LAUNCH_OK("dense_tier_kernel"))
            return false;
    }

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

void ell_set_f32_reduce(bool on)
{
    g_f32_reduce = on;
}

// x2_rows: A is a row view of B (rows of X^2): report overflow as X^2 does,
// on the thresholded width only.
bool ell_multiply_AB(bml_matrix_ellpack_t *A, bml_matrix_ellpack_t *B, bml_matrix_ellpack_t *C,
                     double threshold, double *trace, int *required_M, int x2_rows)
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
    if (!ell_x2_exact())
    {
        bool taken = false;
        bool ok = ell_multiply_dense_tier(A, B, C, threshold, trace, required_M, &taken);
        if (!taken && ell_unordered_fits(A) && ell_unordered_fits(B))
        {
            taken = true;
            ok = ell_multiply_unordered(A, B, C, threshold, trace, required_M, A != B && !x2_rows);
        }
        if (taken)
        {
            ell_mark_device(C);
            return ok;
        }
    }
    MulArgs g{};
    g.Av = A->d_value; g.Ai = A->d_index; g.An = A->d_nnz; g.lda = A->ld; g.NA = A->N;
    g.Bv = B->d_value; g.Bi = B->d_index; g.Bn = B->d_nnz; g.ldb = B->ld; g.NB = B->N;
    g.Cv = C->d_value; g.Ci = C->d_index; g.Cn = C->d_nnz; g.ldc = C->ld; g.Mc = C->M;
    g.thr = threshold;
    g.check_pre = (A != B && !x2_rows) ? 1 : 0;
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
// (A, W8, B1, W16, K4, K8, C; a row handed on is counted in every tier it entered).
extern "C" BML_B200_API int bml_b200_last_tier_counts(int *counts, int n)
{
    for (int t = 0; t < n && t < NTIERS; ++t)
        counts[t] = g_last_tiers[t];
    return NTIERS;
}

// Tier selection for later multiplies (bit t = tier t in the order above; 0
// restores the default).  Also forgets the per-row estimates of the last call.
extern "C" BML_B200_API int bml_b200_set_x2_tiers(int mask)
{
    const int old = g_tier_mask;
    g_tier_mask = mask ? (mask & ((1 << NTIERS) - 1)) : B200_X2_TIERS;
    g_hint_valid = false;
    return old;
}
