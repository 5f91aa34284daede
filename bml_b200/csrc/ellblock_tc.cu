// ELLBLOCK X^2 on the tcgen05 tensor cores, FP16 with a hi/lo split (mixed
// precision; no reference counterpart: the reference multiplies blocks in the
// matrix precision, ellblock/bml_multiply_ellblock_typed.c:246-442).
//
// X is scaled by a power of two 2^s (its largest entry near 2^14) and every
// 32x32 block x is split as hi = fp16(2^s x), lo = fp16(2^s x - hi); X^2 =
// sum_jb X[ib,jb] X[jb,kb] is formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory and scaled back by 2^-2s (lo*lo, about 2^-22
// of the product, is dropped).  The accuracy is then set by the tensor
// cores' FP32 accumulation: one X^2 of the 16^3 block lattice has its trace
// within 7e-6, with BF16 operands (8-bit significands) and FP16 alike.  The
// result is written back in the matrix precision; blocks are kept as in the
// reference (kb == ib, or max |x| > threshold), the traces are FP64 sums.
//
// Work: persistent CTAs, claiming from a counter groups of four consecutive block rows
// ib0..ib0+3, which share most of their block columns jb on a lattice.  For
// the group, with M = 128 = 4 x 32 rows:
//   D[kb] (128 x 32, FP32, in TMEM) += [X[ib0,jb]; ..; X[ib0+3,jb]] X[jb,kb]
// over the union J of the rows' block columns (missing blocks are zero), for
// every output block column kb; 16 output tiles of 32 TMEM columns are live
// at once (a wave), so the group's outputs are made in waves.
// Operands are staged into shared memory in the UMMA canonical K-major
// no-swizzle layout (8-row x 16-byte core matrices).  A split kernel first
// writes every block of X in that layout, as the left operand (rows x k) and
// as the right operand (columns x k, the block transposed), one contiguous
// 2 KB image each, so staging is one bulk copy (cp.async.bulk, completing on
// an mbarrier) per block, issued by one producer thread into rings of left
// and right operand buffers.  One thread issues the MMAs and releases each
// buffer with tcgen05.commit on its "empty" mbarrier.  Everything either
// thread needs per pair is precomputed by the whole CTA when the wave's pair
// list is built (the new-left-operand flag, the rows each tile touches), so
// their loops hold only the waits, the copies and the MMAs.  Every wait is
// bounded.
#include "device_util.cuh"
#include "ellblock.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

using namespace b200;

namespace {

constexpr int TB = 32;            // block size this path handles
constexpr int TC_THREADS = 128;   // 4 warps; warp q owns TMEM lanes 32q..32q+31
constexpr int TC_GROUP = 4;       // block rows per group (M = 128)
constexpr int IMG = TB * TB;      // 16-bit elements per block image (2 KB)
constexpr int TC_NWCAP = 2048;    // bitmap words: up to 65536 block columns
// Two shapes of the kernel: a small one with two CTAs per SM (8 live tiles,
// 256 TMEM columns each, so one CTA's set-up and epilogue overlap the
// other's MMAs) that takes groups up to its capacities, and a large one with
// one CTA per SM that the host falls back to when a group exceeds them.
// ABUF/BBUF: left/right operand buffers; JCAP: union of block columns per
// group; KCAP: output block columns per group; LCAP: product pairs per wave;
// PCAP: product pairs per group.
template <int TILES_, int CTAS_, int ABUF_, int BBUF_, int JCAP_, int KCAP_, int LCAP_, int PCAP_> struct TcCfg
{
    static constexpr int TILES = TILES_, CTAS = CTAS_, ABUF = ABUF_, BBUF = BBUF_;
    static constexpr int JCAP = JCAP_, KCAP = KCAP_, LCAP = LCAP_, PCAP = PCAP_;
    static_assert(CTAS * TILES * 32 <= 512, "tensor memory holds 512 columns per SM");
    static_assert(TILES <= 16, "tile numbers take 4 bits of a pair");
};
#ifndef B200_TCS_SHAPE
#define B200_TCS_SHAPE 8, 2, 3, 8, 512, 1024, 1024, 4096
#endif
using TcSmall = TcCfg<B200_TCS_SHAPE>;
using TcBig = TcCfg<16, 1, 6, 12, 1024, 4096, 2048, 8192>;

// Operand type of the split: FP16 (11-bit significands: hi and lo carry
// about 22 bits, the dropped lo*lo about 2^-22 of a product) with the whole
// matrix scaled by 2^s so that its largest entry is near 2^14 (entries down
// to about 2^-24 of it keep a normal lo); or BF16 (8-bit significands, no
// scaling needed, about 2^-16 per product).
#ifndef B200_TC_F16
#define B200_TC_F16 1
#endif
#if B200_TC_F16
typedef __half tc_t;
__device__ __forceinline__ tc_t tc_from_double(double x) { return __double2half(x); }
__device__ __forceinline__ double tc_to_double(tc_t h) { return (double) __half2float(h); }
#else
typedef __nv_bfloat16 tc_t;
__device__ __forceinline__ tc_t tc_from_double(double x) { return __float2bfloat16_rn((float) x); }
__device__ __forceinline__ double tc_to_double(tc_t h) { return (double) __bfloat162float(h); }
#endif

// Exponent s of the split's scale 2^s, from the bits of max |x| (as float):
// the largest entry lands near 2^14; 0 for an all-zero matrix (BF16: 0).
__device__ __forceinline__ int tc_scale_exp(unsigned maxbits)
{
    if (!B200_TC_F16 || maxbits == 0u)
        return 0;
    int e = 0;
    frexpf(__uint_as_float(maxbits), &e); // max |x| in [2^(e-1), 2^e)
    return min(max(14 - e, -100), 100);
}

// 16-bit image of a block in the K-major no-swizzle layout, as a left operand
// (element (r, k) of the block) or a right operand (element (n, k) = block
// (k, n)): 16-byte rows of 8 k, 8-row core matrices of 128 bytes; the four
// k-chunks of an 8-row group sit next to each other (LBO = 128 B) and the
// row groups follow at SBO = 512 B, so each 32 x 32 block is one contiguous
// 2 KB image and four blocks stack into the 128-row left operand.
constexpr unsigned TC_LBO = 128, TC_SBO = 512;

__device__ __forceinline__ int img_off(int row, int k)
{
    return (row >> 3) * 256 + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}

// max |x| over the stored blocks of X, as float bits (non-negative floats
// order like their bits), into *maxbits.
template <typename T>
__global__ void tc_maxabs_kernel(const T *pool, const int *nnzb, int NB, int MB, long long slot_elems,
                                 unsigned *maxbits)
{
    float m = 0.f;
    for (long long s = blockIdx.x; s < (long long) NB * MB; s += gridDim.x)
    {
        const int ib = (int) (s / MB), jp = (int) (s % MB);
        if (jp >= nnzb[ib])
            continue;
        const T *x = pool + s * slot_elems;
        for (int e = threadIdx.x; e < IMG; e += blockDim.x)
            m = fmaxf(m, fabsf((float) x[e]));
    }
    for (int o = 16; o; o >>= 1)
        m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(maxbits, __float_as_uint(m));
}

// Split every stored block of X, scaled by 2^s, into four images: left hi,
// left lo, right hi, right lo, at img + slot*4*IMG.
template <typename T>
__global__ void tc_split_kernel(const T *pool, const int *nnzb, int NB, int MB, long long slot_elems,
                                const unsigned *maxbits, tc_t *img)
{
    const double scale = ldexp(1.0, tc_scale_exp(*maxbits));
    for (long long s = blockIdx.x; s < (long long) NB * MB; s += gridDim.x)
    {
        const int ib = (int) (s / MB), jp = (int) (s % MB);
        if (jp >= nnzb[ib])
            continue;
        const T *x = pool + s * slot_elems;
        tc_t *o = img + s * 4 * IMG;
        for (int e = threadIdx.x; e < IMG; e += blockDim.x)
        {
            const int r = e >> 5, c = e & 31;
            const double v = (double) x[e] * scale; // a power of two: exact
            const tc_t hi = tc_from_double(v);
            const tc_t lo = tc_from_double(v - tc_to_double(hi));
            o[img_off(r, c)] = hi;           // left: row r, k = c
            o[IMG + img_off(r, c)] = lo;
            o[2 * IMG + img_off(c, r)] = hi; // right: n = c, k = r
            o[3 * IMG + img_off(c, r)] = lo;
        }
    }
}

// --- tcgen05 / mbarrier primitives ---------------------------------------
__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned) __cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t smem_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    // start address, leading (k) and stride (row group) byte offsets in
    // 16-byte units; version 1 (bits 46-47); no swizzle; base offset 0.
    return (uint64_t) ((addr >> 4) & 0x3FFFu) | ((uint64_t) ((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t) ((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D F32, A and B both FP16 (type 0) or
// both BF16 (type 1), both K-major, N = 32, M = 128.
constexpr uint32_t TC_AB_TYPE = B200_TC_F16 ? 0u : 1u;
constexpr uint32_t TC_IDESC =
    (1u << 4) | (TC_AB_TYPE << 7) | (TC_AB_TYPE << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_f16(unsigned tmem_d, uint64_t adesc, uint64_t bdesc, unsigned accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u),
                   "r"(0u), "r"(0u)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init1(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(su32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}

// Bulk copy global -> shared (16-byte aligned, a multiple of 16 bytes),
// completing on bar.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     su32(dst)),
                 "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(su32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of bar, at most about 2 s; false on timeout.
__device__ bool mbar_wait2s(uint64_t *bar, unsigned parity)
{
    if (mbar_test(bar, parity))
        return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_test(bar, parity))
        if (now_ns() - t0 > 2000000000ull)
            return false;
    return true;
}

__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32])
{
    unsigned r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                   "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                   "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
                   "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
                   "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i)
        v[i] = __uint_as_float(r[i]);
}

// Shared memory of the X^2 kernel.
template <class Cfg> struct TcSmem
{
    union
    {
        tc_t a[Cfg::ABUF][2][4 * IMG]; // left operands, hi and lo: 128 x 32 (8 KB each)
        struct
        {
            unsigned jbits[TC_NWCAP]; // the group's block columns jb (bitmap over NB)
            int jpre[TC_NWCAP];       // J entries before each bitmap word: index = rank of jb
            unsigned kbits[TC_NWCAP]; // output block columns of the group (bitmap over NB)
            int kpre[TC_NWCAP];       // tiles before each bitmap word: tile = rank of kb
        } su; // the group's set-up, while the left-operand ring is idle
    };
    union
    {
        tc_t b[Cfg::BBUF][2][IMG]; // right operands, hi and lo: 32 x 32 (2 KB each)
        float stage[TC_GROUP][TB][TB + 1]; // epilogue transpose (the ring is idle then)
    };
    uint64_t full_a[Cfg::ABUF], full_b[Cfg::BBUF]; // bulk copies landed
    uint64_t empty_b[Cfg::BBUF];            // MMAs reading a B buffer (and all before) done
    uint64_t empty_a[Cfg::ABUF];            // MMAs reading an A buffer's fill (and all before) done
    uint64_t done;                        // all MMAs of a wave done
    unsigned tmem;
    int nJ, nK, npairs, ok, dead, grp;
    int jb[Cfg::JCAP];             // union of the group's block columns
    short jslot[Cfg::JCAP][TC_GROUP]; // position of X[ib0+q, jb] in row ib0+q, or -1
    int klist[Cfg::KCAP];          // kb of each output tile
    int jcnt[Cfg::JCAP];           // pairs of the current wave per J entry, then their start
    int list[Cfg::LCAP];           // pairs of the current wave: j << 20 | tile << 16 | kp
    int jstart[Cfg::JCAP + 1];     // first pair of each J entry in ptile
    unsigned short ptile[Cfg::PCAP]; // output tile of every pair (j, kp) of the group
    unsigned char jmask[Cfg::JCAP];  // rows q of the group holding X[ib0+q, jb]
    int touched[Cfg::TILES];         // rows q of the group with a product in the tile
};

template <typename T> struct TcView
{
    const T *pool;
    const int *indexb, *nnzb;
    int NB, MB;
    long long slot;
};

template <typename T> struct TcOut
{
    T *pool;
    int *indexb, *nnzb;
    int MB;
    long long slot;
};

// Slot of key k in an open-addressing table of size 2*cap (cap a power of 2).
__device__ __forceinline__ int tc_find(int *keys, int cap2, int k, bool &found)
{
    unsigned h = ((unsigned) k * 2654435761u) & (unsigned) (cap2 - 1);
    for (int p = 0; p < cap2; ++p)
    {
        if (keys[h] == k)
        {
            found = true;
            return (int) h;
        }
        if (keys[h] == B200_EMPTY_KEY)
        {
            found = false;
            return (int) h;
        }
        h = (h + 1) & (unsigned) (cap2 - 1);
    }
    found = false;
    return -1;
}

// Rank of the set bits of bits[0..nwords): pre[w] = set bits before word w,
// list[rank] = bit position (up to cap entries), *total = bits set.  All
// TC_THREADS threads; `scratch` holds one int per warp.
__device__ void rank_bits(const unsigned *bits, int *pre, int *list, int cap, int nwords, int *scratch, int *total,
                          int tid, int lane, int warp)
{
    const int per = (nwords + TC_THREADS - 1) / TC_THREADS;
    const int w0 = min(tid * per, nwords), w1 = min(w0 + per, nwords);
    int sum = 0;
    for (int w = w0; w < w1; ++w)
        sum += __popc(bits[w]);
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1)
    {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o)
            incl += y;
    }
    if (lane == 31)
        scratch[warp] = incl;
    __syncthreads();
    int run = incl - sum;
    for (int w = 0; w < warp; ++w)
        run += scratch[w];
    for (int w = w0; w < w1; ++w)
    {
        pre[w] = run;
        unsigned b = bits[w];
        while (b)
        {
            const int bt = __ffs(b) - 1;
            b &= b - 1;
            if (run < cap)
                list[run] = (w << 5) + bt;
            ++run;
        }
    }
    if (tid == TC_THREADS - 1)
        *total = run;
}

// flags: [0] row overflow, [1] widest kept row, [2] group over capacity,
// [3] a tensor-core wait timed out, [4] next group to claim
template <typename T, class Cfg>
__global__ void __launch_bounds__(TC_THREADS, Cfg::CTAS)
    tc_x2_kernel(TcView<T> X, TcOut<T> C, const tc_t *img, const tc_t *zimg, double thr,
                 double *dA, double *dC, int *flags)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    constexpr int TC_TILES = Cfg::TILES, TC_ABUF = Cfg::ABUF, TC_BBUF = Cfg::BBUF, TC_JCAP = Cfg::JCAP;
    constexpr int TC_KCAP = Cfg::KCAP, TC_LCAP = Cfg::LCAP, TC_PCAP = Cfg::PCAP;
    TcSmem<Cfg> &S = *reinterpret_cast<TcSmem<Cfg> *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ngroups = (X.NB + TC_GROUP - 1) / TC_GROUP;

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&S.tmem)),
                     "r"(TC_TILES * 32)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0)
    {
        for (int i = 0; i < TC_ABUF; ++i)
        {
            mbar_init1(&S.full_a[i]);
            mbar_init1(&S.empty_a[i]);
        }
        for (int i = 0; i < TC_BBUF; ++i)
        {
            mbar_init1(&S.full_b[i]);
            mbar_init1(&S.empty_b[i]);
        }
        mbar_init1(&S.done);
        S.dead = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tbase = S.tmem;
    const float unscale = ldexpf(1.0f, -2 * tc_scale_exp((unsigned) flags[8]));
    bool dead = false; // a wait timed out: stop issuing work
    // pipeline counters, kept alike by the producer (thread 0) and the MMA
    // issuer (thread 32): pairs and left operands issued so far
    unsigned gp = 0, ga = 0, nwaves = 0;
    unsigned copied_a = 0; // left operands whose copies thread 0 issued

    for (;;)
    {
        // groups are claimed from a counter (they differ in cost), by one
        // thread for the whole CTA
        if (tid == 0)
            S.grp = atomicAdd(&flags[4], 1);
        __syncthreads();
        const int grp = S.grp;
        if (grp >= ngroups || dead)
            break;
        const int ib0 = grp * TC_GROUP;
        // ---- the group's block columns J: a bitmap over NB, index = rank ----
        const int nwords = (X.NB + 31) >> 5;
        const int myrow = ib0 + warp; // block row of this warp (left operand q = warp)
        for (int s2 = tid; s2 < nwords; s2 += TC_THREADS)
        {
            S.su.jbits[s2] = 0u;
            S.su.kbits[s2] = 0u;
        }
        if (tid == 0)
            S.ok = 1;
        __syncthreads();
        int bad = 0;
        if (myrow < X.NB)
            for (int jp = lane; jp < X.nnzb[myrow]; jp += 32)
            {
                const int jb = X.indexb[(size_t) myrow * X.MB + jp];
                if (jb < 0 || jb >= X.NB)
                    bad = 1;
                else
                    atomicOr(&S.su.jbits[jb >> 5], 1u << (jb & 31));
            }
        if (__syncthreads_or(bad))
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        rank_bits(S.su.jbits, S.su.jpre, S.jb, TC_JCAP, nwords, S.jcnt, &S.nJ, tid, lane, warp);
        __syncthreads();
        if (S.nJ > TC_JCAP)
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        for (int j = tid; j < S.nJ; j += TC_THREADS)
            for (int q = 0; q < TC_GROUP; ++q)
                S.jslot[j][q] = -1;
        __syncthreads();
        if (myrow < X.NB)
            for (int jp = lane; jp < X.nnzb[myrow]; jp += 32)
            {
                const int jb = X.indexb[(size_t) myrow * X.MB + jp];
                const int j = S.su.jpre[jb >> 5] + __popc(S.su.jbits[jb >> 5] & ((1u << (jb & 31)) - 1u));
                S.jslot[j][warp] = (short) jp;
            }
        __syncthreads();
        for (int j = tid; j < S.nJ; j += TC_THREADS)
        {
            unsigned char m = 0;
            for (int q = 0; q < TC_GROUP; ++q)
                if (S.jslot[j][q] >= 0)
                    m |= (unsigned char) (1u << q);
            S.jmask[j] = m;
        }
        __syncthreads();
        const int nJ = S.nJ;
        // ---- output block columns K: a bitmap over NB, tiles by rank ----
        int badk = 0;
        for (int j = warp; j < nJ && S.ok; j += TC_THREADS / 32)
        {
            const int jb = S.jb[j];
            for (int kp = lane; kp < X.nnzb[jb]; kp += 32)
            {
                const int kb = X.indexb[(size_t) jb * X.MB + kp];
                if (kb < 0 || kb >= X.NB)
                    badk = 1;
                else
                    atomicOr(&S.su.kbits[kb >> 5], 1u << (kb & 31));
            }
        }
        if (__syncthreads_or(badk))
        {
            if (tid == 0)
                S.ok = 0;
        }
        __syncthreads();
        rank_bits(S.su.kbits, S.su.kpre, S.klist, TC_KCAP, nwords, S.jcnt, &S.nK, tid, lane, warp);
        __syncthreads();
        if (tid == 0 && S.nK > TC_KCAP)
            S.ok = 0;
        __syncthreads();
        if (warp == 0)
        {
            int run = 0;
            for (int j0 = 0; j0 < nJ; j0 += 32)
            {
                const int j = j0 + lane;
                const int n = j < nJ ? X.nnzb[S.jb[j]] : 0;
                int incl = n;
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o)
                        incl += y;
                }
                if (j < nJ)
                    S.jstart[j] = run + incl - n;
                run += __shfl_sync(FULL, incl, 31);
            }
            if (lane == 0)
            {
                S.jstart[nJ] = run;
                if (run > TC_PCAP)
                    S.ok = 0;
            }
        }
        __syncthreads();
        if (!S.ok)
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        // the output tile of every pair (j, kp), once per group
        for (int j = warp; j < nJ; j += TC_THREADS / 32)
        {
            const int jb = S.jb[j];
            for (int kp = lane; kp < X.nnzb[jb]; kp += 32)
            {
                const int kb = X.indexb[(size_t) jb * X.MB + kp];
                S.ptile[S.jstart[j] + kp] =
                    (unsigned short) (S.su.kpre[kb >> 5] + __popc(S.su.kbits[kb >> 5] & ((1u << (kb & 31)) - 1u)));
            }
        }
        // the set-up area is the left-operand ring: order its generic
        // accesses before the bulk copies that refill it
        proxy_fence();
        __syncthreads();
        const int nK = S.nK;
        const int nW = (nK + TC_TILES - 1) / TC_TILES;
        int kept = 0;
        double trc = 0.0;

        // ---- tr X of the group's rows (FP64, row order) ----
        if (myrow < X.NB)
        {
            double s = 0.0;
            for (int j0 = 0; j0 < X.nnzb[myrow]; j0 += 32)
            {
                const int jp = j0 + lane;
                unsigned bal = __ballot_sync(FULL, jp < X.nnzb[myrow] && X.indexb[(size_t) myrow * X.MB + jp] == myrow);
                while (bal)
                {
                    const int d = j0 + __ffs(bal) - 1;
                    bal &= bal - 1;
                    const T *blk = X.pool + ((size_t) myrow * X.MB + d) * X.slot;
                    double v = (double) blk[lane * (TB + 1)];
                    for (int o = 16; o; o >>= 1)
                        v += __shfl_xor_sync(FULL, v, o);
                    s += v;
                }
            }
            if (lane == 0 && dA)
                dA[myrow] = s;
        }

        // ---- waves of TC_TILES output tiles ----
        for (int w = 0; w < nW && !dead; ++w)
        {
            const int t0 = w * TC_TILES;
            const int nt = min(TC_TILES, nK - t0);
            if (tid < TC_TILES)
                S.touched[tid] = 0;
            __syncthreads();
            // pairs (j, kb) of this wave, ordered by j then kp: count per j,
            // prefix, write
            for (int j = warp; j < nJ; j += TC_THREADS / 32)
            {
                const int ps = S.jstart[j], pn = S.jstart[j + 1] - ps;
                int cnt = 0;
                for (int k0 = 0; k0 < pn; k0 += 32)
                {
                    const int kp = k0 + lane;
                    bool in = false;
                    if (kp < pn)
                    {
                        const int t = S.ptile[ps + kp];
                        in = t >= t0 && t < t0 + nt;
                    }
                    cnt += __popc(__ballot_sync(FULL, in));
                }
                if (lane == 0)
                    S.jcnt[j] = cnt;
            }
            __syncthreads();
            if (tid == 0)
            {
                int run = 0;
                for (int j = 0; j < nJ; ++j)
                {
                    const int c = S.jcnt[j];
                    S.jcnt[j] = run;
                    run += c;
                }
                S.npairs = run;
            }
            __syncthreads();
            const int p0 = 0, p1 = S.npairs;
            if (p1 > TC_LCAP)
            {
                if (tid == 0)
                    atomicExch(&flags[2], 1);
                dead = true; // capacity, not a timeout: leave the group set
                break;
            }
            for (int j = warp; j < nJ; j += TC_THREADS / 32)
            {
                const int ps = S.jstart[j], pn = S.jstart[j + 1] - ps;
                int pos = S.jcnt[j];
                for (int k0 = 0; k0 < pn; k0 += 32)
                {
                    const int kp = k0 + lane;
                    bool in = false;
                    int t = 0;
                    if (kp < pn)
                    {
                        t = S.ptile[ps + kp];
                        in = t >= t0 && t < t0 + nt;
                    }
                        const unsigned bal = __ballot_sync(FULL, in);
                    if (in)
                    {
                        const int at = pos + __popc(bal & lanemask_lt());
                        // bit 30: the first pair of this j in the wave (a new left operand)
                        S.list[at] = (at == S.jcnt[j] ? 1 << 30 : 0) | (j << 20) | ((t - t0) << 16) | kp;
                        atomicOr(&S.touched[t - t0], (int) S.jmask[j]);
                    }
                    pos += __popc(bal);
                }
            }
            __syncthreads();
            if (tid == 0)
            {
                // producer (thread 0): for each pair, its right operand into
                // the next B buffer and, on a new j, the group's left operand
                // into the next A buffer, each once the MMAs that read the
                // buffer's previous fill are done
                for (int p = p0; p < p1; ++p)
                {
                    const int pv = S.list[p];
                    const int j = (pv >> 20) & 1023, kp = pv & 0xFFFF;
                    const unsigned b = gp % TC_BBUF, f = gp / TC_BBUF;
                    if (pv >> 30)
                    {
                        const unsigned a = ga % TC_ABUF, fa = ga / TC_ABUF;
                        if (fa >= 1 && !mbar_wait2s(&S.empty_a[a], (fa - 1) & 1))
                        {
                            S.dead = 1;
                            break;
                        }
                        mbar_expect(&S.full_a[a], 2 * 4 * IMG * 2);
#pragma unroll
                        for (int q = 0; q < TC_GROUP; ++q)
                        {
                            const int jp = S.jslot[j][q];
#pragma unroll
                            for (int part = 0; part < 2; ++part)
                            {
                                const tc_t *src =
                                    jp >= 0 ? img + (((size_t) (ib0 + q) * X.MB + jp) * 4 + part) * IMG : zimg;
                                bulk_copy(reinterpret_cast<unsigned char *>(S.a[a][part]) + q * 2048, src, IMG * 2,
                                          &S.full_a[a]);
                            }
                        }
                        ++ga;
                        copied_a = ga;
                    }
                    if (f >= 1 && !mbar_wait2s(&S.empty_b[b], (f - 1) & 1))
                    {
                        S.dead = 1;
                        break;
                    }
                    mbar_expect(&S.full_b[b], 2 * IMG * 2);
                    // the right hi and lo images are adjacent in both places:
                    // one 4 KB copy
                    const tc_t *bsrc = img + ((size_t) S.jb[j] * X.MB + kp) * 4 * IMG;
                    bulk_copy(S.b[b][0], bsrc + 2 * IMG, 2 * IMG * 2, &S.full_b[b]);
                    ++gp;
                }
            }
            else if (tid == 32)
            {
                // MMA issuer (thread 32): the same sequence, consuming the
                // ring; the first MMA into a tile in this wave overwrites it
                unsigned started = 0, acur = 0;
                for (int p = p0; p < p1; ++p)
                {
                    const int pv = S.list[p];
                    const int tile = (pv >> 16) & 15;
                    const unsigned b = gp % TC_BBUF, f = gp / TC_BBUF;
                    if (pv >> 30)
                    {
                        if (p > p0)
                            umma_commit(&S.empty_a[acur]); // the previous left operand is done with
                        acur = ga % TC_ABUF;
                        if (!mbar_wait2s(&S.full_a[acur], (ga / TC_ABUF) & 1))
                        {
                            S.dead = 1;
                            break;
                        }
                        ++ga;
                    }
                    if (!mbar_wait2s(&S.full_b[b], f & 1))
                    {
                        S.dead = 1;
                        break;
                    }
                    tc_fence_after();
                    const unsigned d = tbase + (unsigned) (tile * 32);
                    const unsigned a0 = su32(S.a[acur][0]), a1 = su32(S.a[acur][1]);
                    const unsigned b0 = su32(S.b[b][0]), b1 = su32(S.b[b][1]);
                    unsigned acc = (started >> tile) & 1u;
                    started |= 1u << tile;
#pragma unroll
                    for (int ks = 0; ks < 2; ++ks)
                    {
                        // K = 16: two 8-wide k-chunks per step
                        const uint64_t ah = smem_desc(a0 + ks * 2 * TC_LBO, TC_LBO, TC_SBO);
                        const uint64_t al = smem_desc(a1 + ks * 2 * TC_LBO, TC_LBO, TC_SBO);
                        const uint64_t bh = smem_desc(b0 + ks * 2 * TC_LBO, TC_LBO, TC_SBO);
                        const uint64_t bl = smem_desc(b1 + ks * 2 * TC_LBO, TC_LBO, TC_SBO);
                        umma_f16(d, ah, bh, acc);
                        umma_f16(d, ah, bl, 1u);
                        umma_f16(d, al, bh, 1u);
                        acc = 1u;
                    }
                    umma_commit(&S.empty_b[b]);
                    ++gp;
                }
                // the wave's last left operand, then every MMA of the wave
                // (and before) done -> done barrier
                if (p1 > p0)
                    umma_commit(&S.empty_a[acur]);
                umma_commit(&S.done);
            }
            // the other lanes of warps 0 and 1 wait here, not in a polling
            // loop beside their working lane
            __syncwarp();
            // the producer's and issuer's counters must stay alike: both
            // walked every pair of the wave unless the wave died
            const bool late = !mbar_wait2s(&S.done, nwaves & 1);
            ++nwaves;
            tc_fence_after();
            if (__syncthreads_or(late || *reinterpret_cast<volatile int *>(&S.dead)))
            {
                if (tid == 0)
                    atomicExch(&flags[3], 1);
                dead = true;
                break;
            }
            // ---- epilogue: warp q reads block row ib0+q of every tile ----
            for (int t = 0; t < nt; ++t)
            {
                float v[32];
                tmem_ld32(tbase + ((unsigned) (warp * 32) << 16) + (unsigned) (t * 32), v);
#pragma unroll
                for (int c = 0; c < 32; ++c)
                    v[c] *= unscale; // undo the split's 2^s on both factors
                const int kb = S.klist[t0 + t];
                if (myrow >= X.NB || !((S.touched[t] >> warp) & 1))
                    continue;
                float mx = 0.f, diag = 0.f;
#pragma unroll
                for (int c = 0; c < 32; ++c)
                {
                    mx = fmaxf(mx, fabsf(v[c]));
                    diag = c == lane ? v[c] : diag;
                }
                for (int o = 16; o; o >>= 1)
                    mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, o));
                const bool keep = kb == myrow || (double) mx > thr;
                if (!keep)
                    continue;
                if (kb == myrow)
                {
                    double dd = (double) diag;
                    for (int o = 16; o; o >>= 1)
                        dd += __shfl_xor_sync(FULL, dd, o);
                    trc += dd;
                }
                if (kept < C.MB)
                {
                    // lane = block row; through shared memory so that the
                    // warp writes the row-major block in contiguous runs
#pragma unroll
                    for (int c = 0; c < 32; ++c)
                        S.stage[warp][lane][c] = v[c];
                    __syncwarp();
                    T *dst = C.pool + ((size_t) myrow * C.MB + kept) * C.slot;
#pragma unroll 4
                    for (int r = 0; r < 32; ++r)
                        dst[r * TB + lane] = (T) S.stage[warp][r][lane];
                    __syncwarp();
                    if (lane == 0)
                        C.indexb[(size_t) myrow * C.MB + kept] = kb;
                }
                ++kept;
            }
            // the transpose area is the copy ring: order these generic writes
            // before the next wave's bulk copies
            proxy_fence();
            tc_fence_before();
            __syncthreads();
        }
        if (myrow < X.NB && lane == 0)
        {
            C.nnzb[myrow] = kept < C.MB ? kept : C.MB;
            atomicMax(&flags[1], kept);
            if (kept > C.MB)
                atomicExch(&flags[0], 1);
            if (dC)
                dC[myrow] = trc;
        }
        __syncthreads();
    }
    // after a timeout, give the MMAs in flight one more bounded wait before
    // their tensor memory is released
    if (dead && tid == 32)
    {
        umma_commit(&S.done);
        mbar_wait2s(&S.done, nwaves & 1);
    }
    if (dead && tid == 0)
    {
        // bulk copies still in flight land before the CTA leaves: the last
        // fill of every buffer (bounded waits)
        for (unsigned b = 0; b < TC_BBUF && b < gp; ++b)
        {
            const unsigned last = (gp - 1 - b) / TC_BBUF; // fill index of buffer (gp-1-b) % TC_BBUF
            mbar_wait2s(&S.full_b[(gp - 1 - b) % TC_BBUF], last & 1);
        }
        for (unsigned a = 0; a < TC_ABUF && a < copied_a; ++a)
            mbar_wait2s(&S.full_a[(copied_a - 1 - a) % TC_ABUF], ((copied_a - 1 - a) / TC_ABUF) & 1);
    }
    // release the tensor memory (after every read of it)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TC_TILES * 32)
                     : "memory");
}

} // namespace

template <typename T>
bool tc_split(B200Context *c, const bml_matrix_ellblock_t *X, int sgrid, unsigned *maxbits, tc_t *img)
{
    const T *pool = static_cast<const T *>(X->d_pool);
    tc_maxabs_kernel<T><<<sgrid, 256, 0, c->stream>>>(pool, X->d_nnzb, X->NB, X->MB, X->slot_elems, maxbits);
    if (!LAUNCH_OK("tc_maxabs_kernel"))
        return false;
    tc_split_kernel<T><<<sgrid, 256, 0, c->stream>>>(pool, X->d_nnzb, X->NB, X->MB, X->slot_elems, maxbits, img);
    return LAUNCH_OK("tc_split_kernel");
}

template <typename T, class Cfg>
bool tc_launch(B200Context *c, const bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, const tc_t *img,
               const tc_t *zimg, double threshold, double *dA, double *dC, int *flags)
{
    const size_t smem = sizeof(TcSmem<Cfg>) + 1024;
    auto k = tc_x2_kernel<T, Cfg>;
    if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
        return false;
    k<<<c->sm_count * Cfg::CTAS, TC_THREADS, smem, c->stream>>>(
        TcView<T>{static_cast<const T *>(X->d_pool), X->d_indexb, X->d_nnzb, X->NB, X->MB, X->slot_elems},
        TcOut<T>{static_cast<T *>(X2->d_pool), X2->d_indexb, X2->d_nnzb, X2->MB, X2->slot_elems}, img, zimg,
        threshold, dA, dC, flags);
    return LAUNCH_OK("tc_x2_kernel");
}

// X2 = X*X on the tensor cores (FP16 hi/lo split, FP32 accumulation); X and
// X2 must have blocks of 32 throughout.  Returns false with a status set
// (UNSUPPORTED when the partition or a group's size is outside this path).
bool eb_multiply_x2_tc(bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, double threshold, double *trace)
{
    if (!X || !X2 || X == X2 || X->NB != X2->NB || X->matrix_precision != X2->matrix_precision)
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply_x2_tc: X and X2 must be distinct, of one partition and precision");
        return false;
    }
    for (int ib = 0; ib < X->NB; ++ib)
        if (X->bsize[ib] != TB || X2->bsize[ib] != TB)
        {
            b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply_x2_tc: block %d has size %d (32 needed)", ib,
                           X->bsize[ib]);
            return false;
        }
    if (X->NB > TC_NWCAP * 32)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply_x2_tc: NB=%d above %d", X->NB, TC_NWCAP * 32);
        return false;
    }
    if (X->MB > 32767)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply_x2_tc: MB=%d above 32767", X->MB);
        return false;
    }
    B200Context *c = b200_ctx();
    if (!c || !eb_to_device(X) || !eb_to_device(X2))
        return false;
    const int NB = X->NB, MB = X->MB;
    const size_t n_img = (size_t) NB * MB * 4 * IMG;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t off_tr = al(n_img * sizeof(tc_t));
    const size_t off_flags = al(off_tr + (size_t) 2 * NB * sizeof(double));
    const size_t off_zero = al(off_flags + 64);
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(off_zero + IMG * sizeof(tc_t)));
    if (!scr)
        return false;
    tc_t *img = reinterpret_cast<tc_t *>(scr);
    double *dA = reinterpret_cast<double *>(scr + off_tr);
    double *dC = dA + NB;
    int *flags = reinterpret_cast<int *>(scr + off_flags);
    unsigned *maxbits = reinterpret_cast<unsigned *>(flags + 8); // max |x| of X, for the split's scale
    tc_t *zimg = reinterpret_cast<tc_t *>(scr + off_zero);
    if (!CUDA_OK(cudaMemsetAsync(flags, 0, 64, c->stream)) ||
        !CUDA_OK(cudaMemsetAsync(zimg, 0, IMG * sizeof(tc_t), c->stream)) ||
        !CUDA_OK(cudaMemsetAsync(dA, 0, (size_t) 2 * NB * sizeof(double), c->stream)))
        return false;
    const int sgrid = (int) min((long long) NB * MB, (long long) c->sm_count * 32);
    bool ok = X->matrix_precision == double_real
                  ? tc_split<double>(c, X, sgrid, maxbits, img)
                  : tc_split<float>(c, X, sgrid, maxbits, img);
    if (!ok)
        return false;
    // the two-CTA shape first; the one-CTA shape if a group exceeded it
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 8192;
    int hf[4];
    for (int shape = 0; shape < 2; ++shape)
    {
        if (shape == 1 && !CUDA_OK(cudaMemsetAsync(flags, 0, 20, c->stream)))
            return false;
        if (X->matrix_precision == double_real)
            ok = shape == 0 ? tc_launch<double, TcSmall>(c, X, X2, img, zimg, threshold, dA, dC, flags)
                            : tc_launch<double, TcBig>(c, X, X2, img, zimg, threshold, dA, dC, flags);
        else
            ok = shape == 0 ? tc_launch<float, TcSmall>(c, X, X2, img, zimg, threshold, dA, dC, flags)
                            : tc_launch<float, TcBig>(c, X, X2, img, zimg, threshold, dA, dC, flags);
        if (!ok)
            return false;
        if (!CUDA_OK(cudaMemcpyAsync(pin, flags, 16, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
            return false;
        memcpy(hf, pin, sizeof(hf));
        if (!hf[2] || hf[3])
            break; // fitted (or timed out: reported below)
    }
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 4096 + 256);
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(dA, dC, NB, out);
    if (!LAUNCH_OK("b200_sum_rows_kernel"))
        return false;
    if (!CUDA_OK(cudaMemcpyAsync(pin + 64, out, 16, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    X2->mirror = MIRROR_DEVICE_NEWER;
    if (trace)
        memcpy(trace, pin + 64, 2 * sizeof(double));
    if (hf[3])
    {
        b200_set_error(BML_B200_ERR_TIMEOUT, "multiply_x2_tc: a tensor-core wait timed out");
        return false;
    }
    if (hf[2])
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply_x2_tc: a group of block rows exceeds the kernel's capacity");
        return false;
    }
    if (hf[0])
    {
        b200_set_error(BML_B200_ERR_ROW_OVERFLOW,
                       "Number of non-zeroes blocks per row > MB, Increase MB (need %d, MB = %d)", hf[1], X2->MB);
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int bml_b200_ellblock_multiply_x2_tc(bml_matrix_t *X, bml_matrix_t *X2, double threshold,
                                                double *trace)
{
    if (bml_get_type(X) != ellblock || bml_get_type(X2) != ellblock)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ellblock_multiply_x2_tc: ELLBLOCK matrices expected");
        return BML_B200_ERR_INVALID;
    }
    bml_b200_clear_error();
    double tr[2] = {0.0, 0.0};
    if (!eb_multiply_x2_tc(static_cast<bml_matrix_ellblock_t *>(X), static_cast<bml_matrix_ellblock_t *>(X2),
                           threshold, tr))
        return b200_get_error();
    if (trace)
    {
        trace[0] = tr[0];
        trace[1] = tr[1];
    }
    return BML_B200_OK;
}

extern "C" int bml_b200_ellblock_sp2_mixed(bml_matrix_t *H, bml_matrix_t *D, double threshold, double occupation,
                                           int maxiter, double tol, int stall, int nclose, double *info)
{
    double local[8] = {0, 4, 0, 0, 0, 0, 0, 0};
    double *inf = info ? info : local;
    for (int k = 0; k < 8; ++k)
        inf[k] = local[k];
    if (!H || !D || H == D || bml_get_type(H) != ellblock || bml_get_type(D) != ellblock ||
        bml_get_precision(H) != bml_get_precision(D) || bml_get_N(H) != bml_get_N(D) || nclose < 0 ||
        nclose > maxiter)
    {
        b200_set_error(BML_B200_ERR_INVALID, "ellblock_sp2_mixed: H and D must be distinct ELLBLOCK matrices "
                                             "of one precision and N, 0 <= nclose <= maxiter");
        return BML_B200_ERR_INVALID;
    }
    bml_b200_clear_error();
    bml_copy(H, D);
    double *eb = static_cast<double *>(bml_gershgorin(H));
    if (!eb || bml_b200_last_error())
    {
        free(eb);
        return bml_b200_last_error();
    }
    bml_normalize(D, eb[0], eb[1]);
    free(eb);
    if (bml_b200_last_error())
        return bml_b200_last_error();
    bml_matrix_t *X2 = bml_zero_matrix(ellblock, bml_get_precision(D), bml_get_N(D), bml_get_M(D), sequential);
    if (!X2)
        return bml_b200_last_error();
    int status = BML_B200_OK, rule = 3, it = 0, it_tc = 0, since = 0;
    double best = HUGE_VAL, last = 0.0, x2s = 0.0, x2s_tc = 0.0;
    for (; it < maxiter; ++it)
    {
        const bool closing = it >= maxiter - nclose;
        double tr[2];
        const auto t0 = std::chrono::steady_clock::now();
        bool ok = false, on_tc = false;
        if (!closing)
        {
            // Blocks other than 32 x 32, or a group beyond the tensor-core
            // kernel's capacities, are an expected outcome here: that
            // iteration runs on the exact product, noted as information.
            const int verbose = b200_swap_verbose(0);
            ok = on_tc = eb_multiply_x2_tc(static_cast<bml_matrix_ellblock_t *>(D),
                                           static_cast<bml_matrix_ellblock_t *>(X2), threshold, tr);
            b200_swap_verbose(verbose);
            if (!on_tc && b200_get_error() == BML_B200_ERR_UNSUPPORTED)
            {
                bml_b200_clear_error();
                if (verbose)
                    fprintf(stderr, "[bml_b200 info] ellblock_sp2_mixed: iteration %d runs on the exact block "
                                    "product (outside the tensor-core kernel's capacities)\n", it);
            }
            else if (!on_tc)
                b200_set_error(b200_get_error(), "ellblock_sp2_mixed: tensor-core X^2 failed in iteration %d", it);
        }
        if (closing || (!on_tc && !bml_b200_last_error()))
            ok = eb_multiply_x2(static_cast<bml_matrix_ellblock_t *>(D), static_cast<bml_matrix_ellblock_t *>(X2),
                                threshold, tr);
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        x2s += dt;
        if (on_tc)
        {
            x2s_tc += dt;
            ++it_tc;
        }
        if (!ok)
        {
            status = b200_get_error();
            rule = 4;
            break;
        }
        const double t = tr[0], t2 = tr[1];
        last = fabs(t - t2);
        if (fabs(t2 - occupation) <= fabs(2.0 * t - t2 - occupation))
            bml_copy(X2, D);
        else
            bml_add(D, X2, 2.0, -1.0, threshold);
        if (bml_b200_last_error())
        {
            status = bml_b200_last_error();
            rule = 4;
            ++it;
            break;
        }
        if (!closing && rule == 3)
        {
            // bulk stop rules: jump to the closing iterations
            bool stop = last < tol;
            if (!stop && stall > 0)
            {
                if (last < best)
                {
                    best = last;
                    since = 0;
                }
                else if (++since >= stall)
                    stop = true;
            }
            if (stop)
            {
                rule = last < tol ? 1 : 2;
                const int remaining = maxiter - nclose - it - 1;
                maxiter -= remaining; // the closing iterations follow now
            }
        }
    }
    bml_deallocate(&X2);
    inf[0] = it;
    inf[1] = rule;
    inf[2] = status == BML_B200_OK ? bml_trace(D) : 0.0;
    inf[3] = last;
    inf[4] = 0;
    inf[5] = x2s;
    inf[6] = it_tc;
    inf[7] = x2s_tc;
    return status;
}
