// ELLBLOCK X^2 on the tcgen05 tensor cores, in one of two splits (mixed
// precision; no reference counterpart: the reference multiplies blocks in the
// matrix precision, ellblock/bml_multiply_ellblock_typed.c:246-442): FP16
// hi/lo halves with FP32 accumulation (the default, below), or 8-bit slices
// with exact INT32 accumulation (bml_b200_set_tc_split(1); described with
// its kernels further down).  Both share the group tables, the rings and the
// pipeline; they differ in the operand images, the MMA kind and the epilogue.
//
// FP16 split.  X is scaled by a power of two 2^s (its largest entry near 2^14) and every
// 32x32 block x is split as hi = fp16(2^s x), lo = fp16(2^s x - hi); X^2 =
// sum_jb X[ib,jb] X[jb,kb] is formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory and scaled back by 2^-2s (lo*lo, about 2^-22
// of the product, is dropped).  The accuracy is then set by the tensor
// cores' FP32 accumulation: one X^2 of the 16^3 block lattice has its trace
// within 7e-6, with BF16 operands (8-bit significands) and FP16 alike.  The
// result is written back in the matrix precision; blocks are kept as in the
// reference (kb == ib, or max |x| > threshold), the traces are FP64 sums.
//
// Work: persistent CTAs claim from a counter groups of four consecutive
// block rows ib0..ib0+3, which share most of their block columns jb on a
// lattice.  For the group, with M = 128 = 4 x 32 rows:
//   D[kb] (128 x 32, FP32, in TMEM) += [X[ib0,jb]; ..; X[ib0+3,jb]] X[jb,kb]
// over the union J of the rows' block columns (missing blocks are zero), for
// every output block column kb in K; 8 output tiles of 32 TMEM columns are
// live at once (a wave), so the group's outputs are made in waves.
// The group's tables (J, K, the output tile of every pair (jb, kb), and the
// pairs sorted by wave with a stable counting sort, so that the pairs of one
// jb stay together and share one left operand) are built by the CTA in global
// memory, one set per CTA, sized before the launch by a counting kernel for
// the largest group: the kernel takes groups of any size.
// Operands are staged into shared memory in the UMMA canonical K-major
// no-swizzle layout (8-row x 16-byte core matrices).  A split kernel first
// writes every block of X in that layout, as the left operand (rows x k) and
// as the right operand (columns x k, the block transposed), the parts of each
// interleaved by row group, so staging is one bulk copy (cp.async.bulk,
// completing on an mbarrier) per block.  The pairs
// of one wave and one block column jb form a step: one left operand (the
// group's four blocks of column jb) and at most one right operand per tile.
// A producer warp copies a step's left operand into a ring of buffers and its
// right operands side by side, in tile order, into a ring of slots; an issuer
// warp (one lane) then issues one MMA per run of consecutive tiles and part,
// N = 32 x the run's tiles (up to 256), and releases the buffer and slots
// with tcgen05.commit on their "empty" mbarriers.  Both warps read the sorted
// pairs 32 records per load; every wait is bounded.
#include "device_util.cuh"
#include "ellblock.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <chrono>
#include <climits>
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
// Shape of the kernel: TILES output tiles of 32 TMEM columns live per CTA (a
// wave), CTAS CTAs per SM (two, so that one CTA's set-up and epilogue overlap
// the other's MMAs), ABUF left-operand buffers and BBUF right-operand slots
// (a step takes one slot per pair, side by side).  Measured on the 16^3 block
// lattice's X^2: 8 tiles x 2 CTAs 6.9 ms, 16 tiles x 1 CTA 10.0 ms (with one
// MMA per pair).
template <int TILES_, int CTAS_, int ABUF_, int BBUF_, int ABYTES_ = 16384, int BBYTES_ = 4096> struct TcCfg
{
    static constexpr int TILES = TILES_, CTAS = CTAS_, ABUF = ABUF_, BBUF = BBUF_;
    static constexpr int ABYTES = ABYTES_, BBYTES = BBYTES_; // one left operand / right operand slot
    static_assert(CTAS * TILES * 32 <= 512, "tensor memory holds 512 columns per SM");
    static_assert(TILES <= 16, "a step's tiles take 16 bits of a record");
    static_assert(BBUF >= TILES, "a step's right operands fit the slot ring");
};
#ifndef B200_TC_TILES
#define B200_TC_TILES 8
#endif
#ifndef B200_TC_CTAS
#define B200_TC_CTAS 2
#endif
#ifndef B200_TC_ABUF
#define B200_TC_ABUF 3
#endif
#ifndef B200_TC_BBUF
#define B200_TC_BBUF 14
#endif
using TcShape = TcCfg<B200_TC_TILES, B200_TC_CTAS, B200_TC_ABUF, B200_TC_BBUF>;

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

// 16-bit images of a block in the K-major no-swizzle layout, as a left
// operand (element (row, k) = block (r, k)) or a right operand (element
// (row, k) = block (k, n), row = n): 16-byte rows of 8 k, 8-row core
// matrices of 128 bytes, the four k-chunks of an 8-row group side by side
// (LBO = 128 B); hi and lo of a row group together, row group g at g * 1 KB,
// hi at +0 and lo at +512 B.  A block is then one 4 KB image whose row
// groups follow at a uniform SBO = 1 KB, so four blocks placed one after the
// other form the 128-row left operand, and the images of consecutive output
// tiles side by side one right operand of N = 32 x (tiles).
constexpr unsigned TC_LBO = 128, TC_RSBO = 1024, TC_RLO = 512;

__device__ __forceinline__ int rimg_off(int n, int k, int part)
{
    return (n >> 3) * 512 + part * 256 + (k >> 3) * 64 + (n & 7) * 8 + (k & 7);
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

// Split every stored block of X, scaled by 2^s, into its images at
// img + slot*4*IMG: the left operand's hi and lo interleaved by row group
// (4 KB), then the right operand's (4 KB).  One warp per block: lane c
// holds column c of every row; the right image (n = c) is written from
// registers, the left one (row r) through a shared-memory transpose, both in
// 16-byte stores.
constexpr int TC_SPLIT_WARPS = 8;

template <typename T>
__global__ void __launch_bounds__(TC_SPLIT_WARPS * 32)
    tc_split_kernel(const T *pool, const int *nnzb, int NB, int MB, long long slot_elems, const unsigned *maxbits,
                    tc_t *img)
{
    __shared__ __align__(16) tc_t sh[TC_SPLIT_WARPS][2][TB][TB + 8]; // [part][row][k], rows of 80 B
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const double scale = ldexp(1.0, tc_scale_exp(*maxbits));
    const long long warps = (long long) gridDim.x * TC_SPLIT_WARPS;
    for (long long s = (long long) blockIdx.x * TC_SPLIT_WARPS + wq; s < (long long) NB * MB; s += warps)
    {
        const int ib = (int) (s / MB), jp = (int) (s % MB);
        if (jp >= nnzb[ib])
            continue;
        const T *x = pool + s * slot_elems;
        tc_t *o = img + s * 4 * IMG;
        tc_t hi[TB], lo[TB];
#pragma unroll
        for (int r = 0; r < TB; ++r)
        {
            const double v = (double) x[r * TB + lane] * scale; // a power of two: exact
            hi[r] = tc_from_double(v);
            lo[r] = tc_from_double(v - tc_to_double(hi[r]));
            sh[wq][0][r][lane] = hi[r];
            sh[wq][1][r][lane] = lo[r];
        }
        // right: n = lane, k = r; eight consecutive k per 16-byte store
#pragma unroll
        for (int kc = 0; kc < 4; ++kc)
        {
            uint4 vh, vl;
            tc_t *ph = reinterpret_cast<tc_t *>(&vh), *pl = reinterpret_cast<tc_t *>(&vl);
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
                ph[i] = hi[kc * 8 + i];
                pl[i] = lo[kc * 8 + i];
            }
            *reinterpret_cast<uint4 *>(o + 2 * IMG + rimg_off(lane, kc * 8, 0)) = vh;
            *reinterpret_cast<uint4 *>(o + 2 * IMG + rimg_off(lane, kc * 8, 1)) = vl;
        }
        __syncwarp();
        // left: row r = lane, k = eight consecutive columns per store
#pragma unroll
        for (int part = 0; part < 2; ++part)
#pragma unroll
            for (int kc = 0; kc < 4; ++kc)
                *reinterpret_cast<uint4 *>(o + rimg_off(lane, kc * 8, part)) =
                    *reinterpret_cast<const uint4 *>(&sh[wq][part][lane][kc * 8]);
        __syncwarp();
    }
}

// --- exact mode: 8-bit slices with INT32 accumulation (kind::i8) --------
// Every entry x of scalar row r, as a left operand, is written
//   x = sigma_r 2^-6 (a1 + 2^-7 a2 + 2^-14 a3 + 2^-21 a4 + 2^-28 a5) + e,
// |a_s| <= 64 (signed 8-bit), |e| <= 2^-35 sigma_r, with sigma_r = 2^e_r the
// power of two just above the row's largest entry; as a right operand the
// same with tau_c of its scalar column.  A product of two entries is then
// 2^-12 sigma_r tau_c sum_{s,t} a_s b_t 2^-7(s+t-2); the terms with
// s + t <= 6 (15 MMAs per block pair, each K = 32) are kept, the others are
// below 2^-33 sigma_r tau_c.  Each level L = s + t sums in its own INT32
// accumulator in TMEM, exactly (no rounding at all: a term is at most
// 64 x 64 x 32 = 2^17 per level and pair, five terms at L = 6, so up to
// 3276 pairs per tile fit in 2^31), and the epilogue combines the five
// levels in FP64, exactly.  The result differs from the exact product only
// by the slicing, about 2^-33 sigma_r tau_c per product term, without the
// FP32 accumulation error of the FP16 form.  (Four slices, 2^-27 per term,
// left SP2's trace 1.6e-5 from the exact solve: the error is relative to the
// row and column maxima, not to each entry.)
constexpr int TC8_SLICES = 5;
constexpr int TC8_LEVELS = TC8_SLICES;  // s + t = 2..6
constexpr int TC8_IMG = TB * TB;        // bytes per 8-bit slice image of a block (1 KB)
constexpr int TC8_BLOCK_BYTES = 2 * TC8_SLICES * TC8_IMG; // left slices | right slices
constexpr int TC16_BLOCK_BYTES = 8 * IMG;                 // left hi, lo | right hi, lo
constexpr int TC_ZERO_BYTES = TC8_BLOCK_BYTES / 2;        // a zero left image, either split
constexpr int TC8_MAX_COLS = 3276;      // block columns per group the level sums hold
constexpr unsigned TC8_LBO = 128;

// Byte offset of element (row, k) in an 8-bit image, left or right operand:
// 16-byte rows of 16 k, 8-row core matrices of 128 bytes, the two k-chunks
// of an 8-row group side by side (LBO = 128 B), the five slices of a row
// group together, row group g at g * 1280 B and slice s at +256 s.  A block
// is one 5 KB image with a uniform SBO = 1280 B, so four blocks stack into
// the 128-row left operand and consecutive tiles' images form one wider
// right operand.
constexpr unsigned TC8_RSBO = 1280;

__device__ __forceinline__ int rimg8_off(int n, int k, int s)
{
    return (n >> 3) * 1280 + s * 256 + (k >> 4) * 128 + (n & 7) * 16 + (k & 15);
}

// Exponent e with 2^e > m >= 0 (m given by its bits; 0 for m = 0).
__device__ __forceinline__ int tc8_exp(unsigned long long bits)
{
    const double m = __longlong_as_double((long long) bits);
    if (!(m > 0.0))
        return 0;
    int e = 0;
    frexp(m, &e); // m in [2^(e-1), 2^e)
    return e;
}

// Largest |x| of every scalar row (rowmax) and column (colmax) of X, as
// the bits of non-negative doubles (which order like the values).  One warp
// per stored block: lane = column, a loop over the block's rows.
template <typename T>
__global__ void tc8_max_kernel(const T *pool, const int *indexb, const int *nnzb, int NB, int MB, long long slot_elems,
                               unsigned long long *rowmax, unsigned long long *colmax)
{
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long) gridDim.x * blockDim.x) >> 5;
    for (long long s = ((long long) blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < (long long) NB * MB; s += warps)
    {
        const int ib = (int) (s / MB), jp = (int) (s % MB);
        if (jp >= nnzb[ib])
            continue;
        const int jb = indexb[s];
        const T *x = pool + s * slot_elems;
        double cm = 0.0;
        for (int r = 0; r < TB; ++r)
        {
            const double v = fabs((double) x[r * TB + lane]);
            cm = fmax(cm, v);
            double rm = v;
            for (int o = 16; o; o >>= 1)
                rm = fmax(rm, __shfl_xor_sync(FULL, rm, o));
            if (lane == 0)
                atomicMax(&rowmax[(size_t) ib * TB + r], (unsigned long long) __double_as_longlong(rm));
        }
        atomicMax(&colmax[(size_t) jb * TB + lane], (unsigned long long) __double_as_longlong(cm));
    }
}

// The slices a1..a4 of u (|u| < 1), each in [-64, 64].
__device__ __forceinline__ void tc8_slices(double u, signed char (&a)[TC8_SLICES])
{
    double y = u * 64.0;
#pragma unroll
    for (int s = 0; s < TC8_SLICES; ++s)
    {
        const double q = rint(y);
        a[s] = (signed char) (int) q;
        y = (y - q) * 128.0; // exact: y - q is y's fraction, scaled by a power of two
    }
}

// Slice every stored block of X into its 8-bit images at img + slot * 10 KB:
// the left slices 1..5 (element (r, k) of the block, scaled by sigma of
// scalar row r), then the right slices 1..5 (element (n, k) = block (k, n),
// scaled by tau of scalar column n), each operand interleaved by row group in
// 5 KB.  One warp per block, lane c on column c: the right slices
// are packed in registers, the left ones go through a shared-memory
// transpose; both are written in 16-byte stores.
constexpr int TC8_SPLIT_WARPS = 4; // 30 KB of static shared memory

template <typename T>
__global__ void __launch_bounds__(TC8_SPLIT_WARPS * 32)
    tc8_split_kernel(const T *pool, const int *indexb, const int *nnzb, int NB, int MB, long long slot_elems,
                     const unsigned long long *rowmax, const unsigned long long *colmax, signed char *img)
{
    __shared__ __align__(16) signed char sh[TC8_SPLIT_WARPS][TC8_SLICES][TB][TB + 16]; // rows of 48 B
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const long long warps = (long long) gridDim.x * TC8_SPLIT_WARPS;
    for (long long s = (long long) blockIdx.x * TC8_SPLIT_WARPS + wq; s < (long long) NB * MB; s += warps)
    {
        const int ib = (int) (s / MB), jp = (int) (s % MB);
        if (jp >= nnzb[ib])
            continue;
        const int jb = indexb[s];
        const T *x = pool + s * slot_elems;
        signed char *o = img + s * TC8_BLOCK_BYTES;
        const int ec = -tc8_exp(colmax[(size_t) jb * TB + lane]);
        unsigned rp[TC8_SLICES][2][4]; // right slices: [slice][k-chunk][4 bytes per word]
#pragma unroll
        for (int q = 0; q < TC8_SLICES; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    rp[q][h][i] = 0u;
#pragma unroll
        for (int r = 0; r < TB; ++r)
        {
            const double v = (double) x[r * TB + lane];
            signed char a[TC8_SLICES];
            tc8_slices(ldexp(v, -tc8_exp(rowmax[(size_t) ib * TB + r])), a);
#pragma unroll
            for (int q = 0; q < TC8_SLICES; ++q)
                sh[wq][q][r][lane] = a[q];
            tc8_slices(ldexp(v, ec), a);
            // byte r & 15 of k-chunk r >> 4: word (r & 15) >> 2, shift 8 (r & 3)
#pragma unroll
            for (int q = 0; q < TC8_SLICES; ++q)
                rp[q][r >> 4][(r & 15) >> 2] |= (unsigned) (unsigned char) a[q] << (8 * (r & 3));
        }
        // right: n = lane, sixteen consecutive k per store
#pragma unroll
        for (int q = 0; q < TC8_SLICES; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h)
                *reinterpret_cast<uint4 *>(o + TC8_SLICES * TC8_IMG + rimg8_off(lane, h * 16, q)) =
                    make_uint4(rp[q][h][0], rp[q][h][1], rp[q][h][2], rp[q][h][3]);
        __syncwarp();
        // left: row r = lane, sixteen consecutive columns per store
#pragma unroll
        for (int q = 0; q < TC8_SLICES; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h)
                *reinterpret_cast<uint4 *>(o + rimg8_off(lane, h * 16, q)) =
                    *reinterpret_cast<const uint4 *>(&sh[wq][q][lane][h * 16]);
        __syncwarp();
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
// both BF16 (type 1), both K-major, M = 128; N (bits 17-22, N / 8) is added
// per MMA: 32 per output tile of the run it covers.
constexpr uint32_t TC_AB_TYPE = B200_TC_F16 ? 0u : 1u;
constexpr uint32_t TC_IDESC = (1u << 4) | (TC_AB_TYPE << 7) | (TC_AB_TYPE << 10) | ((128u >> 4) << 24);

// N field of an instruction descriptor for a run of `tiles` output tiles
// (N = 32 tiles: 32..256, a multiple of 16 as M = 128 requires; longer runs
// are split by the caller).
__device__ __forceinline__ uint32_t idesc_n(int tiles) { return (uint32_t) (tiles * 32 >> 3) << 17; }

__device__ __forceinline__ void umma_f16(unsigned tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         unsigned accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
                   "r"(0u), "r"(0u)
                 : "memory");
}

// kind::i8 instruction descriptor: D S32 (2), A and B signed 8-bit (1),
// both K-major, M = 128; N added per MMA as above.
constexpr uint32_t TC8_IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma_i8(unsigned tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        unsigned accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u),
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
        unsigned char a[Cfg::ABUF][Cfg::ABYTES]; // left operands: 128 x 32, every part
        struct
        {
            unsigned jbits[TC_NWCAP]; // the group's block columns jb (bitmap over NB)
            int jpre[TC_NWCAP];       // J entries before each bitmap word: index = rank of jb
            unsigned kbits[TC_NWCAP]; // output block columns of the group (bitmap over NB)
            int kpre[TC_NWCAP];       // tiles before each bitmap word: tile = rank of kb
        } su;                         // the group's set-up, while the left-operand ring is idle
        int wpos[4 * TC_NWCAP];       // then the next free place of every wave in the sorted pairs
    };
    union
    {
        unsigned char b[Cfg::BBUF][Cfg::BBYTES]; // right operand slots: 32 x 32, every part
        float stage[TC_GROUP][TB][TB + 1]; // epilogue transpose (the ring is idle then)
        double dstage[TC_GROUP][TB][17];   // the same for the 8-bit mode's FP64 values, 16 columns at a time
    };
    uint64_t full_a[Cfg::ABUF], full_b[Cfg::BBUF]; // bulk copies landed (B: per step, a ring of BBUF)
    uint64_t empty_b[Cfg::BBUF];                   // MMAs of a step (and all before) done
    uint64_t empty_a[Cfg::ABUF];                   // MMAs reading an A buffer's fill (and all before) done
    uint64_t done;                                 // all MMAs of a wave done
    unsigned sstart[Cfg::BBUF];                    // producer: first slot (a running count) of each live step
    unsigned tmem;
    int nJ, nK, npairs, dead, grp;
    int scratch[TC_THREADS / 32];
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

// A group's tables, in global memory: one set per CTA, each sized for the
// largest group (tc_count_kernel).  A pair (j, kp) is the product of the
// group's left operand for J entry j with the right operand X[jb_j, kb],
// kb the kp-th block column of row jb_j.  The pairs of one wave and one J
// entry (a step: at most one pair per tile) share one left operand and go to
// the tensor cores together.  Records of the sorted pairs:
//   x = tile within the wave (bits 0-3) | j << 4 (bits 4-19; while the
//       tables are built) | 1 << 31 on a step's first pair, whose bits 4-19
//       then hold the step's tiles as a mask,
//   y = slot of the right operand, jb * MB + kp,
//   z, w = position jp of X[ib0+q, jb] in row ib0+q for q = 0..3, 16 bits
//          each (z: q = 0, 1; w: q = 2, 3), 0xFFFF where the row lacks jb.
struct TcTab
{
    int *jb;              // [jcap] J: the group's block columns, ascending
    uint2 *jslot;         // [jcap] positions of X[ib0+q, jb], as z, w above
    unsigned char *jmask; // [jcap] rows q holding jb
    int *jstart;          // [jcap + 1] first pair of each J entry, pairs in (j, kp) order
    int *klist;           // [kcap] K: the output block columns, ascending (tile = rank)
    int *ttouch;          // [kcap] rows q with a product in each tile
    int *ptile;           // [pcap] output tile of every pair, in (j, kp) order
    uint4 *list;          // [pcap] the pairs sorted by wave, in (j, kp) order within a wave
    int *wstart;          // [wcap + 1] first pair of each wave in list
    int jcap, kcap, pcap, wcap;
};

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

// Sizes of every group's tables: |J|, |K| and its pairs sum_{jb in J}
// nnzb[jb].  Their maxima over the groups go to flags[5], [6] and [7], a
// block column outside 0..NB-1 to flags[2].  One group per CTA at a time;
// the rows of J are walked one per warp.
template <typename T>
__global__ void __launch_bounds__(TC_THREADS) tc_count_kernel(TcView<T> X, int *flags)
{
    __shared__ unsigned jbits[TC_NWCAP], kbits[TC_NWCAP];
    __shared__ long long red[TC_THREADS / 32][3];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ngroups = (X.NB + TC_GROUP - 1) / TC_GROUP;
    const int nwords = (X.NB + 31) >> 5;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x)
    {
        for (int w = tid; w < nwords; w += TC_THREADS)
        {
            jbits[w] = 0u;
            kbits[w] = 0u;
        }
        __syncthreads();
        const int row = g * TC_GROUP + warp;
        int bad = 0;
        if (row < X.NB)
            for (int jp = lane; jp < X.nnzb[row]; jp += 32)
            {
                const int jb = X.indexb[(size_t) row * X.MB + jp];
                if (jb < 0 || jb >= X.NB)
                    bad = 1;
                else
                    atomicOr(&jbits[jb >> 5], 1u << (jb & 31));
            }
        __syncthreads();
        long long pairs = 0, nj = 0, nk = 0;
        // warp-strided words of the J bitmap; each set bit's row is walked
        // by the whole warp
        for (int w0 = warp * 32; w0 < nwords; w0 += TC_THREADS)
        {
            const int w = w0 + lane;
            unsigned b = w < nwords ? jbits[w] : 0u;
            nj += __popc(b);
            for (;;)
            {
                const unsigned live = __ballot_sync(FULL, b != 0u);
                if (!live)
                    break;
                const int src = __ffs(live) - 1;
                const unsigned bsrc = __shfl_sync(FULL, b, src);
                const int jb = ((w0 + src) << 5) + __ffs(bsrc) - 1;
                if (lane == src)
                    b &= b - 1;
                const int n = X.nnzb[jb];
                if (lane == 0)
                    pairs += n;
                for (int kp = lane; kp < n; kp += 32)
                {
                    const int kb = X.indexb[(size_t) jb * X.MB + kp];
                    if (kb < 0 || kb >= X.NB)
                        bad = 1;
                    else
                        atomicOr(&kbits[kb >> 5], 1u << (kb & 31));
                }
            }
        }
        __syncthreads();
        for (int w = tid; w < nwords; w += TC_THREADS)
            nk += __popc(kbits[w]);
        for (int o = 16; o; o >>= 1)
        {
            pairs += __shfl_xor_sync(FULL, pairs, o);
            nj += __shfl_xor_sync(FULL, nj, o);
            nk += __shfl_xor_sync(FULL, nk, o);
        }
        if (lane == 0)
        {
            red[warp][0] = pairs;
            red[warp][1] = nj;
            red[warp][2] = nk;
        }
        if (__syncthreads_or(bad) && tid == 0)
            atomicExch(&flags[2], 1);
        if (tid == 0)
        {
            long long s[3] = {0, 0, 0};
            for (int w = 0; w < TC_THREADS / 32; ++w)
                for (int k = 0; k < 3; ++k)
                    s[k] += red[w][k];
            atomicMax(&flags[5], (int) s[1]);
            atomicMax(&flags[6], (int) s[2]);
            atomicMax(&flags[7], (int) min(s[0], (long long) INT_MAX));
        }
        __syncthreads();
    }
}

// Position of X[ib0+q, jb] in row ib0+q from a record's z, w (0xFFFF: none).
__device__ __forceinline__ unsigned rec_slot(const uint4 &r, int q)
{
    const unsigned v = q < 2 ? r.z : r.w;
    return (v >> ((q & 1) * 16)) & 0xFFFFu;
}

// flags: [0] row overflow, [1] widest kept row, [2] a group's tables outside
// their sizes, [3] a tensor-core wait timed out, [4] next group to claim,
// [8] max |x| of X (the split's scale)
// I8: the 8-bit slice mode (kind::i8, four INT32 level accumulators per
// tile, rowmax/colmax give the scales); otherwise the FP16 hi/lo mode.
// img: 8 KB of operand images per block slot, left half then right half.
template <typename T, class Cfg, bool I8>
__global__ void __launch_bounds__(TC_THREADS, Cfg::CTAS)
    tc_x2_kernel(TcView<T> X, TcOut<T> C, TcTab G, const unsigned char *img, const unsigned char *zimg, double thr,
                 const unsigned long long *rowmax, const unsigned long long *colmax, double *dA, double *dC,
                 int *flags)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    constexpr int TC_TILES = Cfg::TILES, TC_ABUF = Cfg::ABUF, TC_BBUF = Cfg::BBUF;
    constexpr int TUSED = TC_TILES * 32 * (I8 ? TC8_LEVELS : 1); // tensor memory columns used
    constexpr int TCOLS = TUSED <= 32 ? 32 : TUSED <= 64 ? 64 : TUSED <= 128 ? 128 : TUSED <= 256 ? 256 : 512;
    constexpr int BLK = I8 ? TC8_BLOCK_BYTES : TC16_BLOCK_BYTES; // image bytes per block slot
    static_assert(TUSED <= 512, "tensor memory holds 512 columns per SM");
    static_assert(Cfg::ABYTES >= TC_GROUP * BLK / 2 && Cfg::BBYTES >= BLK / 2, "operand buffers");
    TcSmem<Cfg> &S = *reinterpret_cast<TcSmem<Cfg> *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ngroups = (X.NB + TC_GROUP - 1) / TC_GROUP;
    {
        const size_t cb = blockIdx.x;
        G.jb += cb * G.jcap;
        G.jslot += cb * G.jcap;
        G.jmask += cb * G.jcap;
        G.jstart += cb * (G.jcap + 1);
        G.klist += cb * G.kcap;
        G.ttouch += cb * G.kcap;
        G.ptile += cb * G.pcap;
        G.list += cb * G.pcap;
        G.wstart += cb * (G.wcap + 1);
    }

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&S.tmem)),
                     "r"(TCOLS)
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
    // pipeline counters, kept alike by the producer (warp 0) and the MMA
    // issuer (warp 1): steps, right-operand slots (a running count) and
    // left operands issued so far; go: the producer's oldest step not yet
    // seen done
    unsigned gs = 0, bh = 0, ga = 0, go = 0, nwaves = 0;
    unsigned copied_a = 0; // left operands whose copies warp 0 issued

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
        rank_bits(S.su.jbits, S.su.jpre, G.jb, G.jcap, nwords, S.scratch, &S.nJ, tid, lane, warp);
        __syncthreads();
        const int nJ = S.nJ;
        if (nJ > G.jcap)
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        for (int j = tid; j < nJ; j += TC_THREADS)
            G.jslot[j] = make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
        __syncthreads();
        if (myrow < X.NB)
            for (int jp = lane; jp < X.nnzb[myrow]; jp += 32)
            {
                const int jb = X.indexb[(size_t) myrow * X.MB + jp];
                const int j = S.su.jpre[jb >> 5] + __popc(S.su.jbits[jb >> 5] & ((1u << (jb & 31)) - 1u));
                reinterpret_cast<unsigned short *>(G.jslot + j)[warp] = (unsigned short) jp;
            }
        __syncthreads();
        for (int j = tid; j < nJ; j += TC_THREADS)
        {
            const uint2 s = G.jslot[j];
            const uint4 r = make_uint4(0u, 0u, s.x, s.y);
            unsigned char m = 0;
            for (int q = 0; q < TC_GROUP; ++q)
                if (rec_slot(r, q) != 0xFFFFu)
                    m |= (unsigned char) (1u << q);
            G.jmask[j] = m;
        }
        // ---- output block columns K: a bitmap over NB, tiles by rank ----
        // (each warp takes 32 J entries at a time, their rows' lengths loaded
        // at once, then walks the rows one by one)
        int badk = 0;
        for (int j0 = warp * 32; j0 < nJ; j0 += TC_THREADS)
        {
            const int jl = j0 + lane;
            const int jbl = jl < nJ ? G.jb[jl] : 0, nl = jl < nJ ? X.nnzb[jbl] : 0;
            for (int i = 0; i < min(32, nJ - j0); ++i)
            {
                const int jb = __shfl_sync(FULL, jbl, i), n = __shfl_sync(FULL, nl, i);
                for (int kp = lane; kp < n; kp += 32)
                {
                    const int kb = X.indexb[(size_t) jb * X.MB + kp];
                    if (kb < 0 || kb >= X.NB)
                        badk = 1;
                    else
                        atomicOr(&S.su.kbits[kb >> 5], 1u << (kb & 31));
                }
            }
        }
        if (__syncthreads_or(badk))
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        rank_bits(S.su.kbits, S.su.kpre, G.klist, G.kcap, nwords, S.scratch, &S.nK, tid, lane, warp);
        if (warp == 0)
        {
            // first pair of every J entry: pairs in (j, kp) order
            int run = 0;
            for (int j0 = 0; j0 < nJ; j0 += 32)
            {
                const int j = j0 + lane;
                const int n = j < nJ ? X.nnzb[G.jb[j]] : 0;
                int incl = n;
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o)
                        incl += y;
                }
                if (j < nJ)
                    G.jstart[j] = run + incl - n;
                run += __shfl_sync(FULL, incl, 31);
            }
            if (lane == 0)
            {
                G.jstart[nJ] = run;
                S.npairs = run;
            }
        }
        __syncthreads();
        const int nK = S.nK, npairs = S.npairs;
        const int nW = (nK + TC_TILES - 1) / TC_TILES;
        if (nK > G.kcap || npairs > G.pcap || nW > G.wcap || nW > 4 * TC_NWCAP)
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        for (int t = tid; t < nK; t += TC_THREADS)
            G.ttouch[t] = 0;
        __syncthreads();
        // the output tile of every pair (j, kp), and the rows each tile touches
        for (int j0 = warp * 32; j0 < nJ; j0 += TC_THREADS)
        {
            const int jl = j0 + lane;
            int jbl = 0, psl = 0, nl = 0, ml = 0;
            if (jl < nJ)
            {
                jbl = G.jb[jl];
                psl = G.jstart[jl];
                nl = G.jstart[jl + 1] - psl;
                ml = G.jmask[jl];
            }
            for (int i = 0; i < min(32, nJ - j0); ++i)
            {
                const int jb = __shfl_sync(FULL, jbl, i), ps = __shfl_sync(FULL, psl, i);
                const int n = __shfl_sync(FULL, nl, i), m = __shfl_sync(FULL, ml, i);
                for (int kp = lane; kp < n; kp += 32)
                {
                    const int kb = X.indexb[(size_t) jb * X.MB + kp];
                    const int t = S.su.kpre[kb >> 5] + __popc(S.su.kbits[kb >> 5] & ((1u << (kb & 31)) - 1u));
                    G.ptile[ps + kp] = t;
                    atomicOr(&G.ttouch[t], m);
                }
            }
        }
        __syncthreads();
        // ---- the pairs sorted by wave (a stable counting sort) ----
        // The J entries are cut into nq ranges of consecutive entries, one
        // per warp (nq = 4 when four rows of wave counters fit, else 1); warp
        // q places its range's pairs, in (j, kp) order, after those of the
        // earlier ranges in every wave: stable.
        const int nq = nW <= TC_NWCAP ? TC_THREADS / 32 : 1;
        int *cnt = S.wpos; // [nq][nW]: pairs per range and wave, then the next free place
        for (int w = tid; w < nq * nW; w += TC_THREADS)
            cnt[w] = 0;
        __syncthreads();
        const int jlo = (int) ((long long) nJ * warp / nq), jhi = (int) ((long long) nJ * (warp + 1) / nq);
        if (nq == 1)
        {
            for (int p = tid; p < npairs; p += TC_THREADS)
                atomicAdd(&cnt[G.ptile[p] / TC_TILES], 1);
        }
        else
        {
            const int pl = G.jstart[jlo], ph = G.jstart[jhi];
            for (int p = pl + lane; p < ph; p += 32)
                atomicAdd(&cnt[warp * nW + G.ptile[p] / TC_TILES], 1);
        }
        __syncthreads();
        if (warp == 0)
        {
            int run = 0;
            for (int w0 = 0; w0 < nW; w0 += 32)
            {
                const int w = w0 + lane;
                int n = 0;
                if (w < nW)
                    for (int q = 0; q < nq; ++q)
                        n += cnt[q * nW + w];
                int incl = n;
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o)
                        incl += y;
                }
                if (w < nW)
                {
                    int base = run + incl - n;
                    G.wstart[w] = base;
                    for (int q = 0; q < nq; ++q)
                    {
                        const int c = cnt[q * nW + w];
                        cnt[q * nW + w] = base;
                        base += c;
                    }
                }
                run += __shfl_sync(FULL, incl, 31);
            }
            if (lane == 0)
                G.wstart[nW] = run;
        }
        __syncthreads();
        if (warp < nq)
        {
            int *wpos = cnt + warp * nW;
            for (int j0 = jlo; j0 < jhi; j0 += 32)
            {
                const int jl = j0 + lane;
                int jbl = 0, psl = 0, nl = 0;
                uint2 sll = make_uint2(0u, 0u);
                if (jl < jhi)
                {
                    jbl = G.jb[jl];
                    psl = G.jstart[jl];
                    nl = G.jstart[jl + 1] - psl;
                    sll = G.jslot[jl];
                }
                for (int i = 0; i < min(32, jhi - j0); ++i)
                {
                    const int j = j0 + i;
                    const int jb = __shfl_sync(FULL, jbl, i), ps = __shfl_sync(FULL, psl, i);
                    const int n = __shfl_sync(FULL, nl, i);
                    const unsigned slx = __shfl_sync(FULL, sll.x, i), sly = __shfl_sync(FULL, sll.y, i);
                    for (int k0 = 0; k0 < n; k0 += 32)
                    {
                        const int kp = k0 + lane;
                        const int t = kp < n ? G.ptile[ps + kp] : -1;
                        const int w = t >= 0 ? t / TC_TILES : -1 - lane;
                        const unsigned peers = __match_any_sync(FULL, w);
                        const int leader = __ffs(peers) - 1;
                        int base = 0;
                        if (lane == leader && t >= 0)
                        {
                            base = wpos[w];
                            wpos[w] = base + __popc(peers);
                        }
                        base = __shfl_sync(FULL, base, leader);
                        if (t >= 0)
                        {
                            const int pos = base + __popc(peers & lanemask_lt());
                            G.list[pos] = make_uint4((unsigned) (t - w * TC_TILES) | ((unsigned) j << 4),
                                                     (unsigned) jb * (unsigned) X.MB + (unsigned) kp, slx, sly);
                        }
                    }
                }
            }
        }
        __syncthreads();
        // a step starts (a new left operand) where j changes within a wave,
        // and at every wave's first pair
        for (int p = tid; p < npairs; p += TC_THREADS)
        {
            const unsigned x = G.list[p].x;
            if (p == 0 || ((x ^ G.list[p - 1].x) & 0x000FFFF0u))
                G.list[p].x = x | 0x80000000u;
        }
        __syncthreads();
        for (int w = tid; w < nW; w += TC_THREADS)
            if (G.wstart[w] < npairs) // every wave has a pair: each tile is some pair's
                G.list[G.wstart[w]].x |= 0x80000000u;
        __syncthreads();
        // every step's tiles, into its first record (ptile is free again: the
        // sort above was its last reader); the pairs of a step have distinct
        // tiles unless a row of X repeats a block column
        int badstep = 0;
        for (int p = tid; p < npairs; p += TC_THREADS)
            if (G.list[p].x >> 31)
            {
                unsigned m = 1u << (G.list[p].x & 15u);
                int n = 1;
                for (int q = p + 1; q < npairs && !(G.list[q].x >> 31); ++q, ++n)
                    m |= 1u << (G.list[q].x & 15u);
                badstep |= __popc(m) != n;
                G.ptile[p] = (int) m;
            }
        if (__syncthreads_or(badstep))
        {
            if (tid == 0)
                atomicExch(&flags[2], 1);
            continue;
        }
        for (int p = tid; p < npairs; p += TC_THREADS)
            if (G.list[p].x >> 31)
                G.list[p].x = (G.list[p].x & 0x8000000Fu) | (unsigned) G.ptile[p] << 4;
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
        // the set-up area is the left-operand ring: order its generic
        // accesses before the bulk copies that refill it
        proxy_fence();
        __syncthreads();

        // ---- waves of TC_TILES output tiles ----
        for (int w = 0; w < nW && !dead; ++w)
        {
            const int t0 = w * TC_TILES;
            const int nt = min(TC_TILES, nK - t0);
            const int p0 = G.wstart[w], p1 = G.wstart[w + 1];
            if (warp == 0)
            {
                // producer (warp 0): 32 records per load; for each step wholly
                // inside them, the group's four blocks of column jb into the
                // next A buffer (a lane per block and part) and the step's
                // right operands into a run of free slots (a lane per pair,
                // slot = rank of its tile among the step's), each once the
                // MMAs that read the buffer's or slots' previous fill are
                // done.  Lane 0 waits and arms the barriers; the counters are
                // alike in all lanes.

                bool quit = false;
                for (int p = p0; p < p1 && !quit;)
                {
                    const int n = min(32, p1 - p);
                    const uint4 r = lane < n ? G.list[p + lane] : make_uint4(0u, 0u, 0u, 0u);
                    unsigned todo = __ballot_sync(FULL, lane < n && (r.x >> 31));
                    int used = 0;
                    while (todo)
                    {
                        const int s0 = __ffs(todo) - 1;
                        todo &= todo - 1;
                        const unsigned mask = (__shfl_sync(FULL, r.x, s0) >> 4) & 0xFFFFu;
                        const int need = __popc(mask);
                        if (s0 + need > n)
                            break; // runs past the loaded records: the next load starts here
                        const unsigned rz = __shfl_sync(FULL, r.z, s0), rw = __shfl_sync(FULL, r.w, s0);
                        const unsigned a = ga % TC_ABUF, fa = ga / TC_ABUF;
                        unsigned h = bh;
                        if (h % TC_BBUF + need > TC_BBUF)
                            h += TC_BBUF - h % TC_BBUF;
                        const unsigned e = gs % TC_BBUF;
                        int late = 0;
                        if (lane == 0)
                        {
                            if (fa >= 1 && !mbar_wait2s(&S.empty_a[a], (fa - 1) & 1))
                                late = 1;
                            // slots [h, h + need) of the ring (a running
                            // count), not across its end: free once the older
                            // steps holding them are done (and this step's
                            // barriers once their previous use is)
                            while (!late && (gs - go >= (unsigned) TC_BBUF ||
                                             (go < gs && h + need - S.sstart[go % TC_BBUF] > (unsigned) TC_BBUF)))
                            {
                                if (!mbar_wait2s(&S.empty_b[go % TC_BBUF], (go / TC_BBUF) & 1))
                                    late = 1;
                                else
                                    ++go;
                            }
                            if (late)
                                S.dead = 1;
                            else
                            {
                                S.sstart[e] = h;
                                mbar_expect(&S.full_a[a], TC_GROUP * BLK / 2);
                                mbar_expect(&S.full_b[e], need * (BLK / 2));
                            }
                        }
                        go = __shfl_sync(FULL, go, 0);
                        if (__shfl_sync(FULL, late, 0))
                        {
                            quit = true;
                            break;
                        }
                        if (lane < TC_GROUP)
                        {
                            // block q's left image (4 KB: hi and lo; or 5 KB:
                            // five slices), one copy; the four stack into the
                            // 128-row operand
                            const int q = lane;
                            const unsigned jp = ((q < 2 ? rz : rw) >> ((q & 1) * 16)) & 0xFFFFu;
                            const unsigned char *src =
                                jp != 0xFFFFu ? img + ((size_t) (ib0 + q) * X.MB + jp) * BLK : zimg;
                            bulk_copy(S.a[a] + q * (BLK / 2), src, BLK / 2, &S.full_a[a]);
                        }
                        if (lane >= s0 && lane < s0 + need)
                        {
                            // the right operand's parts are adjacent in both
                            // places: one copy
                            const unsigned rank = __popc(mask & ((1u << (r.x & 15u)) - 1u));
                            bulk_copy(S.b[h % TC_BBUF] + rank * Cfg::BBYTES, img + (size_t) r.y * BLK + BLK / 2,
                                      BLK / 2, &S.full_b[e]);
                        }
                        ++ga;
                        copied_a = ga;
                        bh = h + need;
                        ++gs;
                        used = s0 + need;
                    }
                    if (used == 0 && !quit)
                    {
                        // a step longer than 32 records: tables out of shape
                        if (lane == 0)
                        {
                            atomicExch(&flags[2], 1);
                            S.dead = 1;
                        }
                        quit = true;
                    }
                    p += used;
                }
            }
            else if (warp == 1)
            {
                // MMA issuer (warp 1; lane 0 issues): the same steps, from 32
                // records per load, consuming the rings.  A step's tiles fall
                // into runs of consecutive tiles whose slots are adjacent: one
                // MMA per run and part, N = 32 x the run's tiles.  The first
                // MMA into a tile in this wave overwrites it, so a run also
                // ends where that changes.
                unsigned started = 0, acur = 0;
                bool any = false, quit = false;
                for (int p = p0; p < p1 && !quit;)
                {
                    const int n = min(32, p1 - p);
                    const unsigned rxl = lane < n ? G.list[p + lane].x : 0u;
                    unsigned todo = __ballot_sync(FULL, lane < n && (rxl >> 31));
                    int used = 0;
                    while (todo)
                    {
                        const int s0 = __ffs(todo) - 1;
                        todo &= todo - 1;
                        const unsigned mask = (__shfl_sync(FULL, rxl, s0) >> 4) & 0xFFFFu;
                        const int need = __popc(mask);
                        if (s0 + need > n)
                            break;
                        unsigned h = bh;
                        if (h % TC_BBUF + need > TC_BBUF)
                            h += TC_BBUF - h % TC_BBUF;
                        const unsigned e = gs % TC_BBUF;
                        int late = 0;
                        if (lane == 0)
                        {
                            if (any)
                                umma_commit(&S.empty_a[acur]); // the previous left operand is done with
                            acur = ga % TC_ABUF;
                            if (!mbar_wait2s(&S.full_a[acur], (ga / TC_ABUF) & 1) ||
                                !mbar_wait2s(&S.full_b[e], (gs / TC_BBUF) & 1))
                                late = 1;
                        }
                        if (__shfl_sync(FULL, late, 0))
                        {
                            if (lane == 0)
                                S.dead = 1;
                            quit = true;
                            break;
                        }
                        if (lane == 0)
                        {
                            tc_fence_after();
                            const unsigned a0 = su32(S.a[acur]), sb0 = su32(S.b[h % TC_BBUF]);
                            unsigned m = mask;
                            while (m)
                            {
                                const int ta = __ffs(m) - 1;
                                const unsigned st = (started >> ta) & 1u;
                                const unsigned x = (m >> ta) & ((st ? started : ~started) >> ta);
                                // x's trailing ones (at least 1), at most 8
                                // tiles: an MMA takes N <= 256
                                const int len = min(__ffs(~x) - 1, 8);
                                m &= ~(((1u << len) - 1u) << ta);
                                const unsigned b0 = sb0 + (unsigned) __popc(mask & ((1u << ta) - 1u)) * Cfg::BBYTES;
                                if (I8)
                                {
                                    // slices s, t (0-based) with s + t <= 4 into
                                    // level s + t's INT32 accumulators,
                                    // [level][tile]; K = 32 per instruction
                                    const uint32_t id = TC8_IDESC | idesc_n(len);
#pragma unroll
                                    for (int sa = 0; sa < TC8_SLICES; ++sa)
#pragma unroll
                                        for (int sb = 0; sb + sa < TC8_LEVELS; ++sb)
                                            umma_i8(tbase + (unsigned) ((sa + sb) * TC_TILES * 32 + ta * 32),
                                                    smem_desc(a0 + sa * 256, TC8_LBO, TC8_RSBO),
                                                    smem_desc(b0 + sb * 256, TC8_LBO, TC8_RSBO), id,
                                                    sa == 0 ? st : 1u);
                                    continue;
                                }
                                const unsigned d = tbase + (unsigned) (ta * 32);
                                const unsigned a1 = a0 + TC_RLO;
                                const uint32_t id = TC_IDESC | idesc_n(len);
                                unsigned acc = st;
#pragma unroll
                                for (int ks = 0; ks < 2; ++ks)
                                {
                                    // K = 16: two 8-wide k-chunks per step
                                    const uint64_t ah = smem_desc(a0 + ks * 2 * TC_LBO, TC_LBO, TC_RSBO);
                                    const uint64_t al = smem_desc(a1 + ks * 2 * TC_LBO, TC_LBO, TC_RSBO);
                                    const uint64_t bh = smem_desc(b0 + ks * 2 * TC_LBO, TC_LBO, TC_RSBO);
                                    const uint64_t bl = smem_desc(b0 + TC_RLO + ks * 2 * TC_LBO, TC_LBO, TC_RSBO);
                                    umma_f16(d, ah, bh, id, acc);
                                    umma_f16(d, ah, bl, id, 1u);
                                    umma_f16(d, al, bh, id, 1u);
                                    acc = 1u;
                                }
                            }
                            umma_commit(&S.empty_b[e]);
                        }
                        __syncwarp();
                        any = true;
                        started |= mask;
                        ++ga;
                        bh = h + need;
                        ++gs;
                        used = s0 + need;
                    }
                    if (used == 0)
                        quit = true; // the producer flagged it
                    p += used;
                }
                // the wave's last left operand, then every MMA of the wave
                // (and before) done -> done barrier
                if (lane == 0)
                {
                    if (any)
                        umma_commit(&S.empty_a[acur]);
                    umma_commit(&S.done);
                }
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
            if (I8)
            {
                const double srow = myrow < X.NB ? ldexp(1.0, tc8_exp(rowmax[(size_t) myrow * TB + lane]) - 12) : 0.0;
                for (int t = 0; t < nt; ++t)
                {
                    // a row without products in the tile skips it (the warp
                    // reads only its own row's lanes of tensor memory)
                    const int kb = G.klist[t0 + t];
                    if (myrow >= X.NB || !((G.ttouch[t0 + t] >> warp) & 1))
                        continue;
                    // the five levels, highest first: v = (((D6 2^-7 + D5) 2^-7 + D4) 2^-7 + D3) 2^-7 + D2
                    double v[32];
                    for (int lev = TC8_LEVELS - 1; lev >= 0; --lev)
                    {
                        float w[32];
                        tmem_ld32(tbase + ((unsigned) (warp * 32) << 16) + (unsigned) (lev * TC_TILES * 32 + t * 32),
                                  w);
#pragma unroll
                        for (int c = 0; c < 32; ++c)
                            v[c] = (lev == TC8_LEVELS - 1 ? 0.0 : v[c] * 0x1p-7) + (double) __float_as_int(w[c]);
                    }
                    // the power of two of scalar column c, from lane c
                    const double cs = ldexp(1.0, tc8_exp(colmax[(size_t) kb * TB + lane]));
                    double mx = 0.0, diag = 0.0;
#pragma unroll
                    for (int c = 0; c < 32; ++c)
                    {
                        v[c] *= srow * __shfl_sync(FULL, cs, c);
                        mx = fmax(mx, fabs(v[c]));
                        diag = c == lane ? v[c] : diag;
                    }
                    for (int o = 16; o; o >>= 1)
                        mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
                    const bool keep = kb == myrow || mx > thr;
                    if (!keep)
                        continue;
                    if (kb == myrow)
                    {
                        double dd = diag;
                        for (int o = 16; o; o >>= 1)
                            dd += __shfl_xor_sync(FULL, dd, o);
                        trc += dd;
                    }
                    if (kept < C.MB)
                    {
                        // lane = block row; through shared memory, 16
                        // columns at a time, so that the warp writes the
                        // row-major block in contiguous runs
                        T *dst = C.pool + ((size_t) myrow * C.MB + kept) * C.slot;
#pragma unroll
                        for (int h = 0; h < 2; ++h)
                        {
#pragma unroll
                            for (int c = 0; c < 16; ++c)
                                S.dstage[warp][lane][c] = v[h * 16 + c];
                            __syncwarp();
#pragma unroll 4
                            for (int e = lane; e < 32 * 16; e += 32)
                            {
                                const int r = e >> 4, c = e & 15;
                                dst[r * TB + h * 16 + c] = (T) S.dstage[warp][r][c];
                            }
                            __syncwarp();
                        }
                        if (lane == 0)
                            C.indexb[(size_t) myrow * C.MB + kept] = kb;
                    }
                    ++kept;
                }
            }
            for (int t = 0; t < (I8 ? 0 : nt); ++t)
            {
                const int kb = G.klist[t0 + t];
                if (myrow >= X.NB || !((G.ttouch[t0 + t] >> warp) & 1))
                    continue;
                float v[32];
                tmem_ld32(tbase + ((unsigned) (warp * 32) << 16) + (unsigned) (t * 32), v);
#pragma unroll
                for (int c = 0; c < 32; ++c)
                    v[c] *= unscale; // undo the split's 2^s on both factors
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
        for (unsigned b = 0; b < TC_BBUF && b < gs; ++b)
            mbar_wait2s(&S.full_b[(gs - 1 - b) % TC_BBUF], ((gs - 1 - b) / TC_BBUF) & 1);
        for (unsigned a = 0; a < TC_ABUF && a < copied_a; ++a)
            mbar_wait2s(&S.full_a[(copied_a - 1 - a) % TC_ABUF], ((copied_a - 1 - a) / TC_ABUF) & 1);
    }
    // release the tensor memory (after every read of it)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TCOLS)
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
    tc_split_kernel<T><<<sgrid, TC_SPLIT_WARPS * 32, 0, c->stream>>>(pool, X->d_nnzb, X->NB, X->MB, X->slot_elems,
                                                                      maxbits, img);
    return LAUNCH_OK("tc_split_kernel");
}

template <typename T> TcView<T> tc_view(const bml_matrix_ellblock_t *X)
{
    return TcView<T>{static_cast<const T *>(X->d_pool), X->d_indexb, X->d_nnzb, X->NB, X->MB, X->slot_elems};
}

template <typename T>
bool tc8_split(B200Context *c, const bml_matrix_ellblock_t *X, int sgrid, unsigned long long *rowmax,
               unsigned long long *colmax, signed char *img)
{
    const T *pool = static_cast<const T *>(X->d_pool);
    tc8_max_kernel<T><<<sgrid, 256, 0, c->stream>>>(pool, X->d_indexb, X->d_nnzb, X->NB, X->MB, X->slot_elems, rowmax,
                                                   colmax);
    if (!LAUNCH_OK("tc8_max_kernel"))
        return false;
    tc8_split_kernel<T><<<sgrid, TC8_SPLIT_WARPS * 32, 0, c->stream>>>(pool, X->d_indexb, X->d_nnzb, X->NB, X->MB,
                                                                        X->slot_elems, rowmax, colmax, img);
    return LAUNCH_OK("tc8_split_kernel");
}

// The 8-bit mode's shape: 3 tiles of five 32-column level accumulators
// (480 of the 512 TMEM columns), one CTA per SM, so the rings take most of
// the SM's shared memory: 5 left buffers and 18 right slots of five slices.
#ifndef B200_TC8_ABUF
#define B200_TC8_ABUF 5
#endif
#ifndef B200_TC8_BBUF
#define B200_TC8_BBUF 18
#endif
using TcShape8 = TcCfg<3, 1, B200_TC8_ABUF, B200_TC8_BBUF, TC_GROUP * TC8_SLICES * TC8_IMG, TC8_SLICES * TC8_IMG>;

template <typename T, class Cfg, bool I8>
bool tc_launch(B200Context *c, const bml_matrix_ellblock_t *X, bml_matrix_ellblock_t *X2, const TcTab &tab,
               const unsigned char *img, const unsigned char *zimg, double threshold, const unsigned long long *rowmax,
               const unsigned long long *colmax, double *dA, double *dC, int *flags, int grid)
{
    // a one-CTA shape holds all of the SM's tensor memory: ask for enough
    // shared memory that a second CTA cannot share the SM
    const size_t smem = std::max(sizeof(TcSmem<Cfg>) + 1024, Cfg::CTAS == 1 ? size_t(120) << 10 : size_t(0));
    auto k = tc_x2_kernel<T, Cfg, I8>;
    if (!CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem)))
        return false;
    k<<<grid, TC_THREADS, smem, c->stream>>>(
        tc_view<T>(X), TcOut<T>{static_cast<T *>(X2->d_pool), X2->d_indexb, X2->d_nnzb, X2->MB, X2->slot_elems}, tab,
        img, zimg, threshold, rowmax, colmax, dA, dC, flags);
    return LAUNCH_OK("tc_x2_kernel");
}

// The split of the tensor-core X^2: 0 FP16 hi/lo with FP32 accumulation, 1
// 8-bit slices with exact INT32 accumulation.
static int g_tc_split = 0;

// Bytes of device memory the tables of one X^2 may take (all CTAs).
constexpr size_t TC_TABLE_BUDGET = size_t(16) << 30;

// X2 = X*X on the tensor cores, in the split g_tc_split selects (FP16 hi/lo
// with FP32 accumulation, or 8-bit slices with INT32 accumulation); X and X2
// must have blocks of 32 throughout.  Returns false with a status set
// (UNSUPPORTED when the partition is outside this path, or the group tables
// would exceed TC_TABLE_BUDGET; in the 8-bit split also NB > 32768, or a
// group with more than TC8_MAX_COLS block columns, whose level sums could
// pass 2^31).
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
    const bool dbl = X->matrix_precision == double_real;
    int *flags = reinterpret_cast<int *>(static_cast<unsigned char *>(c->d_small) + 32768);
    unsigned *maxbits = reinterpret_cast<unsigned *>(flags + 8); // max |x| of X, for the split's scale
    unsigned char *pin = static_cast<unsigned char *>(c->pinned) + 8192;
    // sizes of the group tables
    const int ngroups = (NB + TC_GROUP - 1) / TC_GROUP;
    if (!CUDA_OK(cudaMemsetAsync(flags, 0, 64, c->stream)))
        return false;
    const int cgrid = std::min(ngroups, c->sm_count * 8);
    if (dbl)
        tc_count_kernel<double><<<cgrid, TC_THREADS, 0, c->stream>>>(tc_view<double>(X), flags);
    else
        tc_count_kernel<float><<<cgrid, TC_THREADS, 0, c->stream>>>(tc_view<float>(X), flags);
    if (!LAUNCH_OK("tc_count_kernel"))
        return false;
    int hf[8];
    if (!CUDA_OK(cudaMemcpyAsync(pin, flags, sizeof(hf), cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    memcpy(hf, pin, sizeof(hf));
    if (hf[2])
    {
        b200_set_error(BML_B200_ERR_INVALID, "multiply_x2_tc: a block column outside 0..NB-1");
        return false;
    }
    const bool i8 = g_tc_split == 1;
    if (i8 && (NB > 4 * TC_NWCAP * TcShape8::TILES || hf[5] > TC8_MAX_COLS))
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED,
                       "multiply_x2_tc: the 8-bit split takes NB <= %d and groups of <= %d block columns",
                       4 * TC_NWCAP * TcShape8::TILES, TC8_MAX_COLS);
        return false;
    }
    const int tiles = i8 ? TcShape8::TILES : TcShape::TILES;
    const int grid = c->sm_count * (i8 ? TcShape8::CTAS : TcShape::CTAS);
    TcTab tab{};
    tab.jcap = std::max(hf[5], 1);
    tab.kcap = std::max(hf[6], 1);
    tab.pcap = std::max(hf[7], 1);
    tab.wcap = (tab.kcap + tiles - 1) / tiles;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t J = tab.jcap, K = tab.kcap, P = tab.pcap, W = tab.wcap, g = grid;
    const size_t sz[9] = {g * J * 4, g * J * 8, g * J, g * (J + 1) * 4, g * K * 4, g * K * 4,
                          g * P * 4, g * P * 16, g * (W + 1) * 4};
    size_t tab_bytes = 0;
    for (size_t s : sz)
        tab_bytes += al(s);
    if (hf[7] == INT_MAX || tab_bytes > TC_TABLE_BUDGET)
    {
        b200_set_error(BML_B200_ERR_UNSUPPORTED, "multiply_x2_tc: group tables of %zu bytes above the budget",
                       tab_bytes);
        return false;
    }
    // 8 KB (FP16) or 10 KB (8-bit) of images per block slot, the traces, a zero
    // image, the 8-bit split's row and column maxima, the tables
    const size_t n_img = (size_t) NB * MB * (i8 ? TC8_BLOCK_BYTES : TC16_BLOCK_BYTES);
    const size_t off_tr = al(n_img);
    const size_t off_zero = al(off_tr + (size_t) 2 * NB * sizeof(double));
    const size_t off_max = al(off_zero + TC_ZERO_BYTES);
    const size_t n_scalar = (size_t) NB * TB;
    const size_t off_tab = al(off_max + (i8 ? 2 * n_scalar * sizeof(unsigned long long) : 0));
    unsigned char *scr = static_cast<unsigned char *>(b200_scratch(off_tab + tab_bytes));
    if (!scr)
        return false;
    unsigned char *img = scr;
    double *dA = reinterpret_cast<double *>(scr + off_tr);
    double *dC = dA + NB;
    unsigned char *zimg = scr + off_zero;
    unsigned long long *rowmax = i8 ? reinterpret_cast<unsigned long long *>(scr + off_max) : nullptr;
    unsigned long long *colmax = i8 ? rowmax + n_scalar : nullptr;
    {
        unsigned char *p = scr + off_tab;
        auto take = [&](int i) {
            unsigned char *q = p;
            p += al(sz[i]);
            return q;
        };
        tab.jb = reinterpret_cast<int *>(take(0));
        tab.jslot = reinterpret_cast<uint2 *>(take(1));
        tab.jmask = take(2);
        tab.jstart = reinterpret_cast<int *>(take(3));
        tab.klist = reinterpret_cast<int *>(take(4));
        tab.ttouch = reinterpret_cast<int *>(take(5));
        tab.ptile = reinterpret_cast<int *>(take(6));
        tab.list = reinterpret_cast<uint4 *>(take(7));
        tab.wstart = reinterpret_cast<int *>(take(8));
    }
    if (!CUDA_OK(cudaMemsetAsync(flags, 0, 64, c->stream)) ||
        !CUDA_OK(cudaMemsetAsync(zimg, 0, TC_ZERO_BYTES, c->stream)) ||
        !CUDA_OK(cudaMemsetAsync(dA, 0, (size_t) 2 * NB * sizeof(double), c->stream)) ||
        (i8 && !CUDA_OK(cudaMemsetAsync(rowmax, 0, 2 * n_scalar * sizeof(unsigned long long), c->stream))))
        return false;
    const int sgrid = (int) std::min((long long) NB * MB, (long long) c->sm_count * 32);
    bool ok;
    if (i8)
    {
        signed char *img8 = reinterpret_cast<signed char *>(img);
        ok = dbl ? tc8_split<double>(c, X, sgrid, rowmax, colmax, img8)
                 : tc8_split<float>(c, X, sgrid, rowmax, colmax, img8);
        if (ok)
            ok = dbl ? tc_launch<double, TcShape8, true>(c, X, X2, tab, img, zimg, threshold, rowmax, colmax, dA, dC,
                                                         flags, grid)
                     : tc_launch<float, TcShape8, true>(c, X, X2, tab, img, zimg, threshold, rowmax, colmax, dA, dC,
                                                        flags, grid);
    }
    else
    {
        tc_t *img16 = reinterpret_cast<tc_t *>(img);
        ok = dbl ? tc_split<double>(c, X, sgrid, maxbits, img16) : tc_split<float>(c, X, sgrid, maxbits, img16);
        if (ok)
            ok = dbl ? tc_launch<double, TcShape, false>(c, X, X2, tab, img, zimg, threshold, nullptr, nullptr, dA,
                                                          dC, flags, grid)
                     : tc_launch<float, TcShape, false>(c, X, X2, tab, img, zimg, threshold, nullptr, nullptr, dA, dC,
                                                         flags, grid);
    }
    if (!ok)
        return false;
    double *out = reinterpret_cast<double *>(static_cast<unsigned char *>(c->d_small) + 4096 + 256);
    b200_sum_rows_kernel<<<1, 1024, 0, c->stream>>>(dA, dC, NB, out);
    if (!LAUNCH_OK("b200_sum_rows_kernel"))
        return false;
    if (!CUDA_OK(cudaMemcpyAsync(pin, flags, 16, cudaMemcpyDeviceToHost, c->stream)) ||
        !CUDA_OK(cudaMemcpyAsync(pin + 64, out, 16, cudaMemcpyDeviceToHost, c->stream)) || !b200_sync())
        return false;
    memcpy(hf, pin, 4 * sizeof(int));
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
        b200_set_error(BML_B200_ERR_INVALID, "multiply_x2_tc: a group's tables differ from their counted sizes");
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
extern "C" int bml_b200_set_tc_split(int mode)
{
    const int old = g_tc_split;
    g_tc_split = mode == 1 ? 1 : 0;
    return old;
}

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
            // Blocks other than 32 x 32, or a partition beyond the
            // tensor-core kernel's limits, are an expected outcome here: that
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
                                    "product (outside the tensor-core kernel's limits)\n", it);
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
