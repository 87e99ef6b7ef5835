// Block SpMM on the tensor cores (tcgen05 kind::f16, FP32 accumulation),
// sm_100a.
//
// Y[M][b] = A[M][K] X[K][b] for a sparse FP32 A whose rows are cut into
// blocks of 128 consecutive rows.  Each block keeps the sorted union of its
// rows' column indices (padded to a multiple of 16 with copies of its last
// column, zero-valued) and its values as a dense 128 x union matrix, zero
// where a row lacks a column.  A block is one M = 128 tile: its union
// columns are the K dimension, the b = 128 or 256 probes the N dimension, so
// every gathered row of X feeds 128 rows of products on the tensor core.
// Fill (nonzeros over 128 x union) decides the cost: blocks made of rows
// with overlapping neighbourhoods (slq_block_order) matter.
//
// FP32 accuracy from FP16 operands: each operand is split into two FP16
// parts, hi = rn_f16(v) and lo = rn_f16(v - hi) (22 significant bits
// together), after a power-of-two scaling that keeps the parts in FP16's
// range: row r of A by 2^f_r (its largest |a| to [2^13, 2^14)), probe p of X
// by 2^e_p (its norm 1 / s_p, or its largest |x| when no norm is known, to
// at most 2^14, so every element fits).  Three products per K step, A_lo
// X_hi + A_hi X_lo + A_hi X_hi, accumulate in FP32 in tensor memory; the
// dropped lo x lo term and the rounding of the lo parts leave about 2^-22
// relative error per product.  The epilogue multiplies by 2^-f_r 2^-e_p s_p
// (exact powers of two times s_p).  The tensor core's FP32 accumulation
// truncates; over the ~40 K steps of a block that shrinks |y| by about 1e-6
// relative.
//
// Format (built on the device by k_blk_* below):
//   bstage[nblk + 1]   first 16-column stage of each block (exclusive sum)
//   ucol[16 * stages]  union column indices, stage by stage
//   rsc[nblk * 128]    2^-f_r per stored row (1 for the padding rows)
//   img[stages][2][2048]  FP16 parts (hi then lo) of each stage's scaled
//                      values, 128 rows x 16 columns in the K-major
//                      no-swizzle layout the MMA reads: element (r, k) at
//                      half offset (r % 8) * 8 + (r / 8) * 128 + (k / 8) * 64
//                      + (k % 8) (core matrices of 8 rows x 8 values; leading
//                      byte offset 128 between the two K core matrices,
//                      stride byte offset 256 between 8-row groups)
// so one stage of A is one contiguous 8 KB bulk copy.
//
// Kernel k_spmm_blk (persistent, one CTA per SM; CTA c takes slots c, c +
// grid, ... of the format's slot order, which keeps every wave of grid slots
// to one run of consecutive blocks -- the X rows they gather stay in L2 --
// and balances the CTAs' stage counts within each wave):
//   warp 8        producer: per stage, one cp.async.bulk of the A parts;
//   warps 10-17   converters: load the stage's 16 X rows from global memory
//                 (two stages ahead, into registers), scale and split them
//                 into FP16 parts and store both in the MN-major 128-byte
//                 swizzled layout (atoms of 8 K rows x 64 probes);
//                 with X already split (PRE: the probe block scaled and split
//                 into X16[row] = hi[b] | lo[b] by k_x16_split, once per
//                 Lanczos step) the same warps only copy the rows' 16-byte
//                 chunks into that layout (no arithmetic, half the stores).
//                 TMA gathers of the rows (tile::gather4, four 128-byte box
//                 rows each under the 128-byte swizzle) measured two times
//                 slower than these loads;
//   warp 9        MMA issuer: per stage (K = 16) the three products into an
//                 FP32 accumulator in tensor memory (lane = block row,
//                 column = probe), two accumulators so the epilogue of one
//                 block overlaps the products of the next;
//   warps 0-7     epilogue: the SpMM epilogue of the other kernels (probe
//                 scales, affine shift, three-term subtraction, partial sums
//                 of alpha or |y|^2) on the finished accumulator; its
//                 element arithmetic is FP32 (y rounded once more than the
//                 FP64 form, the terms x y, y y, z y one rounding each), the
//                 sums over a warp's 32 rows FP32 and all further sums FP64,
//                 the per-probe factor applied to the sums.
// Every mbarrier wait is bounded; a wait that runs out sets the error word
// and the CTA drains its copies and MMAs before it leaves.  No multicast: the
// only TMA copies read this GPU's own format buffer.

#ifndef SLQ_BLK_CUH_
#define SLQ_BLK_CUH_

#include <cuda_fp16.h>

#include "slq_kernels.cuh"

namespace slq {

constexpr int BLK_ROWS = 128;
constexpr int BLK_BK = 16;            // union columns per stage (one K step)
// Stages in the ring.  Fewer stages leave more of the SM's shared-memory /
// L1 storage to the L1 cache, which the epilogue's loads use: a thread
// reads 64 of the 128 bytes of a row's X line in one pass and the other 64
// in the next, so the line must survive in L1 in between.  Measured per
// product at b = 256: eight stages 7 % slower than six, seven 1 %, five
// the same, four 2 % slower.
constexpr int BLK_STAGES = 6;
constexpr int BLK_A_PART = BLK_ROWS * BLK_BK * 2;     // 4 KB per FP16 part
constexpr int BLK_IMG_STAGE = 2 * BLK_ROWS * BLK_BK;  // halves per stage image
constexpr int BLK_EPI_WARPS = 8;
constexpr int BLK_PRODUCER = 8;       // warp indices
constexpr int BLK_MMA = 9;
constexpr int BLK_CONV0 = 10;
constexpr int BLK_CONV_WARPS = 8;
constexpr int BLK_THREADS = (BLK_CONV0 + BLK_CONV_WARPS) * 32;  // 576
constexpr int BLK_TAIL = 512;         // barriers, tensor-memory address, flags

__host__ __device__ constexpr uint32_t blk_x_part(int nb)
{
    return static_cast<uint32_t>(nb) * BLK_BK * 2u;   // one FP16 part of X
}

__host__ __device__ constexpr uint32_t blk_stage_bytes(int nb)
{
    return 2u * BLK_A_PART + 2u * blk_x_part(nb);
}

// stages, barriers, partial sums [4][256] (doubles), the per-probe
// constants [4][256] (floats)
__host__ __device__ constexpr size_t blk_smem_bytes(int nb)
{
    return 1023 + static_cast<size_t>(BLK_STAGES) * blk_stage_bytes(nb) + BLK_TAIL +
           4 * 256 * sizeof(double) + 4 * 256 * sizeof(float);
}

// ---------------------------------------------------------------------------
// format build
// ---------------------------------------------------------------------------

// keys[e] = (block of row << cbits) | column, pos[e] = e, rr[e] = row % 128
// (one warp per row)
__global__ void k_blk_keys(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ind,
                           int64_t rows, int cbits, uint64_t* __restrict__ keys,
                           int32_t* __restrict__ pos, uint8_t* __restrict__ rr)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t row = w0; row < rows; row += nw)
    {
        const uint64_t hi = static_cast<uint64_t>(row >> 7) << cbits;
        for (int64_t e = ptr[row] + lane; e < ptr[row + 1]; e += 32)
        {
            keys[e] = hi | static_cast<uint32_t>(ind[e]);
            pos[e] = static_cast<int32_t>(e);
            rr[e] = static_cast<uint8_t>(row & 127);
        }
    }
}

// Block unions by bitmap.  A block's rows are consecutive CSR rows, so its
// entries are one range of the index array; its union columns are the set
// bits of a bitmap over its column range [lo, hi] in shared memory, in
// increasing column order: the order the sorted (block, column) keys give,
// so both ways build the same format.  A block whose columns span more than
// BLK_UNION_SPAN sets *wide and the build takes the sorted-key path.  One
// CTA of BLK_UNION_THREADS threads per block.
constexpr int BLK_UNION_WORDS = 8192;  // 32 KB of bits: spans of up to 262,144 columns
constexpr int64_t BLK_UNION_SPAN = int64_t(BLK_UNION_WORDS) * 32;
constexpr int BLK_UNION_THREADS = 256;
constexpr int BLK_UNION_GROUPS = BLK_UNION_WORDS / 8;  // prefix counts per 8 words

struct BlkUnionSmem {
    uint32_t bits[BLK_UNION_WORDS];
    int32_t pre8[BLK_UNION_GROUPS];  // set bits in words [0, 8 g)
    int32_t red[2 * (BLK_UNION_THREADS / 32) + 2];
};

// the block's smallest and largest column (hi = -1 for an empty block);
// every thread of the CTA receives both
__device__ __forceinline__ void blk_col_range(const int32_t* __restrict__ ind, int64_t e0,
                                              int64_t e1, BlkUnionSmem& sm, int32_t& lo,
                                              int32_t& hi)
{
    constexpr int NW = BLK_UNION_THREADS / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t l = INT_MAX, h = -1;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += BLK_UNION_THREADS)
    {
        const int32_t c = ind[e];
        l = min(l, c);
        h = max(h, c);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        l = min(l, __shfl_xor_sync(FULL_MASK, l, off));
        h = max(h, __shfl_xor_sync(FULL_MASK, h, off));
    }
    if (lane == 0)
    {
        sm.red[w] = l;
        sm.red[NW + w] = h;
    }
    __syncthreads();
    if (w == 0)
    {
        l = lane < NW ? sm.red[lane] : INT_MAX;
        h = lane < NW ? sm.red[NW + lane] : -1;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            l = min(l, __shfl_xor_sync(FULL_MASK, l, off));
            h = max(h, __shfl_xor_sync(FULL_MASK, h, off));
        }
        if (lane == 0)
        {
            sm.red[2 * NW] = l;
            sm.red[2 * NW + 1] = h;
        }
    }
    __syncthreads();
    lo = sm.red[2 * NW];
    hi = sm.red[2 * NW + 1];
    __syncthreads();  // red is written again by the caller
}

// the block's bitmap over `words` words from column lo
__device__ __forceinline__ void blk_bitmap(const int32_t* __restrict__ ind, int64_t e0, int64_t e1,
                                           int32_t lo, int words, BlkUnionSmem& sm)
{
    for (int w = threadIdx.x; w < words; w += BLK_UNION_THREADS) sm.bits[w] = 0u;
    __syncthreads();
    for (int64_t e = e0 + threadIdx.x; e < e1; e += BLK_UNION_THREADS)
    {
        const uint32_t off = static_cast<uint32_t>(ind[e] - lo);
        atomicOr(&sm.bits[off >> 5], 1u << (off & 31));
    }
    __syncthreads();
}

// cnt[b] = union size of block b; *wide = 1 if a block spans too many
// columns (cnt is then rebuilt by the sorted-key path)
__global__ void __launch_bounds__(BLK_UNION_THREADS)
    k_blk_ucount(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ind, int64_t rows,
                 int64_t nblk, int32_t* __restrict__ cnt, int32_t* __restrict__ wide)
{
    __shared__ BlkUnionSmem sm;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const int64_t r0 = b * BLK_ROWS, r1 = min(rows, r0 + BLK_ROWS);
        const int64_t e0 = ptr[r0], e1 = ptr[r1];
        int32_t lo, hi;
        blk_col_range(ind, e0, e1, sm, lo, hi);
        const int64_t span = hi < 0 ? 0 : int64_t(hi) - lo + 1;  // the same in every thread
        if (span == 0 || span > BLK_UNION_SPAN)
        {
            if (threadIdx.x == 0)
            {
                cnt[b] = 0;
                if (span > BLK_UNION_SPAN) atomicOr(wide, 1);
            }
            continue;
        }
        const int words = static_cast<int>((span + 31) >> 5);
        blk_bitmap(ind, e0, e1, lo, words, sm);
        int32_t c = 0;
        for (int k = threadIdx.x; k < words; k += BLK_UNION_THREADS) c += __popc(sm.bits[k]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(FULL_MASK, c, off);
        if (lane == 0) sm.red[w] = c;
        __syncthreads();
        if (threadIdx.x == 0)
        {
            int32_t t = 0;
            for (int k = 0; k < BLK_UNION_THREADS / 32; ++k) t += sm.red[k];
            cnt[b] = t;
        }
        __syncthreads();
    }
}

// union index of the column at offset `off` from lo (bits and pre8 built)
__device__ __forceinline__ int32_t blk_union_index(const BlkUnionSmem& sm, uint32_t off)
{
    const int wd = static_cast<int>(off >> 5);
    int32_t u = sm.pre8[wd >> 3];
    for (int k = wd & ~7; k < wd; ++k) u += __popc(sm.bits[k]);
    return u + __popc(sm.bits[wd] & ((1u << (off & 31)) - 1u));
}

// Per block (spans checked by k_blk_ucount): its union columns into ucol
// from stage bstage[b], the last stage padded with copies of the largest
// union column (0 for an empty block), and its values into the zeroed FP32
// staging images tmp[stage][128][16] (atomic adds only sum duplicate
// (row, column) entries).  One warp per row for the values.
__global__ void __launch_bounds__(BLK_UNION_THREADS)
    k_blk_ufill(const int32_t* __restrict__ ptr, const int32_t* __restrict__ ind,
                const float* __restrict__ vals, int64_t rows, int64_t nblk,
                const int32_t* __restrict__ bstage, int32_t* __restrict__ ucol,
                float* __restrict__ tmp)
{
    __shared__ BlkUnionSmem sm;
    constexpr int NW = BLK_UNION_THREADS / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x)
    {
        const int64_t r0 = b * BLK_ROWS, r1 = min(rows, r0 + BLK_ROWS);
        const int64_t e0 = ptr[r0], e1 = ptr[r1];
        const int64_t base = static_cast<int64_t>(bstage[b]) * BLK_BK;
        const int64_t end = static_cast<int64_t>(bstage[b + 1]) * BLK_BK;
        int32_t lo, hi;
        blk_col_range(ind, e0, e1, sm, lo, hi);
        if (hi < 0)
        {
            for (int64_t j = base + threadIdx.x; j < end; j += BLK_UNION_THREADS) ucol[j] = 0;
            continue;
        }
        const int64_t span = int64_t(hi) - lo + 1;
        if (span > BLK_UNION_SPAN) continue;  // k_blk_ucount flagged it: not this path
        const int words = static_cast<int>((span + 31) >> 5);
        blk_bitmap(ind, e0, e1, lo, words, sm);
        // prefix counts per 8 words: each thread sums whole groups, then one
        // exclusive scan over the threads' totals
        const int groups = (words + 7) >> 3;
        const int per = (groups + BLK_UNION_THREADS - 1) / BLK_UNION_THREADS;
        const int g0 = min(groups, static_cast<int>(threadIdx.x) * per);
        const int g1 = min(groups, g0 + per);
        int32_t t = 0;
        for (int g = g0; g < g1; ++g)
        {
            int32_t s8 = 0;
            for (int k = g * 8; k < min(words, g * 8 + 8); ++k) s8 += __popc(sm.bits[k]);
            sm.pre8[g] = s8;  // group total for now
            t += s8;
        }
        int32_t incl = t;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
        {
            const int32_t v = __shfl_up_sync(FULL_MASK, incl, off);
            if (lane >= off) incl += v;
        }
        if (lane == 31) sm.red[w] = incl;
        __syncthreads();
        int32_t before = incl - t;
        for (int k = 0; k < w; ++k) before += sm.red[k];
        for (int g = g0; g < g1; ++g)
        {
            const int32_t s8 = sm.pre8[g];
            sm.pre8[g] = before;
            before += s8;
        }
        __syncthreads();
        int32_t total = 0;  // the block's union size
        for (int k = 0; k < NW; ++k) total += sm.red[k];
        // union columns in increasing order, then the last stage's padding
        for (int k = threadIdx.x; k < words; k += BLK_UNION_THREADS)
        {
            uint32_t m = sm.bits[k];
            if (!m) continue;
            int32_t u = blk_union_index(sm, static_cast<uint32_t>(k) << 5);
            while (m)
            {
                const int bit = __ffs(m) - 1;
                ucol[base + u++] = lo + k * 32 + bit;
                m &= m - 1u;
            }
        }
        for (int64_t j = base + total + threadIdx.x; j < end; j += BLK_UNION_THREADS) ucol[j] = hi;
        // values
        for (int64_t row = r0 + w; row < r1; row += NW)
        {
            const int rr = static_cast<int>(row & (BLK_ROWS - 1));
            for (int64_t e = ptr[row] + lane; e < ptr[row + 1]; e += 32)
            {
                const int32_t u = blk_union_index(sm, static_cast<uint32_t>(ind[e] - lo));
                const int64_t stage = bstage[b] + u / BLK_BK;
                atomicAdd(&tmp[(stage * BLK_ROWS + rr) * BLK_BK + u % BLK_BK], vals[e]);
            }
        }
        __syncthreads();
    }
}

// flags[i] = 1 where sorted key i starts a new (block, column) pair
__global__ void k_blk_flags(const uint64_t* __restrict__ keys, int64_t nnz,
                            int32_t* __restrict__ flags)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// cnt[block] = union size (atomic counts of the flagged keys: the totals do
// not depend on the order of the additions)
__global__ void k_blk_count(const uint64_t* __restrict__ keys, const int32_t* __restrict__ flags,
                            int64_t nnz, int cbits, int32_t* __restrict__ cnt)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (flags[i]) atomicAdd(&cnt[keys[i] >> cbits], 1);
}

// stg[block] = stages of the block (an empty block keeps one zero stage)
__global__ void k_blk_stages(const int32_t* __restrict__ cnt, int64_t nblk,
                             int32_t* __restrict__ stg)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= nblk;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        stg[i] = (i == nblk) ? 0 : max(1, (cnt[i] + BLK_BK - 1) / BLK_BK);
}

// ucol entries of the unions (uidx = inclusive sum of flags)
__global__ void k_blk_ucol(const uint64_t* __restrict__ keys, const int32_t* __restrict__ flags,
                           const int32_t* __restrict__ uidx, int64_t nnz, int cbits,
                           const int32_t* __restrict__ ufirst, const int32_t* __restrict__ bstage,
                           int32_t* __restrict__ ucol)
{
    const uint64_t cmask = (uint64_t(1) << cbits) - 1;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        if (flags[i])
        {
            const int64_t blk = static_cast<int64_t>(keys[i] >> cbits);
            const int64_t j = uidx[i] - 1 - ufirst[blk];
            ucol[static_cast<int64_t>(bstage[blk]) * BLK_BK + j] =
                static_cast<int32_t>(keys[i] & cmask);
        }
}

// padding of each block's last stage: copies of its last union column (0
// for an empty block); their values stay zero
__global__ void k_blk_pad(const int32_t* __restrict__ cnt, const int32_t* __restrict__ bstage,
                          int64_t nblk, int32_t* __restrict__ ucol)
{
    for (int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < nblk;
         b += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int64_t base = static_cast<int64_t>(bstage[b]) * BLK_BK;
        const int64_t end = static_cast<int64_t>(bstage[b + 1]) * BLK_BK;
        const int32_t fill = cnt[b] > 0 ? ucol[base + cnt[b] - 1] : 0;
        for (int64_t j = base + cnt[b]; j < end; ++j) ucol[j] = fill;
    }
}

// Row scales: fsc[r] = 2^f_r with the row's largest |a| scaled into
// [2^13, 2^14) (f_r = 0 for an empty or all-zero row), rsc[r] = 2^-f_r;
// rows past `rows` (the last block's padding) get 1.  One warp per row.
__global__ void k_blk_rowscale(const int32_t* __restrict__ ptr, const float* __restrict__ val,
                               int64_t rows, int64_t padded, float* __restrict__ fsc,
                               float* __restrict__ rsc)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t row = w0; row < padded; row += nw)
    {
        float mx = 0.0f;
        if (row < rows)
            for (int64_t e = ptr[row] + lane; e < ptr[row + 1]; e += 32)
                mx = fmaxf(mx, fabsf(val[e]));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL_MASK, mx, off));
        if (lane == 0)
        {
            int f = 0;
            if (mx > 0.0f && isfinite(mx))
            {
                int ex = 0;
                frexpf(mx, &ex);  // mx = m 2^ex, m in [0.5, 1)
                f = min(max(14 - ex, -120), 120);
            }
            fsc[row] = ldexpf(1.0f, f);
            rsc[row] = ldexpf(1.0f, -f);
        }
    }
}

// values into FP32 staging images, tmp[stage][128][16] (zeroed first; the
// same 8 KB per stage that the FP16 parts take afterwards); atomic adds only
// sum duplicate (row, column) entries, each slot otherwise receives one
// value
__global__ void k_blk_scatter(const uint64_t* __restrict__ keys, const int32_t* __restrict__ pos,
                              const int32_t* __restrict__ uidx, int64_t nnz, int cbits,
                              const int32_t* __restrict__ ufirst,
                              const int32_t* __restrict__ bstage, const float* __restrict__ vals,
                              const uint8_t* __restrict__ rr, float* __restrict__ tmp)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int64_t blk = static_cast<int64_t>(keys[i] >> cbits);
        const int64_t j = uidx[i] - 1 - ufirst[blk];
        const int32_t e = pos[i];
        const int64_t stage = bstage[blk] + j / BLK_BK;
        atomicAdd(&tmp[(stage * BLK_ROWS + rr[e]) * BLK_BK + j % BLK_BK], vals[e]);
    }
}

// In place, per stage (one CTA of 256 threads per stage at a time): the
// 2048 staged FP32 values of a stage become its FP16 parts, hi =
// rn_f16(a 2^f_r) and lo = rn_f16(a 2^f_r - hi), in the MMA's K-major
// layout; the stage's block comes from a binary search of bstage.
__global__ void __launch_bounds__(256)
k_blk_split(void* __restrict__ img, const int32_t* __restrict__ bstage, int64_t nblk,
            const float* __restrict__ fsc, int64_t stages)
{
    constexpr int PER = BLK_ROWS * BLK_BK / 256;  // values per thread
    for (int64_t st = blockIdx.x; st < stages; st += gridDim.x)
    {
        int64_t lo_b = 0, hi_b = nblk - 1;  // last block with bstage <= st
        while (lo_b < hi_b)
        {
            const int64_t mid = (lo_b + hi_b + 1) / 2;
            if (bstage[mid] <= st) lo_b = mid;
            else hi_b = mid - 1;
        }
        float* src = reinterpret_cast<float*>(img) + st * (BLK_ROWS * BLK_BK);
        float a[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) a[u] = src[threadIdx.x + u * 256];
        __syncthreads();
        __half* dst = reinterpret_cast<__half*>(img) + st * BLK_IMG_STAGE;
#pragma unroll
        for (int u = 0; u < PER; ++u)
        {
            const int i = threadIdx.x + u * 256;
            const int r = i / BLK_BK, k = i % BLK_BK;
            const float v = a[u] * fsc[lo_b * BLK_ROWS + r];
            const __half h = __float2half_rn(v);
            const __half l = __float2half_rn(v - __half2float(h));
            __half* o = dst + (r & 7) * 8 + (r >> 3) * 128 + (k >> 3) * 64 + (k & 7);
            o[0] = h;
            o[BLK_ROWS * BLK_BK] = l;
        }
        __syncthreads();
    }
}

// Per-probe largest |x| of an X whose norms are not known (the products
// that get no probe scale): mx[p] (zeroed first) receives the maximum as the
// bit pattern of a non-negative float, by atomicMax; non-finite values count
// as zero.  Block = 256 threads = 8 rows x 32 probes; grid.y = b / 32.
__global__ void k_blk_colmax(const float* __restrict__ X, int64_t rows, int b,
                             unsigned int* __restrict__ mx)
{
    const int q = blockIdx.y * 32 + (threadIdx.x & 31);
    float m = 0.0f;
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * 8 + (threadIdx.x >> 5); r < rows;
         r += static_cast<int64_t>(gridDim.x) * 8)
    {
        const float v = fabsf(X[r * b + q]);
        if (isfinite(v)) m = fmaxf(m, v);
    }
    atomicMax(&mx[q], __float_as_uint(m));
}

// ---------------------------------------------------------------------------
// the product
// ---------------------------------------------------------------------------

struct BlkArgs {
    int64_t M;                 // rows of Y
    int64_t nblk;              // 128-row blocks
    int NB;                    // probes = b (128 or 256)
    const int32_t* bstage;
    const int32_t* order;      // block of each slot (CTA c takes slots c, c + grid, ...)
    const int32_t* ucol;
    const float* rsc;
    const __half* img;
    const __half* x16;         // PRE: X split into FP16 parts, [K][2 NB] (hi | lo)
    const int32_t* xexp;       // PRE: its per-probe exponents (NULL: from sx)
    const float* X;
    const double* sx;          // per-probe scale s_p of X (norm 1 / s_p), or NULL
    const unsigned int* xmax;  // sx == NULL: per-probe max |x| (float bits)
    double shift;
    float* Y;
    const float* Z;
    const double* zc;
    const double* zs;
    int epi;
    double* partials;          // [grid][NB]
    int32_t* error;
};

// FP16 parts of four scaled values, packed: hi = rn_f16(v), lo =
// rn_f16(v - hi)
__device__ __forceinline__ void split_h4(float4 v, uint2& hi, uint2& lo)
{
    const __half2 h01 = __floats2half2_rn(v.x, v.y);
    const __half2 h23 = __floats2half2_rn(v.z, v.w);
    const float2 f01 = __half22float2(h01);
    const float2 f23 = __half22float2(h23);
    const __half2 l01 = __floats2half2_rn(v.x - f01.x, v.y - f01.y);
    const __half2 l23 = __floats2half2_rn(v.z - f23.x, v.w - f23.y);
    hi = make_uint2(*reinterpret_cast<const uint32_t*>(&h01),
                    *reinterpret_cast<const uint32_t*>(&h23));
    lo = make_uint2(*reinterpret_cast<const uint32_t*>(&l01),
                    *reinterpret_cast<const uint32_t*>(&l23));
}

// The power-of-two exponent e_p that scales probe p of X into FP16 range:
// with the probe's scale s_p (|x|_2 = 1 / s_p) every scaled |x| is at most
// 2^14; without a usable scale, 0.
__device__ __forceinline__ int blk_x_exp(double sxv) { return x16_exp(sxv); }

// X16[r][p] = hi, X16[r][b + p] = lo of 2^e_p X[r][p] (the FP16 parts the
// block SpMM multiplies), for rows x b probes, b a multiple of 8; thread =
// 8 probes of one row (two float4 in, one 16-byte store per part).
__global__ void k_x16_split(const float* __restrict__ X, const double* __restrict__ sx,
                            int64_t rows, int b, __half* __restrict__ X16)
{
    __shared__ float scale[1024];
    for (int p = threadIdx.x; p < b; p += blockDim.x) scale[p] = ldexpf(1.0f, blk_x_exp(sx[p]));
    __syncthreads();
    const int per_row = b >> 3;
    const int64_t total = rows * per_row;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int64_t r = i / per_row;
        const int p = static_cast<int>(i - r * per_row) * 8;
        const float4* src = reinterpret_cast<const float4*>(X + r * b + p);
        float4 a = __ldcs(src), c = __ldcs(src + 1);
        a = make_float4(a.x * scale[p], a.y * scale[p + 1], a.z * scale[p + 2], a.w * scale[p + 3]);
        c = make_float4(c.x * scale[p + 4], c.y * scale[p + 5], c.z * scale[p + 6],
                        c.w * scale[p + 7]);
        uint2 ha, la, hc, lc;
        split_h4(a, ha, la);
        split_h4(c, hc, lc);
        __half* dst = X16 + r * 2 * b + p;
        *reinterpret_cast<uint4*>(dst) = make_uint4(ha.x, ha.y, hc.x, hc.y);
        *reinterpret_cast<uint4*>(dst + b) = make_uint4(la.x, la.y, lc.x, lc.y);
    }
}

// Reduce-scatter of 16 per-lane values over the warp's 32 lanes: on return
// lanes 0-15 hold the sum over all lanes of value blk_col(lane), lanes
// 16-31 the same sums again.  16 shuffles instead of 16 x 5 for 16 separate
// tree reductions; the order of the additions is fixed.
__device__ __forceinline__ int blk_col(int lane)
{
    return 8 * (lane & 1) + 4 * ((lane >> 1) & 1) + 2 * ((lane >> 2) & 1) + ((lane >> 3) & 1);
}

__device__ __forceinline__ float reduce_scatter16(float (&a)[16], int lane)
{
#pragma unroll
    for (int st = 0; st < 4; ++st)
    {
        const int h = 8 >> st;          // values kept after this step
        const bool upper = (lane >> st) & 1;
#pragma unroll
        for (int i = 0; i < h; ++i)
        {
            const float send = upper ? a[i] : a[i + h];
            const float keep = upper ? a[i + h] : a[i];
            a[i] = keep + __shfl_xor_sync(FULL_MASK, send, 1 << st);
        }
    }
    return a[0] + __shfl_xor_sync(FULL_MASK, a[0], 16);
}

// Position in a CTA's stage sequence: its blocks blockIdx.x, + gridDim.x, ...
// and each block's stages in order.
struct BlkCursor {
    int64_t slot;  // this CTA's slots: blockIdx.x, + gridDim.x, ...
    int st, s1;
    const int32_t* order;

    __device__ void start(const int32_t* bstage, const int32_t* ord, int64_t nblk)
    {
        order = ord;
        slot = blockIdx.x;
        st = s1 = 0;
        if (slot < nblk)
        {
            const int64_t blk = order[slot];
            st = bstage[blk];
            s1 = bstage[blk + 1];
        }
    }

    __device__ void advance(const int32_t* bstage, int64_t nblk)
    {
        if (slot >= nblk) return;
        if (++st >= s1)
        {
            slot += gridDim.x;
            if (slot < nblk)
            {
                const int64_t blk = order[slot];
                st = bstage[blk];
                s1 = bstage[blk + 1];
            }
        }
    }

    // union row k of the current stage (-1 past the end)
    __device__ int row(const int32_t* ucol, int64_t nblk, int k) const
    {
        return slot < nblk ? ucol[int64_t(st) * BLK_BK + k] : -1;
    }
};

// Instruction descriptor, kind::f16 with FP16 A and B, FP32 D, M = 128, A
// K-major, B MN-major (transpose bit 16), N = nb
__host__ __device__ constexpr uint32_t blk_idesc(uint32_t nb)
{
    return (1u << 4) | (1u << 16) | ((nb >> 3) << 17) | ((128u >> 4) << 24);
}

template <int NB, bool PRE>
__global__ void __launch_bounds__(BLK_THREADS, 1)
k_spmm_blk(const BlkArgs d)
{
    constexpr int NT = BLK_THREADS;
    extern __shared__ __align__(1024) unsigned char smem_blk[];
    const uint32_t stage_bytes = blk_stage_bytes(NB);
    const uint32_t x_bytes = blk_x_part(NB);
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_blk) + 1023) & ~uintptr_t(1023));
    unsigned char* tail = base + BLK_STAGES * stage_bytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(tail);
    uint64_t* conv = full + BLK_STAGES;
    uint64_t* empty = conv + BLK_STAGES;
    uint64_t* acc_full = empty + BLK_STAGES;   // [2]
    uint64_t* acc_empty = acc_full + 2;        // [2]
    uint64_t* drain = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 2);  // [2]
    double* red = reinterpret_cast<double*>(tail + BLK_TAIL);  // [4][256]
    // per-probe constants in FP32: 2^e_p (X scaling), s_p 2^-e_p, t s_p
    // (affine shift), zc_p zs_p (three-term subtraction)
    float* c_xs = reinterpret_cast<float*>(red + 4 * 256);
    float* c_sx = c_xs + 256;
    float* c_ts = c_sx + 256;
    float* c_zcs = c_ts + 256;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const uint32_t tmem_cols = 2u * static_cast<uint32_t>(NB);
    if (tid == 0)
    {
        for (int s = 0; s < BLK_STAGES; ++s)
        {
            mbar_init(&full[s], 1);
            // one arrival per converter warp, or per copier thread (PRE)
            mbar_init(&conv[s], PRE ? BLK_CONV_WARPS * 32 : BLK_CONV_WARPS);
            mbar_init(&empty[s], 1);
        }
        for (int i = 0; i < 2; ++i)
        {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], BLK_EPI_WARPS);
        }
        mbar_init(drain, 1);
        abort_flag[0] = 0;
        abort_flag[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 4 * 256; i += NT) red[i] = 0.0;
    for (int p = tid; p < NB; p += NT)
    {
        // 2^e_p keeps every scaled |x| <= 2^14: |x| <= |x|_2 = 1 / s_p, or
        // the measured maximum when no scale is given (k_x16_split scales
        // by the same 2^e_p)
        const double sxv = d.sx ? d.sx[p] : 1.0;
        int e = 0;
        if (PRE && d.xexp)
        {
            e = d.xexp[p];  // the exponent the split block was written with
        }
        else if (d.sx)
        {
            e = blk_x_exp(sxv);
        }
        else
        {
            const float m = __uint_as_float(d.xmax[p]);
            if (m > 0.0f)
            {
                int ex = 0;
                frexpf(m, &ex);
                e = min(max(14 - ex, -120), 120);
            }
        }
        c_xs[p] = ldexpf(1.0f, e);
        c_sx[p] = static_cast<float>(ldexp(sxv, -e));
        c_ts[p] = static_cast<float>(d.shift * sxv);
        c_zcs[p] = d.Z ? static_cast<float>(d.zc[p] * d.zs[p]) : 0.0f;
    }
    if (warp == BLK_MMA)
    {
        tc::tmem_alloc(tmem_slot, tmem_cols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    auto give_up = [&]() {
        abort_flag[0] = 1;
        atomicExch(d.error, 1);
    };

    if (warp == BLK_PRODUCER)
    {
        // producer: the A parts of every stage, one 8 KB bulk copy each,
        // read once per product: they leave L2 first, before the X rows
        // that neighbouring blocks gather again
        if (lane == 0)
        {
            const uint64_t a_policy = l2_evict_first_policy();
            int64_t it = 0;
            bool ok = true;
            for (int64_t slot = blockIdx.x; slot < d.nblk && ok; slot += gridDim.x)
            {
                const int64_t blk = d.order[slot];
                const int s0 = d.bstage[blk], s1 = d.bstage[blk + 1];
                for (int st = s0; st < s1; ++st, ++it)
                {
                    const int s = static_cast<int>(it % BLK_STAGES);
                    const uint32_t ph = static_cast<uint32_t>((it / BLK_STAGES) & 1);
                    if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag))
                    {
                        give_up();
                        ok = false;
                        break;
                    }
                    unsigned char* stp = base + static_cast<size_t>(s) * stage_bytes;
                    mbar_expect_tx(&full[s], static_cast<uint32_t>(2 * BLK_A_PART));
                    bulk_copy_g2s_hint(stp, d.img + int64_t(st) * BLK_IMG_STAGE, 2 * BLK_A_PART,
                                       &full[s], a_policy);
                }
            }
            // the copies in flight land before the CTA leaves
            for (int64_t k = it - BLK_STAGES; k < it; ++k)
            {
                if (k < 0) continue;
                mbar_wait(&full[k % BLK_STAGES], static_cast<uint32_t>((k / BLK_STAGES) & 1),
                          abort_flag + 1);
            }
        }
        __syncwarp();
    }
    else if (PRE && warp >= BLK_CONV0)
    {
        // copiers (X split beforehand): thread ct takes union row k = ct / 16
        // of each stage and its 16-byte chunks c = ct % 16 + 16 j of the
        // row's X16 entry (hi | lo: part c / (NB / 8), probes 8 g .. 8 g + 7,
        // g = c % (NB / 8)) and copies them (cp.async, no registers) to MN
        // atom g / 8, K atom k / 8, row k % 8, chunk (g % 8) XOR (k % 8) of
        // the part's region -- the converters' layout.  Each thread's copies
        // of a stage arrive on conv[s] by themselves when they land
        // (cp.async.mbarrier.arrive.noinc; conv counts the 256 threads), so
        // a thread moves on to the next free stage at once and up to
        // BLK_STAGES stages of gathers are in flight; the row indices load
        // four stages before they are needed.
        constexpr int AH = 4;
        const int ct = tid - BLK_CONV0 * 32;
        const int k = ct >> 4;
        constexpr int nj = NB / 64;          // chunks per thread (4 or 2)
        constexpr int gpp = NB / 8;          // 16-byte chunks per part
        uint32_t dst[nj];
#pragma unroll
        for (int j = 0; j < nj; ++j)
        {
            const int c = (ct & 15) + 16 * j;
            const int part = c / gpp, g = c % gpp;
            dst[j] = static_cast<uint32_t>(part) * x_bytes + (g >> 3) * 2048 + (k >> 3) * 1024 +
                     (k & 7) * 128 + (((g & 7) ^ (k & 7)) << 4);
        }
        BlkCursor ix;
        ix.start(d.bstage, d.order, d.nblk);
        int ring[AH];
#pragma unroll
        for (int i = 0; i < AH; ++i)
        {
            ring[i] = ix.row(d.ucol, d.nblk, k);
            ix.advance(d.bstage, d.nblk);
        }
        int64_t it = 0;
        bool ok = true;
        for (int64_t slot = blockIdx.x; slot < d.nblk && ok; slot += gridDim.x)
        {
            const int64_t blk = d.order[slot];
            const int s0 = d.bstage[blk], s1 = d.bstage[blk + 1];
            for (int st = s0; st < s1; ++st, ++it)
            {
                const int s = static_cast<int>(it % BLK_STAGES);
                const uint32_t ph = static_cast<uint32_t>((it / BLK_STAGES) & 1);
                const int row = ring[0];
#pragma unroll
                for (int i = 0; i + 1 < AH; ++i) ring[i] = ring[i + 1];
                ring[AH - 1] = ix.row(d.ucol, d.nblk, k);
                ix.advance(d.bstage, d.nblk);
                bool got = true;
                if (lane == 0) got = mbar_wait(&empty[s], ph ^ 1u, abort_flag);
                if (!__shfl_sync(FULL_MASK, got ? 1 : 0, 0))
                {
                    if (lane == 0) give_up();
                    ok = false;
                    break;
                }
                const uint32_t xs0 =
                    smem_u32(base + static_cast<size_t>(s) * stage_bytes + 2 * BLK_A_PART);
                const __half* src = d.x16 + int64_t(row) * 2 * NB + (ct & 15) * 8;
#pragma unroll
                for (int j = 0; j < nj; ++j)
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
                                 ::"r"(xs0 + dst[j]), "l"(src + 128 * j) : "memory");
                asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];"
                             ::"r"(smem_u32(&conv[s])) : "memory");
            }
        }
        // every copy lands before the thread leaves (also after a failed wait)
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    else if (!PRE && warp >= BLK_CONV0)
    {
        // converters.  Thread ct takes union row k = ct / 16 of each stage
        // and its float4 slices f = ct % 16 + 16 j (probes 4f .. 4f + 3, MN
        // atom j), loaded from global memory two stages ahead (row index one
        // stage before that), scaled by 2^e_p, split into FP16 parts and
        // stored in the MN-major 128-byte swizzled layout: probe n of row k
        // at atom n / 64 (2 KB apart), K atom k / 8 (1 KB apart), row k % 8
        // (128 bytes), 16-byte chunk (n % 64) / 8 XOR k % 8.
        const int ct = tid - BLK_CONV0 * 32;
        const int k = ct >> 4;
        constexpr int nj = NB / 64;        // float4 slices per thread (2 or 4)
        const uint32_t xoff0 = static_cast<uint32_t>(
            (k >> 3) * 1024 + (k & 7) * 128 + ((((ct & 15) >> 1) ^ (k & 7)) << 4) + (ct & 1) * 8);
        auto load_x = [&](int row, float4 (&buf)[4]) {
            if (row < 0) return;
            const float4* src = reinterpret_cast<const float4*>(d.X + int64_t(row) * NB) + (ct & 15);
#pragma unroll
            for (int j = 0; j < nj; ++j) buf[j] = __ldg(src + 16 * j);
        };
        // the scales of this thread's probes
        float4 xs[nj];
#pragma unroll
        for (int j = 0; j < nj; ++j)
            xs[j] = *reinterpret_cast<const float4*>(c_xs + 4 * ((ct & 15) + 16 * j));
        // stage cursors: the one being converted and the one whose row index
        // is loading
        BlkCursor cur, ix;
        cur.start(d.bstage, d.order, d.nblk);
        ix.start(d.bstage, d.order, d.nblk);
        float4 b0[4], b1[4];
        // prologue: rows of stages 0 and 1 loading, the index of stage 2
        load_x(ix.row(d.ucol, d.nblk, k), b0);
        ix.advance(d.bstage, d.nblk);
        load_x(ix.row(d.ucol, d.nblk, k), b1);
        ix.advance(d.bstage, d.nblk);
        int next_row = ix.row(d.ucol, d.nblk, k);
        ix.advance(d.bstage, d.nblk);
        int64_t it = 0;
        bool ok = true;
        auto step = [&](float4 (&buf)[4]) -> bool {
            const int s = static_cast<int>(it % BLK_STAGES);
            const uint32_t ph = static_cast<uint32_t>((it / BLK_STAGES) & 1);
            // the slot is free once the MMAs that read it completed
            bool got = true;
            if (lane == 0) got = mbar_wait(&empty[s], ph ^ 1u, abort_flag);
            if (!__shfl_sync(FULL_MASK, got ? 1 : 0, 0))
            {
                if (lane == 0) give_up();
                return false;
            }
            __syncwarp();
            unsigned char* xh = base + static_cast<size_t>(s) * stage_bytes + 2 * BLK_A_PART;
            unsigned char* xl = xh + x_bytes;
#pragma unroll
            for (int j = 0; j < nj; ++j)
            {
                const float4 v = make_float4(buf[j].x * xs[j].x, buf[j].y * xs[j].y,
                                             buf[j].z * xs[j].z, buf[j].w * xs[j].w);
                uint2 hi, lo;
                split_h4(v, hi, lo);
                *reinterpret_cast<uint2*>(xh + xoff0 + j * 2048) = hi;
                *reinterpret_cast<uint2*>(xl + xoff0 + j * 2048) = lo;
            }
            tc::fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&conv[s]);
            ++it;
            cur.advance(d.bstage, d.nblk);
            // refill: X rows of the stage two ahead, the next index
            load_x(next_row, buf);
            next_row = ix.row(d.ucol, d.nblk, k);
            ix.advance(d.bstage, d.nblk);
            return true;
        };
        while (ok && cur.slot < d.nblk)
        {
            ok = step(b0);
            if (!ok || cur.slot >= d.nblk) break;
            ok = step(b1);
        }
    }
    else if (warp == BLK_MMA)
    {
        if (lane == 0)
        {
            const uint32_t idesc = blk_idesc(static_cast<uint32_t>(NB));
            int64_t it = 0, lb = 0;
            bool ok = true;
            for (int64_t slot = blockIdx.x; slot < d.nblk && ok; slot += gridDim.x, ++lb)
            {
                const int64_t blk = d.order[slot];
                const int buf = static_cast<int>(lb & 1);
                if (lb >= 2 &&
                    !mbar_wait(&acc_empty[buf], static_cast<uint32_t>(((lb >> 1) - 1) & 1),
                               abort_flag))
                {
                    give_up();
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const uint32_t dacc = tmem + static_cast<uint32_t>(buf * NB);
                const int s0 = d.bstage[blk], s1 = d.bstage[blk + 1];
                for (int st = s0; st < s1; ++st, ++it)
                {
                    const int s = static_cast<int>(it % BLK_STAGES);
                    const uint32_t ph = static_cast<uint32_t>((it / BLK_STAGES) & 1);
                    if (!mbar_wait(&full[s], ph, abort_flag) || !mbar_wait(&conv[s], ph, abort_flag))
                    {
                        give_up();
                        ok = false;
                        break;
                    }
                    // the copiers' cp.async writes (generic proxy) before the
                    // MMAs read the stage through the async proxy
                    if (PRE) tc::fence_proxy_async_smem();
                    tc::fence_after_sync();
                    unsigned char* stp = base + static_cast<size_t>(s) * stage_bytes;
                    // A: K-major, no swizzle (K core matrices 128 bytes apart,
                    // 8-row groups 256); X: MN-major, 128-byte swizzle (MN
                    // atoms 2 KB apart, K atoms 1 KB)
                    const uint64_t ah = tc::smem_desc(stp, 128, 256);
                    const uint64_t al = tc::smem_desc(stp + BLK_A_PART, 128, 256);
                    const uint64_t xh =
                        tc::smem_desc(stp + 2 * BLK_A_PART, 2048, 1024) | (uint64_t(2) << 61);
                    const uint64_t xl =
                        tc::smem_desc(stp + 2 * BLK_A_PART + x_bytes, 2048, 1024) |
                        (uint64_t(2) << 61);
                    const uint32_t acc = (st > s0) ? 1u : 0u;
                    tc::mma_f16_ss(dacc, al, xh, idesc, acc);
                    tc::mma_f16_ss(dacc, ah, xl, idesc, 1u);
                    tc::mma_f16_ss(dacc, ah, xh, idesc, 1u);
                    tc::commit(&empty[s]);
                }
                if (!ok) break;
                tc::commit(&acc_full[buf]);
            }
            // every issued MMA completes before the tensor memory is freed
            tc::commit(drain);
            mbar_wait(drain, 0, abort_flag + 1);
        }
        __syncwarp();
    }
    else
    {
        // epilogue: warp w reads lanes 32 (w % 4) .. +31 (block rows) and the
        // probe columns of half w / 4, 16 at a time; thread = block row
        const int qd = warp & 3;
        const int half = warp >> 2;
        const uint32_t lanes = static_cast<uint32_t>(32 * qd) << 16;
        constexpr int cols = NB / 2;
        const int c_begin = half * cols;
        const bool need_x = d.shift != 0.0 || d.epi == 1;
        const bool need_z = d.Z != nullptr;
        // the partial-sum term as a branch-free blend: x y, y y or z y
        const float wx = d.epi == 1 ? 1.0f : 0.0f;
        const float wy = d.epi == 2 ? 1.0f : 0.0f;
        const float wz = d.epi == 3 ? 1.0f : 0.0f;
        const int my_col = blk_col(lane);
        int64_t lb = 0;
        for (int64_t slot = blockIdx.x; slot < d.nblk; slot += gridDim.x, ++lb)
        {
            const int64_t blk = d.order[slot];
            const int buf = static_cast<int>(lb & 1);
            const int64_t row = blk * BLK_ROWS + 32 * qd + lane;
            const float rs = d.rsc[row];  // 2^-f_r (padding rows hold 1)
            bool got = true;
            if (lane == 0)
                got = mbar_wait(&acc_full[buf], static_cast<uint32_t>((lb >> 1) & 1), abort_flag);
            if (!__shfl_sync(FULL_MASK, got ? 1 : 0, 0))
            {
                if (lane == 0) give_up();
                break;
            }
            __syncwarp();
            tc::fence_after_sync();
            const bool live = row < d.M;
            const uint32_t dacc = tmem + static_cast<uint32_t>(buf * NB);
            for (int c0 = c_begin; c0 < c_begin + cols; c0 += 16)
            {
                uint32_t v[16];
                tc::ld_x16(dacc + lanes + static_cast<uint32_t>(c0), v);
                // this row's 16 X and Z values (64 bytes each, 16-byte aligned)
                float xv[16], zv[16];
                const int64_t o = row * NB + c0;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                {
                    float4 x4 = make_float4(0.f, 0.f, 0.f, 0.f), z4 = x4;
                    if (live && need_x) x4 = __ldg(reinterpret_cast<const float4*>(d.X + o) + q);
                    if (live && need_z) z4 = __ldg(reinterpret_cast<const float4*>(d.Z + o) + q);
                    xv[4 * q] = x4.x; xv[4 * q + 1] = x4.y; xv[4 * q + 2] = x4.z; xv[4 * q + 3] = x4.w;
                    zv[4 * q] = z4.x; zv[4 * q + 1] = z4.y; zv[4 * q + 2] = z4.z; zv[4 * q + 3] = z4.w;
                }
                tc::wait_ld();
                // y = s A x (+ t s x) (- zc zs z) in FP32; the partial-sum
                // terms x y, y y or z y in FP32, summed over the warp's 32
                // rows in FP32 and over warps and blocks in FP64 (the
                // per-probe factor s_p or zs_p is applied to the sums)
                float add[16];
                float yv[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    const int p = c0 + j;
                    // the shift and three-term constants are zero where unused
                    float y = __uint_as_float(v[j]) * (c_sx[p] * rs);
                    y = fmaf(c_ts[p], xv[j], y);
                    y = fmaf(-c_zcs[p], zv[j], y);
                    yv[j] = y;
                    add[j] = y * fmaf(wx, xv[j], fmaf(wy, y, wz * zv[j]));
                }
                if (live)
                {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        reinterpret_cast<float4*>(d.Y + o)[q] =
                            make_float4(yv[4 * q], yv[4 * q + 1], yv[4 * q + 2], yv[4 * q + 3]);
                }
                if (!live)
                {
#pragma unroll
                    for (int j = 0; j < 16; ++j) add[j] = 0.0f;
                }
                if (d.epi != 0)
                {
                    const float sum = reduce_scatter16(add, lane);
                    if (lane < 16) red[qd * 256 + c0 + my_col] += static_cast<double>(sum);
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);
        }
    }

    tc::fence_before_sync();
    __syncthreads();
    if (warp == BLK_MMA)
    {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, tmem_cols);
    }
    if (d.epi != 0)
        for (int q = tid; q < NB; q += NT)
        {
            // the per-probe factor of the terms: s_p (alpha), 1 (|y|^2), zs_p
            const double f = d.epi == 1 ? (d.sx ? d.sx[q] : 1.0) : d.epi == 3 ? d.zs[q] : 1.0;
            d.partials[static_cast<int64_t>(blockIdx.x) * NB + q] =
                f * (((red[q] + red[256 + q]) + red[512 + q]) + red[768 + q]);
        }
}

}  // namespace slq

#endif  // SLQ_BLK_CUH_
