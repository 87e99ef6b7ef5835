// Block SpMM on the tensor cores (tcgen05 kind::tf32), sm_100a.
//
// Y[M][b] = A[M][K] X[K][b] for a sparse FP32 A whose rows are cut into
// blocks of 128 consecutive rows.  Each block keeps the sorted union of its
// rows' column indices (padded to a multiple of 16 with copies of its last
// column, zero-valued) and its values as a dense 128 x union matrix, zero
// where a row lacks a column.  A block is one M = 128 tile: its union
// columns are the K dimension, the b <= 256 probes the N dimension, so every
// gathered row of X (1 KB at b = 256) feeds 128 rows of products and the
// tensor core does the multiply-adds.  Fill (nonzeros over 128 x union)
// decides the cost: blocks made of rows with overlapping neighbourhoods
// (slq_block_order) matter.
//
// Format (built on the device by k_blk_* below):
//   bstage[nblk + 1]   first 16-column stage of each block (exclusive sum)
//   ucol[16 * stages]  union column indices, stage by stage
//   img[stages][2][2048]  TF32 parts of each stage's values, hi = rn_tf32(a)
//                      then lo = rn_tf32(a - hi), each 128 rows x 16 columns
//                      in the K-major no-swizzle layout the MMA reads:
//                      element (r, k) at float offset (r % 8) * 4 + (r / 8) *
//                      128 + (k / 4) * 32 + (k % 4) (core matrices of 8 rows
//                      x 4 values; leading byte offset 128 between K-adjacent
//                      core matrices, stride byte offset 512 between 8-row
//                      groups)
// so one stage of A is one contiguous 16 KB bulk copy.
//
// Kernel k_spmm_blk (persistent, one CTA per SM, blocks dealt round-robin):
//   warp 8        producer: per stage, one cp.async.bulk of the A parts;
//   warps 10-17   converters: load the stage's 16 X rows from global memory
//                 (two stages ahead, into registers), split them into TF32
//                 parts, hi = rn_tf32(x) and lo = rn_tf32(x - hi) (integer
//                 rounding of the bit patterns), and store both in the
//                 MN-major 128-byte-swizzle-with-32-byte-atoms layout (4 K
//                 rows x 32 probes per atom).  TMA gathers of the X rows would
//                 need one gather4 per 512 bytes (the swizzle limits a box row
//                 to 128 bytes), which measured slower than these loads;
//   warp 9        MMA issuer: per K step of 8 the three products A_lo X_hi
//                 + A_hi X_lo + A_hi X_hi into an FP32 accumulator in tensor
//                 memory (lane = block row, column = probe), two
//                 accumulators so the epilogue of one block overlaps the
//                 products of the next;
//   warps 0-7     epilogue: the SpMM epilogue of the other kernels (probe
//                 scales, affine shift, three-term subtraction, partial sums
//                 of alpha or |y|^2) on the finished accumulator; its
//                 element arithmetic is FP32 (y = s A x rounded once more
//                 than the FP64 form, the terms x y, y y, z y one rounding
//                 each) and the row sums FP64, the per-probe factor applied
//                 to the sums.
// The dropped A_lo X_lo term and the rounding of the lo parts leave about
// 2^-22 relative error per product; the accumulation runs in the tensor
// core's FP32.  Every mbarrier wait is bounded; a wait that runs out sets
// the error word and the CTA drains its copies and MMAs before it leaves.
// No multicast: every TMA load reads this GPU's own buffers.

#ifndef SLQ_BLK_CUH_
#define SLQ_BLK_CUH_

#include "slq_kernels.cuh"

namespace slq {

constexpr int BLK_ROWS = 128;
constexpr int BLK_BK = 16;            // union columns per stage
constexpr int BLK_STAGES = 4;
constexpr int BLK_A_BYTES = BLK_ROWS * BLK_BK * 4;  // 8 KB per A part
constexpr int BLK_IMG_STAGE = 2 * BLK_ROWS * BLK_BK;   // floats per stage image (hi, lo)
constexpr int BLK_EPI_WARPS = 8;
constexpr int BLK_PRODUCER = 8;       // warp indices
constexpr int BLK_MMA = 9;
constexpr int BLK_CONV0 = 10;
constexpr int BLK_CONV_WARPS = 8;
constexpr int BLK_THREADS = (BLK_CONV0 + BLK_CONV_WARPS) * 32;  // 576
constexpr int BLK_AHEAD = 2;          // stages of X rows loaded ahead

__host__ __device__ constexpr uint32_t blk_stage_bytes(int nb)
{
    return 2u * BLK_A_BYTES + 2u * static_cast<uint32_t>(nb) * BLK_BK * 4u;
}

// stages, barriers (256 bytes), partial sums [4][256] (doubles) and the
// per-probe epilogue constants [3][256] (floats)
__host__ __device__ constexpr size_t blk_smem_bytes(int nb)
{
    return 1023 + static_cast<size_t>(BLK_STAGES) * blk_stage_bytes(nb) + 256 +
           4 * 256 * sizeof(double) + 3 * 256 * sizeof(float);
}

// TF32 parts by integer rounding of the bit patterns (round half away
// from zero on the 13 dropped mantissa bits): hi = rn_tf32(x), lo =
// rn_tf32(x - hi), the x - hi difference exact in FP32.  Integer adds and
// masks keep the conversion off the conversion pipe.
__device__ __forceinline__ float round_tf32_bits(float x)
{
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
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

// values into the stage images (zeroed first); atomic adds only sum
// duplicate (row, column) entries, each slot otherwise receives one value
__global__ void k_blk_scatter(const uint64_t* __restrict__ keys, const int32_t* __restrict__ pos,
                              const int32_t* __restrict__ uidx, int64_t nnz, int cbits,
                              const int32_t* __restrict__ ufirst,
                              const int32_t* __restrict__ bstage, const float* __restrict__ vals,
                              const uint8_t* __restrict__ rr, float* __restrict__ img)
{
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        const int64_t blk = static_cast<int64_t>(keys[i] >> cbits);
        const int64_t j = uidx[i] - 1 - ufirst[blk];
        const int32_t e = pos[i];
        const int r = rr[e];
        const int kk = static_cast<int>(j % BLK_BK);
        const int64_t stage = bstage[blk] + j / BLK_BK;
        const int64_t off = stage * BLK_IMG_STAGE + (r & 7) * 4 + (r >> 3) * 128 +
                            (kk >> 2) * 32 + (kk & 3);
        atomicAdd(&img[off], vals[e]);
    }
}

// TF32 parts of the stage images in place: the values (scattered into the
// hi half) become hi = rn_tf32(a), the lo half rn_tf32(a - hi)

__global__ void k_blk_split(float* __restrict__ img, int64_t stages)
{
    const int64_t total = stages * (BLK_ROWS * BLK_BK);
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    {
        float* h = img + (i / (BLK_ROWS * BLK_BK)) * BLK_IMG_STAGE + i % (BLK_ROWS * BLK_BK);
        const float a = *h;
        const float hi = round_tf32_bits(a);
        h[BLK_ROWS * BLK_BK] = round_tf32_bits(a - hi);
        *h = hi;
    }
}

// ---------------------------------------------------------------------------
// the product
// ---------------------------------------------------------------------------

struct BlkArgs {
    int64_t M;                 // rows of Y
    int64_t nblk;              // 128-row blocks
    int NB;                    // probes = b (128 or 256)
    const int32_t* bstage;
    const int32_t* ucol;
    const float* img;
    const float* X;
    const double* sx;
    double shift;
    float* Y;
    const float* Z;
    const double* zc;
    const double* zs;
    int epi;
    double* partials;          // [grid][NB]
    int32_t* error;
};

__device__ __forceinline__ void split1(float& x, float& lo)
{
    const float h = round_tf32_bits(x);
    lo = round_tf32_bits(x - h);
    x = h;
}

__device__ __forceinline__ void split4(float4& v, float4& lo)
{
    split1(v.x, lo.x);
    split1(v.y, lo.y);
    split1(v.z, lo.z);
    split1(v.w, lo.w);
}

// Reduce-scatter of 16 per-lane values over the warp's 32 lanes: on return
// lanes 0-15 hold the sum over all lanes of value blk_col(lane), lanes
// 16-31 the same sums again.  16 shuffles of doubles instead of 16 x 5 for
// 16 separate tree reductions; the order of the additions is fixed.
__device__ __forceinline__ int blk_col(int lane)
{
    return 8 * (lane & 1) + 4 * ((lane >> 1) & 1) + 2 * ((lane >> 2) & 1) + ((lane >> 3) & 1);
}

__device__ __forceinline__ double reduce_scatter16(double (&a)[16], int lane)
{
#pragma unroll
    for (int st = 0; st < 4; ++st)
    {
        const int h = 8 >> st;          // values kept after this step
        const bool upper = (lane >> st) & 1;
#pragma unroll
        for (int i = 0; i < h; ++i)
        {
            const double send = upper ? a[i] : a[i + h];
            const double keep = upper ? a[i + h] : a[i];
            a[i] = keep + __shfl_xor_sync(FULL_MASK, send, 1 << st);
        }
    }
    return a[0] + __shfl_xor_sync(FULL_MASK, a[0], 16);
}

__global__ void __launch_bounds__(BLK_THREADS, 1)
k_spmm_blk(const BlkArgs d)
{
    extern __shared__ __align__(1024) unsigned char smem_blk[];
    const uint32_t stage_bytes = blk_stage_bytes(d.NB);
    const uint32_t x_bytes = static_cast<uint32_t>(d.NB) * BLK_BK * 4;  // one X part
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
    double* red = reinterpret_cast<double*>(tail + 256);      // [4][256]
    // per-probe epilogue constants in FP32: s_p, t s_p (affine shift) and
    // zc_p zs_p (three-term subtraction)
    float* c_sx = reinterpret_cast<float*>(red + 4 * 256);
    float* c_ts = c_sx + 256;
    float* c_zcs = c_ts + 256;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const uint32_t tmem_cols = 2u * static_cast<uint32_t>(d.NB);
    if (tid == 0)
    {
        for (int s = 0; s < BLK_STAGES; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&conv[s], BLK_CONV_WARPS);  // one arrival per converter warp
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
    for (int i = tid; i < 4 * 256; i += BLK_THREADS) red[i] = 0.0;
    for (int p = tid; p < d.NB; p += BLK_THREADS)
    {
        const double sxv = d.sx ? d.sx[p] : 1.0;
        c_sx[p] = static_cast<float>(sxv);
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
        // producer: the A parts of every stage, one 16 KB bulk copy each
        if (lane == 0)
        {
            int64_t it = 0;
            bool ok = true;
            for (int64_t blk = blockIdx.x; blk < d.nblk && ok; blk += gridDim.x)
            {
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
                    mbar_expect_tx(&full[s], static_cast<uint32_t>(2 * BLK_A_BYTES));
                    bulk_copy_g2s(stp, d.img + int64_t(st) * BLK_IMG_STAGE, 2 * BLK_A_BYTES,
                                  &full[s]);
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
    else if (warp >= BLK_CONV0)
    {
        // converters.  X: thread ct takes union row k = ct / 16 of each stage
        // and its float4 slices f = ct % 16 + 16 j (probes 4f .. 4f + 3),
        // loaded from global memory BLK_AHEAD stages ahead (row index one
        // stage before that), split into TF32 parts and stored in the
        // MN-major layout: probe n of row k at atom n / 32 (2 KB apart), K
        // atom k / 4 (512 bytes apart), row k % 4 (128 bytes), 32-byte chunk
        // (n % 32) / 8 XOR k % 4.
        const int ct = tid - BLK_CONV0 * 32;
        const int k = ct >> 4;
        const int nj = d.NB / 64;          // float4 slices per thread (2 or 4)
        uint32_t xoff[4];                  // byte offsets of the slices in an X part
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int f = (ct & 15) + 16 * j;
            const int c = ((f & 7) >> 1) ^ (k & 3);
            xoff[j] = static_cast<uint32_t>((f >> 3) * 2048 + (k >> 2) * 512 + (k & 3) * 128 +
                                            c * 32 + (f & 1) * 16);
        }
        // stage cursors: the one being converted, the one whose X rows are
        // loading, the one whose row index is loading
        struct Cursor {
            int64_t blk;
            int st, s1;
        };
        auto start = [&](Cursor& c) {
            c.blk = blockIdx.x;
            c.st = c.s1 = 0;
            if (c.blk < d.nblk)
            {
                c.st = d.bstage[c.blk];
                c.s1 = d.bstage[c.blk + 1];
            }
        };
        auto advance = [&](Cursor& c) {
            if (c.blk >= d.nblk) return;
            if (++c.st >= c.s1)
            {
                c.blk += gridDim.x;
                if (c.blk < d.nblk)
                {
                    c.st = d.bstage[c.blk];
                    c.s1 = d.bstage[c.blk + 1];
                }
            }
        };
        auto row_of = [&](const Cursor& c) -> int {
            return c.blk < d.nblk ? d.ucol[int64_t(c.st) * BLK_BK + k] : -1;
        };
        auto load_x = [&](int row, float4 (&buf)[4]) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < nj && row >= 0)
                    buf[j] = __ldg(reinterpret_cast<const float4*>(d.X + int64_t(row) * d.NB) +
                                   (ct & 15) + 16 * j);
        };
        Cursor cur, ix;
        start(cur);
        start(ix);
        float4 b0[4], b1[4];
        // prologue: rows of stages 0 and 1 loading, the index of stage 2
        load_x(row_of(ix), b0);
        advance(ix);
        load_x(row_of(ix), b1);
        advance(ix);
        int next_row = row_of(ix);
        advance(ix);
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
            unsigned char* xh = base + static_cast<size_t>(s) * stage_bytes + 2 * BLK_A_BYTES;
            unsigned char* xl = xh + x_bytes;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                if (j >= nj) continue;
                float4 v = buf[j], lo;
                split4(v, lo);
                *reinterpret_cast<float4*>(xh + xoff[j]) = v;
                *reinterpret_cast<float4*>(xl + xoff[j]) = lo;
            }
            tc::fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&conv[s]);
            ++it;
            advance(cur);
            // refill: X rows of the stage BLK_AHEAD ahead, the next index
            load_x(next_row, buf);
            next_row = row_of(ix);
            advance(ix);
            return true;
        };
        while (ok && cur.blk < d.nblk)
        {
            ok = step(b0);
            if (!ok || cur.blk >= d.nblk) break;
            ok = step(b1);
        }
    }
    else if (warp == BLK_MMA)
    {
        if (lane == 0)
        {
            const uint32_t idesc = tc::idesc_tf32_m128(static_cast<uint32_t>(d.NB)) | (1u << 16);
            int64_t it = 0, lb = 0;
            bool ok = true;
            for (int64_t blk = blockIdx.x; blk < d.nblk && ok; blk += gridDim.x, ++lb)
            {
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
                const uint32_t dacc = tmem + static_cast<uint32_t>(buf * d.NB);
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
                    tc::fence_after_sync();
                    unsigned char* stp = base + static_cast<size_t>(s) * stage_bytes;
                    const uint64_t ah = tc::smem_desc(stp, 128, 512);
                    const uint64_t al = tc::smem_desc(stp + BLK_A_BYTES, 128, 512);
                    // MN-major, 128-byte swizzle with 32-byte atoms: N atoms 2 KB
                    // apart, K atoms (4 rows) 512 bytes apart
                    const uint64_t xh =
                        tc::smem_desc(stp + 2 * BLK_A_BYTES, 2048, 512) | (uint64_t(1) << 61);
                    const uint64_t xl =
                        tc::smem_desc(stp + 2 * BLK_A_BYTES + x_bytes, 2048, 512) |
                        (uint64_t(1) << 61);
#pragma unroll
                    for (int kk = 0; kk < BLK_BK / 8; ++kk)
                    {
                        // K step kk: two K core matrices of A (256 bytes), two K
                        // atoms of X (1 KB)
                        const uint64_t ao = static_cast<uint64_t>(kk * 256) >> 4;
                        const uint64_t xo = static_cast<uint64_t>(kk * 1024) >> 4;
                        const uint32_t acc = (st > s0 || kk > 0) ? 1u : 0u;
                        tc::mma_tf32_ss(dacc, al + ao, xh + xo, idesc, acc);
                        tc::mma_tf32_ss(dacc, ah + ao, xl + xo, idesc, 1u);
                        tc::mma_tf32_ss(dacc, ah + ao, xh + xo, idesc, 1u);
                    }
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
        const int cols = d.NB / 2;
        const int c_begin = half * cols;
        const bool need_x = d.shift != 0.0 || d.epi == 1;
        const int my_col = blk_col(lane);
        int64_t lb = 0;
        for (int64_t blk = blockIdx.x; blk < d.nblk; blk += gridDim.x, ++lb)
        {
            const int buf = static_cast<int>(lb & 1);
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
            const int64_t row = blk * BLK_ROWS + 32 * qd + lane;
            const bool live = row < d.M;
            const uint32_t dacc = tmem + static_cast<uint32_t>(buf * d.NB);
            for (int c0 = c_begin; c0 < c_begin + cols; c0 += 16)
            {
                uint32_t v[16];
                tc::ld_x16(dacc + lanes + static_cast<uint32_t>(c0), v);
                // this row's 16 X and Z values (64 bytes each, 16-byte aligned)
                float xv[16], zv[16];
                const int64_t o = row * d.NB + c0;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                {
                    float4 x4 = make_float4(0.f, 0.f, 0.f, 0.f), z4 = x4;
                    if (live && need_x) x4 = __ldg(reinterpret_cast<const float4*>(d.X + o) + q);
                    if (live && d.Z) z4 = __ldg(reinterpret_cast<const float4*>(d.Z + o) + q);
                    xv[4 * q] = x4.x; xv[4 * q + 1] = x4.y; xv[4 * q + 2] = x4.z; xv[4 * q + 3] = x4.w;
                    zv[4 * q] = z4.x; zv[4 * q + 1] = z4.y; zv[4 * q + 2] = z4.z; zv[4 * q + 3] = z4.w;
                }
                tc::wait_ld();
                // y = s A x (+ t s x) (- zc zs z) in FP32; the partial-sum
                // terms x y, y y or z y in FP32, summed over rows in FP64
                // (the per-probe factor s_p or zs_p is applied to the sums)
                double add[16];
                float yv[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                {
                    const int p = c0 + j;
                    float y = __uint_as_float(v[j]) * c_sx[p];
                    if (d.shift != 0.0) y = fmaf(c_ts[p], xv[j], y);
                    if (d.Z) y = fmaf(-c_zcs[p], zv[j], y);
                    yv[j] = y;
                    float a = 0.0f;
                    if (d.epi == 1) a = xv[j] * y;
                    else if (d.epi == 2) a = y * y;
                    else if (d.epi == 3) a = zv[j] * y;
                    add[j] = live ? static_cast<double>(a) : 0.0;
                }
                if (live)
                {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        reinterpret_cast<float4*>(d.Y + o)[q] =
                            make_float4(yv[4 * q], yv[4 * q + 1], yv[4 * q + 2], yv[4 * q + 3]);
                }
                if (d.epi != 0)
                {
                    const double sum = reduce_scatter16(add, lane);
                    if (lane < 16) red[qd * 256 + c0 + my_col] += sum;
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
        for (int q = tid; q < d.NB; q += BLK_THREADS)
        {
            // the per-probe factor of the terms: s_p (alpha), 1 (|y|^2), zs_p
            const double f = d.epi == 1 ? (d.sx ? d.sx[q] : 1.0) : d.epi == 3 ? d.zs[q] : 1.0;
            d.partials[static_cast<int64_t>(blockIdx.x) * d.NB + q] =
                f * (((red[q] + red[256 + q]) + red[512 + q]) + red[768 + q]);
        }
}

}  // namespace slq

#endif  // SLQ_BLK_CUH_
