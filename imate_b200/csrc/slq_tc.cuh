// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a.
//
// The contraction of a row-group SpMM tile,
//   D[M = 128 probes][N = 16 rows] += A[M][K = 8 union columns] * B[K][N],
// runs as kind::tf32 MMAs with FP32 accumulation in tensor memory.  FP32
// operands are split into TF32 pairs, hi = rn_tf32(x), lo = rn_tf32(x - hi),
// and D = A_lo B_hi + A_hi B_lo + A_hi B_hi; the dropped A_lo B_lo term and
// the rounding of the lo parts leave a relative error of about 2^-21 per
// product.
//
// Encodings (PTX ISA, tcgen05; field layouts as in CUTLASS's
// cute/arch/mma_sm100_desc.hpp):
//   instruction descriptor, kind::tf32, D FP32, M = 128, N = 16, A and B
//     K-major:                                               0x08040910
//   shared-memory descriptor, SWIZZLE_NONE: start >> 4 in bits 0-13,
//     leading byte offset >> 4 in bits 16-29, stride byte offset >> 4 in
//     bits 32-45, version 1 in bits 46-47, layout type 0 in bits 61-63.
//   K-major operand tile in shared memory (no swizzle): core matrices of 8
//     rows x 16 bytes (4 K values); element (r, k) at (r % 8) * 16 +
//     (r / 8) * SBO + (k / 4) * LBO + (k % 4) * 4, here LBO = 128 bytes
//     (the two 4-wide K halves of a core row group side by side) and SBO =
//     256 bytes (next 8 rows).  B (N = 16 rows of the group) is stored this
//     way.  An MN-major TF32 operand (transpose bit 15 for A, 16 for B) reads
//     back as zero without swizzling and with the plain 128-byte swizzle; it
//     needs the 128-byte swizzle with 32-byte atoms (layout type 1, see
//     k_tc_selftest_mn), which TMA writes with
//     CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B.
//   A in tensor memory (TS form): lane m = row m, columns = the K values.
//   Tensor-memory addresses: lane << 16 | column; warp w of a warpgroup
//     reaches lanes 32 (w % 4) .. 32 (w % 4) + 31.

#ifndef SLQ_TC_CUH_
#define SLQ_TC_CUH_

#include <cstdint>
#include <cuda.h>

namespace slq {
namespace tc {

constexpr uint32_t IDESC_TF32_M128_N16 = 0x08040910u;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Whole warp; writes the allocated tensor-memory address to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_addr(dst)), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Whole warp (the allocating one).
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory writes made visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 8 consecutive columns of this thread's lane.
__device__ __forceinline__ void st_x8(uint32_t taddr, const uint32_t (&v)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
                 ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]),
                   "r"(v[6]), "r"(v[7])
                 : "memory");
}

// 16 consecutive columns of this thread's lane.
__device__ __forceinline__ void st_x16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, "
                 "%9, %10, %11, %12, %13, %14, %15, %16};"
                 ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]),
                   "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]),
                   "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
                 : "memory");
}

__device__ __forceinline__ void wait_st()
{
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// 16 consecutive columns of this thread's lane.
__device__ __forceinline__ void ld_x16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, "
                 "%9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                   "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                   "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                 : "r"(taddr)
                 : "memory");
}

__device__ __forceinline__ void wait_ld()
{
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// D (tensor memory) [+]= A (tensor memory) * B (shared memory); one thread.
__device__ __forceinline__ void mma_tf32_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate)
{
    const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "r"(a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2),
          "r"(m3)
        : "memory");
}

// D (tensor memory) [+]= A (shared memory) * B (shared memory); one thread.
__device__ __forceinline__ void mma_tf32_ss(uint32_t d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate)
{
    const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1),
          "r"(m2), "r"(m3)
        : "memory");
}

// kind::f16 (FP16 or BF16 operands as the instruction descriptor says, FP32
// D): D (tensor memory) [+]= A (shared memory) * B (shared memory); one
// thread.
__device__ __forceinline__ void mma_f16_ss(uint32_t d, uint64_t adesc, uint64_t bdesc,
                                           uint32_t idesc, uint32_t accumulate)
{
    const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(m0), "r"(m1),
          "r"(m2), "r"(m3)
        : "memory");
}

// Arrive once on the mbarrier when every MMA this thread issued so far has
// completed (their operand reads included).
__device__ __forceinline__ void commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_addr(bar)) : "memory");
}

// Shared-memory matrix descriptor, SWIZZLE_NONE, version 1.
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo_bytes,
                                              uint32_t sbo_bytes)
{
    const uint64_t start = (smem_addr(p) >> 4) & 0x3FFFu;
    const uint64_t lbo = (lbo_bytes >> 4) & 0x3FFFu;
    const uint64_t sbo = (sbo_bytes >> 4) & 0x3FFFu;
    return start | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// TF32 round-to-nearest (ties away) of an FP32 value, as FP32 bits.
__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo)
{
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}

// Byte offset of element (r, k) of a K-major no-swizzle tile with 8 K
// values per row (LBO = 128, SBO = 256): B (16 x 8) and A (128 x 8).
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k)
{
    return static_cast<uint32_t>((r & 7) * 16 + (r >> 3) * 256 + (k >> 2) * 128 + (k & 3) * 4);
}

// Instruction descriptor, kind::tf32, D FP32, M = 128, A and B K-major, for
// N a multiple of 16 in [16, 256] (N >> 3 in bits 17-22, M >> 4 in 24-28).
__host__ __device__ constexpr uint32_t idesc_tf32_m128(uint32_t n)
{
    return 0x00000910u | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// Shared-memory descriptor of a K-major tile written by a SWIZZLE_128B TMA
// load (rows of 128 bytes = 32 TF32 values, 8-row atoms of 1024 bytes):
// stride byte offset 1024, leading byte offset unused (1), version 1, layout
// type SWIZZLE_128B (2 in bits 61-63).  The tile must start on a 1024-byte
// boundary; a K step of 8 values inside the atom advances the start by 32
// bytes.
__device__ __forceinline__ uint64_t smem_desc_sw128(const void* p)
{
    const uint64_t start = (smem_addr(p) >> 4) & 0x3FFFu;
    return start | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) | (uint64_t(1) << 46) |
           (uint64_t(2) << 61);
}

// 2-D tiled TMA load of box (x, y) .. into shared memory, completing on bar.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
          "r"(smem_addr(bar))
        : "memory");
}

// L2 prefetch of one box of a 2-D tiled tensor map (no completion to wait
// on; coordinates as tma_load_2d)
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int y)
{
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y)
                 : "memory");
}

}  // namespace tc
}  // namespace slq

#endif  // SLQ_TC_CUH_
