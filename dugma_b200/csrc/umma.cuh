// umma.cuh -- the sm_100a tensor-core pieces compi's source-side sums use: tensor-memory (TMEM)
// allocation, per-warp TMEM loads and stores, and the single-thread tcgen05.mma of kind::tf32
// with the A operand in TMEM and the B operand in shared memory.
//
// Layouts (PTX ISA, tcgen05 "Matrix descriptors" and "Instruction descriptor"; the bit
// positions are those of CUTLASS's UMMA::SmemDescriptor / UMMA::InstrDescriptor):
//   * D (M = 128, cta_group::1): row m in TMEM lane m, column n in TMEM column n (FP32).
//   * A in TMEM (kind::tf32): row m in lane m, one K element per 32-bit column.
//   * B in shared memory, K-major, no swizzle: "core matrices" of 8 N-rows x 16 bytes (4 TF32
//     K-elements), each 128 contiguous bytes; the descriptor's stride byte offset (SBO) steps
//     between core matrices along N (8 rows), its leading byte offset (LBO) between the two
//     16-byte K halves of one MMA's K = 8.
//   * A warp reaches only the TMEM lanes 32 (warp % 4) .. 32 (warp % 4) + 31.
#pragma once

#include <stdint.h>

namespace dugma {

// Allocates `ncols` TMEM columns (a power of two >= 32) for this CTA; the whole warp calls it.
// The base address lands in *dst (shared memory).  The permit is given up right away: this
// CTA allocates once.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Frees the CTA's TMEM; the warp that allocated calls it, after every MMA and TMEM access ended.
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// generic-proxy writes to shared memory made visible to the tensor core's (async proxy) reads
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// named barrier `id` (1..15; 0 is __syncthreads) over `n` threads: wait, or arrive without waiting
__device__ __forceinline__ void named_bar_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void named_bar_arrive(int id, int n)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// TMEM address of (lane, column): lane in bits 31..16, column in bits 15..0
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, uint32_t lane, uint32_t col)
{
    return base + (lane << 16) + col;
}

// Each thread of the warp stores 4 consecutive 32-bit columns of its own lane.
__device__ __forceinline__ void tmem_st4(uint32_t taddr, float a, float b, float c, float d)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), "r"(__float_as_uint(a)),
                 "r"(__float_as_uint(b)), "r"(__float_as_uint(c)), "r"(__float_as_uint(d))
                 : "memory");
}

// Each thread of the warp stores 8 consecutive 32-bit columns of its own lane.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8])
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}

// Each thread of the warp loads 16 consecutive 32-bit columns of its own lane (complete after
// tmem_wait_ld).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// Shared-memory descriptor of a K-major, unswizzled operand tile (fields: start address >> 4 in
// bits 0-13, LBO >> 4 in 16-29, SBO >> 4 in 32-45, descriptor version 1 in 46-47, layout 0 =
// no swizzle in 61-63).
__device__ __forceinline__ uint64_t smem_desc_kmajor(const void* p, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    const uint64_t a = (smem_u32(p) >> 4) & 0x3FFFu;
    return a | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) |
           ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::tf32 with FP32 accumulation, A and B K-major, M x N:
// D format F32 (bits 4-5 = 1), A and B format TF32 (7-9, 10-12 = 2), N >> 3 (17-22), M >> 4 (24-28).
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (TMEM) = A (TMEM) x B (shared memory) + (accumulate ? D : 0); issued by one thread.
__device__ __forceinline__ void umma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                             bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate), "r"(0u)
        : "memory");
}

// The mbarrier `bar` receives one arrival when every tcgen05.mma this thread issued before
// has completed (and its operand reads with it).
__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// FP32 -> TF32 (10 explicit mantissa bits), rounded to nearest with ties away from zero, as an
// FP32 bit pattern whose low 13 bits are zero; integer pipe only.  Finite inputs below 2^127.
__device__ __forceinline__ float tf32_rna(float x)
{
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

}  // namespace dugma
