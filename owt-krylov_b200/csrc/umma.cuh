// Fifth-generation tensor core (tcgen05) helpers for sm_100a: shared-memory
// operand descriptors, the f16-kind MMA with FP32 accumulators in tensor
// memory (TMEM), commits to mbarriers, TMEM allocation and loads.
//
// Operands are BF16 tiles in shared memory, K-major with the 128-byte
// swizzle: a tile is rows of 64 elements (128 B); 8 consecutive rows form a
// 1024-byte swizzle atom in which 16-byte chunk c of row r is stored at chunk
// c ^ (r & 7).  Tiles start on 1024-byte boundaries.  The descriptor fields
// (start >> 4 in bits [0,14), leading offset in [16,30), stride offset in
// [32,46), version 1 in [46,48), layout type 2 = 128-byte swizzle in
// [61,64)) and the instruction-descriptor fields follow the public layout
// in CUTLASS's cute/arch/mma_sm100_desc.hpp (SmemDescriptor, InstrDescriptor);
// for this K-major swizzled form the leading offset is 1 and the stride
// offset is one atom (1024 B).  One MMA consumes K = 16 elements (32 bytes of
// each row), so stepping K inside a 64-element block adds 32 bytes to the
// start address.
#pragma once

#include <cstdint>

#include "device_common.cuh"

namespace owtk::dev {

// Byte offset of 16-byte chunk `chunk` (0..7) of row `row` in a swizzled tile.
__device__ __forceinline__ std::uint32_t sw128(int row, int chunk)
{
    return static_cast<std::uint32_t>(row * 128 + ((chunk ^ (row & 7)) << 4));
}

__device__ __forceinline__ std::uint64_t umma_desc_sw128(std::uint32_t smem_addr)
{
    std::uint64_t d = 0;
    d |= static_cast<std::uint64_t>((smem_addr & 0x3FFFFu) >> 4);   // start address
    d |= static_cast<std::uint64_t>(1) << 16;                       // leading byte offset (unused: 1)
    d |= static_cast<std::uint64_t>(1024 >> 4) << 32;               // stride byte offset: one atom
    d |= static_cast<std::uint64_t>(1) << 46;                       // descriptor version
    d |= static_cast<std::uint64_t>(2) << 61;                       // 128-byte swizzle
    return d;
}

// f16-kind instruction descriptor: BF16 A and B (both K-major), FP32 D.
__host__ __device__ constexpr std::uint32_t umma_idesc_bf16(int m, int n)
{
    return (1u << 4)                                      // D format F32
        | (1u << 7)                                       // A format BF16
        | (1u << 10)                                      // B format BF16
        | (static_cast<std::uint32_t>(n >> 3) << 17)      // N / 8
        | (static_cast<std::uint32_t>(m >> 4) << 24);     // M / 16
}

// D[tmem] (+)= A * B^T, issued by one thread.
__device__ __forceinline__ void umma_bf16(std::uint32_t d_tmem, std::uint64_t a_desc, std::uint64_t b_desc,
                                          std::uint32_t idesc, bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(static_cast<std::uint32_t>(accumulate))
        : "memory");
}

// Arrive on `bar` when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(std::uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Warp-collective: allocate `cols` TMEM columns (power of two >= 32); the base
// address is written to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(std::uint32_t dst, std::uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Warp-collective, same warp as the allocation.
__device__ __forceinline__ void tmem_free(std::uint32_t base, std::uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// Warp-collective: 32 lanes x 32 consecutive FP32 columns; lane i of the warp
// receives TMEM lane (taddr lane + i), columns [col, col + 32).
__device__ __forceinline__ void tmem_ld32(std::uint32_t taddr, float (&v)[32])
{
    std::uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Warp-collective: 32 lanes x 16 consecutive FP32 columns.
__device__ __forceinline__ void tmem_ld16(std::uint32_t taddr, float (&v)[16])
{
    std::uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------- tensor loads
// TMA tensor copies global -> shared through a CUtensorMap (a __grid_constant__
// kernel parameter), completing on an mbarrier.  x is the innermost
// coordinate (elements; here always 0, so 16-byte aligned).  No multicast.
__device__ __forceinline__ void tma_load_2d(std::uint32_t dst, const void* tmap, int x, int y, std::uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(tmap), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared -> global tile store through a tensor map (rows past the tensor's
// extent are not written); completion is tracked by bulk groups.
__device__ __forceinline__ void tma_store_2d(const void* tmap, std::uint32_t src, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%2, %3}], [%1];" ::"l"(tmap),
                 "r"(src), "r"(x), "r"(y)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Wait until every committed bulk store has finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Wait until at most the latest committed bulk store may still be reading
// shared memory.
__device__ __forceinline__ void bulk_wait_read_all_but_one()
{
    asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}

// Wait until every committed bulk store has completed.
__device__ __forceinline__ void bulk_wait_all()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Four rows r0..r3 (box one row high) into 4 consecutive box-sized slots.
__device__ __forceinline__ void tma_gather4(std::uint32_t dst, const void* tmap, int x, int r0, int r1, int r2, int r3,
                                            std::uint32_t bar, std::uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7], %8;" ::"r"(dst),
        "l"(tmap), "r"(x), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(bar), "l"(policy)
        : "memory");
}

__device__ __forceinline__ std::uint64_t l2_policy_evict_normal()
{
    std::uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}

}  // namespace owtk::dev
