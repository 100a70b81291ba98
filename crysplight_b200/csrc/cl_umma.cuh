// cl_umma.cuh — 5th-generation tensor-core (tcgen05) building blocks for sm_100a:
// shared-memory matrix descriptors, the BF16 x BF16 -> FP32 MMA with its
// accumulator in tensor memory (TMEM), TMEM allocation and loads, and bounded
// mbarrier waits.
//
// Operand layouts in shared memory.  (1) The canonical K-major layout without
// swizzle (make_desc), staged by ordinary stores.  (2) The K-major layout with
// the 128-byte swizzle (make_desc_sw128), written by TMA: a tile of R rows x
// 64 BF16 is R rows of 128 bytes, 8-row groups 1024 bytes apart (SBO), the
// 16-byte pieces of row r XOR-permuted by (r & 7); a K step of 16 elements
// advances the start address by 32 bytes inside the swizzle atom.
//
// Layout (1) in detail: the canonical K-major layout without
// swizzle.  A core matrix is 8 rows x 16 bytes (8 BF16 along K), its rows
// contiguous (128 bytes).  For a tile of R rows x KC K-elements, core matrix
// (row group g = r/8, K chunk c = k/8) sits at byte ((c * R/8) + g) * 128: row
// groups are 128 bytes apart (stride byte offset, SBO) and K chunks R*16
// bytes apart (leading byte offset, LBO).  One MMA instruction consumes K = 16,
// i.e. two K chunks starting at chunk 2s.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace cl {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) of an R-row K-major tile in the canonical layout.
__device__ __forceinline__ uint32_t tile_offset(uint32_t r, uint32_t k, uint32_t R)
{
    return (((k >> 3) * (R >> 3) + (r >> 3)) * 8u + (r & 7u)) * 16u + (k & 7u) * 2u;
}

// 64-bit shared-memory matrix descriptor (tcgen05 "matrix descriptor"):
// start address >> 4 in bits 0-13, LBO >> 4 in bits 16-29, SBO >> 4 in bits
// 32-45, descriptor version 1 in bits 46-47, base offset 0, no swizzle (0 in
// bits 61-63).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Descriptor of a 128-byte-swizzled K-major tile (1024-byte aligned base):
// LBO unused (1), SBO = 1024 bytes, layout type 2 (SWIZZLE_128B) in bits 61-63.
__device__ __forceinline__ uint64_t make_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Descriptor of a 128-byte-swizzled MN-major tile, as TMA writes boxes of
// 64 MN-elements (128 bytes) x 64 K-rows: swizzle atoms of 64 MN-elements x
// 8 K-rows (1 KB), consecutive 8-row K groups SBO = 1024 bytes apart,
// consecutive 64-element MN groups LBO bytes apart (the box size, 8 KB); a K
// step of 16 advances the start address by two atoms (2 KB).
__device__ __forceinline__ uint64_t make_desc_sw128_mn(uint32_t saddr, uint32_t lbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// 32-bit instruction descriptor for kind::f16: D = F32 (bits 4-5 = 1),
// A = B = BF16 (bits 7-9, 10-12 = 1), A and B K-major (0) or MN-major (1) in
// bits 15 and 16, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t make_idesc_bf16(int M, int N, bool a_mn = false, bool b_mn = false)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on an mbarrier when all previously issued MMAs of this thread complete.
__device__ __forceinline__ void commit(uint64_t* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the mbarrier phase with parity `phase`; gives up after `budget`
// polls and returns false (the caller records an error instead of hanging).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t phase, uint32_t budget)
{
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < budget; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok) : "r"(a), "r"(phase) : "memory");
        if (ok) return true;
    }
    return false;
}

// Same, but also gives up as soon as *abort is set by another thread.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* mbar, uint32_t phase, uint32_t budget,
                                                   volatile int* abort)
{
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < budget; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok) : "r"(a), "r"(phase) : "memory");
        if (ok) return true;
        if ((i & 63u) == 63u && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(mbar)) : "memory");
}

// Arrive and add `bytes` to the transaction count the current phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

// 2-D tiled TMA load of the box at element coordinates (x = inner, y = row)
// into this CTA's shared memory; completion counted on `mbar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int32_t x, int32_t y, uint64_t* mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :: "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(mbar))
        : "memory");
}

// 2-D tiled TMA store of a shared-memory box to element coordinates (x =
// inner, y = row); completion tracked by bulk groups of the issuing thread.
__device__ __forceinline__ void tma_store_2d(const void* tmap, int32_t x, int32_t y, const void* src)
{
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                 :: "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_u32(src)) : "memory");
}

__device__ __forceinline__ void bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Wait until every committed bulk store of this thread has read its source.
__device__ __forceinline__ void bulk_wait_read0()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Wait until every committed bulk store of this thread is complete.
__device__ __forceinline__ void bulk_wait0()
{
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void prefetch_tmap(const void* tmap)
{
    asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}

// Generic-proxy shared-memory writes -> visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// TMEM allocation by one full warp; the column base lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(slot)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32w..32w+31; taddr carries the lane in bits 16-31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace cl
