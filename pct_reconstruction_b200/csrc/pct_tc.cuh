// pct_tc.cuh -- sm_100a tensor-core primitives (tcgen05 + TMEM + mbarrier) used by the learned
// initializer's convolution kernels (pct_unet.cu).
//
// Conventions (PTX ISA, tcgen05 family):
//  * one CTA (cta_group::1) issues M = 128 MMAs; the accumulator D (128 x N fp32) lives in tensor
//    memory, lane i = row i, one 32-bit column per output column;
//  * A and B are read from shared memory through 64-bit matrix descriptors in the canonical
//    no-swizzle layout: the operand is tiled into 8-row x 16-byte core matrices (128 contiguous
//    bytes); LBO is the byte distance between core matrices adjacent along K, SBO between core
//    matrices adjacent along M (or N);
//  * a K-major operand keeps 8 consecutive K elements of one row in a core-matrix row; an
//    MN-major operand keeps 8 consecutive M (N) elements of one K index in a core-matrix row;
//  * an MMA is issued by one thread; tcgen05.commit makes an mbarrier track its completion;
//  * every wait on an mbarrier here is bounded in time and reports expiry to the caller.
#pragma once

#include <cstdint>

namespace pct {
namespace tc {

constexpr int kTileM = 128;
// Bound on a single mbarrier wait: the MMAs it waits for take microseconds.
constexpr unsigned long long kWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// Shared-memory matrix descriptor of a K-major operand in a swizzled layout, as TMA writes it with
// CU_TENSOR_MAP_SWIZZLE_{32,64,128}B when every row holds exactly `row_bytes` = 32, 64 or 128 bytes
// of K: rows are row_bytes apart, 8-row groups 8 * row_bytes apart (SBO), LBO unused; the tile
// base must be aligned to the swizzle atom (8 * row_bytes).  A K step inside the row advances the
// start address by its byte offset.
__device__ __forceinline__ uint64_t smem_desc_swizzled(uint32_t addr, uint32_t row_bytes)
{
    const uint64_t layout = row_bytes == 128 ? 2u : row_bytes == 64 ? 4u : 6u;  // SWIZZLE_128B / 64B / 32B
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(((8u * row_bytes) >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= layout << 61;
    return d;
}

// mbarrier: one arrival that also announces the bytes the TMA copies will deliver
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(bytes) : "memory");
}

// TMA tiled loads of this CTA's own tile into its shared memory, completion counted on mbar.  The innermost
// coordinate must be a multiple of 16 bytes; the others may fall outside the tensor (zero fill).
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void* tmap, uint32_t mbar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        :: "r"(dst), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(mbar), "r"(c0), "r"(c1), "r"(c2) : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* tmap, uint32_t mbar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
        :: "r"(dst), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(mbar), "r"(c0), "r"(c1), "r"(c2), "r"(c3) : "memory");
}

// Instruction descriptor for kind::f16 with bf16 A and B, fp32 D, M = 128, dense.
// mn_major selects MN-major A and B (bits 15 and 16); otherwise both are K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int n, bool mn_major)
{
    return (1u << 4)                                    // D format: f32
         | (1u << 7)                                    // A format: bf16
         | (1u << 10)                                   // B format: bf16
         | (mn_major ? ((1u << 15) | (1u << 16)) : 0u)  // A/B major
         | (static_cast<uint32_t>(n >> 3) << 17)        // N / 8
         | (static_cast<uint32_t>(kTileM >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(mbar) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory stores -> visible to the tensor core's (async proxy) reads.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
    return done != 0;
}

// Wait for the phase of the given parity to complete; false if kWaitNs passed first.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity)
{
    if (mbar_test(mbar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test(mbar, parity)) {
        if (global_ns() - t0 > kWaitNs) return false;
    }
    return true;
}

// TMEM allocation by one full warp; the column base is written to shared memory at slot.
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(slot), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31).
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM columns to allocate for an N-column accumulator: a power of two, at least 32.
__host__ __device__ constexpr uint32_t tmem_columns(int n)
{
    return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : 256u;
}

}  // namespace tc
}  // namespace pct
