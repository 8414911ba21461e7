// umma.cuh -- the Blackwell tensor-core plumbing of the surrogate's kernels: TMA tile loads
// into 128-byte-swizzled shared memory, mbarriers with bounded waits, tcgen05.mma (kind::f16,
// BF16 operands, FP32 accumulators in tensor memory) and tcgen05.ld of the accumulators.
//
// Operand layout.  Every operand tile is K-major: 128 rows (M or N) x 64 K-elements of BF16,
// 128 bytes a row, stored as TMA writes it with CU_TENSOR_MAP_SWIZZLE_128B -- eight-row atoms
// of 1,024 bytes in which the 16-byte chunk c of row r sits at chunk c ^ (r mod 8).  The
// matching shared-memory descriptor has layout type SWIZZLE_128B, a stride of 1,024 bytes
// between eight-row groups and (unused for this layout) a leading offset of 16 bytes; one
// MMA consumes K = 16, and the next K-slice of the same tile starts 32 bytes further on.
// Tiles start on 1,024-byte boundaries so the swizzle phase is zero.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace epsr {
namespace umma {

constexpr int TILE_M = 128;
constexpr int TILE_N = 128;
constexpr int TILE_K = 64;                                  // one 128-byte swizzle row of BF16
constexpr int TILE_BYTES = TILE_M * TILE_K * 2;             // 16 KB per operand tile
constexpr unsigned long long WAIT_NS = 2000000000ull;       // a wait gives up after 2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ----------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase with the given parity to complete; false (and *err set) after WAIT_NS.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (!mbar_try(bar, parity)) {
        if (globaltimer() - t0 > WAIT_NS) {
            if (err) atomicExch(err, 1);
            return false;
        }
    }
    return true;
}

// ----------------------------------------------------------------- TMA
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}
// generic-proxy shared-memory writes made visible to the async proxy (the MMA's operand reads)
// One contiguous copy global -> this CTA's shared memory by the bulk-copy engine, completing
// `bytes` of transaction on the mbarrier (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ----------------------------------------------------------------- tcgen05
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand tile.
__device__ __forceinline__ uint64_t sdesc_sw128(const void *tile) {
    const uint64_t a = (uint64_t)((smem_u32(tile) & 0x3FFFFu) >> 4);
    return a | (1ull << 16)                // leading byte offset 16 B (unused for this layout)
           | ((uint64_t)(1024 >> 4) << 32)  // stride byte offset: 1,024 B between eight-row groups
           | (1ull << 46)                  // descriptor version of tcgen05
           | (2ull << 61);                 // SWIZZLE_128B
}

// Instruction descriptor: kind::f16 with BF16 A and B, FP32 accumulator, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
    return (1u << 4)                      // accumulator F32
           | (1u << 7)                    // A BF16
           | (1u << 10)                   // B BF16
           | ((uint32_t)(n >> 3) << 17)   // N / 8
           | ((uint32_t)(m >> 4) << 24);  // M / 16
}

// D(tmem) (+)= A(smem desc) x B(smem desc)^T; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive once on the mbarrier when every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 columns of 32-bit accumulators: thread t of the warp gets row (lane base + t),
// columns col..col+15.  taddr = tmem base + (lane base << 16) + col.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace epsr
