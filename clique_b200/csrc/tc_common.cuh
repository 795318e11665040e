// tcgen05 / mbarrier / bulk-copy helpers shared by the tensor-core kernels
// (tc_gemm2.cu, tc_panel.cu).  Operand blocks in shared memory use the
// K-major canonical layout without swizzle: 8-row x 16-byte core matrices,
// K-adjacent cores 128 B apart (LBO), 8-row groups 256 B apart (SBO).
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

namespace cliqgpu {
namespace tc2 {

constexpr uint64_t kWaitNs = 200000000ull;   // 0.2 s bound on any mbarrier wait

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t gns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t c) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(c) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ uint32_t mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, int32_t* status, int site) {
    if (mbar_try(b, parity)) return true;
    const uint64_t t0 = gns();
    while (!mbar_try(b, parity)) {
        if (gns() - t0 > kWaitNs) {
            atomicExch(&status[1], 1);
            atomicCAS(&status[2], 0, site);
            return false;
        }
    }
    return true;
}
// 1-D bulk copy global -> shared, completion counted on the mbarrier
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(su32(dst)), "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ uint64_t sdesc(uint32_t a, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool negA) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}
// kind::f16 instruction descriptor: F32 accumulator (bits 4-5 = 1), A and B
// FP16 (format 0 at bits 7-9 and 10-12), negate-A bit 13, N >> 3 at bit 17,
// M >> 4 at bit 24
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool negA) {
    return (1u << 4) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
// C -= v without reading C: one reduction per element per launch, so the
// result equals the load-subtract-store it replaces (same rounding, no race)
__device__ __forceinline__ void red_sub(float* p, float v) {
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(-v) : "memory");
}
__device__ __forceinline__ void red_sub2(float* p, float re, float im) {
    asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(-re), "f"(-im) : "memory");
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }
__device__ __forceinline__ uint32_t core_off(int row, int chunk) { return (row >> 3) * 256 + chunk * 128 + (row & 7) * 16; }

__device__ __forceinline__ uint32_t h2pack(__half a, __half b) {
    return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}
// one plane chunk: 8 consecutive k of one row as fp16 hi and lo
__device__ __forceinline__ void split8(const float* y, uint4& hi, uint4& lo) {
    __half h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        h[q] = __float2half_rn(y[q]);
        l[q] = __float2half_rn(y[q] - __half2float(h[q]));
    }
    hi = make_uint4(h2pack(h[0], h[1]), h2pack(h[2], h[3]), h2pack(h[4], h[5]), h2pack(h[6], h[7]));
    lo = make_uint4(h2pack(l[0], l[1]), h2pack(l[2], l[3]), h2pack(l[4], l[5]), h2pack(l[6], l[7]));
}

}  // namespace tc2
}  // namespace cliqgpu
