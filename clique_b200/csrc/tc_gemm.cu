// Tensor-core (tcgen05, kind::tf32) update kernel for FP32 / complex-FP32 fronts:
//     C[i, j] -= sum_k A[i, k] * d[k] * op(B[j, k])      for i >= j
// which is both the in-panel update and the Schur-complement update
// ABR -= L_B D L_B^T of FrontLDL (include/clique/numeric/ldl/local_front.hpp:67-69).
//
// Precision: every product runs as three TF32 products (the "3xTF32" split
// X = X_hi + X_lo, X_hi = X with the low 13 mantissa bits cleared):
//     A B ~= A_hi B_hi + A_hi B_lo + A_lo B_hi
// accumulated in FP32 in tensor memory, which recovers close to FP32 accuracy
// (the refinement loop then restores FP64 accuracy).
//
// Complex data is split into real planes (planar form): with S = d * op(B),
//     Re C -= Ar Sr^T - Ai Si^T,    Im C -= Ar Si^T + Ai Sr^T,
// the minus sign coming from the instruction descriptor's negate-A bit.  Per
// 8-wide k step a complex tile issues 12 MMAs of 128 x 128 x 8 (2 outputs x 2
// terms x 3 split products); a real tile issues 3.
//
// CTA layout (160 threads): warps 0-3 load their row of A and of B from
// global memory, split and scale it, and write the canonical K-major
// no-swizzle layout into a 3-stage shared-memory ring (core matrices of
// 8 rows x 16 bytes, K-adjacent cores 128 B apart, 8-row groups 256 B apart);
// warp 4 issues tcgen05.mma from one elected thread and releases each stage
// with tcgen05.commit; at the end warps 0-3 read the accumulators with
// tcgen05.ld (each warp owns 32 TMEM lanes = 32 rows) and update C.
// Every mbarrier wait is bounded: on expiry the status word records a
// timeout and the CTA still frees its tensor memory and exits.
#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

namespace tc {

constexpr int kBM = 128, kBN = 128, kKS = 8;     // tile rows, tile columns, k per step
constexpr int kStages = 3;
constexpr int kProducers = 128;                  // warps 0-3
constexpr int kThreads = kProducers + 32;        // + MMA warp
constexpr int kPlaneBytes = kBM * kKS * 4;       // 4 KB: 128 rows x 8 tf32
constexpr uint64_t kWaitNs = 200000000ull;       // 0.2 s bound on any single wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ uint32_t mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wall-clock-bounded wait on an mbarrier phase.  On expiry: status[1] = 1,
// status[2] = the wait site (1 stage full, 2 stage empty, 3 accumulator done),
// and false is returned so that the CTA can release its tensor memory.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* status, int site) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (global_ns() - t0 > kWaitNs) {
            atomicExch(&status[1], 1);
            atomicCAS(&status[2], 0, site);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// shared-memory matrix descriptor: no swizzle, K-major canonical layout
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;    // descriptor version for sm_100
    return d;                   // base offset 0, absolute LBO mode, layout SWIZZLE_NONE
}

// instruction descriptor: kind::tf32, FP32 accumulate, both operands K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool negA) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((negA ? 1u : 0u) << 13) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
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

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// offset of (row, chunk) inside a plane: 8-row groups 256 B apart, K chunks 128 B apart
__device__ __forceinline__ uint32_t plane_off(int row, int chunk) { return (row >> 3) * 256 + chunk * 128 + (row & 7) * 16; }

template <bool C>
struct Planes {
    static constexpr int kA = C ? 4 : 2;   // A: re_hi, re_lo, (im_hi, im_lo)
    static constexpr int kB = C ? 4 : 2;   // S = d op(B): re_hi, re_lo, (im_hi, im_lo)
    static constexpr int kStageBytes = (kA + kB) * kPlaneBytes;
    static constexpr int kTmemCols = C ? 256 : 128;
};

// write hi/lo of 8 values (one row, one k step) into two planes
__device__ __forceinline__ void put_split(uint8_t* hi_plane, uint8_t* lo_plane, int row, const float* v) {
    float h[8], l[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { h[q] = tf32_hi(v[q]); l[q] = v[q] - h[q]; }
    *reinterpret_cast<float4*>(hi_plane + plane_off(row, 0)) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(hi_plane + plane_off(row, 1)) = make_float4(h[4], h[5], h[6], h[7]);
    *reinterpret_cast<float4*>(lo_plane + plane_off(row, 0)) = make_float4(l[0], l[1], l[2], l[3]);
    *reinterpret_cast<float4*>(lo_plane + plane_off(row, 1)) = make_float4(l[4], l[5], l[6], l[7]);
}

template <bool C, bool CJ>
__global__ void __launch_bounds__(kThreads) tc_update_kernel(const GemmProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                             int nprobs, float* __restrict__ L, float* __restrict__ pool0,
                                                             float* __restrict__ pool1, const double* __restrict__ D,
                                                             int32_t* __restrict__ status) {
    using PL = Planes<C>;
    // after a recorded timeout every later CTA returns at once instead of waiting again
    if (*reinterpret_cast<volatile int32_t*>(&status[1]) != 0) return;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * PL::kStageBytes);
    uint64_t* empty = full + kStages;
    uint64_t* done = empty + kStages;
    uint32_t* tmem_base_slot = reinterpret_cast<uint32_t*>(done + 1);

    // ---- which tile ----
    const int64_t bid = blockIdx.x;
    int lo = 0, hi = nprobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= bid) lo = mid; else hi = mid - 1;
    }
    const GemmProb pr = probs[lo];
    int64_t t = bid - prefix[lo];
    const int Mt = (pr.M + kBM - 1) / kBM, Nt = (pr.N + kBN - 1) / kBN;
    int tj = 0;
    while (tj < Nt && t >= Mt - tj) { t -= Mt - tj; ++tj; }
    if (tj >= Nt) {   // inconsistent schedule: record it and do nothing
        if (threadIdx.x == 0) { atomicExch(&status[1], 1); atomicCAS(&status[2], 0, 5); }
        return;
    }
    const int i0 = ((int)t + tj) * kBM, j0 = tj * kBN;
    const int nk = (pr.K + kKS - 1) / kKS;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], kProducers); mbar_init(&empty[s], 1); }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) { tmem_alloc(tmem_base_slot, PL::kTmemCols); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_base_slot;

    if (warp == 4) {
        // ---------------- MMA issuer ----------------
        const uint32_t id_pos = idesc_tf32(kBM, kBN, false), id_neg = idesc_tf32(kBM, kBN, true);
        const uint32_t dre = tmem, dim = tmem + kBN;
        bool ok = true;
        for (int it = 0; it < nk && ok; ++it) {
            const int s = it % kStages;
            ok = mbar_wait(&full[s], (it / kStages) & 1, status, 1);
            if (!ok) break;
            tc_fence_after();
            if (lane == 0) {
                const uint32_t base = smem_u32(smem + s * PL::kStageBytes);
                auto dsc = [&](int plane) { return smem_desc(base + plane * kPlaneBytes, 128, 256); };
                const uint32_t acc = it > 0 ? 1u : 0u;
                // planes: A re_hi 0, re_lo 1, (im_hi 2, im_lo 3); S re_hi kA, re_lo kA+1, (im_hi kA+2, im_lo kA+3)
                constexpr int a_rh = 0, a_rl = 1, a_ih = 2, a_il = 3;
                constexpr int s_rh = PL::kA, s_rl = PL::kA + 1, s_ih = PL::kA + 2, s_il = PL::kA + 3;
                mma_tf32(dre, dsc(a_rh), dsc(s_rh), id_pos, acc);
                mma_tf32(dre, dsc(a_rh), dsc(s_rl), id_pos, 1u);
                mma_tf32(dre, dsc(a_rl), dsc(s_rh), id_pos, 1u);
                if constexpr (C) {
                    mma_tf32(dre, dsc(a_ih), dsc(s_ih), id_neg, 1u);
                    mma_tf32(dre, dsc(a_ih), dsc(s_il), id_neg, 1u);
                    mma_tf32(dre, dsc(a_il), dsc(s_ih), id_neg, 1u);
                    mma_tf32(dim, dsc(a_rh), dsc(s_ih), id_pos, acc);
                    mma_tf32(dim, dsc(a_rh), dsc(s_il), id_pos, 1u);
                    mma_tf32(dim, dsc(a_rl), dsc(s_ih), id_pos, 1u);
                    mma_tf32(dim, dsc(a_ih), dsc(s_rh), id_pos, 1u);
                    mma_tf32(dim, dsc(a_ih), dsc(s_rl), id_pos, 1u);
                    mma_tf32(dim, dsc(a_il), dsc(s_rh), id_pos, 1u);
                }
                mma_commit(&empty[s]);
                if (it == nk - 1) mma_commit(done);
            }
            __syncwarp();
        }
    } else {
        // ---------------- producers ----------------
        const int row = threadIdx.x;            // 0..127
        const int ia = i0 + row, jb = j0 + row;
        const bool va = ia < pr.M, vb = jb < pr.N;
        float* Cbase = pr.cpool < 0 ? L : (pr.cpool == 0 ? pool0 : pool1);
        using X = V<float, C>;
        using W = DV<C>;
        bool ok = true;
        for (int it = 0; it < nk; ++it) {
            const int s = it % kStages;
            X av[kKS], sv[kKS];
            const int k0 = it * kKS;
#pragma unroll
            for (int q = 0; q < kKS; ++q) {
                const int k = k0 + q;
                X a{}, b{};
                if (k < pr.K) {
                    if (va) a = ldv<float, C>(L, pr.A + ia + (int64_t)k * pr.lda);
                    if (vb) {
                        const X dk = conv<X>(reinterpret_cast<const W*>(D)[pr.d + k]);
                        b = dk * opc<CJ>(ldv<float, C>(L, pr.B + jb + (int64_t)k * pr.lda));
                    }
                }
                av[q] = a;
                sv[q] = b;
            }
            if (it >= kStages) {
                ok = mbar_wait(&empty[s], ((it / kStages) - 1) & 1, status, 2);
                if (!ok) break;
            }
            uint8_t* st = smem + s * PL::kStageBytes;
            float v[kKS];
            if constexpr (C) {
#pragma unroll
                for (int q = 0; q < kKS; ++q) v[q] = av[q].r;
                put_split(st + 0 * kPlaneBytes, st + 1 * kPlaneBytes, row, v);
#pragma unroll
                for (int q = 0; q < kKS; ++q) v[q] = av[q].i;
                put_split(st + 2 * kPlaneBytes, st + 3 * kPlaneBytes, row, v);
#pragma unroll
                for (int q = 0; q < kKS; ++q) v[q] = sv[q].r;
                put_split(st + (PL::kA + 0) * kPlaneBytes, st + (PL::kA + 1) * kPlaneBytes, row, v);
#pragma unroll
                for (int q = 0; q < kKS; ++q) v[q] = sv[q].i;
                put_split(st + (PL::kA + 2) * kPlaneBytes, st + (PL::kA + 3) * kPlaneBytes, row, v);
            } else {
#pragma unroll
                for (int q = 0; q < kKS; ++q) v[q] = av[q];
                put_split(st + 0 * kPlaneBytes, st + 1 * kPlaneBytes, row, v);
#pragma unroll
                for (int q = 0; q < kKS; ++q) v[q] = sv[q];
                put_split(st + (PL::kA + 0) * kPlaneBytes, st + (PL::kA + 1) * kPlaneBytes, row, v);
            }
            fence_async_smem();
            mbar_arrive(&full[s]);
        }
        // ---------------- epilogue ----------------
        if (ok) ok = mbar_wait(done, 0, status, 3);
        tc_fence_after();
        if (ok) {
            const int i = ia;   // TMEM lane = row of the tile
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
            for (int c0 = 0; c0 < kBN; c0 += 16) {
                float re[16], im[16];
                tmem_ld16(lane_base + c0, re);
                if constexpr (C) tmem_ld16(lane_base + kBN + c0, im);
                if (va) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const int j = j0 + c0 + q;
                        if (j < pr.N && i >= j) {
                            const int64_t e = pr.C + i + (int64_t)j * pr.ldc;
                            X cv = ldv<float, C>(Cbase, e);
                            if constexpr (C) { cv.r -= re[q]; cv.i -= im[q]; } else { cv -= re[q]; }
                            stv<float, C>(Cbase, e, cv);
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, PL::kTmemCols);
    }
}

}  // namespace tc

size_t tc_update_smem(bool cplx) {
    return (size_t)tc::kStages * (cplx ? tc::Planes<true>::kStageBytes : tc::Planes<false>::kStageBytes) + 1024 + 256;
}

// launch one GEMM-kind schedule entry on the tensor cores (FP32 storage only)
int launch_tc_update(Plan& P, const Launch& ln) {
    float* L = reinterpret_cast<float*>(P.L);
    float* p0 = reinterpret_cast<float*>(P.pool[0]);
    float* p1 = reinterpret_cast<float*>(P.pool[1]);
    const size_t smem = tc_update_smem(P.cplx());
    static bool attr[4] = {false, false, false, false};
    const int key = (P.cplx() ? 2 : 0) + (P.conjugate ? 1 : 0);
    if (P.cplx()) {
        if (P.conjugate) {
            if (!attr[key]) { cudaFuncSetAttribute(tc::tc_update_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); attr[key] = true; }
            tc::tc_update_kernel<true, true><<<(unsigned)ln.nblocks, tc::kThreads, smem, P.stream>>>(
                P.probs + ln.items, P.prefix + ln.prefix, ln.nitems, L, p0, p1, P.D, P.status);
        } else {
            if (!attr[key]) { cudaFuncSetAttribute(tc::tc_update_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); attr[key] = true; }
            tc::tc_update_kernel<true, false><<<(unsigned)ln.nblocks, tc::kThreads, smem, P.stream>>>(
                P.probs + ln.items, P.prefix + ln.prefix, ln.nitems, L, p0, p1, P.D, P.status);
        }
    } else {
        if (!attr[key]) { cudaFuncSetAttribute(tc::tc_update_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); attr[key] = true; }
        tc::tc_update_kernel<false, false><<<(unsigned)ln.nblocks, tc::kThreads, smem, P.stream>>>(
            P.probs + ln.items, P.prefix + ln.prefix, ln.nitems, L, p0, p1, P.D, P.status);
    }
    return CLIQ_OK;
}

}  // namespace cliqgpu
