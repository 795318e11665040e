// Panel of the front LDL^T on the tensor cores (FP32 / complex-FP32 fronts):
//     L21 = A21 W,   W = U D^{-1},   U = op(L11^{-1})^T
// for one 128-row tile of the rows below a 64-wide diagonal block (the Trsm
// of FrontLDL, include/clique/numeric/ldl/local_front.hpp:56-62).
//
// One CTA per tile, 192 threads:
//   warps 0-3  thread = tile row: find the row's largest |Re|, |Im| over
//              its 64 columns, write the row of A21 scaled by a power of two
//              as FP16 hi / lo planes into shared memory; later the
//              epilogue for the same row.
//   warps 4-5  thread = column c of W: the same for row c of the B operand,
//              B[c][t] = W[t][c] = U[t][c] / d_c; warp 4 lane 0 then issues
//              the tcgen05.mma kind::f16 (M = 128, N = 64, K = 16) products.
// The 2xFP16 split and its accuracy are those of the update kernel
// (tc_gemm2.cu): X = X_hi + X_lo after row scaling, three products per
// real product.  The epilogue multiplies by the two inverse scales, writes
// L21 and the row maxima of L21 and of S21 = L21 D that the update kernels'
// operand packing uses, and the row-major copies of the tiles (b+1, b) and
// (b+2, b) for the backward solve.
#include "cliqgpu_internal.h"
#include "device_common.cuh"
#include "tc_common.cuh"

namespace cliqgpu {
namespace tc2 {

constexpr int kPanelRows = 128;
constexpr int kPanelThreads = 192;
constexpr int kPanelK = kTile;                    // 64 columns of the diagonal block
constexpr int kPanelKS = 16;                      // k per kind::f16 MMA
constexpr int kPanelSteps = kPanelK / kPanelKS;   // 4

template <bool C>
struct PanelCfg {
    static constexpr int kPlanes = C ? 4 : 2;
    static constexpr int kABlock = kPanelRows * kPanelKS * 2;   // bytes of one plane, one k step: 4 KB
    static constexpr int kBBlock = kTile * kPanelKS * 2;        // 2 KB
    static constexpr int kABytes = kPlanes * kPanelSteps * kABlock;
    static constexpr int kBBytes = kPlanes * kPanelSteps * kBBlock;
    static constexpr int kTmem = C ? 128 : 64;
};

template <bool C>
__host__ __device__ constexpr size_t panel_tc_smem() {
    // operand planes, inverse scales (A rows, B rows), pivots, mbarrier, TMEM slot, 1 KB alignment slack
    return (size_t)PanelCfg<C>::kABytes + PanelCfg<C>::kBBytes + 4 * (kPanelRows + kTile) + 8 * 2 * kTile + 64 + 1024;
}

__device__ __forceinline__ float cmax(float v) { return fabsf(v); }
__device__ __forceinline__ float cmax(cx<float> v) { return fmaxf(fabsf(v.r), fabsf(v.i)); }

// one operand row (64 k values, already scaled) into the planes at `base`
// (plane stride `pstride`, k-step stride `kstride`)
template <bool C>
__device__ __forceinline__ void put_row16(uint8_t* base, int row, int ks, const V<float, C>* v, int pstride, int kstride) {
    float y[16];
    uint4 h, l;
    uint8_t* b = base + ks * kstride;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        if constexpr (C) y[q] = v[q].r; else y[q] = v[q];
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        split8(y + 8 * c, h, l);
        *reinterpret_cast<uint4*>(b + 0 * pstride + core_off(row, c)) = h;
        *reinterpret_cast<uint4*>(b + 1 * pstride + core_off(row, c)) = l;
    }
    if constexpr (C) {
#pragma unroll
        for (int q = 0; q < 16; ++q) y[q] = v[q].i;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            split8(y + 8 * c, h, l);
            *reinterpret_cast<uint4*>(b + 2 * pstride + core_off(row, c)) = h;
            *reinterpret_cast<uint4*>(b + 3 * pstride + core_off(row, c)) = l;
        }
    }
}

// power-of-two scale s with s * mx in [2^14, 2^15); returns s, stores 1/s
__device__ __forceinline__ float row_scale(float mx, float* inv) {
    int e = mx > 0.f ? ((__float_as_int(mx) >> 23) & 0xff) - 127 : 0;
    e = max(-100, min(100, e));
    *inv = __int_as_float((127 - 14 + e) << 23);
    return __int_as_float((127 + 14 - e) << 23);
}

template <bool C>
__global__ void __launch_bounds__(kPanelThreads, 2) panel_tc_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                                    int k, float* __restrict__ L, const double* __restrict__ D,
                                                                    const float* __restrict__ tinv, uint32_t* __restrict__ eblk,
                                                                    uint32_t* __restrict__ erow, int64_t eblk_total,
                                                                    int64_t erow_total, int32_t* __restrict__ status,
                                                                    const GemmProb* __restrict__ probs, float* __restrict__ pack,
                                                                    int conj) {
    using X = V<float, C>;
    using W = DV<C>;
    using PC = PanelCfg<C>;
    constexpr int nb = kTile;
    if (cta_timed_out(status)) return;   // an earlier wait timed out
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sAop = smem;                                   // A planes: [plane][k step][128 rows x 32 B]
    uint8_t* sBop = sAop + PC::kABytes;                     // B planes: [plane][k step][64 rows x 32 B]
    float* inv_a = reinterpret_cast<float*>(sBop + PC::kBBytes);
    float* inv_b = inv_a + kPanelRows;
    X* s_d = reinterpret_cast<X*>(inv_b + nb);             // pivots (FP32), for S21 = L21 D
    uint64_t* done = reinterpret_cast<uint64_t*>(s_d + nb);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);

    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int slot = it.y, tile = it.z;
    const int kb = min(nb, f.n - k);
    const int r0 = k + kb + kPanelRows * tile;             // first front row of this tile
    const int rows = min(kPanelRows, f.m - r0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // the in-panel update's packing parameters, fetched now so that the
    // epilogue does not wait for them
    __shared__ int64_t s_pk[4];   // packA, packB, scaleA, scaleB (float offsets)
    __shared__ int32_t s_pkn[2];  // K, N
    const bool prepack = probs && it.w >= 0;
    if (threadIdx.x == 0) {
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x == kPanelRows && prepack) {
        const GemmProb& pr = probs[it.w];
        s_pk[0] = pr.packA; s_pk[1] = pr.packB; s_pk[2] = pr.scaleA; s_pk[3] = pr.scaleB;
        s_pkn[0] = pr.K; s_pkn[1] = pr.N;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)), "r"(PC::kTmem) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x < kPanelRows) {
        // ---- A: row i of A21, all 64 columns loaded at once into registers ----
        const int i = threadIdx.x;
        const bool vr = i < rows;
        const int64_t a0 = f.L + r0 + i + (int64_t)k * f.m;
        X v[nb];
#pragma unroll
        for (int t = 0; t < nb; ++t) v[t] = (vr && t < kb) ? ldv<float, C>(L, a0 + (int64_t)t * f.m) : X{};
        float mx = 0.f;
#pragma unroll
        for (int t = 0; t < nb; ++t) mx = fmaxf(mx, cmax(v[t]));
        float inv;
        const float s = row_scale(mx, &inv);
        inv_a[i] = inv;
#pragma unroll
        for (int t = 0; t < nb; ++t) v[t] = v[t] * s;
#pragma unroll
        for (int ks = 0; ks < kPanelSteps; ++ks)
            if (16 * ks < kb) put_row16<C>(sAop, i, ks, v + 16 * ks, kPanelSteps * PC::kABlock, PC::kABlock);
    } else {
        // ---- B: row c of W^T, B[c][t] = U[t][c] / d_c ----
        const int c = threadIdx.x - kPanelRows;
        const X* U = reinterpret_cast<const X*>(tinv) + (int64_t)slot * nb * nb;
        X rd{};
        if (c < kb) {
            const W d = reinterpret_cast<const W*>(D)[f.off + k + c];
            rd = conv<X>(W{} + vone<W>() / d);
            s_d[c] = conv<X>(d);
        } else {
            s_d[c] = X{};
        }
        X v[nb];
#pragma unroll
        for (int t = 0; t < nb; ++t) v[t] = (t < kb && c < kb) ? U[t * nb + c] : X{};
        float mx = 0.f;
#pragma unroll
        for (int t = 0; t < nb; ++t) {
            v[t] = v[t] * rd;
            mx = fmaxf(mx, cmax(v[t]));
        }
        float inv;
        const float s = row_scale(mx, &inv);
        inv_b[c] = inv;
#pragma unroll
        for (int t = 0; t < nb; ++t) v[t] = v[t] * s;
#pragma unroll
        for (int ks = 0; ks < kPanelSteps; ++ks)
            if (16 * ks < kb) put_row16<C>(sBop, c, ks, v + 16 * ks, kPanelSteps * PC::kBBlock, PC::kBBlock);
    }
    // operands written by the generic proxy, read by the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 4) {
        if (lane == 0) {
            const uint32_t idp = idesc_f16(kPanelRows, nb, false), idn = idesc_f16(kPanelRows, nb, true);
            const uint32_t dre = tmem, dim = tmem + nb;
            const uint32_t a = su32(sAop), b = su32(sBop);
            // k steps past the block's kb columns hold zeros: skipped (small fronts, last blocks)
            for (int ks = 0; 16 * ks < kb; ++ks) {
                auto A = [&](int p) { return sdesc(a + (p * kPanelSteps + ks) * PC::kABlock, 128, 256); };
                auto B = [&](int p) { return sdesc(b + (p * kPanelSteps + ks) * PC::kBBlock, 128, 256); };
                const uint32_t acc = ks > 0 ? 1u : 0u;
                mma_f16(dre, A(0), B(0), idp, acc);
                mma_f16(dre, A(0), B(1), idp, 1u);
                mma_f16(dre, A(1), B(0), idp, 1u);
                if constexpr (C) {
                    mma_f16(dre, A(2), B(2), idn, 1u);
                    mma_f16(dre, A(2), B(3), idn, 1u);
                    mma_f16(dre, A(3), B(2), idn, 1u);
                    mma_f16(dim, A(0), B(2), idp, acc);
                    mma_f16(dim, A(0), B(3), idp, 1u);
                    mma_f16(dim, A(1), B(2), idp, 1u);
                    mma_f16(dim, A(2), B(0), idp, 1u);
                    mma_f16(dim, A(2), B(1), idp, 1u);
                    mma_f16(dim, A(3), B(0), idp, 1u);
                }
            }
            mma_commit(done);
        }
        __syncwarp();
    } else if (warp < 4) {
        // ---- epilogue: thread = row i (TMEM lane i) ----
        const bool ok = mbar_wait(done, 0, status, 6);
        tc_fence_after();
        if (ok) {
            const int i = warp * 32 + lane;
            const bool vr = i < rows;
            const float ia = inv_a[i];
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
            const int nT = (f.n + nb - 1) / nb;
            float ml = 0.f, ms = 0.f;
#pragma unroll 1
            for (int c0 = 0; c0 < nb; c0 += 16) {
                float re[16], im[16];
                tmem_ld16(lane_base + c0, re);
                if constexpr (C) tmem_ld16(lane_base + nb + c0, im);
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int c = c0 + q;
                    const float sc = ia * inv_b[c];
                    X v;
                    if constexpr (C) v = X{re[q] * sc, im[q] * sc}; else v = re[q] * sc;
                    if (c >= kb) v = X{};
                    if (vr && c < kb) {
                        stv<float, C>(L, f.L + r0 + i + (int64_t)(k + c) * f.m, v);
                        ml = fmaxf(ml, cmax(v));
                        ms = fmaxf(ms, cmax(v * s_d[c]));
                    }
                }
            }
            if (eblk && vr) {
                const int64_t row = r0 + i;
                const int64_t eb = f.eblk + row * nT + k / nb;
                eblk[eb] = __float_as_uint(ml);
                eblk[eblk_total + eb] = __float_as_uint(ms);
                atomicMax(&erow[f.erow + row], __float_as_uint(ml));
                atomicMax(&erow[erow_total + f.erow + row], __float_as_uint(ms));
            }
            // packed operands of the following in-panel update (rows of this
            // tile are rows tile*128 + i of its problem, K = kb): the A planes
            // scaled by the row maximum ml, and for the first N problem rows
            // the S = D op(L21) planes scaled by ms, in the layout and with
            // the scales the operand packing would produce
            if (prepack) {
                const int64_t packA = s_pk[0], packB = s_pk[1], scaleA = s_pk[2], scaleB = s_pk[3];
                const int pK = s_pkn[0], pN = s_pkn[1];
                const int rp = tile * kPanelRows + i;   // row in the problem
                const int nks = (pK + 15) / 16;
                const bool srow = tile * kPanelRows < pN;
                constexpr int planes = C ? 4 : 2;
                constexpr int64_t plane_bytes = (int64_t)kPanelRows * 16 * 2;
                auto scale_of = [](float mx, float* inv) {
                    int e = mx > 0.f ? ((__float_as_int(mx) >> 23) & 0xff) - 127 : 0;
                    e = max(-100, min(100, e));
                    *inv = __int_as_float((127 - 14 + e) << 23);
                    return __int_as_float((127 + 14 - e) << 23);
                };
                float inv_sa, inv_ss;
                const float sa = scale_of(vr ? ml : 0.f, &inv_sa), ss = scale_of(vr && rp < pN ? ms : 0.f, &inv_ss);
                pack[scaleA + rp] = inv_sa;
                if (srow) pack[scaleB + rp] = inv_ss;
#pragma unroll 1
                for (int ks = 0; ks < nks; ++ks) {
                    float re[16], im[16];
                    tmem_ld16(lane_base + 16 * ks, re);
                    if constexpr (C) tmem_ld16(lane_base + nb + 16 * ks, im);
                    X v[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const int c = 16 * ks + q;
                        const float sc = ia * inv_b[c];
                        if constexpr (C) v[q] = X{re[q] * sc, im[q] * sc}; else v[q] = re[q] * sc;
                        if (c >= kb || !vr) v[q] = X{};
                    }
                    const int64_t blk = (int64_t)tile * nks + ks;
                    uint8_t* base = reinterpret_cast<uint8_t*>(pack + packA) + blk * plane_bytes * planes;
                    float y[16];
                    uint4 h, l;
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        if constexpr (C) y[q] = v[q].r * sa; else y[q] = v[q] * sa;
                    }
#pragma unroll
                    for (int cc = 0; cc < 2; ++cc) {
                        split8(y + 8 * cc, h, l);
                        *reinterpret_cast<uint4*>(base + 0 * plane_bytes + core_off(i, cc)) = h;
                        *reinterpret_cast<uint4*>(base + 1 * plane_bytes + core_off(i, cc)) = l;
                    }
                    if constexpr (C) {
#pragma unroll
                        for (int q = 0; q < 16; ++q) y[q] = v[q].i * sa;
#pragma unroll
                        for (int cc = 0; cc < 2; ++cc) {
                            split8(y + 8 * cc, h, l);
                            *reinterpret_cast<uint4*>(base + 2 * plane_bytes + core_off(i, cc)) = h;
                            *reinterpret_cast<uint4*>(base + 3 * plane_bytes + core_off(i, cc)) = l;
                        }
                    }
                    if (srow) {
#pragma unroll
                        for (int q = 0; q < 16; ++q) {
                            X sv = v[q];
                            if constexpr (C) { if (conj) sv.i = -sv.i; }
                            v[q] = rp < pN ? s_d[16 * ks + q] * sv : X{};
                        }
                        uint8_t* bs = reinterpret_cast<uint8_t*>(pack + packB) + blk * plane_bytes * planes;
#pragma unroll
                        for (int q = 0; q < 16; ++q) {
                            if constexpr (C) y[q] = v[q].r * ss; else y[q] = v[q] * ss;
                        }
#pragma unroll
                        for (int cc = 0; cc < 2; ++cc) {
                            split8(y + 8 * cc, h, l);
                            *reinterpret_cast<uint4*>(bs + 0 * plane_bytes + core_off(i, cc)) = h;
                            *reinterpret_cast<uint4*>(bs + 1 * plane_bytes + core_off(i, cc)) = l;
                        }
                        if constexpr (C) {
#pragma unroll
                            for (int q = 0; q < 16; ++q) y[q] = v[q].i * ss;
#pragma unroll
                            for (int cc = 0; cc < 2; ++cc) {
                                split8(y + 8 * cc, h, l);
                                *reinterpret_cast<uint4*>(bs + 2 * plane_bytes + core_off(i, cc)) = h;
                                *reinterpret_cast<uint4*>(bs + 3 * plane_bytes + core_off(i, cc)) = l;
                            }
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(PC::kTmem) : "memory");
    }
}

}  // namespace tc2

// launch the tensor-core panel for one PANEL step of the schedule
int launch_panel_tc(Plan& P, const Launch& ln, cudaStream_t st, void* pack) {
    const GemmProb* probs = ln.pk_probs >= 0 ? P.probs + ln.pk_probs : nullptr;
    float* L = reinterpret_cast<float*>(P.L);
    const int4* items = reinterpret_cast<const int4*>(P.items) + ln.items;
    static bool attr[2] = {false, false};
    if (P.cplx()) {
        const size_t smem = tc2::panel_tc_smem<true>();
        if (!attr[1]) { cudaFuncSetAttribute(tc2::panel_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); attr[1] = true; }
        tc2::panel_tc_kernel<true><<<(unsigned)ln.nblocks, tc2::kPanelThreads, smem, st>>>(
            P.fronts, items, ln.k, L, P.D, reinterpret_cast<const float*>(P.tinv), P.eblk, P.erow, P.eblk_total, P.erow_total, P.status, probs,
            reinterpret_cast<float*>(pack), P.conjugate);
    } else {
        const size_t smem = tc2::panel_tc_smem<false>();
        if (!attr[0]) { cudaFuncSetAttribute(tc2::panel_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); attr[0] = true; }
        tc2::panel_tc_kernel<false><<<(unsigned)ln.nblocks, tc2::kPanelThreads, smem, st>>>(
            P.fronts, items, ln.k, L, P.D, reinterpret_cast<const float*>(P.tinv), P.eblk, P.erow, P.eblk_total, P.erow_total, P.status, probs,
            reinterpret_cast<float*>(pack), P.conjugate);
    }
    return CLIQ_OK;
}

}  // namespace cliqgpu
