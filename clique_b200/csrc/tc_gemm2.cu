// Tensor-core update for FP32 / complex-FP32 fronts, fed by TMA bulk copies:
//     C[i, j] -= sum_k A[i, k] * d[k] * op(B[j, k])      for i >= j
// (FrontLDL's in-panel Gemm and Schur-complement Trrk,
// include/clique/numeric/ldl/local_front.hpp:67-69).
//
// Two kernels per schedule entry:
//  * pack_kernel writes every operand panel once into a scratch buffer in
//    exactly the shared-memory layout tcgen05.mma reads: planes (Re, Im)
//    x (hi, lo) of the 3xTF32 split, K-major canonical no-swizzle layout
//    (8-row x 16-byte core matrices; K-adjacent cores 128 B apart; 8-row
//    groups 256 B apart), one contiguous block per (row tile, 8-wide k step).
//    The B operand is packed already scaled, S = d * op(B).
//  * tc_gemm_kernel streams those blocks with cp.async.bulk (one elected
//    producer thread, mbarrier transaction counts) through a 4-stage ring,
//    one elected thread issues 12 (complex) or 3 (real) tcgen05.mma of
//    128 x kTcBN per k step into two kTcBN-column TMEM accumulators (Re, Im),
//    and four epilogue warps read them back with tcgen05.ld and update C.
//    With 128 x 128 tiles (256 TMEM columns, 3 stages of 32 KB) two CTAs
//    share an SM, so one CTA's epilogue overlaps the other's products.
// The 3xTF32 split: X = X_hi + X_lo, X_hi = X with the low 13 mantissa bits
// cleared; A B ~= A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated in FP32.
// The 2xFP16 split (default) keeps the same three products at twice the
// tensor rate: each operand row r is scaled by a power of two s_r that puts
// its largest |Re|, |Im| over the GEMM's K range in [2^14, 2^15), then
// X_hi = fp16(s X), X_lo = fp16(s X - X_hi): 22 significant bits like the
// TF32 pair (FP16 and TF32 both carry 10 explicit mantissa bits), and only
// entries below 2^-38 of their row's largest lose relative precision.  The
// blocks hold 16-wide k steps in the same bytes as the 8-wide TF32 steps;
// tcgen05.mma kind::f16 (K = 16, FP32 accumulation) replaces kind::tf32 and
// the epilogue multiplies by 1 / (s_i s_j).
// Complex: Re C -= Ar Sr^T - Ai Si^T (negate-A bit), Im C -= Ar Si^T + Ai Sr^T.
// All waits are bounded by wall-clock time and report a wait site.
#include <cuda_fp16.h>

#include "cliqgpu_internal.h"
#include "device_common.cuh"
#include "tc_common.cuh"

namespace cliqgpu {
namespace tc2 {

constexpr int kBM = kTcBM, kBN = kTcBN, kKS = 8;   // kKS: TF32 k step (an FP16 step is 2 * kKS wide, same bytes)
constexpr int kRatio = kBN / kBM;                  // row tiles per column tile
constexpr int kStages = kBN == 128 ? 3 : 4;        // 3 stages of 32 KB: two CTAs per SM
constexpr int kMinBlocks = kBN == 128 ? 2 : 1;
constexpr int kThreads = 192;                 // warps 0-3 epilogue, 4 TMA producer, 5 MMA issuer

template <bool C>
struct Cfg {
    static constexpr int kPlanes = C ? 4 : 2;                  // (re_hi, re_lo, im_hi, im_lo) or (hi, lo)
    static constexpr int kABytes = kPlanes * kBM * kKS * 4;    // one A block: 128 rows
    static constexpr int kBBytes = kPlanes * kBN * kKS * 4;    // one S block: kBN rows
    static constexpr int kStage = kABytes + kBBytes;
    static constexpr int kTmem = C ? 2 * kBN : kBN;
};


// ---------------------------------------------------------------------------
// pack: one CTA per (row tile, k step) block of one job; thread = row
// ---------------------------------------------------------------------------
template <bool C, bool CJ>
__global__ void __launch_bounds__(kTcBM) pack_kernel(const PackJob* __restrict__ jobs, const int64_t* __restrict__ prefix,
                                                   const int32_t* __restrict__ bmap,
                                                   const float* __restrict__ L, const double* __restrict__ D,
                                                   float* __restrict__ out) {
    using X = V<float, C>;
    using W = DV<C>;
    const int64_t bid = blockIdx.x;
    const int lo = bmap[bid];
    const PackJob jb = jobs[lo];
    const int64_t blk = bid - prefix[lo];
    const int nks = (jb.K + kKS - 1) / kKS;
    const int tile = (int)(blk / nks), ks = (int)(blk % nks);
    const int row = threadIdx.x;
    if (row >= jb.tile_rows) return;
    const int r = tile * jb.tile_rows + row;
    float re[kKS], im[kKS];
#pragma unroll
    for (int q = 0; q < kKS; ++q) {
        const int k = ks * kKS + q;
        X v{};
        if (r < jb.R && k < jb.K) {
            v = ldv<float, C>(L, jb.src + r + (int64_t)k * jb.ld);
            if (jb.d >= 0) v = conv<X>(reinterpret_cast<const W*>(D)[jb.d + k]) * opc<CJ>(v);
        }
        if constexpr (C) { re[q] = v.r; im[q] = v.i; } else { re[q] = v; im[q] = 0.f; }
    }
    const int planes = C ? 4 : 2;
    const int64_t plane_bytes = (int64_t)jb.tile_rows * kKS * 4;
    uint8_t* base = reinterpret_cast<uint8_t*>(out + jb.dst) + blk * plane_bytes * planes;
    float h[kKS], l[kKS];
#pragma unroll
    for (int q = 0; q < kKS; ++q) { h[q] = tf32_hi(re[q]); l[q] = re[q] - h[q]; }
    *reinterpret_cast<float4*>(base + 0 * plane_bytes + core_off(row, 0)) = make_float4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<float4*>(base + 0 * plane_bytes + core_off(row, 1)) = make_float4(h[4], h[5], h[6], h[7]);
    *reinterpret_cast<float4*>(base + 1 * plane_bytes + core_off(row, 0)) = make_float4(l[0], l[1], l[2], l[3]);
    *reinterpret_cast<float4*>(base + 1 * plane_bytes + core_off(row, 1)) = make_float4(l[4], l[5], l[6], l[7]);
    if constexpr (C) {
#pragma unroll
        for (int q = 0; q < kKS; ++q) { h[q] = tf32_hi(im[q]); l[q] = im[q] - h[q]; }
        *reinterpret_cast<float4*>(base + 2 * plane_bytes + core_off(row, 0)) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(base + 2 * plane_bytes + core_off(row, 1)) = make_float4(h[4], h[5], h[6], h[7]);
        *reinterpret_cast<float4*>(base + 3 * plane_bytes + core_off(row, 0)) = make_float4(l[0], l[1], l[2], l[3]);
        *reinterpret_cast<float4*>(base + 3 * plane_bytes + core_off(row, 1)) = make_float4(l[4], l[5], l[6], l[7]);
    }
}

// ---------------------------------------------------------------------------
// 2xFP16 pack: one CTA per (row tile, 16-wide k step) block of one job;
// thread = row.  The row's scale comes from the largest |component| over the
// job's K columns, which the panel kernel recorded per (row, 64-column
// block) and as a running maximum per row; the CTA of the first k step also
// stores the row's inverse scale for the GEMM epilogue.
// ---------------------------------------------------------------------------
constexpr int kKS16 = 2 * kKS;

__device__ __forceinline__ float absmax(float v) { return fabsf(v); }
__device__ __forceinline__ float absmax(cx<float> v) { return fmaxf(fabsf(v.r), fabsf(v.i)); }

// scale and split one row's 16 values of block blk into the FP16 planes at
// float offset dst (inverse row scale at dst_scale + r when ks == 0); the
// row maxima come from eblk (nkb blocks from emax) or erow
// largest |component| of row r over the job's K columns (0 beyond R)
__device__ __forceinline__ float pack_row_max(const PackJob& jb, int64_t emax, int R, int r, const uint32_t* __restrict__ eblk,
                                              const uint32_t* __restrict__ erow) {
    float mx = 0.f;
    if (r < R) {
        if (jb.nkb > 0) {
#pragma unroll 4
            for (int b = 0; b < jb.nkb; ++b) mx = fmaxf(mx, __uint_as_float(eblk[emax + (int64_t)r * jb.enT + b]));
        } else {
            mx = __uint_as_float(erow[emax + r]);
        }
    }
    return mx;
}

template <bool C>
__device__ __forceinline__ void pack_f16_planes(const PackJob& jb, const V<float, C> (&v)[kKS16], int64_t dst, int64_t dst_scale,
                                                float mx, int64_t blk, int ks, int row, int r, float* __restrict__ out) {
    // s = 2^(14 - e) for mx in [2^e, 2^(e+1)): s * mx in [2^14, 2^15)
    int e = mx > 0.f ? ((__float_as_int(mx) >> 23) & 0xff) - 127 : 0;
    e = max(-100, min(100, e));
    const float s = __int_as_float((127 + 14 - e) << 23);
    if (ks == 0) out[dst_scale + r] = __int_as_float((127 - 14 + e) << 23);
    // planes (re_hi, re_lo, im_hi, im_lo) of this k step
    constexpr int planes = C ? 4 : 2;
    const int64_t plane_bytes = (int64_t)jb.tile_rows * kKS16 * 2;
    uint8_t* base = reinterpret_cast<uint8_t*>(out + dst) + blk * plane_bytes * planes;
    float y[kKS16];
    uint4 h, l;
#pragma unroll
    for (int q = 0; q < kKS16; ++q) {
        if constexpr (C) y[q] = v[q].r * s; else y[q] = v[q] * s;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        split8(y + 8 * c, h, l);
        *reinterpret_cast<uint4*>(base + 0 * plane_bytes + core_off(row, c)) = h;
        *reinterpret_cast<uint4*>(base + 1 * plane_bytes + core_off(row, c)) = l;
    }
    if constexpr (C) {
#pragma unroll
        for (int q = 0; q < kKS16; ++q) y[q] = v[q].i * s;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            split8(y + 8 * c, h, l);
            *reinterpret_cast<uint4*>(base + 2 * plane_bytes + core_off(row, c)) = h;
            *reinterpret_cast<uint4*>(base + 3 * plane_bytes + core_off(row, c)) = l;
        }
    }
}

// S = D op(L) of one row over the k step when D has 2 x 2 blocks (pivoted
// fronts): e[q + 1] = D(k + 1, k) of a block starting at k = k0 + q (index 0
// is k0 - 1), D(k, k + 1) = op(e); vm / vp are L at k0 - 1 and k0 + 16
template <bool CJ, class X>
__device__ __forceinline__ void quasi_scale(X (&v)[kKS16], const X* d, const X* e, X vm, X vp) {
    X w[kKS16];
#pragma unroll
    for (int q = 0; q < kKS16; ++q) {
        const X lo = q > 0 ? v[q - 1] : vm, hi = q + 1 < kKS16 ? v[q + 1] : vp;
        X y = d[q] * opc<CJ>(v[q]);
        if (!is_zero(e[q + 1])) y += opc<CJ>(e[q + 1]) * opc<CJ>(hi);
        if (!is_zero(e[q])) y += e[q] * opc<CJ>(lo);
        w[q] = y;
    }
#pragma unroll
    for (int q = 0; q < kKS16; ++q) v[q] = w[q];
}

// PV: the fronts were factored with intra-front pivoting; E (like D) holds
// D(k + 1, k) of each 2 x 2 block of D, and the D-scaled operands mix the
// two rows of a block (the Schur complements of such fronts)
template <bool C, bool CJ, bool PV = false>
__global__ void __launch_bounds__(kTcBM) pack_f16_kernel(const PackJob* __restrict__ jobs, const int64_t* __restrict__ prefix,
                                                       const int32_t* __restrict__ bmap,
                                                       const float* __restrict__ L, const double* __restrict__ D,
                                                       const uint32_t* __restrict__ eblk, const uint32_t* __restrict__ erow,
                                                       float* __restrict__ out, const double* __restrict__ E = nullptr) {
    using X = V<float, C>;
    using W = DV<C>;
    __shared__ X s_da[kKS16], s_ds[kKS16];   // pivots of this k step: A scaling (jb.d) and S = D op(rows) (jb.dS)
    __shared__ X s_ea[kKS16 + 2], s_es[kKS16 + 2];   // PV: 2 x 2 block entries from k0 - 1 to k0 + 16
    const int64_t bid = blockIdx.x;
    const int lo = bmap[bid];
    const PackJob jb = jobs[lo];
    const int64_t blk = bid - prefix[lo];
    const int nks = (jb.K + kKS16 - 1) / kKS16;
    const int tile = (int)(blk / nks), ks = (int)(blk % nks);
    const int row = threadIdx.x;
    const int r = tile * jb.tile_rows + row;
    const bool sjob = jb.RS > 0 && tile * jb.tile_rows < jb.RS;
    // every load of the block is issued up front: the L row, the row maxima
    // of both operands and the k step's pivots (one load per k, shared)
    X v[kKS16];
#pragma unroll
    for (int q = 0; q < kKS16; ++q) {
        const int k = ks * kKS16 + q;
        v[q] = (row < jb.tile_rows && r < jb.R && k < jb.K) ? ldv<float, C>(L, jb.src + r + (int64_t)k * jb.ld) : X{};
    }
    const float mxa = row < jb.tile_rows ? pack_row_max(jb, jb.emax, jb.R, r, eblk, erow) : 0.f;
    const float mxs = (sjob && row < jb.tile_rows) ? pack_row_max(jb, jb.emaxS, jb.RS, r, eblk, erow) : 0.f;
    if (row < kKS16) {
        const int k = ks * kKS16 + row;
        s_da[row] = (jb.d >= 0 && k < jb.K) ? conv<X>(reinterpret_cast<const W*>(D)[jb.d + k]) : X{};
        s_ds[row] = (sjob && k < jb.K) ? conv<X>(reinterpret_cast<const W*>(D)[jb.dS + k]) : X{};
    }
    X vm{}, vp{};
    if constexpr (PV) {
        if (row < kKS16 + 2) {
            const int k = ks * kKS16 + row - 1;
            const bool in = k >= 0 && k < jb.K;
            s_ea[row] = (jb.d >= 0 && in) ? conv<X>(reinterpret_cast<const W*>(E)[jb.d + k]) : X{};
            s_es[row] = (sjob && in) ? conv<X>(reinterpret_cast<const W*>(E)[jb.dS + k]) : X{};
        }
        const int k0 = ks * kKS16;
        if (row < jb.tile_rows && r < jb.R) {
            if (k0 > 0) vm = ldv<float, C>(L, jb.src + r + (int64_t)(k0 - 1) * jb.ld);
            if (k0 + kKS16 < jb.K) vp = ldv<float, C>(L, jb.src + r + (int64_t)(k0 + kKS16) * jb.ld);
        }
    }
    __syncthreads();
    if (row >= jb.tile_rows) return;
    if (jb.d >= 0) {
        if constexpr (PV) {
            quasi_scale<CJ>(v, s_da, s_ea, vm, vp);
        } else {
#pragma unroll
            for (int q = 0; q < kKS16; ++q) v[q] = s_da[q] * opc<CJ>(v[q]);
        }
    }
    pack_f16_planes<C>(jb, v, jb.dst, jb.dst_scale, mxa, blk, ks, row, r, out);
    // the S operand from the same rows (a prefix of this job's rows)
    if (sjob) {
        if constexpr (PV) {
            if (r < jb.RS) quasi_scale<CJ>(v, s_ds, s_es, vm, vp);
#pragma unroll
            for (int q = 0; q < kKS16; ++q) {
                const int k = ks * kKS16 + q;
                if (!(r < jb.RS && k < jb.K)) v[q] = X{};
            }
        } else {
#pragma unroll
            for (int q = 0; q < kKS16; ++q) {
                const int k = ks * kKS16 + q;
                v[q] = (r < jb.RS && k < jb.K) ? s_ds[q] * opc<CJ>(v[q]) : X{};
            }
        }
        pack_f16_planes<C>(jb, v, jb.dstS, jb.dst_scaleS, mxs, blk, ks, row, r, out);
    }
}

// ---------------------------------------------------------------------------
// GEMM on packed operands
// ---------------------------------------------------------------------------
template <bool C, bool F16>
__global__ void __launch_bounds__(kThreads, kMinBlocks) tc_gemm_kernel(const GemmProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                              const int32_t* __restrict__ bmap, const float* __restrict__ pack,
                                                              float* __restrict__ L,
                                                              float* __restrict__ pool0, float* __restrict__ pool1,
                                                              int32_t* __restrict__ status) {
    using CF = Cfg<C>;
    if (cta_timed_out(status)) return;   // an earlier wait timed out
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * CF::kStage);
    uint64_t* empty = full + kStages;
    uint64_t* done = empty + kStages;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ float s_sb[kBN];   // 2xFP16: inverse row scales of the tile's S columns

    // tile of this CTA: kBM-row tiles ti, kBN-column tiles tj, needed when ti >= kRatio tj
    const int64_t bid = blockIdx.x;
    const int lo = bmap[bid];   // this tile's problem
    const GemmProb pr = probs[lo];
    int64_t t = bid - prefix[lo];
    const int Mt = (pr.M + kBM - 1) / kBM, Nt = (pr.N + kBN - 1) / kBN;
    int tj = 0;
    while (tj < Nt && t >= Mt - kRatio * tj) { t -= Mt - kRatio * tj; ++tj; }
    if (tj >= Nt) {
        if (threadIdx.x == 0) { atomicExch(&status[1], 1); atomicCAS(&status[2], 0, 5); }
        return;
    }
    const int ti = kRatio * tj + (int)t;
    const int i0 = ti * kBM, j0 = tj * kBN;
    constexpr int kstep = F16 ? 2 * kKS : kKS;
    const int nk = (pr.K + kstep - 1) / kstep;
    const uint8_t* packA = reinterpret_cast<const uint8_t*>(pack + pr.packA) + (int64_t)ti * nk * CF::kABytes;
    const uint8_t* packB = reinterpret_cast<const uint8_t*>(pack + pr.packB) + (int64_t)tj * nk * CF::kBBytes;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)), "r"(CF::kTmem) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 4) {
        // ---- TMA producer ----
        if (lane == 0) {
            for (int it = 0; it < nk; ++it) {
                const int s = it % kStages;
                if (it >= kStages && !mbar_wait(&empty[s], ((it / kStages) - 1) & 1, status, 2)) break;
                uint8_t* st = smem + s * CF::kStage;
                mbar_expect_tx(&full[s], CF::kStage);
                bulk_g2s(st, packA + (int64_t)it * CF::kABytes, CF::kABytes, &full[s]);
                bulk_g2s(st + CF::kABytes, packB + (int64_t)it * CF::kBBytes, CF::kBBytes, &full[s]);
            }
        }
        __syncwarp();
    } else if (warp == 5) {
        // ---- MMA issuer ----
        const uint32_t idp = F16 ? idesc_f16(kBM, kBN, false) : idesc_tf32(kBM, kBN, false);
        const uint32_t idn = F16 ? idesc_f16(kBM, kBN, true) : idesc_tf32(kBM, kBN, true);
        auto mma = [](uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
            if constexpr (F16) mma_f16(d, a, b, id, acc); else mma_tf32(d, a, b, id, acc);
        };
        const uint32_t dre = tmem, dim = tmem + kBN;
        for (int it = 0; it < nk; ++it) {
            const int s = it % kStages;
            if (!mbar_wait(&full[s], (it / kStages) & 1, status, 1)) break;
            tc_fence_after();
            if (lane == 0) {
                const uint32_t a = su32(smem + s * CF::kStage), b = a + CF::kABytes;
                const uint32_t pa = kBM * kKS * 4, pb = kBN * kKS * 4;   // plane strides
                auto A = [&](int p) { return sdesc(a + p * pa, 128, 256); };
                auto B = [&](int p) { return sdesc(b + p * pb, 128, 256); };
                const uint32_t acc = it > 0 ? 1u : 0u;
                mma(dre, A(0), B(0), idp, acc);
                mma(dre, A(0), B(1), idp, 1u);
                mma(dre, A(1), B(0), idp, 1u);
                if constexpr (C) {
                    mma(dre, A(2), B(2), idn, 1u);
                    mma(dre, A(2), B(3), idn, 1u);
                    mma(dre, A(3), B(2), idn, 1u);
                    mma(dim, A(0), B(2), idp, acc);
                    mma(dim, A(0), B(3), idp, 1u);
                    mma(dim, A(1), B(2), idp, 1u);
                    mma(dim, A(2), B(0), idp, 1u);
                    mma(dim, A(2), B(1), idp, 1u);
                    mma(dim, A(3), B(0), idp, 1u);
                }
                mma_commit(&empty[s]);
                if (it == nk - 1) mma_commit(done);
            }
            __syncwarp();
        }
    } else {
        // ---- epilogue (warps 0-3 own TMEM lanes 32w .. 32w+31) ----
        // 2xFP16: the row scales of A (this thread's row) and of the tile's S
        // columns are fetched while the products run
        const int i = i0 + warp * 32 + lane;
        const bool vrow = i < pr.M;
        const float sa = F16 && vrow ? pack[pr.scaleA + i] : 1.f;
        if constexpr (F16) {
            static_assert(kBN == 128, "one S column per epilogue thread");
            const int jt = warp * 32 + lane;
            s_sb[jt] = j0 + jt < pr.N ? pack[pr.scaleB + j0 + jt] : 0.f;
            asm volatile("bar.sync 1, 128;" ::: "memory");   // the four epilogue warps
        }
        const bool ok = mbar_wait(done, 0, status, 3);
        tc_fence_after();
        if (ok) {
            float* Cb = pr.cpool < 0 ? L : (pr.cpool == 0 ? pool0 : pool1);
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
            for (int c0 = 0; c0 < kBN; c0 += 16) {
                if (j0 + c0 >= pr.N || j0 + c0 > i0 + kBM - 1) break;   // warp-uniform: nothing left in this tile row block
                float re[16], im[16];
                tmem_ld16(lane_base + c0, re);
                if constexpr (C) tmem_ld16(lane_base + kBN + c0, im);
                if (vrow) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const int j = j0 + c0 + q;
                        if (j < pr.N && i >= j) {
                            const int64_t e = pr.C + i + (int64_t)j * pr.ldc;
                            float f = 1.f;
                            if constexpr (F16) f = sa * s_sb[j - j0];
                            if constexpr (C) red_sub2(Cb + 2 * e, re[q] * f, im[q] * f);
                            else red_sub(Cb + e, re[q] * f);
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CF::kTmem) : "memory");
    }
}

}  // namespace tc2

size_t tc2_smem(bool cplx) {
    return (size_t)tc2::kStages * (cplx ? tc2::Cfg<true>::kStage : tc2::Cfg<false>::kStage) + 1024 + 256;
}

// pack the launch's operands, then run the tensor-core GEMM
template <bool C, bool CJ, bool F16>
static void launch_pair(Plan& P, const Launch& ln, cudaEvent_t between, cudaStream_t st, void* pack) {
    float* L = reinterpret_cast<float*>(P.L);
    float* p0 = reinterpret_cast<float*>(P.pool[0]);
    float* p1 = reinterpret_cast<float*>(P.pool[1]);
    float* pk = reinterpret_cast<float*>(pack);
    const PackJob* jobs = P.packjobs + ln.pack_items;
    const int64_t* jpre = P.prefix + ln.pack_prefix;
    if (ln.pack_blocks <= 0 && !ln.prepacked) return;   // nothing to update
    if (ln.pack_blocks <= 0) {
        // operands written by the panel kernel
    } else if constexpr (F16) {
        if (P.pivoted)   // Schur complements of pivoted fronts: D with 2 x 2 blocks
            tc2::pack_f16_kernel<C, CJ, true><<<(unsigned)ln.pack_blocks, kTcBM, 0, st>>>(
                jobs, jpre, P.bmap + ln.pack_map, L, P.D, P.eblk, P.erow, pk, P.E);
        else
            tc2::pack_f16_kernel<C, CJ><<<(unsigned)ln.pack_blocks, kTcBM, 0, st>>>(jobs, jpre, P.bmap + ln.pack_map, L, P.D, P.eblk,
                                                                                       P.erow, pk);
    } else
        tc2::pack_kernel<C, CJ><<<(unsigned)ln.pack_blocks, kTcBM, 0, st>>>(jobs, jpre, P.bmap + ln.pack_map, L, P.D, pk);
    if (between) cudaEventRecord(between, st);
    const size_t smem = tc2_smem(C);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(tc2::tc_gemm_kernel<C, F16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    tc2::tc_gemm_kernel<C, F16><<<(unsigned)ln.nblocks, tc2::kThreads, smem, st>>>(
        P.probs + ln.items, P.prefix + ln.prefix, P.bmap + ln.gemm_map, pk, L, p0, p1, P.status);
}

int launch_tc2(Plan& P, const Launch& ln, cudaEvent_t between, cudaStream_t st, void* pack) {
    const bool f16 = P.split_f16 != 0;
    if (P.cplx()) {
        if (P.conjugate) {
            if (f16) launch_pair<true, true, true>(P, ln, between, st, pack); else launch_pair<true, true, false>(P, ln, between, st, pack);
        } else {
            if (f16) launch_pair<true, false, true>(P, ln, between, st, pack); else launch_pair<true, false, false>(P, ln, between, st, pack);
        }
    } else {
        if (f16) launch_pair<false, false, true>(P, ln, between, st, pack); else launch_pair<false, false, false>(P, ln, between, st, pack);
    }
    if (ln.pack_blocks > 0) P.total_launches += 1;   // the pack kernel (the caller counts the GEMM)
    return CLIQ_OK;
}

}  // namespace cliqgpu
