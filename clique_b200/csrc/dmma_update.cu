// FP64 Schur-complement and trailing updates of the plain form on the FP64
// tensor cores (DMMA, mma.sync m8n8k4 .f64).
//
// The update is the one FrontLDL performs with Gemm + Trrk
// (include/clique/numeric/ldl/local_front.hpp:67-69):
//     C -= A diag(d) op(B)^T      on the lower trapezoid i >= j,
// with A, B column-major panels of the factor arena (leading dimension = the
// front's height), d the FP64 pivots, op = conjugation for LDL^H.  The work
// decomposition is the same as the CUDA-core kernel's: 64 x 64 tiles of the
// lower trapezoid of every problem of the launch, one CTA per tile, the
// problem found through the host-built block map.
//
// Per CTA: four warps in a 2 x 2 grid, each owning a 32 x 32 block of the
// tile (4 x 4 DMMA fragments of 8 x 8).  Operand k-slices (64 rows x BK
// columns of A and of B, plus the BK pivots) are staged into shared memory
// with cp.async through a three-stage ring, so the loads of slice k + 2
// overlap the products of slice k.  The pivot scaling d[k] op(B) is applied
// to the B fragments as they are read from shared memory.  Complex products
// use four real DMMAs (Re += ar br - ai bi, Im += ar bi + ai br).  The
// epilogue subtracts the accumulators with one reduction per element, as the
// CUDA-core kernel does.
//
// Shared-memory layout: slice element (k, r) at k * LD + r.  LD = 68 doubles
// (real) or 66 complex elements makes every fragment read conflict-free: a
// DMMA operand fragment reads rows r0 + lane / 4 at k = k0 + lane % 4.
#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {
namespace dmma {

constexpr int kBM = 64;          // CTA tile edge (same tiles as the CUDA-core kernel)
constexpr int kThreads = 128;    // four warps
constexpr int kStages = 3;

template <bool C>
struct Cfg {
    static constexpr int BK = C ? 8 : 16;         // k columns per stage
    static constexpr int LD = C ? 66 : 68;        // elements per staged k row
    static constexpr int EB = C ? 16 : 8;         // bytes per element
    static constexpr int SLICE = BK * LD;         // elements per operand per stage
    static constexpr size_t smem() { return (size_t)kStages * (2 * SLICE + BK) * EB; }
    // pivoted fronts: also the B rows on either side of the slice and the
    // 2 x 2 blocks' D(k + 1, k) from k0 - 1 to k0 + BK
    static constexpr size_t smem_pv() { return (size_t)kStages * (2 * SLICE + BK + 2 * kBM + BK + 2) * EB; }
};

__device__ __forceinline__ uint32_t sptr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// cp.async of one element (8 or 16 bytes); bytes = 0 fills the destination with zeros
template <int EB>
__device__ __forceinline__ void cp_elem(void* dst, const void* src, bool valid) {
    const uint32_t n = valid ? EB : 0;
    if constexpr (EB == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sptr(dst)), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sptr(dst)), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// D (8 x 8) += A (8 x 4, row) * B (4 x 8, col), FP64
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// PV: the fronts were factored with intra-front pivoting; D has 2 x 2 blocks
// (E holds D(k + 1, k) of a block starting at k, D(k, k + 1) = op of it), so
// D op(B) mixes the two rows of a block -- the neighbour across a slice edge
// comes from the staged halo rows.
// FRONT: the in-front update of a pivoted panel step, whose extents the
// panels wrote on the device: CTA b updates front fl[b / tpf] (tile
// b % tpf) with C -= A D op(A)^T over the columns j0 .. j1 - 1 of the
// panel (state[2 s], state[2 s + 1]), rows and columns from j1, in place
template <bool C, bool CJ, bool PV = false, bool FRONT = false>
__global__ void __launch_bounds__(kThreads) dmma_update_kernel(const GemmProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                               const int32_t* __restrict__ bmap, double* __restrict__ L,
                                                               double* __restrict__ pool0, double* __restrict__ pool1,
                                                               const double* __restrict__ D, const double* __restrict__ E = nullptr,
                                                               const FrontDev* __restrict__ F = nullptr,
                                                               const int32_t* __restrict__ fl = nullptr, int64_t tpf = 0,
                                                               const int32_t* __restrict__ state = nullptr) {
    using X = V<double, C>;
    using G = Cfg<C>;
    constexpr int BK = G::BK, LD = G::LD;
    static_assert(kThreads == 2 * kBM, "one halo element per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    X* sOp = reinterpret_cast<X*>(smem_raw);                       // [stage][A slice | B slice]
    X* sDv = sOp + (size_t)kStages * 2 * G::SLICE;                 // [stage][BK] pivots
    X* sBh = sDv + (size_t)kStages * BK;                           // PV: [stage][2][kBM] B rows k0 - 1, k0 + BK
    X* sEv = sBh + (size_t)kStages * 2 * kBM;                      // PV: [stage][BK + 2] D(k + 1, k), k0 - 1 .. k0 + BK

    const int64_t bid = blockIdx.x;
    GemmProb pr{};
    int64_t t;
    if constexpr (FRONT) {
        const int s = fl[bid / tpf];
        const FrontDev f = F[s];
        const int pj0 = state[2 * s], pj1 = state[2 * s + 1];
        t = bid % tpf;
        pr.A = f.L + pj1 + (int64_t)pj0 * f.m;
        pr.B = pr.A;
        pr.C = f.L + pj1 + (int64_t)pj1 * f.m;
        pr.d = f.off + pj0;
        pr.lda = pr.ldc = f.m;
        pr.M = f.m - pj1;
        pr.N = f.n - pj1;
        pr.K = pj1 - pj0;
        pr.cpool = -1;
        if (pr.K <= 0 || pr.M <= 0 || pr.N <= 0) return;
    } else {
        const int lo = bmap[bid];
        pr = probs[lo];
        t = bid - prefix[lo];
    }
    const int Mt = (pr.M + kBM - 1) / kBM, Nt = (pr.N + kBM - 1) / kBM;
    int tj = 0;
    while (tj < Nt && t >= Mt - tj) { t -= Mt - tj; ++tj; }
    if (tj >= Nt) return;   // FRONT: tiles beyond the actual extents; otherwise cannot happen
    const int ti = tj + (int)t;
    const int i0 = ti * kBM, j0 = tj * kBM;
    double* Cbase = pr.cpool < 0 ? L : (pr.cpool == 0 ? pool0 : pool1);
    const X* Lx = reinterpret_cast<const X*>(L);
    const X* Dx = reinterpret_cast<const X*>(D);
    const X* Ex = reinterpret_cast<const X*>(E);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    const int nk = (pr.K + BK - 1) / BK;

    auto load_stage = [&](int kt, int slot) {
        X* sA = sOp + (size_t)slot * 2 * G::SLICE;
        X* sB = sA + G::SLICE;
        const int k0 = kt * BK;
#pragma unroll
        for (int q = 0; q < kBM * BK / kThreads; ++q) {
            const int idx = tid + kThreads * q;
            const int r = idx % kBM, kk = idx / kBM;
            const bool kin = k0 + kk < pr.K;
            const bool va = kin && i0 + r < pr.M, vb = kin && j0 + r < pr.N;
            const X* srcA = va ? Lx + pr.A + (i0 + r) + (int64_t)(k0 + kk) * pr.lda : Lx;
            const X* srcB = vb ? Lx + pr.B + (j0 + r) + (int64_t)(k0 + kk) * pr.lda : Lx;
            cp_elem<G::EB>(sA + kk * LD + r, srcA, va);
            cp_elem<G::EB>(sB + kk * LD + r, srcB, vb);
        }
        if (tid < BK) {
            const bool v = k0 + tid < pr.K;
            cp_elem<G::EB>(sDv + slot * BK + tid, v ? Dx + pr.d + k0 + tid : Dx, v);
        }
        if constexpr (PV) {
            X* sh = sBh + (size_t)slot * 2 * kBM;
            const int h = tid / kBM, r = tid % kBM;
            const int kh = h == 0 ? k0 - 1 : k0 + BK;
            const bool vh = kh >= 0 && kh < pr.K && j0 + r < pr.N;
            cp_elem<G::EB>(sh + h * kBM + r, vh ? Lx + pr.B + (j0 + r) + (int64_t)kh * pr.lda : Lx, vh);
            if (tid < BK + 2) {
                const int ke = k0 - 1 + tid;
                const bool ve = ke >= 0 && ke < pr.K;
                cp_elem<G::EB>(sEv + (size_t)slot * (BK + 2) + tid, ve ? Ex + pr.d + ke : Ex, ve);
            }
        }
    };

    double acc[4][4][2];                 // real part (or the real value)
    double aci[4][4][C ? 2 : 1];         // imaginary part (complex only)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            acc[a][b][0] = acc[a][b][1] = 0.0;
            aci[a][b][0] = 0.0;
            if constexpr (C) aci[a][b][1] = 0.0;
        }

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) load_stage(s, s);
        cp_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_wait<kStages - 2>();
        __syncthreads();   // slice kt landed for every thread; slot (kt - 1) % kStages is free again
        if (kt + kStages - 1 < nk) load_stage(kt + kStages - 1, (kt + kStages - 1) % kStages);
        cp_commit();
        const int slot = kt % kStages;
        const X* sA = sOp + (size_t)slot * 2 * G::SLICE;
        const X* sB = sA + G::SLICE;
        const X* sd = sDv + slot * BK;
#pragma unroll
        for (int k4 = 0; k4 < BK; k4 += 4) {
            const int k = k4 + tg;
            const X dk = sd[k];
            X af[4], bf[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) af[a] = sA[k * LD + wr + 8 * a + g];
            if constexpr (PV) {
                const X* se = sEv + (size_t)slot * (BK + 2);
                const X* sh = sBh + (size_t)slot * 2 * kBM;
                const X ek = se[k + 1], ekm1 = se[k];   // D(k+1, k) of a block at k; D(k, k-1) of one at k - 1
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int col = wc + 8 * b + g;
                    X v = dk * opc<CJ>(sB[k * LD + col]);
                    if (!is_zero(ek)) v += opc<CJ>(ek) * opc<CJ>(k + 1 < BK ? sB[(k + 1) * LD + col] : sh[kBM + col]);
                    if (!is_zero(ekm1)) v += ekm1 * opc<CJ>(k > 0 ? sB[(k - 1) * LD + col] : sh[col]);
                    bf[b] = v;
                }
            } else {
#pragma unroll
                for (int b = 0; b < 4; ++b) bf[b] = dk * opc<CJ>(sB[k * LD + wc + 8 * b + g]);
            }
            if constexpr (C) {
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const double nai = -af[a].i;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        dmma(acc[a][b][0], acc[a][b][1], af[a].r, bf[b].r);
                        dmma(acc[a][b][0], acc[a][b][1], nai, bf[b].i);
                        if constexpr (C) {
                            dmma(aci[a][b][0], aci[a][b][1], af[a].r, bf[b].i);
                            dmma(aci[a][b][0], aci[a][b][1], af[a].i, bf[b].r);
                        }
                    }
                }
            } else {
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) dmma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
            }
        }
    }
    cp_wait<0>();
    // epilogue: element (row g, columns 2 tg, 2 tg + 1) of every 8 x 8 fragment
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + wr + 8 * a + g;
        if (i >= pr.M) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int j = j0 + wc + 8 * b + 2 * tg + e;
                if (j >= pr.N || i < j) continue;
                const int64_t o = pr.C + i + (int64_t)j * pr.ldc;
                if constexpr (C) {
                    atomicAdd(Cbase + 2 * o, -acc[a][b][e]);
                    atomicAdd(Cbase + 2 * o + 1, -aci[a][b][C ? e : 0]);
                } else {
                    atomicAdd(Cbase + o, -acc[a][b][e]);
                }
            }
        }
    }
}

template <bool C, bool CJ, bool PV>
static void launch_t(const Plan& P, const Launch& ln, cudaStream_t st) {
    const size_t smem = PV ? Cfg<C>::smem_pv() : Cfg<C>::smem();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(dmma_update_kernel<C, CJ, PV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    dmma_update_kernel<C, CJ, PV><<<(unsigned)ln.nblocks, kThreads, smem, st>>>(
        P.probs + ln.items, P.prefix + ln.prefix, P.bmap + ln.gemm_map, reinterpret_cast<double*>(P.L),
        reinterpret_cast<double*>(P.pool[0]), reinterpret_cast<double*>(P.pool[1]), P.D, PV ? P.E : nullptr);
}

}  // namespace dmma

namespace dmma {
template <bool C, bool CJ>
static void launch_front_t(const Plan& P, const int32_t* fl, int64_t nfronts, int64_t tpf, cudaStream_t st) {
    const size_t smem = Cfg<C>::smem_pv();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(dmma_update_kernel<C, CJ, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    dmma_update_kernel<C, CJ, true, true><<<(unsigned)(nfronts * tpf), kThreads, smem, st>>>(
        nullptr, nullptr, nullptr, reinterpret_cast<double*>(P.L), nullptr, nullptr, P.D, P.E, P.fronts, fl, tpf, P.pstate);
}
}  // namespace dmma

// the in-front update of one pivoted panel step of a level (FP64 plans):
// nfronts x tpf CTAs, tpf the 64 x 64 lower-trapezoid tiles of the largest
// trailing block the planned panel widths allow
int launch_dmma_front_update(Plan& P, const int32_t* fl, int64_t nfronts, int64_t tpf, cudaStream_t st) {
    if (nfronts <= 0 || tpf <= 0) return CLIQ_OK;
    if (P.cplx()) {
        if (P.conjugate) dmma::launch_front_t<true, true>(P, fl, nfronts, tpf, st);
        else dmma::launch_front_t<true, false>(P, fl, nfronts, tpf, st);
    } else {
        dmma::launch_front_t<false, false>(P, fl, nfronts, tpf, st);
    }
    return CLIQ_OK;
}

int launch_dmma_update(Plan& P, const Launch& ln, cudaStream_t st) {
    const bool pv = P.pivoted;   // (the Schur complements of pivoted fronts)
    if (P.cplx()) {
        if (P.conjugate) pv ? dmma::launch_t<true, true, true>(P, ln, st) : dmma::launch_t<true, true, false>(P, ln, st);
        else pv ? dmma::launch_t<true, false, true>(P, ln, st) : dmma::launch_t<true, false, false>(P, ln, st);
    } else {
        pv ? dmma::launch_t<false, false, true>(P, ln, st) : dmma::launch_t<false, false, false>(P, ln, st);
    }
    return CLIQ_OK;
}

}  // namespace cliqgpu
