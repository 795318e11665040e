// Intra-front pivoting: the LDL_INTRAPIV_1D / LDL_INTRAPIV_2D front types
// (ldl/local.hpp:31-33,106-111; FrontLDLIntraPiv, ldl/local_front.hpp:74-94).
//
// Each front's pivot block A11 is factored with Bunch-Kaufman partial
// pivoting restricted to the front's own pivot rows: P A11 P^T = L D op(L)^T
// with D block diagonal (1 x 1 and 2 x 2 blocks, alpha = (1 + sqrt 17) / 8,
// magnitudes |re| + |im|), the columns of A21 permuted with P, and the Schur
// complement ABR -= L21 D op(L21)^T passed up as in the unpivoted form.  The
// reference gets this from Elemental's El::LDL( A11, dSub, p, conjugate,
// BUNCH_KAUFMAN_A ), PermuteCols, Trsm, QuasiDiagonalSolve and Trrk.
//
// GPU form, per tree level after its extend-add and assembly, right-looking
// in panels of 64 (65 when a 2 x 2 block closes the panel) columns:
//   bk_panel_kernel   one CTA per front (1024 threads, 512 for FP64; on the
//                     top levels a cluster of 8 CTAs per front): the panel's pivots one column at a
//                     time.  The candidate columns are formed with the
//                     panel's pending update (A(:,k) - L(:,panel) B(k,panel)^T,
//                     B = D op(L)^T built from L and D on the fly), the pivot
//                     search runs over the front's remaining pivot rows, a
//                     chosen interchange swaps rows and columns of the whole
//                     front (the factored columns of L and the columns of A21
//                     included), and the pivot columns of L are written for
//                     the pivot rows;
//   bk_lower_kernel   rows below the pivots (A21): L21(:,panel) = A21(:,panel)
//                     op(L11)^{-T} D^{-1} for the panel's diagonal block, one
//                     thread per row;
//   bk_update2_kernel the panel's rank-kb update of the front's remaining
//                     columns (pivot rows and A21 rows, lower part) for FP32
//                     plans, CUDA cores; FP64 plans run it on DMMA (the
//                     DMMA update kernel's FRONT mode, extents read from the
//                     panel state), bk_update_kernel without DMMA.
// At the end of the level the Schur complements (K = n) go into the update
// pool through the plan's own Schur launches -- tcgen05 for FP32 plans
// (bk_rowmax_kernel gives the 2xFP16 split's row maxima; the packing's
// pivoted variant forms S = D op(L) with the 2 x 2 terms), DMMA for FP64
// plans (halo rows for the 2 x 2 terms) -- or through bk_update_kernel.
// Then the 64 x 64 diagonal-block inverses the sweeps use, and the index
// maps the solves read are rewritten for the pivoted row order (the
// reference's PermuteRows / InversePermuteRows around each front solve,
// lower_solve/local_front.hpp:53-93, become a relabelling of the front's
// pivot rows).
#include "cliqgpu_internal.h"
#include "device_common.cuh"

#include <climits>
#include <cmath>
#include <cstdlib>
#include <string>

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

#ifndef TRY
#define TRY(x)                          \
    do {                                \
        int _st = (x);                  \
        if (_st != CLIQ_OK) return _st; \
    } while (0)
#endif

namespace cliqgpu {
namespace piv {

constexpr int kNb = 64;                 // panel width (one more when a 2 x 2 block closes it)
constexpr int kMaxPanel = kNb + 1;
// threads of a panel CTA: as many loads in flight as the registers allow
// (FP32: 51-62 registers a thread, 1024 threads; FP64: up to 126, 512)
template <class T> constexpr int panel_threads() { return sizeof(T) == 4 ? 1024 : 512; }
constexpr int kClusterCTAs = 8;         // CTAs sharing a front's panel on the top levels
constexpr int kLowerRows = 128;         // rows of A21 per bk_lower_kernel CTA
constexpr int kUpdThreads = 256;
constexpr int kUpdTile = 64;
constexpr double kAlpha = 0.64038820320220756872767623199676;   // (1 + sqrt(17)) / 8

static inline unsigned grid1d(int64_t work, int threads) {
    const int64_t g = (work + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

template <class T> __device__ __forceinline__ T mag1(T a) { return fabs(a); }
template <class T> __device__ __forceinline__ T mag1(cx<T> a) { return fabs(a.r) + fabs(a.i); }
template <class T> __device__ __forceinline__ T realpart(T a) { return a; }
template <class T> __device__ __forceinline__ cx<T> realpart(cx<T> a) { return {a.r, T(0)}; }
template <class X> __device__ __forceinline__ X neg(X a) { return X{} - a; }

// B(j, p) = sum_l D(p, l) op(L(j, l)) over the block of D that holds p:
// D(p, p) = d[p]; D(p, p + 1) = op(e[p]) when a 2 x 2 block starts at p;
// D(p, p - 1) = e[p - 1] when one starts at p - 1.  Lrow(q) reads L(j, q).
template <bool CJ, class X, class Get>
__device__ __forceinline__ X bval(int p, X d, X e, X em1, bool first, Get Lrow) {
    X b = d * opc<CJ>(Lrow(p));
    if (!is_zero(e)) b += opc<CJ>(e) * opc<CJ>(Lrow(p + 1));
    if (first && !is_zero(em1)) b += em1 * opc<CJ>(Lrow(p - 1));
    return b;
}

// sum_p L(i, j0 + p) w[p] over the panel's factored columns (row element
// offset e0 of column j0, column stride m): eight loads in flight, two
// partial sums
// (L1: false reads from L2, for entries other CTAs of the cluster wrote)
template <bool L1, class T, class X>
__device__ __forceinline__ X panel_dot(const T* L, int64_t e0, int m, int np, const X* w) {
    constexpr bool C = !std::is_same<X, T>::value;
    auto ld = [&](int64_t e) -> X {
        if constexpr (L1) return ldv<T, C>(L, e);
        else return ldv_cg<T, C>(L, e);
    };
    X s0{}, s1{};
    int p = 0;
    for (; p + 8 <= np; p += 8) {
        X l[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) l[q] = ld(e0 + (int64_t)(p + q) * m);
#pragma unroll
        for (int q = 0; q < 8; q += 2) {
            mac(s0, l[q], w[p + q]);
            mac(s1, l[q + 1], w[p + q + 1]);
        }
    }
    for (; p < np; ++p) mac(s0, ld(e0 + (int64_t)p * m), w[p]);
    return s0 + s1;
}

// the CTAs' block-argmax results combined across a cluster (G > 1): each
// CTA's thread 0 writes its partial into the first CTA's slots, and after the
// cluster barrier every thread reduces the G slots in the same order
template <int G, class T>
__device__ __forceinline__ void cluster_argmax(T& v, int& idx, T* slot_v, int* slot_i) {
    if constexpr (G > 1) {
        cg::cluster_group cl = cg::this_cluster();
        if (threadIdx.x == 0) {
            cl.map_shared_rank(slot_v, 0)[cl.block_rank()] = v;
            cl.map_shared_rank(slot_i, 0)[cl.block_rank()] = idx;
        }
        cl.sync();
        const T* rv = cl.map_shared_rank(slot_v, 0);
        const int* ri = cl.map_shared_rank(slot_i, 0);
        v = rv[0];
        idx = ri[0];
        for (int q = 1; q < G; ++q) {
            const T ov = rv[q];
            const int oi = ri[q];
            if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
        }
    }
}

// block-wide max with the smallest index on ties, one barrier: every warp
// reduces the per-warp partials itself (the partials are rewritten only
// after a later barrier of the caller)
template <class T>
__device__ __forceinline__ void block_argmax(T& v, int& idx, T* sv, int* si) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
    if (lane == 0) { sv[w] = v; si[w] = idx; }
    __syncthreads();
    v = lane < nw ? sv[lane] : T(-1);
    idx = lane < nw ? si[lane] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
}

// ---------------------------------------------------------------------------
// one panel of Bunch-Kaufman pivots per front: one CTA (G = 1), or a
// cluster of G CTAs sharing the front's rows (the top levels, whose few
// large fronts would leave most SMs idle).  With G > 1 every CTA takes the
// rows k + rank nt + tid + q G nt, the argmax partials meet in the first
// CTA's shared memory, every CTA reaches the same pivot decisions from the
// same combined values (so all pass the same cluster barriers), the entries
// other CTAs wrote are read from L2 (ld.global.cg), and the first CTA's
// thread 0 does the single-entry work
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ, int G = 1>
__global__ void __launch_bounds__(panel_threads<T>()) bk_panel_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl,
                                                                 T* __restrict__ L, double* __restrict__ D, double* __restrict__ E,
                                                                 int32_t* __restrict__ pivg, T* __restrict__ cvec, T* __restrict__ vvec,
                                                                 int32_t* __restrict__ state, int32_t* __restrict__ status) {
    using X = V<T, C>;
    using W = DV<C>;
    __shared__ X s_d[kMaxPanel], s_e[kMaxPanel];   // the panel's D (diagonal, and D(p+1,p) of 2 x 2 blocks)
    __shared__ X s_w[kMaxPanel];                   // B(k, p)
    __shared__ X s_lr[kMaxPanel], s_wi[kMaxPanel]; // L(imax, p), B(imax, p)
    __shared__ T s_rv[32], s_rv2[32];   // per-warp partials of the two reductions of a column step
    __shared__ int s_ri[32], s_ri2[32];
    __shared__ X s_akk, s_ar;
    __shared__ T s_slot_v[G], s_slot2_v[G];   // G > 1: the CTAs' argmax partials (in the first CTA)
    __shared__ int s_slot_i[G], s_slot2_i[G];
    int rank = 0;
    if constexpr (G > 1) rank = (int)cg::this_cluster().block_rank();
    const int s = fl[blockIdx.x / G];
    const FrontDev f = F[s];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int t0 = rank * nt + tid, ntot = G * nt;
    const bool lead = tid == 0 && rank == 0;
    const int n = f.n, m = f.m;
    const int j0 = state[2 * s + 1];
    if (j0 >= n) {   // (the same for every CTA of a cluster)
        if (lead) state[2 * s] = j0;
        return;
    }
    const int64_t base = f.L;
    auto at = [&](int i, int j) -> int64_t { return base + i + (int64_t)j * m; };
    auto ld = [&](const T* p, int64_t e) -> X {
        if constexpr (G > 1) return ldv_cg<T, C>(p, e);
        else return ldv<T, C>(p, e);
    };
    auto sync = [&]() {
        if constexpr (G > 1) cg::this_cluster().sync();
        else __syncthreads();
    };
    auto bcast = [&](X* p, X v) {   // a value every CTA needs, into every CTA's copy
        if constexpr (G > 1) {
            for (int q = 0; q < G; ++q) *cg::this_cluster().map_shared_rank(p, q) = v;
        } else {
            *p = v;
        }
    };
    if (j0 == 0)
        for (int i = t0; i < n; i += ntot) pivg[f.off + i] = f.off + i;
    const int jend = min(n, j0 + kNb);
    int k = j0;
    while (k < jend) {
        const int np = k - j0;
        // B(k, p) for the panel's factored columns
        if (tid < np) {
            const int p = j0 + tid;
            s_w[tid] = bval<CJ>(p, s_d[tid], s_e[tid], tid > 0 ? s_e[tid - 1] : X{}, tid > 0,
                                [&](int q) { return ld(L, at(k, q)); });
        }
        __syncthreads();
        // candidate column k with the panel's pending update; column maximum below the diagonal
        T best = T(-1);
        int bi = INT_MAX;
        for (int i = k + t0; i < n; i += ntot) {
            X a = ld(L, at(i, k)) - panel_dot<G == 1>(L, at(i, j0), m, np, s_w);
            if (i == k) {
                if constexpr (CJ) a = realpart(a);
                bcast(&s_akk, a);
            } else {
                const T g = mag1(a);
                if (g > best) { best = g; bi = i; }
            }
            stv<T, C>(cvec, f.off + i, a);
        }
        block_argmax(best, bi, s_rv, s_ri);   // (its barrier publishes s_akk)
        cluster_argmax<G>(best, bi, s_slot_v, s_slot_i);
        const T colmax = best > T(0) ? best : T(0);
        const int imax = bi == INT_MAX ? k : bi;
        const T absakk = mag1(s_akk);
        int kp = k, kstep = 1;
        bool use_v = false, zero = false;
        if (fmax((double)absakk, (double)colmax) == 0.0) {
            zero = true;
        } else if (absakk >= (T)kAlpha * colmax) {
            kp = k;
        } else {
            // candidate column imax (the full matrix's column, rows k .. n-1)
            if (tid < np) {
                const int p = j0 + tid;
                s_lr[tid] = ld(L, at(imax, p));
                s_wi[tid] = bval<CJ>(p, s_d[tid], s_e[tid], tid > 0 ? s_e[tid - 1] : X{}, tid > 0,
                                     [&](int q) { return ld(L, at(imax, q)); });
            }
            __syncthreads();
            T rbest = T(-1);
            int rbi = INT_MAX;
            // (the rows of vvec follow the same thread mapping as those of cvec)
            for (int j = k + t0; j < n; j += ntot) {
                X a;
                if (j < imax) {
                    a = ld(L, at(imax, j));
                    for (int p = 0; p < np; ++p) {
                        const X b = bval<CJ>(j0 + p, s_d[p], s_e[p], p > 0 ? s_e[p - 1] : X{}, p > 0,
                                             [&](int q) { return ld(L, at(j, q)); });
                        a -= s_lr[p] * b;
                    }
                    a = opc<CJ>(a);
                } else if (j == imax) {
                    a = ld(L, at(imax, imax));
                    for (int p = 0; p < np; ++p) a -= s_lr[p] * s_wi[p];
                    if constexpr (CJ) a = realpart(a);
                    bcast(&s_ar, a);
                } else {
                    a = ld(L, at(j, imax)) - panel_dot<G == 1>(L, at(j, j0), m, np, s_wi);
                }
                stv<T, C>(vvec, f.off + j, a);
                if (j != imax) {
                    const T g = mag1(a);
                    if (g > rbest) { rbest = g; rbi = j; }
                }
            }
            block_argmax(rbest, rbi, s_rv2, s_ri2);   // (publishes s_ar)
            cluster_argmax<G>(rbest, rbi, s_slot2_v, s_slot2_i);
            const T rowmax = rbest > T(0) ? rbest : T(0);
            if (absakk >= (T)kAlpha * colmax * (colmax / rowmax)) {
                kp = k;
            } else if (mag1(s_ar) >= (T)kAlpha * rowmax) {
                kp = imax;
                use_v = true;
            } else {
                kp = imax;
                kstep = 2;
            }
        }
        if (zero && lead) atomicMin(&status[0], __ldcg(pivg + f.off + k) + 1);   // the row's ND index (no interchange here)
        // symmetric interchange of a = kk and b = kp over the whole front
        const int kk = k + kstep - 1;
        if (kp != kk) {
            const int a = kk, b = kp;
            for (int j = t0; j < a; j += ntot) {   // factored columns: rows a and b
                const X t = ld(L, at(a, j));
                stv<T, C>(L, at(a, j), ld(L, at(b, j)));
                stv<T, C>(L, at(b, j), t);
            }
            for (int i = a + 1 + t0; i < b; i += ntot) {   // column a between the two, row b between the two
                const X t = ld(L, at(i, a));
                stv<T, C>(L, at(i, a), opc<CJ>(ld(L, at(b, i))));
                stv<T, C>(L, at(b, i), opc<CJ>(t));
            }
            for (int i = b + 1 + t0; i < m; i += ntot) {   // rows below b (A21 included): columns a and b
                const X t = ld(L, at(i, a));
                stv<T, C>(L, at(i, a), ld(L, at(i, b)));
                stv<T, C>(L, at(i, b), t);
            }
            if (lead) {
                const X t = ld(L, at(a, a));
                stv<T, C>(L, at(a, a), ld(L, at(b, b)));
                stv<T, C>(L, at(b, b), t);
                stv<T, C>(L, at(b, a), opc<CJ>(ld(L, at(b, a))));
                const int32_t g = __ldcg(pivg + f.off + a);
                pivg[f.off + a] = __ldcg(pivg + f.off + b);
                pivg[f.off + b] = g;
                const X c0 = ld(cvec, f.off + a);
                stv<T, C>(cvec, f.off + a, ld(cvec, f.off + b));
                stv<T, C>(cvec, f.off + b, c0);
                const X v0 = ld(vvec, f.off + a);
                stv<T, C>(vvec, f.off + a, ld(vvec, f.off + b));
                stv<T, C>(vvec, f.off + b, v0);
            }
        }
        // the common step (1 x 1 pivot at k, no interchange) needs no barrier
        // here: each thread divides the column entries it formed itself (the
        // rows k + tid + q nt of both candidate columns), and the pivot is in
        // shared memory
        const bool plain = kstep == 1 && kp == k;
        if (!plain) sync();
        // pivot columns of L (pivot rows), D and E
        if (kstep == 1) {
            const T* col = use_v ? vvec : cvec;
            X d = plain ? s_akk : ld(col, f.off + k);
            if constexpr (CJ) d = realpart(d);
            for (int i = k + t0; i < n; i += ntot) {
                if (i == k) continue;
                const X c = ld(col, f.off + i);
                stv<T, C>(L, at(i, k), is_zero(d) ? X{} : c / d);
            }
            if (lead) {
                stv<T, C>(L, at(k, k), vone<X>());
                reinterpret_cast<W*>(D)[f.off + k] = conv<W>(d);
                reinterpret_cast<W*>(E)[f.off + k] = W{};
            }
            if (tid == 0) {
                s_d[np] = d;
                s_e[np] = X{};
            }
        } else {
            X d11 = ld(cvec, f.off + k), d21 = ld(cvec, f.off + k + 1), d22 = ld(vvec, f.off + k + 1);
            if constexpr (CJ) { d11 = realpart(d11); d22 = realpart(d22); }
            const X det = d11 * d22 - d21 * opc<CJ>(d21);
            for (int i = k + 2 + t0; i < n; i += ntot) {
                const X c = ld(cvec, f.off + i), v = ld(vvec, f.off + i);
                stv<T, C>(L, at(i, k), (c * d22 - v * d21) / det);
                stv<T, C>(L, at(i, k + 1), (v * d11 - c * opc<CJ>(d21)) / det);
            }
            if (lead) {
                stv<T, C>(L, at(k, k), vone<X>());
                stv<T, C>(L, at(k + 1, k + 1), vone<X>());
                stv<T, C>(L, at(k + 1, k), X{});
                reinterpret_cast<W*>(D)[f.off + k] = conv<W>(d11);
                reinterpret_cast<W*>(D)[f.off + k + 1] = conv<W>(d22);
                reinterpret_cast<W*>(E)[f.off + k] = conv<W>(d21);
                reinterpret_cast<W*>(E)[f.off + k + 1] = W{};
            }
            if (tid == 0) {
                s_d[np] = d11;
                s_e[np] = d21;
                s_d[np + 1] = d22;
                s_e[np + 1] = X{};
            }
        }
        sync();
        k += kstep;
    }
    if (lead) {
        state[2 * s] = j0;
        state[2 * s + 1] = k;
    }
}

// ---------------------------------------------------------------------------
// rows below the pivots: L21(:, panel) = A21(:, panel) op(L11)^{-T} D^{-1}
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kLowerRows) bk_lower_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl, int chunks,
                                                              T* __restrict__ L, const double* __restrict__ D,
                                                              const double* __restrict__ E, const int32_t* __restrict__ state) {
    using X = V<T, C>;
    using W = DV<C>;
    extern __shared__ __align__(16) unsigned char bk_smem[];
    X* s_l = reinterpret_cast<X*>(bk_smem);   // L11 of the panel, kMaxPanel x kMaxPanel, column-major, then the rows' y
    __shared__ X s_d[kMaxPanel], s_e[kMaxPanel];
    const int fi = blockIdx.x / chunks, ch = blockIdx.x % chunks;
    const int s = fl[fi];
    const FrontDev f = F[s];
    const int j0 = state[2 * s], j1 = state[2 * s + 1], kb = j1 - j0;
    const int u = f.m - f.n;
    if (kb <= 0 || ch * kLowerRows >= u) return;
    const int64_t base = f.L;
    for (int idx = threadIdx.x; idx < kb * kb; idx += blockDim.x) {
        const int r = idx % kb, c = idx / kb;
        s_l[r + c * kMaxPanel] = r > c ? ldv<T, C>(L, base + (j0 + r) + (int64_t)(j0 + c) * f.m) : X{};
    }
    for (int q = threadIdx.x; q < kb; q += blockDim.x) {
        s_d[q] = conv<X>(reinterpret_cast<const W*>(D)[f.off + j0 + q]);
        s_e[q] = conv<X>(reinterpret_cast<const W*>(E)[f.off + j0 + q]);
    }
    __syncthreads();
    const int i = f.n + ch * kLowerRows + threadIdx.x;
    if (i >= f.m) return;
    const int64_t row = base + i;
    // this thread's row of the panel in shared memory (column q at q * kLowerRows + tid): all loads first
    X* y = s_l + kMaxPanel * kMaxPanel + threadIdx.x;
    for (int q = 0; q < kb; ++q) y[q * kLowerRows] = ldv<T, C>(L, row + (int64_t)(j0 + q) * f.m);
    // y(q) = a(q) - sum_{p<q} y(p) op(L11(q, p))
    for (int q = 1; q < kb; ++q) {
        X a = y[q * kLowerRows];
        for (int p = 0; p < q; ++p) a -= y[p * kLowerRows] * opc<CJ>(s_l[q + p * kMaxPanel]);
        y[q * kLowerRows] = a;
    }
    // l = y D^{-1}
    for (int q = 0; q < kb; ++q) {
        const int64_t e0 = row + (int64_t)(j0 + q) * f.m;
        if (!is_zero(s_e[q])) {
            const X d11 = s_d[q], d22 = s_d[q + 1], d21 = s_e[q];
            const X det = d11 * d22 - d21 * opc<CJ>(d21);
            const X y0 = y[q * kLowerRows], y1 = y[(q + 1) * kLowerRows];
            stv<T, C>(L, e0, (y0 * d22 - y1 * d21) / det);
            stv<T, C>(L, e0 + f.m, (y1 * d11 - y0 * opc<CJ>(d21)) / det);
            ++q;
        } else {
            const X d = s_d[q];
            stv<T, C>(L, e0, is_zero(d) ? X{} : y[q * kLowerRows] / d);
        }
    }
}

// ---------------------------------------------------------------------------
// C -= A B^T on the lower part, B(j, p) = sum_l D(p, l) op(L(j, l)):
//   kind 0: the front's remaining columns after its latest panel
//           (rows and columns from j1, K = the panel);
//   kind 1: the Schur complement ABR -= L21 D op(L21)^T (K = n) into the pool.
// One 64 x 64 tile per CTA; tiles beyond the front's actual extent return.
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kUpdThreads, (sizeof(T) == 8 && C) ? 2 : 3) bk_update_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl,
                                                                int64_t tiles_per_front, int kind, T* __restrict__ L,
                                                                T* __restrict__ pool0, T* __restrict__ pool1,
                                                                const double* __restrict__ D, const double* __restrict__ E,
                                                                const int32_t* __restrict__ state) {
    using X = V<T, C>;
    using W = DV<C>;
    constexpr int BM = kUpdTile, BK = C ? 8 : 16, PAD = 1;
    __shared__ X sA[BK][BM + PAD];
    __shared__ X sB[BK][BM + PAD];
    __shared__ X s_d[BK], s_e[BK], s_em1[BK];
    const int64_t fi = blockIdx.x / tiles_per_front;
    int64_t t = blockIdx.x % tiles_per_front;
    const int s = fl[fi];
    const FrontDev f = F[s];
    int r0, c0, k0, K, M, N;
    if (kind == 0) {
        const int j0 = state[2 * s], j1 = state[2 * s + 1];
        r0 = j1; c0 = j1; k0 = j0; K = j1 - j0; M = f.m - j1; N = f.n - j1;
    } else {
        r0 = f.n; c0 = f.n; k0 = 0; K = f.n; M = N = f.m - f.n;
    }
    if (K <= 0 || M <= 0 || N <= 0) return;
    const int Mt = (M + BM - 1) / BM, Nt = (N + BM - 1) / BM;
    int tj = 0;
    while (tj < Nt && t >= Mt - tj) { t -= Mt - tj; ++tj; }
    if (tj >= Nt) return;
    const int ti = tj + (int)t;
    const int i0 = ti * BM, jb0 = tj * BM;
    const int64_t base = f.L;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    X acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = X{};
    for (int kq = 0; kq < K; kq += BK) {
        if (threadIdx.x < BK) {
            const int p = k0 + kq + threadIdx.x;
            const bool in = kq + (int)threadIdx.x < K;
            s_d[threadIdx.x] = in ? conv<X>(reinterpret_cast<const W*>(D)[f.off + p]) : X{};
            s_e[threadIdx.x] = in ? conv<X>(reinterpret_cast<const W*>(E)[f.off + p]) : X{};
            s_em1[threadIdx.x] = (in && p > 0) ? conv<X>(reinterpret_cast<const W*>(E)[f.off + p - 1]) : X{};
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < (BM * BK) / kUpdThreads; ++q) {
            const int idx = threadIdx.x + kUpdThreads * q;
            const int r = idx % BM, kk = idx / BM;
            const int kg = kq + kk;
            X av{}, bv{};
            if (kg < K) {
                const int p = k0 + kg;
                if (i0 + r < M) av = ldv<T, C>(L, base + (r0 + i0 + r) + (int64_t)p * f.m);
                if (jb0 + r < N) {
                    const int64_t rowj = base + (c0 + jb0 + r);
                    bv = bval<CJ>(p, s_d[kk], s_e[kk], s_em1[kk], p > 0,
                                  [&](int qq) { return ldv<T, C>(L, rowj + (int64_t)qq * f.m); });
                }
            }
            sA[kk][r] = av;
            sB[kk][r] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            X av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = sA[kk][ty + 16 * a];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = sB[kk][tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) mac(acc[a][b], av[a], bv[b]);
        }
        __syncthreads();
    }
    T* Cb;
    int64_t cbase, ldc;
    if (kind == 0) {
        Cb = L; cbase = base + r0 + (int64_t)c0 * f.m; ldc = f.m;
    } else {
        Cb = f.pool == 0 ? pool0 : pool1; cbase = f.U; ldc = f.m - f.n;
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = jb0 + tx + 16 * b;
        if (j >= N) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + ty + 16 * a;
            if (i < M && i >= j) {   // one tile writes each entry per launch
                const int64_t e = cbase + i + (int64_t)j * ldc;
                stv<T, C>(Cb, e, ldv<T, C>(Cb, e) - acc[a][b]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// FP32 plans' in-front update (kind 0 above): 128 x 64 tiles, 8 x 4 entries
// a thread, lanes along the rows (coalesced read-modify-write of L), the
// next k slice's operands loaded into registers while the current slice is
// multiplied out of shared memory (two buffers, one barrier a slice).
// Column block tj (64 columns) holds the row tiles tj / 2 .. Mt - 1, so the
// two column blocks of pair u hold Mt - u row tiles each, and the tiles
// before pair u number S(u) = u (2 Mt + 1) - u^2.
// ---------------------------------------------------------------------------
constexpr int kU2M = 128, kU2N = 64;

__host__ __device__ __forceinline__ int64_t upd2_tiles_dev(int64_t M, int64_t N) {
    if (M <= 0 || N <= 0) return 0;
    const int64_t Mt = (M + kU2M - 1) / kU2M, Nt = (N + kU2N - 1) / kU2N;
    const int64_t pairs = Nt / 2;
    return pairs * (2 * Mt + 1) - pairs * pairs + ((Nt & 1) ? Mt - pairs : 0);
}

template <bool C, bool CJ>
__global__ void __launch_bounds__(kUpdThreads, 2) bk_update2_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl,
                                                                    int64_t tiles_per_front, float* __restrict__ L,
                                                                    const double* __restrict__ D, const double* __restrict__ E,
                                                                    const int32_t* __restrict__ state) {
    using X = V<float, C>;
    using W = DV<C>;
    constexpr int BK = C ? 8 : 16;
    constexpr int LA = kU2M * BK / kUpdThreads, LB = kU2N * BK / kUpdThreads;
    static_assert(LA * kUpdThreads == kU2M * BK && LB * kUpdThreads == kU2N * BK, "slice split");
    __shared__ __align__(16) X sA[2][BK][kU2M];
    __shared__ __align__(16) X sB[2][BK][kU2N];
    const int64_t fi = blockIdx.x / tiles_per_front;
    const int64_t t = blockIdx.x % tiles_per_front;
    const int s = fl[fi];
    const FrontDev f = F[s];
    const int j0 = state[2 * s], j1 = state[2 * s + 1];
    const int K = j1 - j0, M = f.m - j1, N = f.n - j1;
    if (K <= 0 || M <= 0 || N <= 0) return;
    if (t >= upd2_tiles_dev(M, N)) return;
    // pair u: the largest with S(u) <= t (the smaller root of u^2 - (2 Mt + 1) u + t, then corrected)
    const int64_t Mt = (M + kU2M - 1) / kU2M, Nt = (N + kU2N - 1) / kU2N;
    const double b2 = 2.0 * (double)Mt + 1.0;
    int64_t u = (int64_t)floor((b2 - sqrt(fmax(b2 * b2 - 4.0 * (double)t, 0.0))) * 0.5);
    auto S = [&](int64_t v) { return v * (2 * Mt + 1) - v * v; };
    if (u < 0) u = 0;
    for (int it = 0; it < 3 && u > 0 && S(u) > t; ++it) --u;
    for (int it = 0; it < 3 && S(u + 1) <= t; ++it) ++u;
    const int64_t rem = t - S(u);
    int64_t tj, ti;
    if (rem < Mt - u) { tj = 2 * u; ti = u + rem; }
    else { tj = 2 * u + 1; ti = u + rem - (Mt - u); }
    if (rem < 0 || tj >= Nt || ti >= Mt || ti < tj / 2) return;
    const int i0 = (int)ti * kU2M, jb0 = (int)tj * kU2N;
    const int64_t base = f.L;
    const int64_t arow = base + j1 + i0;          // row i0 of the trailing block
    const int64_t brow = base + j1 + jb0;         // row (= column of C) jb0
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const W* Dw = reinterpret_cast<const W*>(D) + f.off;
    const W* Ew = reinterpret_cast<const W*>(E) + f.off;

    X ra[LA], rl[LB], rd[LB], re[LB], rem1[LB];
    auto fetch = [&](int kq) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            const int idx = threadIdx.x + kUpdThreads * q;
            const int r = idx % kU2M, kg = kq + idx / kU2M;
            ra[q] = (kg < K && i0 + r < M) ? ldv<float, C>(L, arow + r + (int64_t)(j0 + kg) * f.m) : X{};
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int idx = threadIdx.x + kUpdThreads * q;
            const int r = idx % kU2N, kg = kq + idx / kU2N;
            const int p = j0 + kg;
            const bool in = kg < K && jb0 + r < N;
            rl[q] = in ? ldv<float, C>(L, brow + r + (int64_t)p * f.m) : X{};
            rd[q] = in ? conv<X>(Dw[p]) : X{};
            re[q] = in ? conv<X>(Ew[p]) : X{};
            rem1[q] = (in && p > 0) ? conv<X>(Ew[p - 1]) : X{};
        }
    };
    auto stage = [&](int buf, int kq) {
#pragma unroll
        for (int q = 0; q < LA; ++q) {
            const int idx = threadIdx.x + kUpdThreads * q;
            sA[buf][idx / kU2M][idx % kU2M] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < LB; ++q) {
            const int idx = threadIdx.x + kUpdThreads * q;
            const int r = idx % kU2N, kg = kq + idx / kU2N;
            X bv = rd[q] * opc<CJ>(rl[q]);   // B(j, p) as bval forms it; the 2 x 2 terms are rare
            if (kg + 1 < K && !is_zero(re[q]))
                bv += opc<CJ>(re[q]) * opc<CJ>(ldv<float, C>(L, brow + r + (int64_t)(j0 + kg + 1) * f.m));
            if (kg >= 1 && !is_zero(rem1[q])) bv += rem1[q] * opc<CJ>(ldv<float, C>(L, brow + r + (int64_t)(j0 + kg - 1) * f.m));
            sB[buf][idx / kU2N][r] = bv;
        }
    };

    X acc[8][4];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = X{};
    const int ns = (K + BK - 1) / BK;
    fetch(0);
    stage(0, 0);
    __syncthreads();
    for (int sl = 0; sl < ns; ++sl) {
        const int buf = sl & 1;
        if (sl + 1 < ns) fetch((sl + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            X av[8], bv[4];
            // rows 32 h + 2 tx + {0, 1} (h < 4), columns 4 ty .. 4 ty + 3
            if constexpr (C) {
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const float4 v = *reinterpret_cast<const float4*>(&sA[buf][kk][32 * h + 2 * tx]);
                    av[2 * h] = X{v.x, v.y};
                    av[2 * h + 1] = X{v.z, v.w};
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const float4 v = *reinterpret_cast<const float4*>(&sB[buf][kk][4 * ty + 2 * h]);
                    bv[2 * h] = X{v.x, v.y};
                    bv[2 * h + 1] = X{v.z, v.w};
                }
            } else {
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const float2 v = *reinterpret_cast<const float2*>(&sA[buf][kk][32 * h + 2 * tx]);
                    av[2 * h] = v.x;
                    av[2 * h + 1] = v.y;
                }
                const float4 v = *reinterpret_cast<const float4*>(&sB[buf][kk][4 * ty]);
                bv[0] = v.x; bv[1] = v.y; bv[2] = v.z; bv[3] = v.w;
            }
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) mac(acc[a][b], av[a], bv[b]);
        }
        if (sl + 1 < ns) stage(buf ^ 1, (sl + 1) * BK);
        __syncthreads();
    }
    const int64_t cbase = base + j1 + (int64_t)j1 * f.m;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = jb0 + 4 * ty + b;
        if (j >= N) continue;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int i = i0 + 32 * (a >> 1) + 2 * tx + (a & 1);
            if (i < M && i >= j) {   // one tile writes each entry per launch
                const int64_t e = cbase + i + (int64_t)j * f.m;
                stv<float, C>(L, e, ldv<float, C>(L, e) - acc[a][b]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// inverses of the 64 x 64 diagonal blocks of the unit lower L11 (the sweeps'
// dinv / dinvT blocks), one CTA of 64 threads per block
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void __launch_bounds__(kTile) bk_dinv_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                        const T* __restrict__ L, T* __restrict__ dinv, T* __restrict__ dinvT) {
    using X = V<T, C>;
    extern __shared__ __align__(16) unsigned char bk_dinv_smem[];
    X* s_a = reinterpret_cast<X*>(bk_dinv_smem);   // the block's strictly lower part, kTile x (kTile + 1)
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int b = it.y, k = b * kTile, kb = min(kTile, f.n - k);
    const int c = threadIdx.x;
    for (int r = 0; r < kTile; ++r)
        s_a[r + c * (kTile + 1)] = (r > c && r < kb && c < kb) ? ldv<T, C>(L, f.L + (k + r) + (int64_t)(k + c) * f.m) : X{};
    __syncthreads();
    // column c of the inverse, written in place: x(c) = 1, x(r) = -sum_{c <= t < r} L(r, t) x(t)
    X* Dv = reinterpret_cast<X*>(dinv) + f.dinv + (int64_t)b * kTile * kTile;
    for (int r = 0; r < kTile; ++r) {
        X x{};
        if (c < kb && r == c) x = vone<X>();
        else if (c < kb && r > c && r < kb) {
            for (int t = c; t < r; ++t) mac(x, s_a[r + t * (kTile + 1)], Dv[t + c * kTile]);
            x = neg(x);
        }
        Dv[r + c * kTile] = x;
    }
    if (dinvT) {
        __syncthreads();
        X* DvT = reinterpret_cast<X*>(dinvT) + f.dinv + (int64_t)b * kTile * kTile;
        for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
            const int cc = idx % kTile, i = idx / kTile;
            DvT[cc + i * kTile] = Dv[i + cc * kTile];
        }
    }
}

// ---------------------------------------------------------------------------
// 2xFP16 split of a level's Schur complements on the tensor cores: largest
// |component| of each row of L21 and of S21 = B = L21 D (D with its 2 x 2
// blocks), over the front's n columns, into the two halves of erow (float
// bits), one thread per row below the pivots
// ---------------------------------------------------------------------------
template <bool C, bool CJ>
__global__ void __launch_bounds__(256) bk_rowmax_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl, int chunks,
                                                        const float* __restrict__ L, const double* __restrict__ D,
                                                        const double* __restrict__ E, uint32_t* __restrict__ erow, int64_t erow_total) {
    using X = V<float, C>;
    using W = DV<C>;
    const int fi = blockIdx.x / chunks, ch = blockIdx.x % chunks;
    const FrontDev f = F[fl[fi]];
    const int i = f.n + ch * 256 + threadIdx.x;
    if (i >= f.m) return;
    const int64_t row = f.L + i;
    float ml = 0.f, ms = 0.f;
    X prev{}, cur = f.n > 0 ? ldv<float, C>(L, row) : X{};
    X em1{};
    for (int k = 0; k < f.n; ++k) {
        const X next = k + 1 < f.n ? ldv<float, C>(L, row + (int64_t)(k + 1) * f.m) : X{};
        const X d = conv<X>(reinterpret_cast<const W*>(D)[f.off + k]);
        const X e = conv<X>(reinterpret_cast<const W*>(E)[f.off + k]);
        X b = d * opc<CJ>(cur);
        if (!is_zero(e)) b += opc<CJ>(e) * opc<CJ>(next);
        if (!is_zero(em1)) b += em1 * opc<CJ>(prev);
        if constexpr (C) {
            ml = fmaxf(ml, fmaxf(fabsf(cur.r), fabsf(cur.i)));
            ms = fmaxf(ms, fmaxf(fabsf(b.r), fabsf(b.i)));
        } else {
            ml = fmaxf(ml, fabsf(cur));
            ms = fmaxf(ms, fabsf(b));
        }
        prev = cur;
        cur = next;
        em1 = e;
    }
    erow[f.erow + i] = __float_as_uint(ml);
    erow[erow_total + f.erow + i] = __float_as_uint(ms);
}

// ---------------------------------------------------------------------------
// index maps for the solves in the pivoted order
// ---------------------------------------------------------------------------
__global__ void remap_positions_kernel(int64_t n, const int32_t* __restrict__ pivg, const int32_t* __restrict__ perm,
                                       int32_t* __restrict__ qpos, int32_t* __restrict__ perm_piv) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t g = pivg[q];
        qpos[g] = (int32_t)q;
        perm_piv[q] = perm[g];
    }
}

__global__ void remap_lower_kernel(int64_t cnt, const int32_t* __restrict__ qpos, const int32_t* __restrict__ lower_orig,
                                   int32_t* __restrict__ lower) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < cnt; r += (int64_t)gridDim.x * blockDim.x)
        lower[r] = qpos[lower_orig[r]];
}

// parent row i < n gathers / scatters what the assembled row pivg[off + i] did
__global__ void remap_cmaps_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ pivg,
                                   const int32_t* __restrict__ cmaps_orig, int32_t* __restrict__ cmaps) {
    const FrontDev f = F[blockIdx.x];
    if (f.cmap < 0) return;
    for (int i = threadIdx.x; i < f.n; i += blockDim.x) {
        const int src = pivg[f.off + i] - f.off;
        cmaps[f.cmap + i] = cmaps_orig[f.cmap + src];
        cmaps[f.cmap + f.m + i] = cmaps_orig[f.cmap + f.m + src];
    }
}

// quasi-diagonal solve X := D^{-1} X (diagonal_solve.hpp:53-59): a 2 x 2
// block [[d11, op(e)], [e, d22]] starting at p is solved by p's thread
template <class T, bool C, bool CJ>
__global__ void quasi_diag_kernel(T* __restrict__ X, int64_t ldx, int64_t n, int nrhs, const double* __restrict__ D,
                                  const double* __restrict__ E) {
    using Xv = V<T, C>;
    using W = DV<C>;
    const W* d = reinterpret_cast<const W*>(D);
    const W* e = reinterpret_cast<const W*>(E);
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        if (p > 0 && !is_zero(e[p - 1])) continue;   // second row of a 2 x 2 block
        if (!is_zero(e[p])) {
            const W d11 = d[p], d22 = d[p + 1], d21 = e[p];
            const W det = d11 * d22 - d21 * opc<CJ>(d21);
            for (int j = 0; j < nrhs; ++j) {
                const W b0 = conv<W>(ldv<T, C>(X, p + j * ldx)), b1 = conv<W>(ldv<T, C>(X, p + 1 + j * ldx));
                stv<T, C>(X, p + j * ldx, conv<Xv>((d22 * b0 - opc<CJ>(d21) * b1) / det));
                stv<T, C>(X, p + 1 + j * ldx, conv<Xv>((d11 * b1 - d21 * b0) / det));
            }
        } else {
            const W dp = d[p];
            for (int j = 0; j < nrhs; ++j) stv<T, C>(X, p + j * ldx, conv<Xv>(conv<W>(ldv<T, C>(X, p + j * ldx)) / dp));
        }
    }
}

template <class T, bool C, bool CJ>
static int level_t(Plan& P, int depth, cudaStream_t st, bool schur) {
    const SolveLevel& lv = P.solve_levels[depth];
    if (lv.nfronts <= 0) return CLIQ_OK;
    const int32_t* fl = P.level_fronts + lv.fronts;
    int max_n = 0, max_u = 0;
    for (int s : P.level_list[depth]) {
        max_n = std::max(max_n, P.hfronts[s].n);
        max_u = std::max(max_u, P.hfronts[s].m - P.hfronts[s].n);
    }
    T* L = reinterpret_cast<T*>(P.L);
    T* p0 = reinterpret_cast<T*>(P.pool[0]);
    T* p1 = reinterpret_cast<T*>(P.pool[1]);
    T* cvec = reinterpret_cast<T*>(P.pvec);
    T* vvec = cvec + (C ? 2 : 1) * P.n;
    const size_t smem_lower = sizeof(V<T, C>) * kMaxPanel * (kMaxPanel + kLowerRows);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(bk_lower_kernel<T, C, CJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_lower);
        attr = true;
    }
    const int chunks = std::max(1, (max_u + kLowerRows - 1) / kLowerRows);
    auto tiles = [](int64_t M, int64_t N) -> int64_t {
        if (M <= 0 || N <= 0) return 0;
        const int64_t Mt = (M + kUpdTile - 1) / kUpdTile, Nt = (N + kUpdTile - 1) / kUpdTile;
        return Nt * Mt - Nt * (Nt - 1) / 2;
    };
    const int steps = (max_n + kNb - 1) / kNb;
    // FP32: the in-front updates on bk_update2_kernel (CLIQGPU_PIV_UPDATE=tile64 keeps bk_update_kernel)
    const char* upd_env = std::getenv("CLIQGPU_PIV_UPDATE");
    const bool tile64 = upd_env && std::string(upd_env) == "tile64";
    const bool wide = std::is_same<T, float>::value && !tile64;
    // FP64: the in-front updates on DMMA where the plan's FP64 updates are
    const bool dmma_front = std::is_same<T, double>::value && P.fp64_dmma && !tile64;
    // the top levels (a few large fronts): each front's panels on a cluster
    // of kClusterCTAs CTAs; a refused cluster launch falls back to one CTA a front
    const bool clustered = (int64_t)lv.nfronts * kClusterCTAs <= 148 && max_n >= 512;
    // one CTA a front otherwise; a column step works over the front's pivot
    // rows only, so fronts of at most 128 / 256 pivots take CTAs of that many
    // threads (several CTAs a SM on the deep levels' many small fronts; at
    // least kMaxPanel threads, which the panel's per-column loads need)
    const int narrow = max_n <= 128 ? 128 : max_n <= 256 ? 256 : panel_threads<T>();
    static_assert(kMaxPanel <= 128, "panel CTAs of 128 threads");
    for (int step = 0; step < steps; ++step) {
        bool done = false;
        if (clustered) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)(lv.nfronts * kClusterCTAs));
            cfg.blockDim = dim3(panel_threads<T>());
            cfg.dynamicSmemBytes = 0;
            cfg.stream = st;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = kClusterCTAs;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            done = cudaLaunchKernelEx(&cfg, bk_panel_kernel<T, C, CJ, kClusterCTAs>, (const FrontDev*)P.fronts, fl, L, P.D, P.E,
                                      P.pivg, cvec, vvec, P.pstate, P.status) == cudaSuccess;
            if (!done) cudaGetLastError();
        }
        if (!done)
            bk_panel_kernel<T, C, CJ><<<(unsigned)lv.nfronts, narrow, 0, st>>>(P.fronts, fl, L, P.D, P.E, P.pivg, cvec, vvec,
                                                                           P.pstate, P.status);
        if (max_u > 0)
            bk_lower_kernel<T, C, CJ><<<(unsigned)((int64_t)lv.nfronts * chunks), kLowerRows, smem_lower, st>>>(
                P.fronts, fl, chunks, L, P.D, P.E, P.pstate);
        // every panel is at least kNb wide until the front is done, so the
        // trailing extents below bound the ones the kernels read from pstate
        int64_t tpf = 0;
        for (int s : P.level_list[depth]) {
            const FrontDev& f = P.hfronts[s];
            const int64_t jb = std::min<int64_t>(f.n, (int64_t)(step + 1) * kNb);
            tpf = std::max(tpf, wide ? upd2_tiles_dev(f.m - jb, f.n - jb) : tiles(f.m - jb, f.n - jb));
        }
        if (tpf > 0) {
            if constexpr (std::is_same<T, double>::value) {
                if (dmma_front) {   // 64 x 64 tiles, the same tile count as bk_update_kernel's
                    TRY(launch_dmma_front_update(P, fl, lv.nfronts, tpf, st));
                    P.total_launches += 3;
                    continue;
                }
            }
            if constexpr (std::is_same<T, float>::value) {
                if (wide) {
                    bk_update2_kernel<C, CJ><<<(unsigned)((int64_t)lv.nfronts * tpf), kUpdThreads, 0, st>>>(
                        P.fronts, fl, tpf, L, P.D, P.E, P.pstate);
                    P.total_launches += 3;
                    continue;
                }
            }
            bk_update_kernel<T, C, CJ><<<(unsigned)((int64_t)lv.nfronts * tpf), kUpdThreads, 0, st>>>(
                P.fronts, fl, tpf, 0, L, p0, p1, P.D, P.E, P.pstate);
        }
        P.total_launches += 3;
    }
    if (!schur) return check_cuda("pivoted level");   // the Schur complements go to the tensor cores
    // the Schur complement of every front of the level, K = n
    int64_t tpf = 0;
    for (int s : P.level_list[depth]) tpf = std::max(tpf, tiles(P.hfronts[s].m - P.hfronts[s].n, P.hfronts[s].m - P.hfronts[s].n));
    if (tpf > 0)
        bk_update_kernel<T, C, CJ><<<(unsigned)((int64_t)lv.nfronts * tpf), kUpdThreads, 0, st>>>(P.fronts, fl, tpf, 1, L, p0, p1,
                                                                                                   P.D, P.E, P.pstate);
    P.total_launches += 1;
    return check_cuda("pivoted level");
}

template <class T, bool C, bool CJ>
static int finish_t(Plan& P, cudaStream_t st) {
    const size_t smem = sizeof(V<T, C>) * kTile * (kTile + 1);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(bk_dinv_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    if (P.pivot_dinv_items > 0)
        bk_dinv_kernel<T, C><<<(unsigned)P.pivot_dinv_items, kTile, smem, st>>>(P.fronts, reinterpret_cast<const int4*>(P.pivot_items),
                                                                            reinterpret_cast<const T*>(P.L), reinterpret_cast<T*>(P.dinv),
                                                                            reinterpret_cast<T*>(P.dinvT));
    const unsigned g = grid1d(P.n, 256);
    remap_positions_kernel<<<g, 256, 0, st>>>(P.n, P.pivg, P.perm, P.qpos, P.perm_piv);
    if (P.lower_len > 0) remap_lower_kernel<<<grid1d(P.lower_len, 256), 256, 0, st>>>(P.lower_len, P.qpos, P.lower_orig, P.lower);
    if (P.num_fronts > 0) remap_cmaps_kernel<<<(unsigned)P.num_fronts, 256, 0, st>>>(P.fronts, P.pivg, P.cmaps_orig, P.cmaps);
    P.total_launches += 4;
    return check_cuda("pivoted maps");
}

}  // namespace piv

// allocations on first use; the extend-add's maps in assembled order
int pivot_begin(Plan& P, cudaStream_t st) {
    const int w = P.cplx() ? 2 : 1;
    auto alloc = [&](void** p, size_t bytes) -> int {
        if (*p) return CLIQ_OK;
        if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("cudaMalloc failed for the pivoted factorization's buffers");
            return CLIQ_ERR_OOM;
        }
        P.device_bytes += (int64_t)std::max<size_t>(bytes, 16);
        return CLIQ_OK;
    };
    const bool first = P.E == nullptr;
    TRY(alloc((void**)&P.E, sizeof(double) * w * (size_t)P.n));
    TRY(alloc((void**)&P.pivg, sizeof(int32_t) * (size_t)P.n));
    TRY(alloc((void**)&P.qpos, sizeof(int32_t) * (size_t)P.n));
    TRY(alloc((void**)&P.perm_piv, sizeof(int32_t) * (size_t)P.n));
    TRY(alloc((void**)&P.cmaps_orig, sizeof(int32_t) * (size_t)P.cmaps_len));
    TRY(alloc((void**)&P.lower_orig, sizeof(int32_t) * (size_t)P.lower_len));
    TRY(alloc((void**)&P.pstate, sizeof(int32_t) * 2 * (size_t)P.num_fronts));
    TRY(alloc(&P.pvec, (size_t)P.elem_bytes() * 2 * (size_t)P.n));
    if (first) {
        if (P.cmaps_len > 0) cudaMemcpyAsync(P.cmaps_orig, P.cmaps, sizeof(int32_t) * P.cmaps_len, cudaMemcpyDeviceToDevice, st);
        if (P.lower_len > 0) cudaMemcpyAsync(P.lower_orig, P.lower, sizeof(int32_t) * P.lower_len, cudaMemcpyDeviceToDevice, st);
        // the 64-blocks of every front, for the diagonal-block inverses
        std::vector<int32_t> items;
        for (int s = 0; s < P.num_fronts; ++s)
            for (int b = 0; b * kTile < P.hfronts[s].n; ++b) { items.push_back(s); items.push_back(b); items.push_back(0); items.push_back(0); }
        P.pivot_dinv_items = (int32_t)(items.size() / 4);
        if (items.empty()) items.assign(4, 0);
        TRY(alloc((void**)&P.pivot_items, sizeof(int32_t) * items.size()));
        if (cudaMemcpyAsync(P.pivot_items, items.data(), sizeof(int32_t) * items.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return check_cuda("pivot items");
        if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("pivot items");   // items is host memory
    }
    cudaMemsetAsync(P.pstate, 0, sizeof(int32_t) * 2 * (size_t)P.num_fronts, st);
    return check_cuda("pivoted factorization setup");
}

// the solves' maps back in assembled order (an unpivoted factorization after a pivoted one)
int pivot_restore_maps(Plan& P, cudaStream_t st) {
    if (!P.maps_pivoted) return CLIQ_OK;
    if (P.cmaps_len > 0) cudaMemcpyAsync(P.cmaps, P.cmaps_orig, sizeof(int32_t) * P.cmaps_len, cudaMemcpyDeviceToDevice, st);
    if (P.lower_len > 0) cudaMemcpyAsync(P.lower, P.lower_orig, sizeof(int32_t) * P.lower_len, cudaMemcpyDeviceToDevice, st);
    P.maps_pivoted = false;
    return check_cuda("restore maps");
}

int pivot_level(Plan& P, int depth, cudaStream_t st, bool schur) {
    if (depth < 0 || depth > P.max_depth) return CLIQ_OK;
    const bool cj = P.conjugate && P.cplx();
    if (P.precision == CLIQ_FP64) {
        if (!P.cplx()) return piv::level_t<double, false, false>(P, depth, st, schur);
        return cj ? piv::level_t<double, true, true>(P, depth, st, schur) : piv::level_t<double, true, false>(P, depth, st, schur);
    }
    if (!P.cplx()) return piv::level_t<float, false, false>(P, depth, st, schur);
    return cj ? piv::level_t<float, true, true>(P, depth, st, schur) : piv::level_t<float, true, false>(P, depth, st, schur);
}

// row maxima of the level's Schur operands for the 2xFP16 split (FP32 plans)
int pivot_rowmax(Plan& P, int depth, cudaStream_t st) {
    const SolveLevel& lv = P.solve_levels[depth];
    if (lv.nfronts <= 0 || !P.erow || P.precision != CLIQ_FP32) return CLIQ_OK;
    int max_u = 0;
    for (int s : P.level_list[depth]) max_u = std::max(max_u, P.hfronts[s].m - P.hfronts[s].n);
    if (max_u <= 0) return CLIQ_OK;
    const int chunks = (max_u + 255) / 256;
    const unsigned g = (unsigned)((int64_t)lv.nfronts * chunks);
    const int32_t* fl = P.level_fronts + lv.fronts;
    const float* L = reinterpret_cast<const float*>(P.L);
    if (!P.cplx()) piv::bk_rowmax_kernel<false, false><<<g, 256, 0, st>>>(P.fronts, fl, chunks, L, P.D, P.E, P.erow, P.erow_total);
    else if (P.conjugate) piv::bk_rowmax_kernel<true, true><<<g, 256, 0, st>>>(P.fronts, fl, chunks, L, P.D, P.E, P.erow, P.erow_total);
    else piv::bk_rowmax_kernel<true, false><<<g, 256, 0, st>>>(P.fronts, fl, chunks, L, P.D, P.E, P.erow, P.erow_total);
    P.total_launches += 1;
    return check_cuda("pivoted row maxima");
}

int pivot_finish(Plan& P, cudaStream_t st) {
    const bool cj = P.conjugate && P.cplx();
    int r;
    if (P.precision == CLIQ_FP64) {
        if (!P.cplx()) r = piv::finish_t<double, false, false>(P, st);
        else r = cj ? piv::finish_t<double, true, true>(P, st) : piv::finish_t<double, true, false>(P, st);
    } else {
        if (!P.cplx()) r = piv::finish_t<float, false, false>(P, st);
        else r = cj ? piv::finish_t<float, true, true>(P, st) : piv::finish_t<float, true, false>(P, st);
    }
    if (r == CLIQ_OK) P.maps_pivoted = true;
    return r;
}

int launch_quasi_diag(Plan& P, void* X, int64_t ldx, int nrhs) {
    const unsigned g = 1184;
    const bool cj = P.conjugate && P.cplx();
    if (P.precision == CLIQ_FP64) {
        if (!P.cplx()) piv::quasi_diag_kernel<double, false, false><<<g, 256, 0, P.stream>>>((double*)X, ldx, P.n, nrhs, P.D, P.E);
        else if (cj) piv::quasi_diag_kernel<double, true, true><<<g, 256, 0, P.stream>>>((double*)X, ldx, P.n, nrhs, P.D, P.E);
        else piv::quasi_diag_kernel<double, true, false><<<g, 256, 0, P.stream>>>((double*)X, ldx, P.n, nrhs, P.D, P.E);
    } else {
        if (!P.cplx()) piv::quasi_diag_kernel<float, false, false><<<g, 256, 0, P.stream>>>((float*)X, ldx, P.n, nrhs, P.D, P.E);
        else if (cj) piv::quasi_diag_kernel<float, true, true><<<g, 256, 0, P.stream>>>((float*)X, ldx, P.n, nrhs, P.D, P.E);
        else piv::quasi_diag_kernel<float, true, false><<<g, 256, 0, P.stream>>>((float*)X, ldx, P.n, nrhs, P.D, P.E);
    }
    return check_cuda("quasi-diagonal solve");
}

}  // namespace cliqgpu
