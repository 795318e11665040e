// Numeric multifrontal factorization on the device.
//
// The reference factors one front at a time in post-order (LocalLDL,
// include/clique/numeric/ldl/local.hpp:25-122): zero the update, extend-add
// the two children's updates through leftRelInds/rightRelInds, then
// FrontLDL (ldl/local_front.hpp:30-71) -- a right-looking loop over nb-wide
// column blocks doing LDL of the diagonal block, a TRSM of the panel, the
// in-front GEMM update of the remaining panel columns and a rank-nb Trrk
// update of ABR.
//
// Here every tree level (all fronts at one depth) is processed at once:
//   1. extend_add_kernel  -- gather form of the extend-add: each entry of the
//      parent's lower triangle is written exactly once (frontL := children,
//      ABR := children, zero where no child contributes), using per-front
//      inverse maps of the relative indices; then A's entries of the level's
//      fronts are added (assemble_add_kernel), so the fronts are never
//      cleared or read before this point.
//   2. for k in steps of nb over the level's widest front:
//        diag_ldl_kernel  -- LDL of the kb x kb diagonal block in shared memory
//                            (FP64 arithmetic for FP64 storage, FP32 for FP32
//                            storage), writes L11, D (FP64), U = L11^{-T} and
//                            L11^{-1} for the solves.
//        panel_kernel     -- S21 = A21 U, L21 = S21 D^{-1} (row blocks of 64).
//        gemm (trailing)  -- A22 -= L21 D L21^T over the remaining panel columns.
//   3. gemm (Schur)       -- ABR -= L_B D L_B^T once with K = n, instead of the
//      reference's n/nb rank-nb Trrk passes (same sum, one pass over ABR).
// D is kept in FP64 for every storage precision.
#include <climits>
#include <mutex>
#include <string>
#include <vector>
#include <cstdio>
#include <type_traits>

#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

constexpr int kThreads = 256;

__device__ __forceinline__ float cabsmax(float v) { return fabsf(v); }
__device__ __forceinline__ float cabsmax(double v) { return (float)fabs(v); }
__device__ __forceinline__ float cabsmax(cx<float> v) { return fmaxf(fabsf(v.r), fabsf(v.i)); }
__device__ __forceinline__ float cabsmax(cx<double> v) { return (float)fmax(fabs(v.r), fabs(v.i)); }

// ---------------------------------------------------------------------------
// 1. extend-add (gather form)
//
// Work item (front, j0, i0): columns j0 .. j0+15, rows i0 .. i0+kEARows-1 on
// or below the diagonal.  The children's maps of the item's rows and
// columns are staged in shared memory once; the CTA then sweeps one column at a time
// down a contiguous run of rows (consecutive threads, consecutive rows: few
// DRAM pages open per CTA), each thread issuing the gathers of all its rows
// of the column before any store.
// ---------------------------------------------------------------------------
constexpr int kEAPer = kEARows / kThreads;   // rows of a column per thread
static_assert(kEARows % kThreads == 0, "whole rows per thread");

template <class T, bool C>
__global__ void __launch_bounds__(kThreads) extend_add_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                              T* __restrict__ L, T* __restrict__ pool0, T* __restrict__ pool1,
                                                              const int32_t* __restrict__ cmaps) {
    using X = V<T, C>;
    __shared__ int32_t s_map[2][kEARows];
    __shared__ int32_t s_cmap[2][kEACols];
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int j0 = it.y, i0 = it.z;
    T* up = f.pool == 0 ? pool0 : pool1;
    const T* cp = f.pool == 0 ? pool1 : pool0;
    const int32_t* lm = f.cmap >= 0 ? cmaps + f.cmap : nullptr;
    const int32_t* rm = lm ? lm + f.m : nullptr;
    const int i_end = min(f.m, i0 + kEARows);
    const int j_end = min(f.m, j0 + kEACols);
    for (int i = max(j0, i0) + threadIdx.x; i < i_end; i += kThreads) {
        s_map[0][i - i0] = lm ? lm[i] : -1;
        s_map[1][i - i0] = rm ? rm[i] : -1;
    }
    if (threadIdx.x < kEACols) {
        const int j = j0 + threadIdx.x;
        s_cmap[0][threadIdx.x] = (lm && j < j_end) ? lm[j] : -1;
        s_cmap[1][threadIdx.x] = (rm && j < j_end) ? rm[j] : -1;
    }
    __syncthreads();
    for (int j = j0; j < j_end; ++j) {
        const int lj = s_cmap[0][j - j0], rj = s_cmap[1][j - j0];
        const int ib = max(j, i0) + threadIdx.x;
        X v[kEAPer];
#pragma unroll
        for (int u = 0; u < kEAPer; ++u) {
            const int i = ib + u * kThreads;
            X t = X{};
            if (i < i_end) {
                const int li = lj >= 0 ? s_map[0][i - i0] : -1, ri = rj >= 0 ? s_map[1][i - i0] : -1;
                if (li >= 0) t += ldv<T, C>(cp, f.CU[0] + li + (int64_t)lj * f.cu[0]);
                if (ri >= 0) t += ldv<T, C>(cp, f.CU[1] + ri + (int64_t)rj * f.cu[1]);
            }
            v[u] = t;
        }
#pragma unroll
        for (int u = 0; u < kEAPer; ++u) {
            const int i = ib + u * kThreads;
            if (i >= i_end) break;
            if (j < f.n) stv<T, C>(L, f.L + i + (int64_t)j * f.m, v[u]);
            else stv<T, C>(up, f.U + (i - f.n) + (int64_t)(j - f.n) * f.u, v[u]);
        }
    }
}

// ---------------------------------------------------------------------------
// 2a. LDL of the diagonal block (one CTA per front), FP64 in shared memory
//
// The kb x kb block (padded to 64 with an identity block) is factored in
// four 16-column steps p.  In each step the 256 threads hold the 16 x 16
// diagonal sub-block one entry each (full symmetric copy) together with the
// matching entry of a running inverse (Gaussian elimination on [P | I]);
// one barrier per pivot, the working copies double-buffered by pivot
// parity, and the reciprocal of the next pivot computed by its owner right
// after its own update, so the per-pivot critical path is one update, one
// reciprocal and one barrier.  Then G = A_ip op(L_pp^{-1})^T,
// L_ip = G D_p^{-1} and the rank-16 update A_22 -= G op(L_2p)^T (2 x 2
// register tiles).  Finally the off-diagonal 16 x 16 blocks of L^{-1}:
//   Linv_ij = -Linv_ii * sum_{k=j}^{i-1} L_ik Linv_kj,   i > j.
// Storage: sA holds A / L column-major in its lower triangle and, once
// formed, Linv(r, c) (r > c) at the mirrored position sA[r * 65 + c].
// Outputs: L11 (unit diagonal) and D to global memory, U = op(L11^{-1})^T
// for the panel kernel, and L11^{-1} column-major (forward sweep) and
// row-major (backward sweep).
// ---------------------------------------------------------------------------
constexpr int kDiagLd = kTile + 1;
constexpr int kSub = 16;
constexpr int kSubLd = kSub + 1;

// working type of the diagonal-block factorization: WT real or complex
template <class WT, bool C>
using DiagW = typename std::conditional<C, cx<WT>, WT>::type;

template <class WT, bool C>
__host__ __device__ constexpr size_t diag_smem_bytes() {
    // sA, sG, 2 x (P, X) sub-block buffers, d, 1/d
    return sizeof(DiagW<WT, C>) * (size_t)(kTile * kDiagLd + kTile * kSub + 4 * kSub * kSubLd + 2 * kTile);
}

// Reciprocal of a pivot, on the critical path of every elimination step.
// 1/x for x within float range: Newton-Raphson iteration y <- y (2 - x y)
// from the single-precision reciprocal (about 23 correct bits, two steps
// give full double precision); outside that range the IEEE reciprocal.
// Complex: conj(d) / |d|^2, with d scaled by a power of two when |d|^2
// would leave the range.
__device__ __forceinline__ double recip_nr(double x) {
    const double ax = fabs(x);
    if (!(ax > 1e-30 && ax < 1e30)) return __drcp_rn(x);
    double y = (double)__frcp_rn((float)x);
    y = y * fma(-x, y, 2.0);
    y = y * fma(-x, y, 2.0);
    return y;
}
__device__ __forceinline__ float pivot_recip(float d) { return __frcp_rn(d); }
__device__ __forceinline__ cx<float> pivot_recip(cx<float> d) {
    const float n2 = fmaf(d.r, d.r, d.i * d.i);
    if (n2 > 1e-36f && n2 < 1e36f) {
        const float s = __frcp_rn(n2);
        return {d.r * s, -d.i * s};
    }
    const float mx = fmaxf(fabsf(d.r), fabsf(d.i));
    const int e = ((__float_as_int(mx) >> 23) & 0xff) - 127;
    const float sc = __int_as_float((127 - e) << 23);   // 2^-e
    const float xr = d.r * sc, xi = d.i * sc;
    const float s = __frcp_rn(fmaf(xr, xr, xi * xi)) * sc;
    return {xr * s, -xi * s};
}
__device__ __forceinline__ double pivot_recip(double d) { return recip_nr(d); }
__device__ __forceinline__ cx<double> pivot_recip(cx<double> d) {
    const double n2 = fma(d.r, d.r, d.i * d.i);
    if (n2 > 1e-30 && n2 < 1e30) {
        const double s = recip_nr(n2);
        return {d.r * s, -d.i * s};
    }
    const double mx = fmax(fabs(d.r), fabs(d.i));
    const int e = ((__double2hiint(mx) >> 20) & 0x7ff) - 1023;
    const double sc = __hiloint2double((1023 - e) << 20, 0);   // 2^-e
    const double xr = d.r * sc, xi = d.i * sc;
    const double s = __drcp_rn(fma(xr, xr, xi * xi)) * sc;
    return {xr * s, -xi * s};
}

template <class T, bool C, bool CJ, class WT>
__global__ void __launch_bounds__(kThreads, 2) diag_ldl_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items, int k,
                                                               T* __restrict__ L, double* __restrict__ D, T* __restrict__ tinv,
                                                               T* __restrict__ dinv, T* __restrict__ dinvT, int32_t* __restrict__ status) {
    using W = DiagW<WT, C>;
    using X = V<T, C>;
    constexpr int nb = kTile, ld = kDiagLd;
    static_assert(kThreads == kSub * kSub, "one thread per sub-block entry");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    W* sA = reinterpret_cast<W*>(smem_raw);        // 64 x 65, column-major
    W* sG = sA + nb * ld;                           // 64 x 16 scratch
    W* sP = sG + nb * kSub;                         // 2 x 16 x 17: sub-block working copy (by pivot parity)
    W* sX = sP + 2 * kSub * kSubLd;                 // 2 x 16 x 17: running inverse
    W* s_d = sX + 2 * kSub * kSubLd;
    W* s_rd = s_d + nb;
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int slot = it.y;
    const int kb = min(nb, f.n - k);
    const int tid = threadIdx.x;
    // lower triangle of the block, identity beyond kb; all 16 loads of a
    // thread are issued before the first one is used
    {
        constexpr int kPer = nb * nb / kThreads;
        X v[kPer];
        const int r = tid % nb;
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int c = tid / nb + (kThreads / nb) * q;
            v[q] = (r < kb && c < kb && r >= c) ? ldv<T, C>(L, f.L + (k + r) + (int64_t)(k + c) * f.m) : X{};
        }
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int c = tid / nb + (kThreads / nb) * q;
            if (r < c) continue;
            W w = conv<W>(v[q]);
            if (r >= kb && r == c) w = vone<W>();
            sA[c * ld + r] = w;
        }
    }
    __syncthreads();
    const int sr = tid % kSub, sc = tid / kSub;    // this thread's sub-block entry
    // unrolled: the rows below each sub-block (R = 48, 32, 16) become
    // compile-time constants in the index arithmetic of the panel and update loops
#pragma unroll
    for (int p = 0; p < nb / kSub; ++p) {
        const int b0 = kSub * p;
        if (b0 >= kb) break;   // the rest is the identity padding (kb < 64: small fronts, last blocks)
        // ---- 16 x 16 sub-block: LDL and inverse ----
        W a = sr >= sc ? sA[(b0 + sc) * ld + b0 + sr] : opc<CJ>(sA[(b0 + sr) * ld + b0 + sc]);
        W x = sr == sc ? vone<W>() : W{};
        sP[sc * kSubLd + sr] = a;
        sX[sc * kSubLd + sr] = x;
        if (tid == 0) {
            s_d[b0] = a;
            s_rd[b0] = pivot_recip(a);
            if (b0 < kb && is_zero(a)) atomicMin(&status[0], f.off + k + b0 + 1);
        }
        __syncthreads();
#pragma unroll 1
        for (int j = 0; j < kSub; ++j) {
            const W* P0 = sP + (j & 1) * kSub * kSubLd;
            const W* X0 = sX + (j & 1) * kSub * kSubLd;
            W* P1 = sP + ((j + 1) & 1) * kSub * kSubLd;
            W* X1 = sX + ((j + 1) & 1) * kSub * kSubLd;
            if (sr > j) {
                const W rd = s_rd[b0 + j];
                const W prj = P0[j * kSubLd + sr];                  // P[r][j]
                const W lrj = prj * rd;
                if (sc > j) a -= lrj * P0[sc * kSubLd + j];          // P[r][c] -= L[r][j] P[j][c]
                else if (sc == j) a = lrj;
                x -= lrj * X0[sc * kSubLd + j];                      // row r -= L[r][j] row j
            }
            P1[sc * kSubLd + sr] = a;
            X1[sc * kSubLd + sr] = x;
            if (sr == j + 1 && sc == j + 1) {
                s_d[b0 + j + 1] = a;
                s_rd[b0 + j + 1] = pivot_recip(a);
                if (b0 + j + 1 < kb && is_zero(a)) atomicMin(&status[0], f.off + k + b0 + j + 2);
            }
            __syncthreads();
        }
        if (sr > sc) {
            sA[(b0 + sc) * ld + b0 + sr] = a;      // L_pp
            sA[(b0 + sr) * ld + b0 + sc] = x;      // Linv_pp, mirrored
        }
        __syncthreads();
        const int R = nb - b0 - kSub;     // rows below the sub-block
        if (R == 0) break;
        const int i0 = b0 + kSub;
        // ---- panel: G = A_ip op(Linv_pp)^T, then L_ip = G D_p^{-1} ----
        for (int idx = tid; idx < R * kSub; idx += kThreads) {
            const int i = i0 + idx % R, c = idx / R;
            W g = sA[(b0 + c) * ld + i];
            for (int t = 0; t < c; ++t) g += sA[(b0 + t) * ld + i] * opc<CJ>(sA[(b0 + c) * ld + b0 + t]);
            sG[c * nb + i] = g;
        }
        __syncthreads();
        for (int idx = tid; idx < R * kSub; idx += kThreads) {
            const int i = i0 + idx % R, c = idx / R;
            sA[(b0 + c) * ld + i] = sG[c * nb + i] * s_rd[b0 + c];
        }
        __syncthreads();
        // ---- A_22 -= G op(L_2p)^T on the lower triangle, 2 x 2 tiles ----
        const int T2 = R / 2, ntile = T2 * (T2 + 1) / 2;
        for (int tt = tid; tt < ntile; tt += kThreads) {
            int ti = (int)((sqrtf(8.f * tt + 1.f) - 1.f) * 0.5f);
            while (ti * (ti + 1) / 2 > tt) --ti;
            while ((ti + 1) * (ti + 2) / 2 <= tt) ++ti;
            const int tj = tt - ti * (ti + 1) / 2;
            const int ri = i0 + 2 * ti, cj = i0 + 2 * tj;
            W a00{}, a01{}, a10{}, a11{};
#pragma unroll 4
            for (int t = 0; t < kSub; ++t) {
                const W g0 = sG[t * nb + ri], g1 = sG[t * nb + ri + 1];
                const W l0 = opc<CJ>(sA[(b0 + t) * ld + cj]), l1 = opc<CJ>(sA[(b0 + t) * ld + cj + 1]);
                a00 += g0 * l0; a01 += g0 * l1; a10 += g1 * l0; a11 += g1 * l1;
            }
            sA[cj * ld + ri] -= a00;
            sA[cj * ld + ri + 1] -= a10;
            sA[(cj + 1) * ld + ri + 1] -= a11;
            if (ri > cj) sA[(cj + 1) * ld + ri] -= a01;
        }
        __syncthreads();
    }
    // ---- off-diagonal blocks of L^{-1}, one block row at a time ----
    // Linv_ij = -Linv_ii sum_{k=j}^{i-1} L_ik Linv_kj; thread (r, c) forms entry
    // (r, c) of every block j < i of the row at once (independent sums)
    {
        const int r = tid % kSub, c = tid / kSub;
#pragma unroll
        for (int i = 1; i < nb / kSub; ++i) {
            if (kSub * i >= kb) break;   // block rows of the identity padding are not output
            const int R = kSub * i + r;
            W acc[nb / kSub - 1];
#pragma unroll
            for (int j = 0; j < i; ++j) acc[j] = W{};
#pragma unroll
            for (int kk = 0; kk < i; ++kk) {
#pragma unroll 4
                for (int t = 0; t < kSub; ++t) {
                    const W lik = sA[(kSub * kk + t) * ld + R];                   // L[R][16 kk + t]
#pragma unroll
                    for (int j = 0; j <= kk; ++j) {
                        // Linv[16 kk + t][16 j + c]; Linv_jj is unit lower triangular
                        const W lv = j < kk ? sA[(kSub * kk + t) * ld + kSub * j + c]
                                            : (t == c ? vone<W>() : (t > c ? sA[(kSub * kk + t) * ld + kSub * j + c] : W{}));
                        acc[j] += lik * lv;
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < i; ++j) sG[(j * kSub + c) * kSub + r] = acc[j];
            __syncthreads();
#pragma unroll
            for (int j = 0; j < i; ++j) acc[j] = sG[(j * kSub + c) * kSub + r];
            for (int t = 0; t < r; ++t) {
                const W lit = sA[R * ld + kSub * i + t];                            // Linv_ii[r][t]
#pragma unroll
                for (int j = 0; j < i; ++j) acc[j] += lit * sG[(j * kSub + c) * kSub + t];
            }
#pragma unroll
            for (int j = 0; j < i; ++j) sA[R * ld + kSub * j + c] = W{} - acc[j];
            __syncthreads();
        }
    }
    // ---- outputs, each written with consecutive threads on consecutive addresses ----
    X* U = reinterpret_cast<X*>(tinv) + (int64_t)slot * nb * nb;
    X* Dv = reinterpret_cast<X*>(dinv) + f.dinv + (int64_t)(k / nb) * nb * nb;
#pragma unroll 4
    for (int idx = tid; idx < nb * nb; idx += kThreads) {
        const int i = idx % nb, c = idx / nb;
        const bool in = i < kb && c < kb && i >= c;
        const W linv = i == c ? vone<W>() : (i > c ? sA[i * ld + c] : W{});
        U[c * nb + i] = in ? conv<X>(opc<CJ>(linv)) : X{};
        Dv[i + c * nb] = in ? conv<X>(linv) : X{};
        if (in) stv<T, C>(L, f.L + (k + i) + (int64_t)(k + c) * f.m, i == c ? vone<X>() : conv<X>(sA[c * ld + i]));
    }
    if (dinvT) {
        X* DvT = reinterpret_cast<X*>(dinvT) + f.dinv + (int64_t)(k / nb) * nb * nb;
#pragma unroll 4
        for (int idx = tid; idx < nb * nb; idx += kThreads) {
            const int c = idx % nb, i = idx / nb;
            const bool in = i < kb && c < kb && i >= c;
            const W linv = i == c ? vone<W>() : (i > c ? sA[i * ld + c] : W{});
            DvT[c + i * nb] = in ? conv<X>(linv) : X{};
        }
    }
    if (tid < kb) reinterpret_cast<DV<C>*>(D)[f.off + k + tid] = conv<DV<C>>(s_d[tid]);
}

// ---------------------------------------------------------------------------
// 2b. panel: S21 = A21 U, L21 = S21 D^{-1} for one 64-row block
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void __launch_bounds__(kThreads) panel_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items, int k,
                                                         T* __restrict__ L, const double* __restrict__ D, const T* __restrict__ tinv,
                                                         uint32_t* __restrict__ eblk,
                                                         uint32_t* __restrict__ erow,
                                                         int64_t eblk_total, int64_t erow_total) {
    using X = V<T, C>;
    using W = DV<C>;
    constexpr int nb = kTile, ldA = kTile + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    X* sU = reinterpret_cast<X*>(smem_raw);      // nb x nb row-major
    X* sA = sU + nb * nb;                          // 64 x ldA
    X* sR = sA + kTile * ldA;                      // reciprocal pivots
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int slot = it.y, rb = it.z;
    const int kb = min(nb, f.n - k);
    const int r0 = k + kb + kTile * rb;
    const int rows = min(kTile, f.m - r0);
    const X* U = reinterpret_cast<const X*>(tinv) + (int64_t)slot * nb * nb;
    for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) sU[idx] = U[idx];
    for (int idx = threadIdx.x; idx < kTile * nb; idx += blockDim.x) {
        const int r = idx % kTile, t = idx / kTile;
        X v{};
        if (r < rows && t < kb) v = ldv<T, C>(L, f.L + (r0 + r) + (int64_t)(k + t) * f.m);
        sA[r * ldA + t] = v;
    }
    if (threadIdx.x < kb) {
        const W d = reinterpret_cast<const W*>(D)[f.off + k + threadIdx.x];
        sR[threadIdx.x] = conv<X>(W{} + vone<W>() / d);
    }
    __syncthreads();
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    X acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = X{};
    for (int t = 0; t < kb; ++t) {
        X av[4], uv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) av[a] = sA[(ty + 16 * a) * ldA + t];
#pragma unroll
        for (int b = 0; b < 4; ++b) uv[b] = sU[t * nb + tx + 16 * b];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) mac(acc[a][b], av[a], uv[b]);
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int c = tx + 16 * b;
        if (c >= kb) continue;
        const X rd = sR[c];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int r = ty + 16 * a;
            if (r < rows) stv<T, C>(L, f.L + (r0 + r) + (int64_t)(k + c) * f.m, acc[a][b] * rd);
        }
    }
    // 2xFP16 split: largest |component| of each row of L21 and of S21 = D L21
    // over this block's columns (float bits, order-preserving for >= 0), per
    // block and as a running maximum over the front's blocks
    if (eblk) {
        const int nT = (f.n + nb - 1) / nb;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            float ml = 0.f, ms = 0.f;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int c = tx + 16 * b;
                if (c < kb) {
                    const X v = acc[a][b];
                    ms = fmaxf(ms, cabsmax(v));
                    ml = fmaxf(ml, cabsmax(v * sR[c]));
                }
            }
#pragma unroll
            for (int o = 8; o >= 1; o >>= 1) {
                ml = fmaxf(ml, __shfl_xor_sync(0xffffffffu, ml, o, 16));
                ms = fmaxf(ms, __shfl_xor_sync(0xffffffffu, ms, o, 16));
            }
            const int r = ty + 16 * a;
            if (tx == 0 && r < rows) {
                const int64_t row = r0 + r;
                const int64_t eb = f.eblk + row * nT + k / nb;
                eblk[eb] = __float_as_uint(ml);
                eblk[eblk_total + eb] = __float_as_uint(ms);
                atomicMax(&erow[f.erow + row], __float_as_uint(ml));
                atomicMax(&erow[erow_total + f.erow + row], __float_as_uint(ms));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// 2c. chain tiles for the triangular sweeps, formed once after the whole
// factorization.  For pivot block b >= 1 of a front, with the coupling tile
// S = L_{b,b-1} (rows of block b, columns of block b-1):
//   m1_b     = L_bb^{-1} S                          (forward chain)
//   n1_{b-1} = op(L_{b-1,b-1}^{-1})^T op(S)^T       (backward chain)
// both 64 x 64 column-major, zero outside the rows (m1) / columns (n1) of
// block b.  With them a chain step needs one 64 x 64 product with the newest
// solved block instead of two dependent ones.  One CTA per (front, b); each
// thread forms a 4 x 4 register tile of both products from shared memory.
// ---------------------------------------------------------------------------
template <class T, bool C>
__host__ __device__ constexpr size_t chain_tiles_smem_bytes() {
    return sizeof(V<T, C>) * 2 * kTile * (kTile + 1);
}

template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kThreads) chain_tiles_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                               const T* __restrict__ L, const T* __restrict__ dinv,
                                                               T* __restrict__ m1, T* __restrict__ n1) {
    using X = V<T, C>;
    constexpr int nb = kTile, ld = kTile + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    X* sS = reinterpret_cast<X*>(smem_raw);     // S(r, c) at sS[r + c * ld]
    X* sD = sS + nb * ld;                         // inverse block (r, c) at sD[r + c * ld]
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int b = it.y;
    const int db = min(nb, f.n - b * nb);         // rows of block b (block b - 1 is full)
    const int tid = threadIdx.x, ty = tid / 16, tx = tid % 16;
    const X* Dv = reinterpret_cast<const X*>(dinv) + f.dinv;
    for (int idx = tid; idx < nb * nb; idx += kThreads) {
        const int r = idx % nb, c = idx / nb;
        sS[r + c * ld] = r < db ? ldv<T, C>(L, f.L + (int64_t)(b * nb + r) + (int64_t)((b - 1) * nb + c) * f.m) : X{};
        sD[r + c * ld] = Dv[(int64_t)b * nb * nb + r + c * nb];
    }
    __syncthreads();
    X acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = X{};
    // m1_b(i, j) = sum_k Dinv_b(i, k) S(k, j)
    for (int k = 0; k < db; ++k) {
        X a[4], s[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = sD[ty + 16 * i + k * ld];
#pragma unroll
        for (int j = 0; j < 4; ++j) s[j] = sS[k + (tx + 16 * j) * ld];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) mac(acc[i][j], a[i], s[j]);
    }
    X* M = reinterpret_cast<X*>(m1) + f.chain + (int64_t)b * nb * nb;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) M[(ty + 16 * i) + (tx + 16 * j) * nb] = acc[i][j];
    __syncthreads();
    for (int idx = tid; idx < nb * nb; idx += kThreads) {
        const int r = idx % nb, c = idx / nb;
        sD[r + c * ld] = Dv[(int64_t)(b - 1) * nb * nb + r + c * nb];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = X{};
    // n1_{b-1}(i, j) = op(sum_k Dinv_{b-1}(k, i) S(j, k))
    for (int k = 0; k < nb; ++k) {
        X a[4], s[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = sD[k + (ty + 16 * i) * ld];
#pragma unroll
        for (int j = 0; j < 4; ++j) s[j] = sS[(tx + 16 * j) + k * ld];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) mac(acc[i][j], a[i], s[j]);
    }
    X* N = reinterpret_cast<X*>(n1) + f.chain + (int64_t)(b - 1) * nb * nb;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) N[(ty + 16 * i) + (tx + 16 * j) * nb] = opc<CJ>(acc[i][j]);
}

// ---------------------------------------------------------------------------
// 3. tiled update C -= A diag(d) op(B)^T on the lower trapezoid (i >= j)
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kThreads) gemm_update_kernel(const GemmProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                               int nprobs, const int32_t* __restrict__ bmap, T* __restrict__ L,
                                                               T* __restrict__ pool0, T* __restrict__ pool1, const double* __restrict__ D) {
    using X = V<T, C>;
    using W = DV<C>;
    constexpr int BM = 64, BK = C ? 8 : 16, PAD = 1;
    __shared__ X sA[BK][BM + PAD];
    __shared__ X sB[BK][BM + PAD];
    const int64_t bid = blockIdx.x;
    int lo = 0;
    if (bmap) {
        lo = bmap[bid];   // this tile's problem
    } else {
        int hi = nprobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= bid) lo = mid; else hi = mid - 1;
        }
    }
    const GemmProb pr = probs[lo];
    int64_t t = bid - prefix[lo];
    const int Mt = (pr.M + BM - 1) / BM, Nt = (pr.N + BM - 1) / BM;
    int tj = 0;
    while (tj < Nt && t >= Mt - tj) { t -= Mt - tj; ++tj; }
    if (tj >= Nt) return;   // cannot happen with a consistent schedule
    const int ti = tj + (int)t;
    const int i0 = ti * BM, j0 = tj * BM;
    T* Cbase = pr.cpool < 0 ? L : (pr.cpool == 0 ? pool0 : pool1);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    X acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = X{};
    for (int k0 = 0; k0 < pr.K; k0 += BK) {
#pragma unroll
        for (int q = 0; q < (BM * BK) / kThreads; ++q) {
            const int idx = threadIdx.x + kThreads * q;
            const int r = idx % BM, kk = idx / BM;
            const int kg = k0 + kk;
            X av{}, bv{};
            if (kg < pr.K) {
                if (i0 + r < pr.M) av = ldv<T, C>(L, pr.A + (i0 + r) + (int64_t)kg * pr.lda);
                if (j0 + r < pr.N) {
                    const X dv = conv<X>(reinterpret_cast<const W*>(D)[pr.d + kg]);
                    bv = dv * opc<CJ>(ldv<T, C>(L, pr.B + (j0 + r) + (int64_t)kg * pr.lda));
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
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int j = j0 + tx + 16 * b;
        if (j >= pr.N) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = i0 + ty + 16 * a;
            if (i < pr.M && i >= j) {
                // one reduction per element per launch: same result as load-subtract-store
                const int64_t e = pr.C + i + (int64_t)j * pr.ldc;
                if constexpr (C) {
                    atomicAdd(Cbase + 2 * e, -acc[a][b].r);
                    atomicAdd(Cbase + 2 * e + 1, -acc[a][b].i);
                } else {
                    atomicAdd(Cbase + e, -acc[a][b]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
// Working precision of the diagonal-block LDL: FP64 for FP64 storage; for
// FP32 storage FP32 unless the plan asks for FP64 (CLIQGPU_DIAG_FP64=1).
// The pivots are stored in FP64 either way.
template <class T, bool C, bool CJ, class WT>
static void launch_diag(const Plan& P, const Launch& ln, T* L, const int4* items, cudaStream_t st) {
    diag_ldl_kernel<T, C, CJ, WT><<<(unsigned)ln.nblocks, kThreads, diag_smem_bytes<WT, C>(), st>>>(
        P.fronts, items + ln.items, ln.k, L, P.D, reinterpret_cast<T*>(P.tinv), reinterpret_cast<T*>(P.dinv),
        reinterpret_cast<T*>(P.dinvT), P.status);
}

// captured: issue for a graph captured from stream1 (no dependency on the
// caller's stream inside; the replay wrapper forks and joins it)
template <class T, bool C, bool CJ>
static int64_t issue_factor(Plan& P, bool captured = false) {
    using X = V<T, C>;
    using W = DV<C>;
    const size_t smem_diag = diag_smem_bytes<double, C>();
    const size_t smem_panel = sizeof(X) * (kTile * kTile + kTile * (kTile + 1) + kTile);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(diag_ldl_kernel<T, C, CJ, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_diag);
        cudaFuncSetAttribute(diag_ldl_kernel<T, C, CJ, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)diag_smem_bytes<T, C>());
        cudaFuncSetAttribute(panel_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_panel);
        attr_done = true;
    }
    T* L = reinterpret_cast<T*>(P.L);
    T* p0 = reinterpret_cast<T*>(P.pool[0]);
    T* p1 = reinterpret_cast<T*>(P.pool[1]);
    const int4* items = reinterpret_cast<const int4*>(P.items);
    int64_t launches = 0;
    if (P.profile && P.events.size() < 3 * P.launches.size()) {
        const size_t old = P.events.size();
        P.events.resize(3 * P.launches.size());
        for (size_t i = old; i < P.events.size(); ++i) cudaEventCreate(&P.events[i]);
    }
    // Lookahead: the critical path (extend-add, diagonal blocks, panels,
    // in-panel and next-outer-block updates) on the high-priority stream1,
    // the updates of the columns two outer blocks and more to the right on
    // stream2.  Before the first diagonal block of outer block K the main
    // stream waits for the lookahead update of outer block K - 2 nbo (the
    // last one that writes columns of K); it joins stream2 completely before
    // each extend-add, each Schur update and the chain tiles.
    const bool la = P.stream2 != nullptr;
    cudaStream_t s1 = la ? P.stream1 : P.stream;
    const int nbo = std::max(P.nb, P.outer_nb / P.nb * P.nb);
    size_t next_ev = 0;
    cudaEvent_t last_done = nullptr, last_done3 = nullptr;
    struct Pending { int depth, k0; cudaEvent_t done; };
    std::vector<Pending> pending;
    if (la) {
        cudaEvent_t fork = P.sync_events[next_ev++];
        cudaEventRecord(fork, captured ? s1 : P.stream);
        if (!captured) cudaStreamWaitEvent(s1, fork, 0);
        cudaStreamWaitEvent(P.stream2, fork, 0);
        if (P.pack3) cudaStreamWaitEvent(P.stream3, fork, 0);   // stream3 only carries Schur chunks
    }
    auto join = [&]() {
        if (last_done) cudaStreamWaitEvent(s1, last_done, 0);
        if (last_done3) cudaStreamWaitEvent(s1, last_done3, 0);
        last_done = last_done3 = nullptr;
        pending.clear();
    };
    if (P.erow) cudaMemsetAsync(P.erow, 0, sizeof(uint32_t) * 2 * (size_t)P.erow_total, s1);
    for (size_t li = 0; li < P.launches.size(); ++li) {
        const Launch& ln = P.launches[li];
        if (ln.nblocks <= 0) continue;
        if (la) {
            if (ln.kind == Launch::EXTEND_ADD || (ln.kind == Launch::GEMM && ln.schur && !ln.bulk)) join();
            if (ln.kind == Launch::DIAG && ln.k % nbo == 0 && ln.k >= 2 * nbo)
                for (const Pending& pd : pending)
                    if (pd.depth == ln.depth && pd.k0 == ln.k - 2 * nbo) cudaStreamWaitEvent(s1, pd.done, 0);
        }
        const bool on2 = la && ln.bulk;
        cudaStream_t sb = ln.bulk == 2 ? P.stream3 : P.stream2;
        cudaStream_t st = on2 ? sb : s1;
        if (on2) {   // the lookahead update reads panels produced on stream1 so far
            cudaEvent_t fork = P.sync_events[next_ev++];
            cudaEventRecord(fork, s1);
            cudaStreamWaitEvent(sb, fork, 0);
        }
        if (P.profile) cudaEventRecord(P.events[3 * li], st);
        switch (ln.kind) {
            case Launch::EXTEND_ADD:
                extend_add_kernel<T, C><<<(unsigned)ln.nblocks, kThreads, 0, st>>>(P.fronts, items + ln.items, L, p0, p1, P.cmaps);
                launch_assemble_level(P, ln.depth, st);   // A's entries of this level's fronts
                break;
            case Launch::DIAG:
                if (std::is_same<T, float>::value && !P.diag_fp64) launch_diag<T, C, CJ, T>(P, ln, L, items, st);
                else launch_diag<T, C, CJ, double>(P, ln, L, items, st);
                break;
            case Launch::PANEL:
                if (std::is_same<T, float>::value && P.f16_scales()) {
                    launch_panel_tc(P, ln, st, P.pack);
                    break;
                }
                panel_kernel<T, C><<<(unsigned)ln.nblocks, kThreads, smem_panel, st>>>(
                    P.fronts, items + ln.items, ln.k, L, P.D, reinterpret_cast<const T*>(P.tinv), P.eblk, P.erow, P.eblk_total,
                    P.erow_total);
                break;
            case Launch::GEMM:
                if (std::is_same<T, float>::value && P.tensor_path() && !ln.simt)
                    launch_tc2(P, ln, P.profile ? P.events[3 * li + 2] : nullptr, st,
                               on2 ? (ln.bulk == 2 ? P.pack3 : P.pack2) : P.pack);
                else if (std::is_same<T, double>::value && P.fp64_dmma && !ln.simt)
                    launch_dmma_update(P, ln, st);
                else {   // CUDA cores, on the launch's 64 x 64 tiling
                    const bool alt = ln.alt_prefix >= 0;
                    gemm_update_kernel<T, C, CJ><<<(unsigned)(alt ? ln.alt_nblocks : ln.nblocks), kThreads, 0, st>>>(
                        P.probs + ln.items, P.prefix + (alt ? ln.alt_prefix : ln.prefix), ln.nitems,
                        P.bmap + (alt ? ln.alt_gemm_map : ln.gemm_map), L, p0, p1, P.D);
                }
                break;
        }
        if (P.profile) cudaEventRecord(P.events[3 * li + 1], st);
        if (on2) {
            cudaEvent_t done = P.sync_events[next_ev++];
            cudaEventRecord(done, sb);
            if (ln.bulk == 2) {
                last_done3 = done;
            } else {
                pending.push_back({ln.depth, ln.k, done});
                last_done = done;
            }
        }
        ++launches;
    }
    if (la) join();
    if (P.nchain_items > 0 && !P.solve_exact) {
        static bool ct_attr = false;
        if (!ct_attr) {
            cudaFuncSetAttribute(chain_tiles_kernel<T, C, CJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)chain_tiles_smem_bytes<T, C>());
            ct_attr = true;
        }
        chain_tiles_kernel<T, C, CJ><<<(unsigned)P.nchain_items, kThreads, chain_tiles_smem_bytes<T, C>(), s1>>>(
            P.fronts, reinterpret_cast<const int4*>(P.chain_items), L, reinterpret_cast<const T*>(P.dinv),
            reinterpret_cast<T*>(P.m1), reinterpret_cast<T*>(P.n1));
        ++launches;
    }
    if (la && !captured) {   // the caller's stream continues after the whole factorization
        cudaEvent_t end = P.sync_events[next_ev++];
        cudaEventRecord(end, s1);
        cudaStreamWaitEvent(P.stream, end, 0);
    }
    return launches;
}

#ifndef TRY
#define TRY(x)                          \
    do {                                \
        int _st = (x);                  \
        if (_st != CLIQ_OK) return _st; \
    } while (0)
#endif

// Intra-front pivoting (LDL_INTRAPIV_*): per tree level its extend-add and
// assembly, then the level's Bunch-Kaufman panels and updates (pivot_ldl.cu),
// all on the plan's stream; the extend-add reads the child maps in assembled
// order.  Afterwards the sweeps' diagonal-block inverses, the solves' maps in
// the pivoted order and, for the product form, the chain tiles.
template <class T, bool C, bool CJ>
static int issue_factor_pivoted(Plan& P, int64_t* nlaunch) {
    T* L = reinterpret_cast<T*>(P.L);
    T* p0 = reinterpret_cast<T*>(P.pool[0]);
    T* p1 = reinterpret_cast<T*>(P.pool[1]);
    const int4* items = reinterpret_cast<const int4*>(P.items);
    cudaStream_t st = P.stream;
    const int64_t before = P.total_launches;
    int64_t launches = 0;
    TRY(pivot_begin(P, st));
    // Each level's Schur complements (fixed shapes, K = n) run as the plan's
    // own Schur launches: tcgen05 for FP32 plans with the 2xFP16 split (the
    // S operand packed with D's 2 x 2 blocks), DMMA for FP64 plans (the
    // 2 x 2 terms formed from staged halo rows); otherwise (and for launches
    // the autotuner moved to the CUDA cores) on the CUDA cores with the panels
    const bool tc = ((std::is_same<T, float>::value && P.f16_scales()) || (std::is_same<T, double>::value && P.fp64_dmma)) &&
                    P.schur_chunk == 0;
    std::vector<std::vector<size_t>> schur(P.max_depth + 1);
    std::vector<char> tc_ok(P.max_depth + 1, tc ? 1 : 0);
    for (size_t li = 0; li < P.launches.size(); ++li) {
        const Launch& ln = P.launches[li];
        if (ln.kind != Launch::GEMM || !ln.schur || ln.nblocks <= 0) continue;
        schur[ln.depth].push_back(li);
        if (ln.simt || ln.bulk || ln.prepacked) tc_ok[ln.depth] = 0;
    }
    for (const Launch& ln : P.launches) {
        if (ln.kind != Launch::EXTEND_ADD || ln.nblocks <= 0) continue;
        extend_add_kernel<T, C><<<(unsigned)ln.nblocks, kThreads, 0, st>>>(P.fronts, items + ln.items, L, p0, p1, P.cmaps_orig);
        ++launches;
        TRY(launch_assemble_level(P, ln.depth, st));
        const bool on_tc = tc_ok[ln.depth] != 0;
        TRY(pivot_level(P, ln.depth, st, !on_tc));
        if (on_tc && !schur[ln.depth].empty()) {
            if (std::is_same<T, float>::value) TRY(pivot_rowmax(P, ln.depth, st));
            for (size_t li : schur[ln.depth]) {
                if (std::is_same<T, float>::value) launch_tc2(P, P.launches[li], nullptr, st, P.pack);
                else launch_dmma_update(P, P.launches[li], st);
                ++launches;
            }
        }
    }
    TRY(pivot_finish(P, st));
    if (P.nchain_items > 0 && !P.solve_exact) {
        static bool ct_attr = false;
        if (!ct_attr) {
            cudaFuncSetAttribute(chain_tiles_kernel<T, C, CJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)chain_tiles_smem_bytes<T, C>());
            ct_attr = true;
        }
        chain_tiles_kernel<T, C, CJ><<<(unsigned)P.nchain_items, kThreads, chain_tiles_smem_bytes<T, C>(), st>>>(
            P.fronts, reinterpret_cast<const int4*>(P.chain_items), L, reinterpret_cast<const T*>(P.dinv),
            reinterpret_cast<T*>(P.m1), reinterpret_cast<T*>(P.n1));
        ++launches;
    }
    // the pivoted launchers counted theirs in total_launches
    launches += P.total_launches - before;
    P.total_launches = before;
    *nlaunch = launches;
    return check_cuda("pivoted factor launch");
}

// Direct launches for the first factorization of a plan and for profiled
// ones; otherwise the launch sequence (static for a plan: same grids, items
// and buffers every time) is captured once from the plan's stream, across
// both internal streams, and replayed as one graph.
template <class T, bool C, bool CJ>
static int run_factor_impl(Plan& P) {
    int64_t launches = 0;
    if (P.pivoted) {
        const int st = issue_factor_pivoted<T, C, CJ>(P, &launches);
        if (st != CLIQ_OK) return st;
        P.prof_pending = false;
        ++P.factor_runs;
        P.last_launches = launches;
        P.total_launches += launches;
        return CLIQ_OK;
    }
    TRY(pivot_restore_maps(P, P.stream));
    const bool graphs = P.use_graph && P.stream1 && P.stream2 && P.sync_events.size() >= 2;
    if (graphs && !P.profile && P.factor_runs > 0 && !P.factor_exec) {
        if (cudaStreamBeginCapture(P.stream1, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            // the launchers count their side launches (operand packing) in
            // total_launches: nothing ran yet, so keep that count for the replays
            const int64_t before = P.total_launches;
            const int64_t n = issue_factor<T, C, CJ>(P, true);
            const int64_t side = P.total_launches - before;
            P.total_launches = before;
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(P.stream1, &g);
            if (e == cudaSuccess && g && cudaGraphInstantiate(&P.factor_exec, g, 0) == cudaSuccess) P.graph_launches = n + side;
            else P.factor_exec = nullptr;
            if (g) cudaGraphDestroy(g);
        }
        cudaGetLastError();
        if (!P.factor_exec) P.use_graph = 0;   // capture refused: direct launches from now on
    }
    if (graphs && !P.profile && P.factor_exec) {
        // the last two sync events are not used inside the graph
        cudaEvent_t fork = P.sync_events[P.sync_events.size() - 2], end = P.sync_events.back();
        cudaEventRecord(fork, P.stream);
        cudaStreamWaitEvent(P.stream1, fork, 0);
        if (cudaGraphLaunch(P.factor_exec, P.stream1) != cudaSuccess) return check_cuda("factor graph launch");
        cudaEventRecord(end, P.stream1);
        cudaStreamWaitEvent(P.stream, end, 0);
        launches = P.graph_launches;
        P.prof_pending = false;
    } else {
        launches = issue_factor<T, C, CJ>(P);
        P.prof_pending = P.profile != 0;
    }
    ++P.factor_runs;
    P.last_launches = launches;
    P.total_launches += launches;
    return check_cuda("factor launch");
}

template <class T, bool C>
int run_factor(Plan& P) {
    if (P.conjugate && C) return run_factor_impl<T, C, true>(P);
    return run_factor_impl<T, C, false>(P);
}

template int run_factor<float, false>(Plan&);
template int run_factor<float, true>(Plan&);
template int run_factor<double, false>(Plan&);
template int run_factor<double, true>(Plan&);

}  // namespace cliqgpu


// ===========================================================================
// cliqgpu_front_ldl_noalloc: FrontLDL on one dense front without any device
// allocation.
//
// Some callers cannot allocate device memory while they run: code that owns
// its memory pool and forbids cudaMalloc / cudaFree during a solve phase (a
// cudaFree synchronises the whole device), or code running inside another
// library's critical section.  For them this entry point keeps all of its
// scratch -- D, the inverse diagonal blocks, the work descriptors and the
// status word -- in one file-scope device array of fixed size, and otherwise
// runs the same diagonal-block, panel and CUDA-core update kernels as the
// tree factorization (plain right-looking 64-column steps, Schur update with
// K = n).  The caller passes the front in place: AL (m x n, leading dimension
// exactly m) and ABR ((m-n) x (m-n), leading dimension >= m-n).
//
// Limits: n <= 1024 pivots and m <= 16384 rows.  The array (about 1.2 MB)
// is held by every GPU that loads the library until the process exits.  The
// first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.  Every call waits for its stream and
// reads the status word back before it returns.  All calls share the array and it
// keeps the previous call's contents, so calls that overlap on the GPU (other
// streams, other host threads) race: serialise them.
// ===========================================================================
namespace cliqgpu {
namespace noalloc {

constexpr int kMaxN = 1024;
constexpr int kMaxM = 16384;
constexpr int kMaxSteps = kMaxN / kTile;
constexpr int kMaxItems = kMaxSteps * (1 + (kMaxM + kTile - 1) / kTile);
constexpr int kMaxProbs = kMaxSteps + 1;
constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
// byte offsets inside the scratch array (sized for complex FP64, the widest element)
constexpr size_t kOffStatus = 0;
constexpr size_t kOffFront = align256(kOffStatus + 4 * sizeof(int32_t));
constexpr size_t kOffD = align256(kOffFront + sizeof(FrontDev));
constexpr size_t kOffTinv = align256(kOffD + (size_t)kMaxN * 16);
constexpr size_t kOffDinv = align256(kOffTinv + (size_t)kTile * kTile * 16);
constexpr size_t kOffItems = align256(kOffDinv + (size_t)kMaxSteps * kTile * kTile * 16);
constexpr size_t kOffProbs = align256(kOffItems + (size_t)kMaxItems * sizeof(int4));
constexpr size_t kOffPrefix = align256(kOffProbs + (size_t)kMaxProbs * sizeof(GemmProb));
constexpr size_t kBytes = align256(kOffPrefix + (size_t)kMaxProbs * sizeof(int64_t));

static __device__ __align__(256) unsigned char g_scratch[kBytes];

// device address of g_scratch per device, looked up once with that device current
static std::mutex g_mu;
static void* g_addr[64] = {nullptr};

static int scratch_address(void** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return check_cuda("front_ldl_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= 64) {
        set_last_error("front_ldl_noalloc: device ordinal out of range");
        return CLIQ_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_last_error(std::string("front_ldl_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return CLIQ_ERR_CUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return CLIQ_OK;
}

template <class T, bool C>
__global__ void put_diag(T* __restrict__ A, int64_t lda, int n, const double* __restrict__ D) {
    using W = DV<C>;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
        stv<T, C>(A, j + (int64_t)j * lda, conv<V<T, C>>(reinterpret_cast<const W*>(D)[j]));
}

// one 64-column step: diagonal block, panel row blocks, trailing update (if any)
struct Step {
    int k;
    int64_t diag_item, panel_item;
    int panel_blocks;
    int prob;            // index of the trailing update problem, -1 if none
    int64_t tiles;
};

template <class T, bool C, bool CJ>
static void launch_all(unsigned char* base, int m, int n, T* AL, T* ABR, const std::vector<Step>& steps, int schur_prob,
                       int64_t schur_tiles, cudaStream_t st) {
    using X = V<T, C>;
    const size_t smem_panel = sizeof(X) * (kTile * kTile + kTile * (kTile + 1) + kTile);
    cudaFuncSetAttribute(panel_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_panel);
    cudaFuncSetAttribute(diag_ldl_kernel<T, C, CJ, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)diag_smem_bytes<T, C>());
    const FrontDev* F = reinterpret_cast<const FrontDev*>(base + kOffFront);
    double* D = reinterpret_cast<double*>(base + kOffD);
    T* tinv = reinterpret_cast<T*>(base + kOffTinv);
    T* dinv = reinterpret_cast<T*>(base + kOffDinv);
    const int4* items = reinterpret_cast<const int4*>(base + kOffItems);
    const GemmProb* probs = reinterpret_cast<const GemmProb*>(base + kOffProbs);
    const int64_t* prefix = reinterpret_cast<const int64_t*>(base + kOffPrefix);
    int32_t* status = reinterpret_cast<int32_t*>(base + kOffStatus);
    for (const Step& s : steps) {
        diag_ldl_kernel<T, C, CJ, T><<<1, kThreads, diag_smem_bytes<T, C>(), st>>>(F, items + s.diag_item, s.k, AL, D, tinv, dinv, nullptr, status);
        if (s.panel_blocks > 0)
            panel_kernel<T, C><<<s.panel_blocks, kThreads, smem_panel, st>>>(F, items + s.panel_item, s.k, AL, D, tinv, nullptr,
                                                                               nullptr, 0, 0);
        if (s.prob >= 0)
            gemm_update_kernel<T, C, CJ><<<(unsigned)s.tiles, kThreads, 0, st>>>(probs + s.prob, prefix + s.prob, 1, nullptr, AL, ABR,
                                                                               ABR, D);
    }
    if (schur_prob >= 0)
        gemm_update_kernel<T, C, CJ><<<(unsigned)schur_tiles, kThreads, 0, st>>>(probs + schur_prob, prefix + schur_prob, 1, nullptr, AL,
                                                                               ABR, ABR, D);
    put_diag<T, C><<<(n + 255) / 256, 256, 0, st>>>(AL, (int64_t)m, n, D);
}

}  // namespace noalloc
}  // namespace cliqgpu

using namespace cliqgpu;

extern "C" int cliqgpu_front_ldl_noalloc(int32_t field, int32_t precision, int32_t conjugate, int32_t m, int32_t n, void* AL,
                                         int64_t lda, void* ABR, int64_t ldabr, void* stream) {
    using namespace noalloc;
    if (m < 0 || n < 0 || n > m || !AL || (m > n && (!ABR || ldabr < m - n))) {
        set_last_error("front_ldl_noalloc: invalid sizes or pointers");
        return CLIQ_ERR_ARG;
    }
    if (n > kMaxN || m > kMaxM) {
        set_last_error("front_ldl_noalloc: front too large for the fixed scratch (n <= " + std::to_string(kMaxN) +
                       ", m <= " + std::to_string(kMaxM) + ")");
        return CLIQ_ERR_ARG;
    }
    if (lda != m) {
        set_last_error("front_ldl_noalloc: AL must be stored with leading dimension m");
        return CLIQ_ERR_ARG;
    }
    if (ldabr > INT_MAX) {   // the update problem stores ABR's leading dimension as int32
        set_last_error("front_ldl_noalloc: ldabr must not exceed INT_MAX");
        return CLIQ_ERR_ARG;
    }
    if (n == 0) return CLIQ_OK;
    void* scratch = nullptr;
    int st = scratch_address(&scratch);
    if (st != CLIQ_OK) return st;
    unsigned char* base = reinterpret_cast<unsigned char*>(scratch);
    cudaStream_t s = (cudaStream_t)stream;
    const bool cplx = field == CLIQ_COMPLEX;
    const bool fp32 = precision == CLIQ_FP32;
    const int u = m - n;

    // host-side schedule for the single front (the whole tree has one node)
    FrontDev f{};
    f.L = 0; f.U = 0; f.CU[0] = f.CU[1] = -1; f.cmap = -1; f.lower = 0; f.W = 0;
    f.m = m; f.n = n; f.off = 0; f.u = u; f.pool = 0; f.flag_base = 0; f.dinv = 0; f.chain = -1;
    std::vector<int4> items;
    std::vector<GemmProb> probs;
    std::vector<int64_t> prefix;
    std::vector<Step> steps;
    auto tiles_of = [](int M, int N) -> int64_t {
        const int64_t Mt = (M + kTile - 1) / kTile, Nt = (N + kTile - 1) / kTile;
        return Nt * Mt - Nt * (Nt - 1) / 2;
    };
    for (int k = 0; k < n; k += kTile) {
        Step sp{};
        sp.k = k;
        const int kb = std::min(kTile, n - k);
        sp.diag_item = (int64_t)items.size();
        items.push_back(make_int4(0, 0, 0, 0));
        sp.panel_item = (int64_t)items.size();
        const int rows = m - k - kb;
        for (int rb = 0; rb * kTile < rows; ++rb) items.push_back(make_int4(0, 0, rb, 0));
        sp.panel_blocks = (int)(items.size() - sp.panel_item);
        const int N = n - k - kb;
        sp.prob = -1;
        if (N > 0) {
            GemmProb pr{};
            pr.A = (k + kb) + (int64_t)k * m;
            pr.B = pr.A;
            pr.C = (k + kb) + (int64_t)(k + kb) * m;
            pr.d = k;
            pr.lda = m; pr.ldc = m; pr.M = rows; pr.N = N; pr.K = kb; pr.cpool = -1;
            sp.prob = (int)probs.size();
            sp.tiles = tiles_of(pr.M, pr.N);
            probs.push_back(pr);
            prefix.push_back(0);
        }
        steps.push_back(sp);
    }
    int schur_prob = -1;
    int64_t schur_tiles = 0;
    if (u > 0) {
        GemmProb pr{};
        pr.A = n; pr.B = n; pr.C = 0; pr.d = 0;
        pr.lda = m; pr.ldc = (int32_t)ldabr; pr.M = u; pr.N = u; pr.K = n; pr.cpool = 0;
        schur_prob = (int)probs.size();
        schur_tiles = tiles_of(u, u);
        probs.push_back(pr);
        prefix.push_back(0);
    }
    // descriptors and a cleared status word into the scratch array (no allocation)
    const int32_t st0[4] = {INT_MAX, 0, 0, 0};
    cudaMemcpyAsync(base + kOffStatus, st0, sizeof(st0), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(base + kOffFront, &f, sizeof(f), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(base + kOffItems, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, s);
    if (!probs.empty()) {
        cudaMemcpyAsync(base + kOffProbs, probs.data(), sizeof(GemmProb) * probs.size(), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(base + kOffPrefix, prefix.data(), sizeof(int64_t) * prefix.size(), cudaMemcpyHostToDevice, s);
    }
    if (fp32) {
        if (cplx && conjugate) launch_all<float, true, true>(base, m, n, (float*)AL, (float*)ABR, steps, schur_prob, schur_tiles, s);
        else if (cplx) launch_all<float, true, false>(base, m, n, (float*)AL, (float*)ABR, steps, schur_prob, schur_tiles, s);
        else launch_all<float, false, false>(base, m, n, (float*)AL, (float*)ABR, steps, schur_prob, schur_tiles, s);
    } else {
        if (cplx && conjugate) launch_all<double, true, true>(base, m, n, (double*)AL, (double*)ABR, steps, schur_prob, schur_tiles, s);
        else if (cplx) launch_all<double, true, false>(base, m, n, (double*)AL, (double*)ABR, steps, schur_prob, schur_tiles, s);
        else launch_all<double, false, false>(base, m, n, (double*)AL, (double*)ABR, steps, schur_prob, schur_tiles, s);
    }
    st = check_cuda("front_ldl_noalloc");
    if (st != CLIQ_OK) return st;
    int32_t out[4];
    if (cudaMemcpyAsync(out, base + kOffStatus, sizeof(out), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return check_cuda("front_ldl_noalloc: status");
    if (out[1]) {
        set_last_error("front_ldl_noalloc: a device-side wait timed out");
        return CLIQ_ERR_TIMEOUT;
    }
    if (out[0] != INT_MAX) {
        set_last_error("front_ldl_noalloc: zero pivot at column " + std::to_string(out[0] - 1));
        return CLIQ_ERR_ZERO_PIVOT;
    }
    return CLIQ_OK;
}
