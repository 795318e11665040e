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
//      parent's lower triangle is written exactly once (frontL += children,
//      ABR := children), using per-front inverse maps of the relative indices.
//   2. for k in steps of nb over the level's widest front:
//        diag_ldl_kernel  -- LDL of the kb x kb diagonal block in shared memory
//                            in FP64, writes L11, D (FP64) and U = L11^{-T}.
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

// ---------------------------------------------------------------------------
// 1. extend-add (gather form)
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void __launch_bounds__(kThreads) extend_add_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                              T* __restrict__ L, T* __restrict__ pool0, T* __restrict__ pool1,
                                                              const int32_t* __restrict__ cmaps) {
    using X = V<T, C>;
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int j0 = it.y;
    T* up = f.pool == 0 ? pool0 : pool1;
    const T* cp = f.pool == 0 ? pool1 : pool0;
    const int32_t* lm = f.cmap >= 0 ? cmaps + f.cmap : nullptr;
    const int32_t* rm = lm ? lm + f.m : nullptr;
    for (int jj = 0; jj < kEACols; ++jj) {
        const int j = j0 + jj;
        if (j >= f.m) break;
        const int lj = lm ? lm[j] : -1, rj = rm ? rm[j] : -1;
        if (j < f.n && lj < 0 && rj < 0) continue;
        for (int i = j + threadIdx.x; i < f.m; i += blockDim.x) {
            X v = X{};
            if (lj >= 0) {
                const int li = lm[i];
                if (li >= 0) v += ldv<T, C>(cp, f.CU[0] + li + (int64_t)lj * f.cu[0]);
            }
            if (rj >= 0) {
                const int ri = rm[i];
                if (ri >= 0) v += ldv<T, C>(cp, f.CU[1] + ri + (int64_t)rj * f.cu[1]);
            }
            if (j < f.n) {
                const int64_t e = f.L + i + (int64_t)j * f.m;
                stv<T, C>(L, e, ldv<T, C>(L, e) + v);
            } else {
                stv<T, C>(up, f.U + (i - f.n) + (int64_t)(j - f.n) * f.u, v);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// 2a. LDL of the diagonal block (one CTA per front), FP64 in shared memory
//
// Right-looking elimination of the kb x kb block; the same row operations
// are applied to an identity block, which therefore ends as L11^{-1}
// (Gaussian elimination on [A | I]).  Two barriers per pivot.  Outputs:
// L11 (unit diagonal) and D back to global memory, U = op(L11^{-1})^T for the
// panel kernel, and L11^{-1} itself into the per-front inverse store used by
// the triangular solves.
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kThreads, 1) diag_ldl_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items, int k,
                                                               T* __restrict__ L, double* __restrict__ D, T* __restrict__ tinv,
                                                               T* __restrict__ dinv, T* __restrict__ dinvT, int32_t* __restrict__ status) {
    using W = DV<C>;
    using X = V<T, C>;
    constexpr int nb = kTile;
    // thread (tr, tc) owns rows tr + 16a and columns tc + 16b (a, b < 4) of the
    // block A and of the running inverse Xm, both held in registers
    __shared__ W s_a[nb], s_l[nb], s_xr[nb], s_d[nb];
    const int4 it = items[blockIdx.x];
    const FrontDev f = F[it.x];
    const int slot = it.y;
    const int kb = min(nb, f.n - k);
    const int tr = threadIdx.x & 15, tc = threadIdx.x >> 4;
    W A[4][4], Xm[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int i = tr + 16 * a, c = tc + 16 * b;
            W v{};
            if (i < kb && c < kb && i >= c) v = conv<W>(ldv<T, C>(L, f.L + (k + i) + (int64_t)(k + c) * f.m));
            A[a][b] = v;
            Xm[a][b] = (i == c) ? vone<W>() : W{};
            if (i == c && i < kb) s_d[i] = v;
        }
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
        const W d = s_d[j];
        if (threadIdx.x == 0 && is_zero(d)) atomicMin(&status[0], f.off + k + j + 1);
        const W rd = vone<W>() / d;
        // publish the pivot column (scaled and unscaled) and row j of the inverse
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int i = tr + 16 * a, c = tc + 16 * b;
                if (c == j && i > j && i < kb) {
                    const W l = A[a][b] * rd;
                    s_a[i] = A[a][b];
                    s_l[i] = l;
                    A[a][b] = l;
                }
                if (i == j && c <= j) s_xr[c] = Xm[a][b];
            }
        __syncthreads();
        W la[4], ab[4], xb[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = tr + 16 * a;
            la[a] = (i > j && i < kb) ? s_l[i] : W{};
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int c = tc + 16 * b;
            ab[b] = (c > j && c < kb) ? opc<CJ>(s_a[c]) : W{};
            xb[b] = (c <= j) ? s_xr[c] : W{};
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int i = tr + 16 * a, c = tc + 16 * b;
                if (i > j && i < kb) {
                    if (c > j) {
                        if (i >= c) A[a][b] -= la[a] * ab[b];
                    } else {
                        Xm[a][b] -= la[a] * xb[b];
                    }
                    if (i == j + 1 && c == j + 1) s_d[j + 1] = A[a][b];
                }
            }
        __syncthreads();
    }
    // outputs: U = op(L11^{-1})^T (row-major, for the panel), L11^{-1}
    // (column-major for the forward sweep, row-major for the backward sweep),
    // L11 with unit diagonal, and D
    X* U = reinterpret_cast<X*>(tinv) + (int64_t)slot * nb * nb;
    X* Dv = reinterpret_cast<X*>(dinv) + f.dinv + (int64_t)(k / nb) * nb * nb;
    X* DvT = dinvT ? reinterpret_cast<X*>(dinvT) + f.dinv + (int64_t)(k / nb) * nb * nb : nullptr;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int i = tr + 16 * a, c = tc + 16 * b;
            const bool in = i < kb && c < kb && i >= c;
            U[c * nb + i] = in ? conv<X>(opc<CJ>(Xm[a][b])) : X{};
            Dv[i + c * nb] = in ? conv<X>(Xm[a][b]) : X{};
            if (DvT) DvT[i * nb + c] = in ? conv<X>(Xm[a][b]) : X{};
            if (in) {
                if (i > c) stv<T, C>(L, f.L + (k + i) + (int64_t)(k + c) * f.m, conv<X>(A[a][b]));
                else {
                    stv<T, C>(L, f.L + (k + i) + (int64_t)(k + c) * f.m, vone<X>());
                    reinterpret_cast<W*>(D)[f.off + k + i] = A[a][b];
                }
            }
        }
}

// ---------------------------------------------------------------------------
// 2b. panel: S21 = A21 U, L21 = S21 D^{-1} for one 64-row block
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void __launch_bounds__(kThreads) panel_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items, int k,
                                                         T* __restrict__ L, const double* __restrict__ D, const T* __restrict__ tinv,
                                                         T* __restrict__ subT) {
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
    // the first row block under a full diagonal block is tile (b+1, b) of the
    // pivot rows: keep a row-major copy (zero outside the pivot rows) for the
    // backward sweep
    if (subT && rb == 0 && kb == nb && r0 < f.n) {
        X* S = reinterpret_cast<X*>(subT) + f.dinv + (int64_t)(k / nb) * nb * nb;
        const int prow = min(rows, f.n - r0);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = ty + 16 * a, c = tx + 16 * b;
                S[r * nb + c] = r < prow ? acc[a][b] * sR[c] : X{};
            }
    }
}

// ---------------------------------------------------------------------------
// 3. tiled update C -= A diag(d) op(B)^T on the lower trapezoid (i >= j)
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kThreads) gemm_update_kernel(const GemmProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                               int nprobs, T* __restrict__ L, T* __restrict__ pool0,
                                                               T* __restrict__ pool1, const double* __restrict__ D) {
    using X = V<T, C>;
    using W = DV<C>;
    constexpr int BM = 64, BK = C ? 8 : 16, PAD = 1;
    __shared__ X sA[BK][BM + PAD];
    __shared__ X sB[BK][BM + PAD];
    const int64_t bid = blockIdx.x;
    int lo = 0, hi = nprobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= bid) lo = mid; else hi = mid - 1;
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
template <class T, bool C, bool CJ>
static int run_factor_impl(Plan& P) {
    using X = V<T, C>;
    using W = DV<C>;
    const size_t smem_diag = 0;
    const size_t smem_panel = sizeof(X) * (kTile * kTile + kTile * (kTile + 1) + kTile);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(panel_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_panel);
        attr_done = true;
    }
    T* L = reinterpret_cast<T*>(P.L);
    T* p0 = reinterpret_cast<T*>(P.pool[0]);
    T* p1 = reinterpret_cast<T*>(P.pool[1]);
    const int4* items = reinterpret_cast<const int4*>(P.items);
    int64_t launches = 0;
    if (P.profile && P.events.size() < 2 * P.launches.size()) {
        const size_t old = P.events.size();
        P.events.resize(2 * P.launches.size());
        for (size_t i = old; i < P.events.size(); ++i) cudaEventCreate(&P.events[i]);
    }
    for (size_t li = 0; li < P.launches.size(); ++li) {
        const Launch& ln = P.launches[li];
        if (ln.nblocks <= 0) continue;
        if (P.profile) cudaEventRecord(P.events[2 * li], P.stream);
        switch (ln.kind) {
            case Launch::EXTEND_ADD:
                extend_add_kernel<T, C><<<(unsigned)ln.nblocks, kThreads, 0, P.stream>>>(P.fronts, items + ln.items, L, p0, p1, P.cmaps);
                break;
            case Launch::DIAG:
                diag_ldl_kernel<T, C, CJ><<<(unsigned)ln.nblocks, kThreads, smem_diag, P.stream>>>(
                    P.fronts, items + ln.items, ln.k, L, P.D, reinterpret_cast<T*>(P.tinv), reinterpret_cast<T*>(P.dinv),
                    reinterpret_cast<T*>(P.dinvT), P.status);
                break;
            case Launch::PANEL:
                panel_kernel<T, C><<<(unsigned)ln.nblocks, kThreads, smem_panel, P.stream>>>(
                    P.fronts, items + ln.items, ln.k, L, P.D, reinterpret_cast<const T*>(P.tinv), reinterpret_cast<T*>(P.subT));
                break;
            case Launch::GEMM:
                if (std::is_same<T, float>::value && P.tensor_path())
                    launch_tc2(P, ln);
                else
                    gemm_update_kernel<T, C, CJ><<<(unsigned)ln.nblocks, kThreads, 0, P.stream>>>(
                        P.probs + ln.items, P.prefix + ln.prefix, ln.nitems, L, p0, p1, P.D);
                break;
        }
        if (P.profile) cudaEventRecord(P.events[2 * li + 1], P.stream);
        ++launches;
    }
    P.prof_pending = P.profile != 0;
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
// first call before any stream capture.  All calls share the array and it
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
    const FrontDev* F = reinterpret_cast<const FrontDev*>(base + kOffFront);
    double* D = reinterpret_cast<double*>(base + kOffD);
    T* tinv = reinterpret_cast<T*>(base + kOffTinv);
    T* dinv = reinterpret_cast<T*>(base + kOffDinv);
    const int4* items = reinterpret_cast<const int4*>(base + kOffItems);
    const GemmProb* probs = reinterpret_cast<const GemmProb*>(base + kOffProbs);
    const int64_t* prefix = reinterpret_cast<const int64_t*>(base + kOffPrefix);
    int32_t* status = reinterpret_cast<int32_t*>(base + kOffStatus);
    for (const Step& s : steps) {
        diag_ldl_kernel<T, C, CJ><<<1, kThreads, 0, st>>>(F, items + s.diag_item, s.k, AL, D, tinv, dinv, nullptr, status);
        if (s.panel_blocks > 0)
            panel_kernel<T, C><<<s.panel_blocks, kThreads, smem_panel, st>>>(F, items + s.panel_item, s.k, AL, D, tinv, nullptr);
        if (s.prob >= 0)
            gemm_update_kernel<T, C, CJ><<<(unsigned)s.tiles, kThreads, 0, st>>>(probs + s.prob, prefix + s.prob, 1, AL, ABR,
                                                                               ABR, D);
    }
    if (schur_prob >= 0)
        gemm_update_kernel<T, C, CJ><<<(unsigned)schur_tiles, kThreads, 0, st>>>(probs + schur_prob, prefix + schur_prob, 1, AL,
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
    f.m = m; f.n = n; f.off = 0; f.u = u; f.pool = 0; f.flag_base = 0; f.dinv = 0;
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
    return out[0] == INT_MAX ? CLIQ_OK : CLIQ_ERR_ZERO_PIVOT;
}
