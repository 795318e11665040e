// Front-tree triangular solves on the device.
//
// Reference: Solve (include/clique/numeric/solve.hpp:41-65) = forward sweep
// (LocalLowerForwardSolve, lower_solve/local.hpp:42-119), diagonal solve
// (LocalDiagonalSolve, diagonal_solve.hpp:49-69) and backward sweep (root
// front in DistLowerBackwardSolve, lower_solve/dist.hpp:374-387, then
// LocalLowerBackwardSolve, lower_solve/local.hpp:203-277).  Per front the
// reference calls Trsm + Gemm (lower_solve/local_front.hpp:36-82).
//
// Here each tree level is one pair of launches:
//   forward:  gather (children's W_B into this front's rows)  then
//             fwd_chain: the front's rows in 64-row blocks.  Each block
//             accumulates L[rows, T-block] * x[T-block] over the already
//             solved blocks, then either solves its own diagonal block and
//             publishes it, or subtracts into W_B.  One pass over L.
//   backward: bwd_chain: per 64-column block of L_T, reduce L_B^T x_B (x_B
//             gathered straight from the solution at the front's lowerStruct
//             indices, which the ancestors have finished) and the later
//             T-blocks, then solve the transposed diagonal block.
// Blocks of one front depend on earlier blocks; CTAs take work items from
// an atomic ticket counter in order, so every block a CTA waits for was
// taken by a CTA that is already running.  Waits are bounded: on expiry the
// kernel records a timeout in the status word and finishes without hanging.
#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

constexpr int kSolveThreads = 256;
constexpr int kMaxRhsChunk = 16;     // right-hand sides per sweep
constexpr int kGatherRows = 1024;    // front rows per gather CTA (grid y of the gather launch)
constexpr uint64_t kSpinNs = 500000000ull;   // 0.5 s bound on any single wait

__device__ __forceinline__ int ld_acquire(const int32_t* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// thread 0 waits for flag == epoch; returns false (and records a timeout,
// wait site 4) once the wall-clock bound expires
__device__ __forceinline__ bool wait_flag(const int32_t* flag, int epoch, int32_t* status) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_acquire(flag) != epoch) {
            const uint64_t t0 = global_ns();
            while (ld_acquire(flag) != epoch) {
                if (global_ns() - t0 > kSpinNs) { atomicExch(&status[1], 1); atomicCAS(&status[2], 0, 4); ok = 0; break; }
                __nanosleep(64);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void publish_flag(int32_t* flag, int epoch) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(flag, epoch);
}

// A 64 x 64 tile of a front, loaded into registers one step ahead of its use
// (L does not depend on the chain flags, so its load overlaps the waits).
constexpr int kPre = kTile * kTile / kSolveThreads;   // 16 elements per thread
template <class T, bool C>
__device__ __forceinline__ void tile_fetch(V<T, C>* pre, const T* L, const FrontDev& f, int r0, int nr, int c0, int nc) {
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
        const int idx = threadIdx.x + kSolveThreads * q;
        const int rr = idx % kTile, cc = idx / kTile;
        pre[q] = (rr < nr && cc < nc) ? ldv<T, C>(L, f.L + (r0 + rr) + (int64_t)(c0 + cc) * f.m) : V<T, C>{};
    }
}
template <class X>
__device__ __forceinline__ void tile_store(X* sL, const X* pre) {
#pragma unroll
    for (int q = 0; q < kPre; ++q) {
        const int idx = threadIdx.x + kSolveThreads * q;
        sL[(idx % kTile) * (kTile + 1) + idx / kTile] = pre[q];
    }
}

// ---------------------------------------------------------------------------
// forward gather: X_T += children's W_B (rows < n), W_B := children's W_B
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void __launch_bounds__(kSolveThreads) fwd_gather_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl,
                                                                   T* __restrict__ X, int64_t ldx, T* __restrict__ w0, T* __restrict__ w1,
                                                                   const int32_t* __restrict__ cmaps, int nrhs) {
    using Xv = V<T, C>;
    const FrontDev f = F[fl[blockIdx.x]];
    const int i0 = blockIdx.y * kGatherRows;       // this CTA's chunk of the front's rows
    if (i0 >= f.m) return;
    const int ni = min(kGatherRows, f.m - i0);
    T* wb = f.pool == 0 ? w0 : w1;
    const T* cw = f.pool == 0 ? w1 : w0;
    const int32_t* lm = f.cmap >= 0 ? cmaps + f.cmap : nullptr;
    const int32_t* rm = lm ? lm + f.m : nullptr;
    const int64_t total = (int64_t)ni * nrhs;
    for (int64_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int i = i0 + (int)(idx % ni), j = (int)(idx / ni);
        if (i < f.n && !lm) continue;
        Xv v{};
        if (lm) {
            const int li = lm[i], ri = rm[i];
            if (li >= 0) v += ldv<T, C>(cw, f.CW[0] * nrhs + li + (int64_t)j * f.cu[0]);
            if (ri >= 0) v += ldv<T, C>(cw, f.CW[1] * nrhs + ri + (int64_t)j * f.cu[1]);
        }
        if (i < f.n) {
            const int64_t e = f.off + i + (int64_t)j * ldx;
            stv<T, C>(X, e, ldv<T, C>(X, e) + v);
        } else {
            stv<T, C>(wb, f.W * nrhs + (i - f.n) + (int64_t)j * f.u, v);
        }
    }
}

// ---------------------------------------------------------------------------
// forward chain
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void __launch_bounds__(kSolveThreads) fwd_chain_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                                  int32_t* __restrict__ ticket, int32_t* __restrict__ flags, int epoch,
                                                                  const T* __restrict__ L, const T* __restrict__ dinv,
                                                                  T* __restrict__ X, int64_t ldx,
                                                                  T* __restrict__ w0, T* __restrict__ w1, int nrhs,
                                                                  int32_t* __restrict__ status) {
    using Xv = V<T, C>;
    constexpr int ldl = kTile + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Xv* sL = reinterpret_cast<Xv*>(smem_raw);         // 64 x 65
    Xv* sD = sL + kTile * ldl;                          // 64 x 65: inverse of the diagonal block, sD[r*65+c] = Linv[r][c]
    Xv* sx = sD + kTile * ldl;                          // 64 x kMaxRhsChunk
    __shared__ int s_item;
    if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1);
    __syncthreads();
    if (*reinterpret_cast<volatile int32_t*>(&status[1]) != 0) return;   // an earlier wait timed out
    const int4 it = items[s_item];
    const FrontDev f = F[it.x];
    const int rb = it.y;
    const int r0 = kTile * rb;
    const int rows = min(kTile, f.m - r0);
    const int nT = (f.n + kTile - 1) / kTile;
    const int r = threadIdx.x % kTile, q = threadIdx.x / kTile;   // row, rhs lane
    Xv acc[kMaxRhsChunk / 4];
#pragma unroll
    for (int a = 0; a < kMaxRhsChunk / 4; ++a) acc[a] = Xv{};
    const int cb_end = min(rb, nT);
    Xv pre[kPre];
    if (cb_end > 0) tile_fetch<T, C>(pre, L, f, r0, rows, 0, min(kTile, f.n));
    for (int cb = 0; cb < cb_end; ++cb) {
        const int c0 = kTile * cb, ncols = min(kTile, f.n - c0);
        tile_store(sL, pre);
        if (cb + 1 < cb_end) tile_fetch<T, C>(pre, L, f, r0, rows, c0 + kTile, min(kTile, f.n - c0 - kTile));
        if (!wait_flag(&flags[f.flag_base + cb], epoch, status)) break;
        for (int idx = threadIdx.x; idx < kTile * nrhs; idx += blockDim.x) {
            const int cc = idx % kTile, j = idx / kTile;
            sx[cc * kMaxRhsChunk + j] = cc < ncols ? ldv_cg<T, C>(X, f.off + c0 + cc + (int64_t)j * ldx) : Xv{};
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs) {
                Xv s = acc[a];
                for (int cc = 0; cc < ncols; ++cc) mac(s, sL[r * ldl + cc], sx[cc * kMaxRhsChunk + j]);
                acc[a] = s;
            }
        }
        __syncthreads();
    }
    if (rb < nT) {
        const int dcols = min(kTile, f.n - r0);
        const Xv* Dv = reinterpret_cast<const Xv*>(dinv) + f.dinv + (int64_t)rb * kTile * kTile;
        for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
            const int rr = idx % kTile, cc = idx / kTile;
            sL[rr * ldl + cc] = (rr < rows && cc < dcols) ? ldv<T, C>(L, f.L + (r0 + rr) + (int64_t)(r0 + cc) * f.m) : Xv{};
            sD[rr * ldl + cc] = Dv[idx];
        }
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs && r < dcols) sx[r * kMaxRhsChunk + j] = ldv<T, C>(X, f.off + r0 + r + (int64_t)j * ldx) - acc[a];
        }
        __syncthreads();
        // x = L11^{-1} b with the inverse kept by the factorization
        Xv y[kMaxRhsChunk / 4];
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            Xv sacc{};
            if (j < nrhs && r < dcols)
                for (int cc = 0; cc <= r; ++cc) mac(sacc, sD[r * ldl + cc], sx[cc * kMaxRhsChunk + j]);
            y[a] = sacc;
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs && r < dcols) sx[r * kMaxRhsChunk + j] = y[a];
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs && r < dcols) stv<T, C>(X, f.off + r0 + r + (int64_t)j * ldx, sx[r * kMaxRhsChunk + j]);
        }
        publish_flag(&flags[f.flag_base + rb], epoch);
        // rows of this block below the pivots (rows >= n) take this block's contribution
        if (r >= dcols && r < rows) {
#pragma unroll
            for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
                const int j = q + 4 * a;
                if (j < nrhs) {
                    Xv s = acc[a];
                    for (int cc = 0; cc < dcols; ++cc) mac(s, sL[r * ldl + cc], sx[cc * kMaxRhsChunk + j]);
                    acc[a] = s;
                }
            }
        }
    }
    if (r0 + r >= f.n && r < rows) {
        T* wb = f.pool == 0 ? w0 : w1;
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs) {
                const int64_t e = f.W * nrhs + (r0 + r - f.n) + (int64_t)j * f.u;
                stv<T, C>(wb, e, ldv<T, C>(wb, e) - acc[a]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// diagonal solve X := D^{-1} X (FP64 pivots)
// ---------------------------------------------------------------------------
template <class T, bool C>
__global__ void diag_scale_kernel(T* __restrict__ X, int64_t ldx, int64_t n, int nrhs, const double* __restrict__ D) {
    using Xv = V<T, C>;
    using W = DV<C>;
    const int64_t total = n * nrhs;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = idx % n, j = idx / n;
        const W d = reinterpret_cast<const W*>(D)[p];
        const int64_t e = p + j * ldx;
        const W x = conv<W>(ldv<T, C>(X, e));
        stv<T, C>(X, e, conv<Xv>(x / d));
    }
}

// ---------------------------------------------------------------------------
// backward chain
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
__global__ void __launch_bounds__(kSolveThreads) bwd_chain_kernel(const FrontDev* __restrict__ F, const int4* __restrict__ items,
                                                                  int32_t* __restrict__ ticket, int32_t* __restrict__ flags, int epoch,
                                                                  const T* __restrict__ L, const T* __restrict__ dinv,
                                                                  T* __restrict__ X, int64_t ldx,
                                                                  const int32_t* __restrict__ lower, int nrhs,
                                                                  int32_t* __restrict__ status) {
    using Xv = V<T, C>;
    constexpr int ldl = kTile + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Xv* sL = reinterpret_cast<Xv*>(smem_raw);
    Xv* sD = sL + kTile * ldl;
    Xv* sx = sD + kTile * ldl;
    __shared__ int s_item;
    if (threadIdx.x == 0) s_item = atomicAdd(ticket, 1);
    __syncthreads();
    if (*reinterpret_cast<volatile int32_t*>(&status[1]) != 0) return;   // an earlier wait timed out
    const int4 it = items[s_item];
    const FrontDev f = F[it.x];
    const int rb = it.y;
    const int c0 = kTile * rb;
    const int dcols = min(kTile, f.n - c0);
    const int nT = (f.n + kTile - 1) / kTile;
    const int c = threadIdx.x % kTile, q = threadIdx.x / kTile;
    Xv acc[kMaxRhsChunk / 4];
#pragma unroll
    for (int a = 0; a < kMaxRhsChunk / 4; ++a) acc[a] = Xv{};
    // rows below the pivots: x gathered from the (final) ancestor entries
    Xv pre[kPre];
    if (f.n < f.m) tile_fetch<T, C>(pre, L, f, f.n, min(kTile, f.m - f.n), c0, dcols);
    for (int rr0 = f.n; rr0 < f.m; rr0 += kTile) {
        const int nr = min(kTile, f.m - rr0);
        tile_store(sL, pre);
        if (rr0 + kTile < f.m) tile_fetch<T, C>(pre, L, f, rr0 + kTile, min(kTile, f.m - rr0 - kTile), c0, dcols);
        else if (nT - 1 > rb) tile_fetch<T, C>(pre, L, f, kTile * (nT - 1), min(kTile, f.n - kTile * (nT - 1)), c0, dcols);
        for (int idx = threadIdx.x; idx < kTile * nrhs; idx += blockDim.x) {
            const int rr = idx % kTile, j = idx / kTile;
            Xv v{};
            if (rr < nr) v = ldv<T, C>(X, (int64_t)lower[f.lower + rr0 + rr - f.n] + (int64_t)j * ldx);
            sx[rr * kMaxRhsChunk + j] = v;
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs) {
                Xv s = acc[a];
                for (int rr = 0; rr < nr; ++rr) mac(s, opc<CJ>(sL[rr * ldl + c]), sx[rr * kMaxRhsChunk + j]);
                acc[a] = s;
            }
        }
        __syncthreads();
    }
    if (f.n >= f.m && nT - 1 > rb) tile_fetch<T, C>(pre, L, f, kTile * (nT - 1), min(kTile, f.n - kTile * (nT - 1)), c0, dcols);
    // later pivot blocks of this front
    for (int ib = nT - 1; ib > rb; --ib) {
        const int rr0 = kTile * ib, nr = min(kTile, f.n - rr0);
        tile_store(sL, pre);
        if (ib - 1 > rb) tile_fetch<T, C>(pre, L, f, rr0 - kTile, kTile, c0, dcols);
        if (!wait_flag(&flags[f.flag_base + ib], epoch, status)) break;
        for (int idx = threadIdx.x; idx < kTile * nrhs; idx += blockDim.x) {
            const int rr = idx % kTile, j = idx / kTile;
            sx[rr * kMaxRhsChunk + j] = rr < nr ? ldv_cg<T, C>(X, f.off + rr0 + rr + (int64_t)j * ldx) : Xv{};
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
            const int j = q + 4 * a;
            if (j < nrhs) {
                Xv s = acc[a];
                for (int rr = 0; rr < nr; ++rr) mac(s, opc<CJ>(sL[rr * ldl + c]), sx[rr * kMaxRhsChunk + j]);
                acc[a] = s;
            }
        }
        __syncthreads();
    }
    // diagonal block, transposed: x = op(L11^{-1})^T b
    const Xv* Dv = reinterpret_cast<const Xv*>(dinv) + f.dinv + (int64_t)rb * kTile * kTile;
    for (int idx = threadIdx.x; idx < kTile * kTile; idx += blockDim.x) {
        const int rr = idx % kTile, cc = idx / kTile;
        sD[rr * ldl + cc] = Dv[idx];
    }
#pragma unroll
    for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
        const int j = q + 4 * a;
        if (j < nrhs && c < dcols) sx[c * kMaxRhsChunk + j] = ldv<T, C>(X, f.off + c0 + c + (int64_t)j * ldx) - acc[a];
    }
    __syncthreads();
    Xv y[kMaxRhsChunk / 4];
#pragma unroll
    for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
        const int j = q + 4 * a;
        Xv sacc{};
        if (j < nrhs && c < dcols)
            for (int rr = c; rr < dcols; ++rr) mac(sacc, opc<CJ>(sD[rr * ldl + c]), sx[rr * kMaxRhsChunk + j]);
        y[a] = sacc;
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
        const int j = q + 4 * a;
        if (j < nrhs && c < dcols) sx[c * kMaxRhsChunk + j] = y[a];
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < kMaxRhsChunk / 4; ++a) {
        const int j = q + 4 * a;
        if (j < nrhs && c < dcols) stv<T, C>(X, f.off + c0 + c + (int64_t)j * ldx, sx[c * kMaxRhsChunk + j]);
    }
    publish_flag(&flags[f.flag_base + rb], epoch);
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ>
static int run_solve_impl(Plan& P, T* xn, int nrhs_total) {
    using Xv = V<T, C>;
    const size_t smem = sizeof(Xv) * (2 * kTile * (kTile + 1) + kTile * kMaxRhsChunk);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(fwd_chain_kernel<T, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(bwd_chain_kernel<T, C, CJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_done = true;
    }
    const int4* items = reinterpret_cast<const int4*>(P.items);
    T* L = reinterpret_cast<T*>(P.L);
    T* w0 = reinterpret_cast<T*>(P.wpool[0]);
    T* w1 = reinterpret_cast<T*>(P.wpool[1]);
    const int nlev = P.max_depth + 1;
    int64_t launches = 0;
    for (int j0 = 0; j0 < nrhs_total; j0 += kMaxRhsChunk) {
        const int nrhs = nrhs_total - j0 < kMaxRhsChunk ? nrhs_total - j0 : kMaxRhsChunk;
        T* X = xn + (C ? 2 : 1) * (int64_t)j0 * P.n;
        cudaMemsetAsync(P.tickets, 0, sizeof(int32_t) * 2 * nlev, P.stream);
        for (int d = P.max_depth; d >= 0; --d) {
            const SolveLevel& lv = P.solve_levels[d];
            if (lv.nfronts == 0) continue;
            fwd_gather_kernel<T, C><<<dim3(lv.nfronts, lv.gather_chunks), kSolveThreads, 0, P.stream>>>(P.fronts, P.level_fronts + lv.fronts, X, P.n, w0, w1,
                                                                               P.cmaps, nrhs);
            ++launches;
            if (lv.nfwd > 0) {
                const int epoch = ++P.epoch;
                fwd_chain_kernel<T, C><<<lv.nfwd, kSolveThreads, smem, P.stream>>>(P.fronts, items + lv.fwd_items, P.tickets + 2 * d,
                                                                                   P.flags, epoch, L, reinterpret_cast<const T*>(P.dinv), X, P.n, w0, w1, nrhs, P.status);
                ++launches;
            }
        }
        diag_scale_kernel<T, C><<<1184, 256, 0, P.stream>>>(X, P.n, P.n, nrhs, P.D);
        ++launches;
        for (int d = 0; d <= P.max_depth; ++d) {
            const SolveLevel& lv = P.solve_levels[d];
            if (lv.nbwd == 0) continue;
            const int epoch = ++P.epoch;
            bwd_chain_kernel<T, C, CJ><<<lv.nbwd, kSolveThreads, smem, P.stream>>>(P.fronts, items + lv.bwd_items, P.tickets + 2 * d + 1,
                                                                                    P.flags, epoch, L, reinterpret_cast<const T*>(P.dinv), X, P.n, P.lower, nrhs, P.status);
            ++launches;
        }
    }
    P.last_launches += launches;
    P.total_launches += launches;
    return check_cuda("solve launch");
}

template <class T, bool C>
int run_solve_nodal(Plan& P, void* xn, int nrhs) {
    if (P.conjugate && C) return run_solve_impl<T, C, true>(P, reinterpret_cast<T*>(xn), nrhs);
    return run_solve_impl<T, C, false>(P, reinterpret_cast<T*>(xn), nrhs);
}

template int run_solve_nodal<float, false>(Plan&, void*, int);
template int run_solve_nodal<float, true>(Plan&, void*, int);
template int run_solve_nodal<double, false>(Plan&, void*, int);
template int run_solve_nodal<double, true>(Plan&, void*, int);

}  // namespace cliqgpu
