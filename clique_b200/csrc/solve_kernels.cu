// Front-tree triangular solves on the device.
//
// Reference: Solve (include/clique/numeric/solve.hpp:41-65) = forward sweep
// (LocalLowerForwardSolve, lower_solve/local.hpp:42-119), diagonal solve
// (LocalDiagonalSolve, diagonal_solve.hpp:49-69) and backward sweep (root
// front in DistLowerBackwardSolve, lower_solve/dist.hpp:374-387, then
// LocalLowerBackwardSolve, lower_solve/local.hpp:203-277).  Per front the
// reference calls Trsm + Gemm (lower_solve/local_front.hpp:36-82).
//
// Each tree level is one gather launch plus one sweep launch (forward), or
// one sweep launch (backward).  Inside a sweep launch every front gets
//   * one chain CTA, which walks the front's 64-wide pivot blocks in order.
//     Step s needs the block's right-hand side minus the contributions of
//     all solved blocks.  The newest block's contribution is the only
//     product on the chain's critical path (x_{s-1} stays in its shared
//     memory, the 64x64 tile was prefetched into registers during the
//     previous step); the second newest, q_s, the chain formed right after
//     publishing x_{s-2}; the older ones arrive from a worker as one
//     finished 64 x nrhs partial sum, which the worker had two chain steps
//     to produce.  Then the chain applies the stored inverse of the diagonal
//     block and publishes x_s: two 64x64 products and one flag per step, with
//     no global-memory round trip for x.
//   * workers, which stream the rest of the front's L tiles as the chain
//     publishes solved blocks: forward, one per 64-row block of pivot rows
//     (its partial feeds the chain) and one per 64-row block below the
//     pivots (subtracts into the update vector W_B); backward, one per
//     pivot column block (the first 16 tiles of rows below the pivots, the
//     sums of its helpers in chunk order, then the later pivot blocks), and
//     helpers for the further 16-tile chunks of rows below the pivots.
// Work items are taken from an atomic ticket counter in the order helpers
// (which wait for nothing), then each chain followed by its workers in the
// order the chain consumes them, so every CTA a resident CTA waits for was
// either issued before it or is a worker whose own waits only reach back to
// earlier tickets: the sweep finishes with any number of resident CTAs >= 2.
// Waits are bounded: on expiry a CTA records a timeout in the status word
// and returns, and every other wait gives up as soon as it sees that word
// set.
#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

constexpr int kSolveThreads = 256;
constexpr int kQ = kSolveThreads / kTile;   // slices per tile row (4)
constexpr int kE = kTile / kQ;              // tile elements per thread and slice (16)
constexpr int kLag = kSolveLag;             // blocks the chain adds itself (the two newest)
constexpr int kMaxRhsChunk = kSolveRhsChunk;   // right-hand sides per sweep
constexpr int kPartialStride = kTile * kMaxRhsChunk;   // elements per pivot block in the partial store
constexpr int kGatherRows = 1024;           // front rows per gather CTA (grid y of the gather launch)
constexpr uint64_t kSpinNs = 500000000ull;  // 0.5 s bound on any single wait

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
// wait site 4) once the wall-clock bound expires, or at once when another
// CTA has recorded one
__device__ __forceinline__ bool wait_flag(const int32_t* flag, int epoch, int32_t* status) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_acquire(flag) != epoch) {
            const uint64_t t0 = global_ns();
            while (ld_acquire(flag) != epoch) {
                if (*reinterpret_cast<volatile int32_t*>(&status[1]) != 0) { ok = 0; break; }
                if (global_ns() - t0 > kSpinNs) { atomicExch(&status[1], 1); atomicCAS(&status[2], 0, 4); ok = 0; break; }
                __nanosleep(100);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// thread 0 reads the flag once (no wait); the CTA learns whether it is set
__device__ __forceinline__ bool test_flag(const int32_t* flag, int epoch) {
    __shared__ int s_set;
    if (threadIdx.x == 0) s_set = ld_acquire(flag) == epoch;
    __syncthreads();
    return s_set != 0;
}

__device__ __forceinline__ void publish_flag(int32_t* flag, int epoch) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicExch(flag, epoch);
}

// v[k] = A(r, q*kE + k) of a column-major tile at element offset a0 with
// leading dimension ld, zero outside nr rows / nc columns.  With ld = 64 on
// a row-major tile this reads element (q*kE + k, r) instead.
template <class T, bool C>
__device__ __forceinline__ void row_slice(V<T, C>* v, const T* __restrict__ A, int64_t a0, int64_t ld, int r, int q, int nr,
                                          int nc) {
#pragma unroll
    for (int k = 0; k < kE; ++k) {
        const int c = q * kE + k;
        v[k] = (r < nr && c < nc) ? ldv<T, C>(A, a0 + r + (int64_t)c * ld) : V<T, C>{};
    }
}

// acc[j] += sum_k op(v[k]) * s[(q*kE + k) * NR + j]; s is a 64 x NR tile in
// shared memory, read as a broadcast by the 32 threads of a warp (same q)
template <bool CJ, int NR, class Xv>
__device__ __forceinline__ void slice_mac(Xv (&acc)[NR], const Xv* v, const Xv* s, int q) {
#pragma unroll
    for (int k = 0; k < kE; ++k) {
        const Xv a = opc<CJ>(v[k]);
        const Xv* sr = s + (q * kE + k) * NR;
#pragma unroll
        for (int j = 0; j < NR; ++j) mac(acc[j], a, sr[j]);
    }
}

// Sum the kQ slice partials of each (row, rhs): thread (r, q) gets the
// totals for rhs j = q + kQ*a.  Ends with red still being read: the caller
// synchronises before red is written again.
template <int NR, class Xv>
__device__ __forceinline__ void reduce_slices(const Xv (&acc)[NR], Xv* red, Xv (&out)[NR / kQ], int r, int q) {
#pragma unroll
    for (int j = 0; j < NR; ++j) red[(q * NR + j) * kTile + r] = acc[j];
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NR / kQ; ++a) {
        const int j = q + kQ * a;
        Xv s{};
#pragma unroll
        for (int qq = 0; qq < kQ; ++qq) s += red[(qq * NR + j) * kTile + r];
        out[a] = s;
    }
}

// 64 x NR tile of right-hand sides from X (column-major, ldx) starting at
// row x0, zero beyond nr rows or nrhs columns; L2-coherent loads for values
// another CTA of this launch published
template <class T, bool C, int NR>
__device__ __forceinline__ void load_x_tile(V<T, C>* s, const T* X, int64_t x0, int64_t ldx, int nr, int nrhs) {
    for (int idx = threadIdx.x; idx < kTile * NR; idx += kSolveThreads) {
        const int rr = idx % kTile, j = idx / kTile;
        s[rr * NR + j] = (rr < nr && j < nrhs) ? ldv_cg<T, C>(X, x0 + rr + (int64_t)j * ldx) : V<T, C>{};
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
// sweep launches
// ---------------------------------------------------------------------------
struct SweepArgs {
    const FrontDev* F;
    const int4* items;      // {front, kind, block, 0}
    int32_t* ticket;
    int32_t* xflags;        // per pivot block: x_b published (chain)
    int32_t* pflags;        // per pivot block: partial sum published (worker)
    int epoch;
    const void* L;
    const void* dinv;       // L11^{-1} per 64-block, column-major
    const void* dinvT;      // the same, row-major
    const void* subT;       // tile (b+1, b) of L per pivot block, row-major
    const void* subT2;      // tile (b+2, b) of L per pivot block, row-major
    void* partial;          // kPartialStride elements per pivot block
    void* hpart;            // backward helpers' partial sums, kPartialStride each
    int32_t* hflags;        // backward helpers' flags
    void* X;                // n x nrhs, ND order, ld ldx
    int64_t ldx;
    void* w0;
    void* w1;
    const int32_t* lower;
    int nrhs;
    int32_t* status;
};

// One L tile of a forward worker: wait for x_t, stage it, accumulate.
template <class T, bool C, int NR>
__device__ __forceinline__ bool fwd_tile(const SweepArgs& a, const FrontDev& f, int t, const V<T, C>* lt, V<T, C> (&acc)[NR],
                                         V<T, C>* sx, int q) {
    V<T, C>* sb = sx + (t & 1) * kTile * NR;
    if (!wait_flag(&a.xflags[f.flag_base + t], a.epoch, a.status)) return false;
    load_x_tile<T, C, NR>(sb, reinterpret_cast<const T*>(a.X), f.off + (int64_t)t * kTile, a.ldx, min(kTile, f.n - t * kTile), a.nrhs);
    __syncthreads();
    slice_mac<false, NR>(acc, lt, sb, q);
    return true;
}

// Forward chain of one front:
//   x_s = L_ss^{-1} (b_s - partial_s - q_s - L_{s,s-1} x_{s-1}),
// partial_s from the pivot-row worker (blocks < s - 2), q_s = L_{s,s-2} x_{s-2}
// formed by the chain right after it published x_{s-2}.
template <class T, bool C, int NR>
__device__ void fwd_chain(const SweepArgs& a, const FrontDev& f, int nT, int r, int q, V<T, C>* sx, V<T, C>* red, V<T, C>* sq) {
    using Xv = V<T, C>;
    static_assert(kLag == 2, "the chain adds the two newest blocks");
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* Dinv = reinterpret_cast<const T*>(a.dinv);
    const T* Part = reinterpret_cast<const T*>(a.partial);
    T* X = reinterpret_cast<T*>(a.X);
    Xv* sprev = sx;                 // x_{s-1}
    Xv* st = sx + kTile * NR;       // right-hand side of the diagonal block
    Xv lp[kE], dv[kE];
    row_slice<T, C>(dv, Dinv, f.dinv, kTile, r, q, kTile, kTile);
    // b_s - partial_s for the next step, gathered after each publish when the
    // worker has already finished (then the step starts without a global
    // round trip)
    Xv nxt[NR / kQ];
    bool have_next = false;
    for (int s = 0; s < nT; ++s) {
        const int r0 = s * kTile, ds = min(kTile, f.n - r0);
        const bool fed = s > kLag;  // a worker holds the contributions of blocks < s - kLag
        Xv tv[NR / kQ];
        if (have_next) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] = nxt[b];
        } else {
            if (fed && !wait_flag(&a.pflags[f.flag_base + s], a.epoch, a.status)) return;
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                Xv v{};
                if (r < ds && j < a.nrhs) {
                    v = ldv<T, C>(X, f.off + r0 + r + (int64_t)j * a.ldx);
                    if (fed) v -= ldv_cg<T, C>(Part, (int64_t)(f.flag_base + s) * kPartialStride + j * kTile + r);
                }
                tv[b] = v;
            }
        }
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (s >= 2 && r < ds && j < a.nrhs) tv[b] -= sq[(s & 1) * kTile * NR + r * NR + j];
        }
        if (s > 0) {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<false, NR>(acc, lp, sprev, q);
            Xv u[NR / kQ];
            reduce_slices<NR>(acc, red, u, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] -= u[b];
        }
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = tv[b];
        __syncthreads();
        {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<false, NR>(acc, dv, st, q);
            Xv xs[NR / kQ];
            reduce_slices<NR>(acc, red, xs, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                const bool in = r < ds && j < a.nrhs;
                if (in) stv<T, C>(X, f.off + r0 + r + (int64_t)j * a.ldx, xs[b]);
                sprev[r * NR + j] = in ? xs[b] : Xv{};
            }
        }
        if (s + 1 < nT) {
            row_slice<T, C>(lp, L, f.L + (r0 + kTile) + (int64_t)r0 * f.m, f.m, r, q, min(kTile, f.n - r0 - kTile), kTile);
            row_slice<T, C>(dv, Dinv, f.dinv + (int64_t)(s + 1) * kTile * kTile, kTile, r, q, kTile, kTile);
        }
        // tile of the off-path product, in flight during the publish
        Xv lq[kE];
        if (s + 2 < nT)
            row_slice<T, C>(lq, L, f.L + (r0 + 2 * kTile) + (int64_t)r0 * f.m, f.m, r, q, min(kTile, f.n - r0 - 2 * kTile), kTile);
        publish_flag(&a.xflags[f.flag_base + s], a.epoch);
        have_next = false;
        if (s + 1 < nT) {
            const int s1 = s + 1, r1 = s1 * kTile, d1 = min(kTile, f.n - r1);
            const bool fed1 = s1 > kLag;
            if (!fed1 || test_flag(&a.pflags[f.flag_base + s1], a.epoch)) {
#pragma unroll
                for (int b = 0; b < NR / kQ; ++b) {
                    const int j = q + kQ * b;
                    Xv v{};
                    if (r < d1 && j < a.nrhs) {
                        v = ldv<T, C>(X, f.off + r1 + r + (int64_t)j * a.ldx);
                        if (fed1) v -= ldv_cg<T, C>(Part, (int64_t)(f.flag_base + s1) * kPartialStride + j * kTile + r);
                    }
                    nxt[b] = v;
                }
                have_next = true;
            }
        }
        // off the critical path: q_{s+2} = L_{s+2,s} x_s
        if (s + 2 < nT) {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<false, NR>(acc, lq, sprev, q);
            Xv qv[NR / kQ];
            reduce_slices<NR>(acc, red, qv, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) sq[(s & 1) * kTile * NR + r * NR + q + kQ * b] = qv[b];
            __syncthreads();
        }
    }
}

// Forward sweep of a small front (at most two pivot blocks, kWholeLowerRows
// rows below) by one CTA: both blocks, then every 64-row tile below the
// pivots, with the solved blocks kept in shared memory (no flags).
template <class T, bool C, int NR>
__device__ void fwd_whole(const SweepArgs& a, const FrontDev& f, int nT, int r, int q, V<T, C>* sx, V<T, C>* red, V<T, C>* sq) {
    using Xv = V<T, C>;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* Dinv = reinterpret_cast<const T*>(a.dinv);
    T* X = reinterpret_cast<T*>(a.X);
    Xv* st = sx;                     // right-hand side of the diagonal block
    Xv* xb = sq;                     // x_0, x_1
    for (int s = 0; s < nT; ++s) {
        const int r0 = s * kTile, ds = min(kTile, f.n - r0);
        Xv tv[NR / kQ];
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            tv[b] = (r < ds && j < a.nrhs) ? ldv<T, C>(X, f.off + r0 + r + (int64_t)j * a.ldx) : Xv{};
        }
        Xv dv[kE];
        row_slice<T, C>(dv, Dinv, f.dinv + (int64_t)s * kTile * kTile, kTile, r, q, kTile, kTile);
        if (s == 1) {
            Xv lp[kE];
            row_slice<T, C>(lp, L, f.L + kTile, f.m, r, q, ds, kTile);   // L_{1,0}
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<false, NR>(acc, lp, xb, q);
            Xv u[NR / kQ];
            reduce_slices<NR>(acc, red, u, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] -= u[b];
        }
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = tv[b];
        __syncthreads();
        Xv acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        slice_mac<false, NR>(acc, dv, st, q);
        Xv xs[NR / kQ];
        reduce_slices<NR>(acc, red, xs, r, q);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            const bool in = r < ds && j < a.nrhs;
            if (in) stv<T, C>(X, f.off + r0 + r + (int64_t)j * a.ldx, xs[b]);
            xb[s * kTile * NR + r * NR + j] = in ? xs[b] : Xv{};
        }
        __syncthreads();
    }
    // rows below the pivots: W_B -= L_B x_T
    T* wb = reinterpret_cast<T*>(f.pool == 0 ? a.w0 : a.w1);
    for (int R0 = f.n; R0 < f.m; R0 += kTile) {
        const int nr = min(kTile, f.m - R0);
        Xv acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        for (int t = 0; t < nT; ++t) {
            Xv lt[kE];
            row_slice<T, C>(lt, L, f.L + R0 + (int64_t)t * kTile * f.m, f.m, r, q, nr, min(kTile, f.n - t * kTile));
            slice_mac<false, NR>(acc, lt, xb + t * kTile * NR, q);
        }
        Xv out[NR / kQ];
        reduce_slices<NR>(acc, red, out, r, q);
        if (r < nr) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                if (j < a.nrhs) {
                    const int64_t e = f.W * a.nrhs + (R0 - f.n + r) + (int64_t)j * f.u;
                    stv<T, C>(wb, e, ldv<T, C>(wb, e) - out[b]);
                }
            }
        }
        __syncthreads();
    }
}

template <class T, bool C, int NR>
__global__ void __launch_bounds__(kSolveThreads, NR <= 4 ? 2 : 1) fwd_sweep_kernel(SweepArgs a) {
    using Xv = V<T, C>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Xv* sx = reinterpret_cast<Xv*>(smem_raw);     // 2 x [64][NR]
    Xv* red = sx + 2 * kTile * NR;                // [kQ][NR][64]
    Xv* sq = red + kQ * NR * kTile;               // 2 x [64][NR]: the chain's off-path products
    __shared__ int s_item;
    if (threadIdx.x == 0) s_item = atomicAdd(a.ticket, 1);
    __syncthreads();
    if (*reinterpret_cast<volatile int32_t*>(&a.status[1]) != 0) return;   // an earlier wait gave up
    const int4 it = a.items[s_item];
    const FrontDev f = a.F[it.x];
    const int r = threadIdx.x % kTile, q = threadIdx.x / kTile;
    const int nT = (f.n + kTile - 1) / kTile;
    if (it.y == kItemChain) {
        fwd_chain<T, C, NR>(a, f, nT, r, q, sx, red, sq);
        return;
    }
    if (it.y == kItemWhole) {
        fwd_whole<T, C, NR>(a, f, nT, r, q, sx, red, sq);
        return;
    }
    // worker: rows [R0, R0 + nr) against the pivot blocks t < t_end
    const T* L = reinterpret_cast<const T*>(a.L);
    int R0, nr, t_end;
    if (it.y == kItemPivotRows) { R0 = kTile * it.z; nr = min(kTile, f.n - R0); t_end = it.z - kLag; }
    else { R0 = f.n + kTile * it.z; nr = min(kTile, f.m - R0); t_end = nT; }
    Xv acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = Xv{};
    Xv la[kE], lb[kE];
    row_slice<T, C>(la, L, f.L + R0, f.m, r, q, nr, min(kTile, f.n));
    for (int t = 0; t < t_end; t += 2) {
        // two tiles in flight: the next one loads while this one waits for its x block
        if (t + 1 < t_end)
            row_slice<T, C>(lb, L, f.L + R0 + (int64_t)(t + 1) * kTile * f.m, f.m, r, q, nr, min(kTile, f.n - (t + 1) * kTile));
        if (!fwd_tile<T, C, NR>(a, f, t, la, acc, sx, q)) return;
        if (t + 1 >= t_end) break;
        if (t + 2 < t_end)
            row_slice<T, C>(la, L, f.L + R0 + (int64_t)(t + 2) * kTile * f.m, f.m, r, q, nr, min(kTile, f.n - (t + 2) * kTile));
        if (!fwd_tile<T, C, NR>(a, f, t + 1, lb, acc, sx, q)) return;
    }
    Xv out[NR / kQ];
    reduce_slices<NR>(acc, red, out, r, q);
    if (it.y == kItemPivotRows) {
        T* Part = reinterpret_cast<T*>(a.partial);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) stv<T, C>(Part, (int64_t)(f.flag_base + it.z) * kPartialStride + j * kTile + r, out[b]);
        }
        publish_flag(&a.pflags[f.flag_base + it.z], a.epoch);
    } else if (r < nr) {
        T* wb = reinterpret_cast<T*>(f.pool == 0 ? a.w0 : a.w1);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) {
                const int64_t e = f.W * a.nrhs + (R0 - f.n + r) + (int64_t)j * f.u;
                stv<T, C>(wb, e, ldv<T, C>(wb, e) - out[b]);
            }
        }
    }
}

// Backward chain of one front, last pivot block first:
//   x_c = op(L_cc^{-1})^T (y_c - partial_c - q_c - op(L_{c+1,c})^T x_{c+1}),
// partial_c from the column worker (rows below the pivots and pivot blocks
// after c + 2), q_c = op(L_{c+2,c})^T x_{c+2} formed right after x_{c+2}.
template <class T, bool C, bool CJ, int NR>
__device__ void bwd_chain(const SweepArgs& a, const FrontDev& f, int nT, int r, int q, V<T, C>* sx, V<T, C>* red, V<T, C>* sq) {
    using Xv = V<T, C>;
    static_assert(kLag == 2, "the chain adds the two newest blocks");
    const T* DinvT = reinterpret_cast<const T*>(a.dinvT);
    const T* SubT = reinterpret_cast<const T*>(a.subT);
    const T* SubT2 = reinterpret_cast<const T*>(a.subT2);
    const T* Part = reinterpret_cast<const T*>(a.partial);
    T* X = reinterpret_cast<T*>(a.X);
    Xv* sprev = sx;                 // x_{c+1}
    Xv* st = sx + kTile * NR;
    // thread (r, q) holds column r, rows q*kE .. q*kE+kE-1 of the row-major tiles
    Xv lp[kE], dv[kE];
    row_slice<T, C>(dv, DinvT, f.dinv + (int64_t)(nT - 1) * kTile * kTile, kTile, r, q, kTile, kTile);
    // y_c - partial_c for the next step, gathered after each publish when the
    // worker has already finished
    Xv nxt[NR / kQ];
    bool have_next = false;
    for (int c = nT - 1; c >= 0; --c) {
        const int c0 = c * kTile, dc = min(kTile, f.n - c0);
        const bool fed = f.m > f.n || c + kLag + 1 <= nT - 1;
        Xv tv[NR / kQ];
        if (have_next) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] = nxt[b];
        } else {
            if (fed && !wait_flag(&a.pflags[f.flag_base + c], a.epoch, a.status)) return;
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                Xv v{};
                if (r < dc && j < a.nrhs) {
                    v = ldv<T, C>(X, f.off + c0 + r + (int64_t)j * a.ldx);
                    if (fed) v -= ldv_cg<T, C>(Part, (int64_t)(f.flag_base + c) * kPartialStride + j * kTile + r);
                }
                tv[b] = v;
            }
        }
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (c + 2 < nT && r < dc && j < a.nrhs) tv[b] -= sq[(c & 1) * kTile * NR + r * NR + j];
        }
        if (c + 1 < nT) {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<CJ, NR>(acc, lp, sprev, q);
            Xv u[NR / kQ];
            reduce_slices<NR>(acc, red, u, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] -= u[b];
        }
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = tv[b];
        __syncthreads();
        {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<CJ, NR>(acc, dv, st, q);
            Xv xs[NR / kQ];
            reduce_slices<NR>(acc, red, xs, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                const bool in = r < dc && j < a.nrhs;
                if (in) stv<T, C>(X, f.off + c0 + r + (int64_t)j * a.ldx, xs[b]);
                sprev[r * NR + j] = in ? xs[b] : Xv{};
            }
        }
        if (c > 0) {
            const int64_t blk = f.dinv + (int64_t)(c - 1) * kTile * kTile;
            row_slice<T, C>(lp, SubT, blk, kTile, r, q, kTile, kTile);
            row_slice<T, C>(dv, DinvT, blk, kTile, r, q, kTile, kTile);
        }
        // tile of the off-path product, in flight during the publish
        Xv lq[kE];
        if (c >= 2) row_slice<T, C>(lq, SubT2, f.dinv + (int64_t)(c - 2) * kTile * kTile, kTile, r, q, kTile, kTile);
        publish_flag(&a.xflags[f.flag_base + c], a.epoch);
        have_next = false;
        if (c >= 1) {
            const int c1 = c - 1, o1 = c1 * kTile;
            const bool fed1 = f.m > f.n || c1 + kLag + 1 <= nT - 1;
            if (!fed1 || test_flag(&a.pflags[f.flag_base + c1], a.epoch)) {
#pragma unroll
                for (int b = 0; b < NR / kQ; ++b) {
                    const int j = q + kQ * b;
                    Xv v{};
                    if (j < a.nrhs) {   // blocks before the last are full
                        v = ldv<T, C>(X, f.off + o1 + r + (int64_t)j * a.ldx);
                        if (fed1) v -= ldv_cg<T, C>(Part, (int64_t)(f.flag_base + c1) * kPartialStride + j * kTile + r);
                    }
                    nxt[b] = v;
                }
                have_next = true;
            }
        }
        // off the critical path: q_{c-2} = op(L_{c,c-2})^T x_c
        if (c >= 2) {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<CJ, NR>(acc, lq, sprev, q);
            Xv qv[NR / kQ];
            reduce_slices<NR>(acc, red, qv, r, q);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) sq[(c & 1) * kTile * NR + r * NR + q + kQ * b] = qv[b];
            __syncthreads();
        }
    }
}

// Backward sweep of a small front by one CTA: for each pivot block, last
// first, the contributions of the rows below the pivots (x gathered at
// lowerStruct; tiles staged through shared memory for the transposed
// product) and of the later block, then the transposed inverse.
template <class T, bool C, bool CJ, int NR>
__device__ void bwd_whole(const SweepArgs& a, const FrontDev& f, int nT, int r, int q, V<T, C>* sx, V<T, C>* red, V<T, C>* sq,
                          V<T, C>* sL) {
    using Xv = V<T, C>;
    constexpr int ldl = kTile + 1;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* DinvT = reinterpret_cast<const T*>(a.dinvT);
    const T* SubT = reinterpret_cast<const T*>(a.subT);
    T* X = reinterpret_cast<T*>(a.X);
    Xv* st = sx;
    Xv* xs = sx + kTile * NR;        // gathered x of one tile below the pivots
    Xv* x1 = sq;                     // x_1 once solved
    for (int c = nT - 1; c >= 0; --c) {
        const int c0 = c * kTile, dc = min(kTile, f.n - c0);
        Xv acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        for (int R0 = f.n; R0 < f.m; R0 += kTile) {
            const int nr = min(kTile, f.m - R0);
            Xv pre[kE];
#pragma unroll
            for (int p = 0; p < kE; ++p) {
                const int cc = q + kQ * p;
                pre[p] = (r < nr && cc < dc) ? ldv<T, C>(L, f.L + R0 + r + (int64_t)(c0 + cc) * f.m) : Xv{};
            }
            __syncthreads();   // previous readers of sL / xs are done
#pragma unroll
            for (int p = 0; p < kE; ++p) sL[(q + kQ * p) * ldl + r] = pre[p];
            for (int idx = threadIdx.x; idx < kTile * NR; idx += kSolveThreads) {
                const int rr = idx % kTile, j = idx / kTile;
                xs[rr * NR + j] = (rr < nr && j < a.nrhs)
                                      ? ldv<T, C>(X, (int64_t)a.lower[f.lower + R0 - f.n + rr] + (int64_t)j * a.ldx) : Xv{};
            }
            __syncthreads();
            Xv v[kE];
#pragma unroll
            for (int k = 0; k < kE; ++k) v[k] = sL[r * ldl + q * kE + k];
            slice_mac<CJ, NR>(acc, v, xs, q);
        }
        if (c + 1 < nT) {
            Xv lp[kE];
            row_slice<T, C>(lp, SubT, f.dinv + (int64_t)c * kTile * kTile, kTile, r, q, kTile, kTile);   // tile (c+1, c)
            slice_mac<CJ, NR>(acc, lp, x1, q);
        }
        Xv u[NR / kQ];
        reduce_slices<NR>(acc, red, u, r, q);
        Xv tv[NR / kQ];
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            tv[b] = (r < dc && j < a.nrhs) ? ldv<T, C>(X, f.off + c0 + r + (int64_t)j * a.ldx) - u[b] : Xv{};
            st[r * NR + j] = tv[b];
        }
        __syncthreads();
        Xv dv[kE];
        row_slice<T, C>(dv, DinvT, f.dinv + (int64_t)c * kTile * kTile, kTile, r, q, kTile, kTile);
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        slice_mac<CJ, NR>(acc, dv, st, q);
        Xv xv[NR / kQ];
        reduce_slices<NR>(acc, red, xv, r, q);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            const bool in = r < dc && j < a.nrhs;
            if (in) stv<T, C>(X, f.off + c0 + r + (int64_t)j * a.ldx, xv[b]);
            x1[r * NR + j] = in ? xv[b] : Xv{};
        }
        __syncthreads();
    }
}

template <class T, bool C, bool CJ, int NR>
__global__ void __launch_bounds__(kSolveThreads, NR <= 4 ? 2 : 1) bwd_sweep_kernel(SweepArgs a) {
    using Xv = V<T, C>;
    constexpr int ldl = kTile + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Xv* sx = reinterpret_cast<Xv*>(smem_raw);     // 2 x [64][NR]
    Xv* red = sx + 2 * kTile * NR;                // [kQ][NR][64]
    Xv* sq = red + kQ * NR * kTile;               // 2 x [64][NR]: the chain's off-path products
    Xv* sL = sq + 2 * kTile * NR;                 // [64 columns][65]
    __shared__ int s_item;
    if (threadIdx.x == 0) s_item = atomicAdd(a.ticket, 1);
    __syncthreads();
    if (*reinterpret_cast<volatile int32_t*>(&a.status[1]) != 0) return;   // an earlier wait gave up
    const int4 it = a.items[s_item];
    const FrontDev f = a.F[it.x];
    const int r = threadIdx.x % kTile, q = threadIdx.x / kTile;
    const int nT = (f.n + kTile - 1) / kTile;
    if (it.y == kItemChain) {
        bwd_chain<T, C, CJ, NR>(a, f, nT, r, q, sx, red, sq);
        return;
    }
    if (it.y == kItemWhole) {
        bwd_whole<T, C, CJ, NR>(a, f, nT, r, q, sx, red, sq, sL);
        return;
    }
    // column worker (kItemColumns) or helper (kItemLowerChunk, chunk it.w >= 1):
    // op(L[R, c-block])^T x_R over rows R below the pivots (x gathered at
    // lowerStruct, final since the ancestors are solved); the worker then adds
    // the helpers' sums and the pivot blocks after c + kLag as the chain
    // publishes them
    const bool helper = it.y == kItemLowerChunk;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* X = reinterpret_cast<const T*>(a.X);
    const int c = it.z, c0 = c * kTile, dc = min(kTile, f.n - c0);
    const int nlow = (f.m - f.n + kTile - 1) / kTile;
    const int low0 = helper ? it.w * kLowerChunkTiles : 0;
    const int low1 = min(nlow, low0 + kLowerChunkTiles);
    const int nl = max(0, low1 - low0);
    const int npiv = helper ? 0 : max(0, nT - 1 - (c + kLag));
    const int ntiles = nl + npiv;
    // coalesced staging: element p of this thread is (row r, column q + kQ*p)
    auto tile_of = [&](int i, int& R0, int& nr) {
        if (i < nl) { R0 = f.n + kTile * (low0 + i); nr = min(kTile, f.m - R0); }
        else { R0 = kTile * (nT - 1 - (i - nl)); nr = min(kTile, f.n - R0); }
    };
    Xv pre[kE];
    auto fetch = [&](int i) {
        int R0, nr;
        tile_of(i, R0, nr);
#pragma unroll
        for (int p = 0; p < kE; ++p) {
            const int cc = q + kQ * p;
            pre[p] = (r < nr && cc < dc) ? ldv<T, C>(L, f.L + R0 + r + (int64_t)(c0 + cc) * f.m) : Xv{};
        }
    };
    Xv acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = Xv{};
    if (ntiles > 0) fetch(0);
    for (int i = 0; i < ntiles; ++i) {
        int R0, nr;
        tile_of(i, R0, nr);
        __syncthreads();   // the previous tile's readers are done with sL and sx
#pragma unroll
        for (int p = 0; p < kE; ++p) sL[(q + kQ * p) * ldl + r] = pre[p];
        if (i + 1 < ntiles) fetch(i + 1);
        if (i >= nl) {
            if (!wait_flag(&a.xflags[f.flag_base + R0 / kTile], a.epoch, a.status)) return;
            load_x_tile<T, C, NR>(sx, X, f.off + R0, a.ldx, nr, a.nrhs);
        } else {
            for (int idx = threadIdx.x; idx < kTile * NR; idx += kSolveThreads) {
                const int rr = idx % kTile, j = idx / kTile;
                sx[rr * NR + j] = (rr < nr && j < a.nrhs)
                                      ? ldv<T, C>(X, (int64_t)a.lower[f.lower + R0 - f.n + rr] + (int64_t)j * a.ldx) : Xv{};
            }
        }
        __syncthreads();
        Xv v[kE];
#pragma unroll
        for (int k = 0; k < kE; ++k) v[k] = sL[r * ldl + q * kE + k];
        slice_mac<CJ, NR>(acc, v, sx, q);
    }
    Xv out[NR / kQ];
    reduce_slices<NR>(acc, red, out, r, q);
    if (helper) {
        T* HP = reinterpret_cast<T*>(a.hpart);
        const int64_t h = f.hbase + (int64_t)c * (f.nch - 1) + (it.w - 1);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) stv<T, C>(HP, h * kPartialStride + j * kTile + r, out[b]);
        }
        publish_flag(&a.hflags[h], a.epoch);
        return;
    }
    // the helpers of this column block were issued before this CTA; add
    // their sums in chunk order
    const T* HP = reinterpret_cast<const T*>(a.hpart);
    for (int ch = 1; ch < f.nch; ++ch) {
        const int64_t h = f.hbase + (int64_t)c * (f.nch - 1) + (ch - 1);
        if (!wait_flag(&a.hflags[h], a.epoch, a.status)) return;
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) out[b] += ldv_cg<T, C>(HP, h * kPartialStride + j * kTile + r);
        }
    }
    T* Part = reinterpret_cast<T*>(a.partial);
#pragma unroll
    for (int b = 0; b < NR / kQ; ++b) {
        const int j = q + kQ * b;
        if (j < a.nrhs) stv<T, C>(Part, (int64_t)(f.flag_base + c) * kPartialStride + j * kTile + r, out[b]);
    }
    publish_flag(&a.pflags[f.flag_base + c], a.epoch);
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ, int NR>
static int64_t run_sweeps(Plan& P, T* X, int nrhs) {
    using Xv = V<T, C>;
    const size_t smem_fwd = sizeof(Xv) * (4 + kQ) * kTile * NR;
    const size_t smem_bwd = smem_fwd + sizeof(Xv) * kTile * (kTile + 1);
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(fwd_sweep_kernel<T, C, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fwd);
        cudaFuncSetAttribute(bwd_sweep_kernel<T, C, CJ, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bwd);
        attr_done = true;
    }
    const int4* items = reinterpret_cast<const int4*>(P.items);
    SweepArgs a{};
    a.F = P.fronts;
    a.xflags = P.flags;
    a.pflags = P.flags + P.flags_total;
    a.L = P.L;
    a.dinv = P.dinv;
    a.dinvT = P.dinvT;
    a.subT = P.subT;
    a.subT2 = P.subT2;
    a.partial = P.partial;
    a.hpart = P.hpart;
    a.hflags = P.flags + 2 * P.flags_total;
    a.X = X;
    a.ldx = P.n;
    a.w0 = P.wpool[0];
    a.w1 = P.wpool[1];
    a.lower = P.lower;
    a.nrhs = nrhs;
    a.status = P.status;
    T* w0 = reinterpret_cast<T*>(P.wpool[0]);
    T* w1 = reinterpret_cast<T*>(P.wpool[1]);
    const int nlev = P.max_depth + 1;
    int64_t launches = 0;
    cudaMemsetAsync(P.tickets, 0, sizeof(int32_t) * 2 * nlev, P.stream);
    for (int d = P.max_depth; d >= 0; --d) {
        const SolveLevel& lv = P.solve_levels[d];
        if (lv.nfronts == 0) continue;
        fwd_gather_kernel<T, C><<<dim3(lv.nfronts, lv.gather_chunks), kSolveThreads, 0, P.stream>>>(
            P.fronts, P.level_fronts + lv.fronts, X, P.n, w0, w1, P.cmaps, nrhs);
        ++launches;
        if (lv.nfwd > 0) {
            a.items = items + lv.fwd_items;
            a.ticket = P.tickets + 2 * d;
            a.epoch = ++P.epoch;
            fwd_sweep_kernel<T, C, NR><<<lv.nfwd, kSolveThreads, smem_fwd, P.stream>>>(a);
            ++launches;
        }
    }
    diag_scale_kernel<T, C><<<1184, 256, 0, P.stream>>>(X, P.n, P.n, nrhs, P.D);
    ++launches;
    for (int d = 0; d <= P.max_depth; ++d) {
        const SolveLevel& lv = P.solve_levels[d];
        if (lv.nbwd == 0) continue;
        a.items = items + lv.bwd_items;
        a.ticket = P.tickets + 2 * d + 1;
        a.epoch = ++P.epoch;
        bwd_sweep_kernel<T, C, CJ, NR><<<lv.nbwd, kSolveThreads, smem_bwd, P.stream>>>(a);
        ++launches;
    }
    return launches;
}

template <class T, bool C, bool CJ>
static int run_solve_impl(Plan& P, T* xn, int nrhs_total) {
    // complex double sweeps take at most 8 right-hand sides at a time (the
    // 16-wide accumulators would not fit in registers)
    constexpr int kChunk = (C && sizeof(T) == 8) ? 8 : kMaxRhsChunk;
    int64_t launches = 0;
    for (int j0 = 0; j0 < nrhs_total; j0 += kChunk) {
        const int nrhs = nrhs_total - j0 < kChunk ? nrhs_total - j0 : kChunk;
        T* X = xn + (C ? 2 : 1) * (int64_t)j0 * P.n;
        if (nrhs <= 4) launches += run_sweeps<T, C, CJ, 4>(P, X, nrhs);
        else if constexpr (kChunk == 8) launches += run_sweeps<T, C, CJ, 8>(P, X, nrhs);
        else if (nrhs <= 8) launches += run_sweeps<T, C, CJ, 8>(P, X, nrhs);
        else launches += run_sweeps<T, C, CJ, 16>(P, X, nrhs);
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
