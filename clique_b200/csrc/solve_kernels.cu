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
//   * one chain CTA, which walks the front's 64-wide pivot blocks in order:
//         forward   x_s = y_s - M_s x_{s-1},   M_s = L_ss^{-1} L_{s,s-1},
//         backward  x_c = z_c - N_c x_{c+1},   N_c = op(L_cc^{-1})^T op(L_{c+1,c})^T,
//     with y_s / z_c from the block's worker and M, N formed once per
//     factorization.  One 64 x 64 product per step is the chain's whole
//     critical path: x_{s-1} stays in its shared memory and the tile was
//     loaded into registers two steps earlier.  After each block the chain
//     publishes its progress, one word per front.
//   * workers, which stream the rest of the front's L tiles as the chain
//     publishes solved blocks.  Forward: one per 64-row block of pivot rows,
//         y_s = L_ss^{-1} (b_s - sum_{t <= s-2} L_st x_t),
//     and one per 64-row block below the pivots (subtracts into the update
//     vector W_B).  Backward: one per pivot column block c,
//         z_c = op(L_cc^{-1})^T (y_c - sum_{r below the pivots} op(L_rc)^T x_r
//                                    - sum_{r >= c+2} op(L_rc)^T x_r),
//     taking the first 16 tiles of rows below the pivots itself and the sums
//     of helpers for the further 16-tile chunks (issued first, no waits).
//   Every worker keeps the next L tile and, once published, the next x tile
//   in flight while it multiplies the current one.
// Work items are taken from an atomic ticket counter in the order helpers
// (which wait for nothing), then each chain followed by its workers in the
// order the chain consumes them, so every CTA a resident CTA waits for was
// either issued before it or is a worker whose own waits only reach back to
// earlier tickets: the sweep finishes with any number of resident CTAs >= 2.
// Waits are bounded: on expiry a CTA records a timeout in the status word
// and returns, and every other wait gives up as soon as it sees that word
// set.
#include <climits>
#include <type_traits>

#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {

constexpr int kSolveThreads = 256;
constexpr int kQ = kSolveThreads / kTile;   // slices per tile row (4)
constexpr int kE = kTile / kQ;              // tile elements per thread and slice (16)
constexpr int kLag = kSolveLag;             // worker s adds the blocks t <= s - kLag
constexpr int kMaxRhsChunk = kSolveRhsChunk;   // right-hand sides per sweep
constexpr int kPartialStride = kTile * kMaxRhsChunk;   // elements per pivot block in the partial store
constexpr int kGatherRows = 1024;           // front rows per gather CTA (grid y of the gather launch)
constexpr uint64_t kSpinNs = 500000000ull;  // 0.5 s bound on any single wait

__device__ __forceinline__ int ld_acquire(const int32_t* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
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
__device__ __forceinline__ bool wait_flag(const int32_t* flag, int epoch, int32_t* status, uint64_t limit_ns = kSpinNs) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        if (ld_acquire(flag) != epoch) {
            const uint64_t t0 = global_ns();
            while (ld_acquire(flag) != epoch) {
                if (*reinterpret_cast<volatile int32_t*>(&status[1]) != 0) { ok = 0; break; }
                if (global_ns() - t0 > limit_ns) { atomicExch(&status[1], 1); atomicCAS(&status[2], 0, 4); ok = 0; break; }
                __nanosleep(100);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Publish after the CTA's stores: the barrier orders every thread's stores
// before thread 0's fence, which makes them visible at device scope before
// the flag.
__device__ __forceinline__ void publish_flag(int32_t* flag, int epoch) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicExch(flag, epoch);
    }
}

// Chain progress word of a front: (epoch << 32) | number of solved blocks
// published in this launch.  A word from an older launch counts as zero.
__device__ __forceinline__ int progress_count(unsigned long long w, int epoch) {
    return (int)(w >> 32) == epoch ? (int)(w & 0xffffffffu) : 0;
}

// Chain: publish `count` solved blocks (thread 0) and meanwhile test the
// flag of the next worker result (thread 32, null: none); returns whether
// that flag is set, the same for the whole CTA.
__device__ __forceinline__ bool publish_and_test(unsigned long long* word, int count, int epoch, const int32_t* next_flag) {
    __shared__ int s_set;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicExch(word, ((unsigned long long)(unsigned)epoch << 32) | (unsigned)count);
    } else if (threadIdx.x == 32) {
        s_set = next_flag != nullptr && ld_acquire(next_flag) == epoch;
    }
    __syncthreads();
    return s_set != 0;
}

// thread 0 waits until the chain has published at least `need` blocks; the
// CTA gets the count seen (every block below it is readable), or -1 after a
// timeout (wait site 4) or another CTA's timeout
__device__ __forceinline__ int wait_progress(const unsigned long long* word, int need, int epoch, int32_t* status) {
    __shared__ int s_cnt;
    if (threadIdx.x == 0) {
        int cnt = progress_count(ld_acquire64(word), epoch);
        if (cnt < need) {
            const uint64_t t0 = global_ns();
            while ((cnt = progress_count(ld_acquire64(word), epoch)) < need) {
                if (*reinterpret_cast<volatile int32_t*>(&status[1]) != 0) { cnt = -1; break; }
                if (global_ns() - t0 > kSpinNs) { atomicExch(&status[1], 1); atomicCAS(&status[2], 0, 4); cnt = -1; break; }
                __nanosleep(64);
            }
        }
        s_cnt = cnt;
    }
    __syncthreads();
    return s_cnt;
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

// resident CTAs per SM the sweeps ask for: two when the L tiles of a thread
// fit in half the register file (real or FP32 complex, up to 4 right-hand sides)
template <class T, bool C, int NR>
constexpr int sweep_min_blocks() { return (NR <= 4 && !(C && sizeof(T) == 8)) ? 2 : 1; }

// Register staging of a 64 x NR tile of right-hand sides: element e of this
// thread is (row (tid + 256 e) % 64, rhs (tid + 256 e) / 64).
template <int NR>
struct XStage {
    static constexpr int kN = kTile * NR / kSolveThreads;
    __device__ __forceinline__ static int row(int e) { return (threadIdx.x + kSolveThreads * e) % kTile; }
    __device__ __forceinline__ static int rhs(int e) { return (threadIdx.x + kSolveThreads * e) / kTile; }
};

// x rows x0 .. x0 + nr - 1 of X (column-major, ldx) into registers, zero
// beyond nr rows or nrhs columns; L2-coherent loads for values another CTA
// of this launch published
template <class T, bool C, int NR>
__device__ __forceinline__ void stage_x(V<T, C> (&xr)[XStage<NR>::kN], const T* X, int64_t x0, int64_t ldx, int nr, int nrhs) {
#pragma unroll
    for (int e = 0; e < XStage<NR>::kN; ++e) {
        const int rr = XStage<NR>::row(e), j = XStage<NR>::rhs(e);
        xr[e] = (rr < nr && j < nrhs) ? ldv_cg<T, C>(X, x0 + rr + (int64_t)j * ldx) : V<T, C>{};
    }
}

template <int NR, class Xv>
__device__ __forceinline__ void put_x(const Xv (&xr)[XStage<NR>::kN], Xv* s) {
#pragma unroll
    for (int e = 0; e < XStage<NR>::kN; ++e) s[XStage<NR>::row(e) * NR + XStage<NR>::rhs(e)] = xr[e];
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
// tiny fronts (one pivot block, at most kTinyLowerRows rows below): one warp
// per front, kTinyWarps fronts per CTA, no flags.  Lane = pivot row / column
// (lane and lane + 32); the right-hand-side rows a product needs are staged
// in the warp's slice of shared memory and read as broadcasts.
//   forward   x_T = L11^{-1} x_T,   W_B -= L21 x_T
//   backward  z = x_T - op(L21)^T X[lowerStruct],   x_T = op(L11^{-1})^T z
// ---------------------------------------------------------------------------
constexpr int kTinyWarps = 8;

template <class T, bool C, int NR>
__global__ void __launch_bounds__(32 * kTinyWarps) tiny_fwd_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl,
                                                                   int nf, T* __restrict__ X, int64_t ldx, T* __restrict__ w0,
                                                                   T* __restrict__ w1, const T* __restrict__ L,
                                                                   const T* __restrict__ dinv, int nrhs) {
    using Xv = V<T, C>;
    extern __shared__ __align__(16) unsigned char tiny_smem[];
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int fi = blockIdx.x * kTinyWarps + w;
    if (fi >= nf) return;   // warp-uniform; only warp barriers below
    Xv* sb = reinterpret_cast<Xv*>(tiny_smem) + (int64_t)w * kTile * NR;
    const FrontDev f = F[fl[fi]];
    const int n = f.n, u = f.m - f.n;
    for (int e = lane; e < n * NR; e += 32) {
        const int k = e % n, j = e / n;
        sb[k * NR + j] = j < nrhs ? ldv<T, C>(X, f.off + k + (int64_t)j * ldx) : Xv{};
    }
    __syncwarp();
    // x_T = L11^{-1} b: rows lane and lane + 32 (column k of the inverse is contiguous)
    const Xv* Dv = reinterpret_cast<const Xv*>(dinv) + f.dinv;
    Xv a0[NR], a1[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) a0[j] = a1[j] = Xv{};
    for (int k = 0; k < n; ++k) {
        const Xv d0 = lane < n ? Dv[lane + k * kTile] : Xv{};
        const Xv d1 = lane + 32 < n ? Dv[lane + 32 + k * kTile] : Xv{};
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            const Xv bv = sb[k * NR + j];
            mac(a0[j], d0, bv);
            mac(a1[j], d1, bv);
        }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        if (lane < n) {
            if (j < nrhs) stv<T, C>(X, f.off + lane + (int64_t)j * ldx, a0[j]);
            sb[lane * NR + j] = a0[j];
        }
        if (lane + 32 < n) {
            if (j < nrhs) stv<T, C>(X, f.off + lane + 32 + (int64_t)j * ldx, a1[j]);
            sb[(lane + 32) * NR + j] = a1[j];
        }
    }
    __syncwarp();
    // W_B -= L21 x_T, 32 rows at a time (row i of L21: stride m between columns)
    T* wb = f.pool == 0 ? w0 : w1;
    const Xv* Lf = reinterpret_cast<const Xv*>(L) + f.L + f.n;
    for (int i0 = 0; i0 < u; i0 += 32) {
        const int i = i0 + lane;
        Xv acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        for (int k = 0; k < n; ++k) {
            const Xv l = i < u ? Lf[i + (int64_t)k * f.m] : Xv{};
#pragma unroll
            for (int j = 0; j < NR; ++j) mac(acc[j], l, sb[k * NR + j]);
        }
        if (i < u) {
#pragma unroll
            for (int j = 0; j < NR; ++j) {
                if (j >= nrhs) break;
                const int64_t e = f.W * nrhs + i + (int64_t)j * f.u;
                stv<T, C>(wb, e, ldv<T, C>(wb, e) - acc[j]);
            }
        }
    }
}

template <class T, bool C, bool CJ, int NR>
__global__ void __launch_bounds__(32 * kTinyWarps) tiny_bwd_kernel(const FrontDev* __restrict__ F, const int32_t* __restrict__ fl,
                                                                   int nf, T* __restrict__ X, int64_t ldx, const T* __restrict__ L,
                                                                   const T* __restrict__ dinvT, const int32_t* __restrict__ lower,
                                                                   int nrhs) {
    using Xv = V<T, C>;
    extern __shared__ __align__(16) unsigned char tiny_smem[];
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int fi = blockIdx.x * kTinyWarps + w;
    if (fi >= nf) return;   // warp-uniform; only warp barriers below
    Xv* sb = reinterpret_cast<Xv*>(tiny_smem) + (int64_t)w * kTile * NR;
    const FrontDev f = F[fl[fi]];
    const int n = f.n, u = f.m - f.n;
    Xv a0[NR], a1[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        a0[j] = (lane < n && j < nrhs) ? ldv<T, C>(X, f.off + lane + (int64_t)j * ldx) : Xv{};
        a1[j] = (lane + 32 < n && j < nrhs) ? ldv<T, C>(X, f.off + lane + 32 + (int64_t)j * ldx) : Xv{};
    }
    // z = y - op(L21)^T x_B, the solved rows below staged 32 at a time
    const Xv* Lf = reinterpret_cast<const Xv*>(L) + f.L + f.n;
    for (int i0 = 0; i0 < u; i0 += 32) {
        const int i = i0 + lane;
        const int gi = i < u ? lower[f.lower + i] : -1;
        __syncwarp();
#pragma unroll
        for (int j = 0; j < NR; ++j) sb[lane * NR + j] = (gi >= 0 && j < nrhs) ? ldv<T, C>(X, gi + (int64_t)j * ldx) : Xv{};
        __syncwarp();
        const int cn = min(32, u - i0);
        for (int t = 0; t < cn; ++t) {
            const Xv l0 = lane < n ? opc<CJ>(Lf[i0 + t + (int64_t)lane * f.m]) : Xv{};
            const Xv l1 = lane + 32 < n ? opc<CJ>(Lf[i0 + t + (int64_t)(lane + 32) * f.m]) : Xv{};
#pragma unroll
            for (int j = 0; j < NR; ++j) {
                const Xv xv = sb[t * NR + j];
                a0[j] -= l0 * xv;
                a1[j] -= l1 * xv;
            }
        }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        if (lane < n) sb[lane * NR + j] = a0[j];
        if (lane + 32 < n) sb[(lane + 32) * NR + j] = a1[j];
    }
    __syncwarp();
    // x_T[k] = sum_t op(Linv[t][k]) z[t]; Linv[t][k] is element k + 64 t of the row-major copy
    const Xv* DvT = reinterpret_cast<const Xv*>(dinvT) + f.dinv;
    Xv r0[NR], r1[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) r0[j] = r1[j] = Xv{};
    for (int t = 0; t < n; ++t) {
        const Xv d0 = lane < n ? opc<CJ>(DvT[lane + t * kTile]) : Xv{};
        const Xv d1 = lane + 32 < n ? opc<CJ>(DvT[lane + 32 + t * kTile]) : Xv{};
#pragma unroll
        for (int j = 0; j < NR; ++j) {
            const Xv zv = sb[t * NR + j];
            mac(r0[j], d0, zv);
            mac(r1[j], d1, zv);
        }
    }
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        if (j >= nrhs) break;
        if (lane < n) stv<T, C>(X, f.off + lane + (int64_t)j * ldx, r0[j]);
        if (lane + 32 < n) stv<T, C>(X, f.off + lane + 32 + (int64_t)j * ldx, r1[j]);
    }
}

// ---------------------------------------------------------------------------
// diagonal solve X := D^{-1} X (FP64 pivots)
// ---------------------------------------------------------------------------
// thread = row p: its pivot is read once for all right-hand sides, the
// columns' loads issued before the divisions
template <class T, bool C>
__global__ void diag_scale_kernel(T* __restrict__ X, int64_t ldx, int64_t n, int nrhs, const double* __restrict__ D) {
    using Xv = V<T, C>;
    using W = DV<C>;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const W d = reinterpret_cast<const W*>(D)[p];
        Xv x[kMaxRhsChunk];
#pragma unroll
        for (int j = 0; j < kMaxRhsChunk; ++j)
            if (j < nrhs) x[j] = ldv<T, C>(X, p + j * ldx);
#pragma unroll
        for (int j = 0; j < kMaxRhsChunk; ++j)
            if (j < nrhs) stv<T, C>(X, p + j * ldx, conv<Xv>(conv<W>(x[j]) / d));
    }
}


// ---------------------------------------------------------------------------
// sweep launches
// ---------------------------------------------------------------------------
struct SweepArgs {
    const FrontDev* F;
    const int4* items;      // {front, kind, block, chunk}
    int32_t* ticket;
    unsigned long long* xprog;   // per front: the chain's progress word
    int32_t* pflags;        // per pivot block: the worker's y / z published
    int epoch;
    const void* L;
    const void* dinv;       // L11^{-1} per 64-block, column-major
    const void* dinvT;      // the same, row-major
    const void* m1;         // forward chain tiles L_ss^{-1} L_{s,s-1}
    const void* n1;         // backward chain tiles op(L_cc^{-1})^T op(L_{c+1,c})^T
    void* partial;          // kPartialStride elements per pivot block: y_s / z_c
    void* hpart;            // backward helpers' partial sums, kPartialStride each
    int32_t* hflags;        // backward helpers' flags
    void* X;                // n x nrhs, ND order, ld ldx
    int64_t ldx;
    void* w0;
    void* w1;
    const int32_t* lower;
    int nrhs;
    int32_t* status;
    // 1: substitution form of the chain steps, x_s = L_ss^{-1} (t_s - L_{s,s-1} x_{s-1})
    // (and its backward counterpart) with the workers publishing t_s; 0: the
    // product form x_s = y_s - M_s x_{s-1} through the stored chain tiles
    int exact;
};

// Forward chain of front fi: x_s = y_s - M_s x_{s-1}.  Step s multiplies the
// tile M_s (in registers since step s-2) with x_{s-1} (in shared memory),
// subtracts the product from y_s (the worker's result, loaded right after
// publishing x_{s-1} when the worker had finished, else waited for now),
// stores and publishes x_s.
// Substitution form (a.exact): the tile is L_{s,s-1} itself and the worker
// publishes t_s = b_s - sum_{t <= s-2} L_st x_t; the step forms
// v = t_s - L_{s,s-1} x_{s-1} in shared memory (sv) and x_s = L_ss^{-1} v,
// with L_ss^{-1} loaded one step ahead.  Two dependent products per step
// instead of one, but the rounding of the inverse enters after the
// cancellation between t_s and L_{s,s-1} x_{s-1}, as in a triangular solve.
template <class T, bool C, int NR>
__device__ void fwd_chain(const SweepArgs& a, const FrontDev& f, int fi, int nT, int r, int q, V<T, C>* sx, V<T, C>* red,
                          V<T, C>* sv) {
    using Xv = V<T, C>;
    const T* M1 = reinterpret_cast<const T*>(a.m1);
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* Dinv = reinterpret_cast<const T*>(a.dinv);
    const T* Part = reinterpret_cast<const T*>(a.partial);
    T* X = reinterpret_cast<T*>(a.X);
    const bool exact = a.exact != 0;
    Xv nxt[NR / kQ];
    bool have_next = false;
    Xv dt[kE];   // exact form: L_ss^{-1} of the current step
    auto load_m = [&](int s, Xv (&dst)[kE]) {   // the coupling tile of step s >= 1
        if (exact)
            row_slice<T, C>(dst, L, f.L + (int64_t)s * kTile + (int64_t)(s - 1) * kTile * f.m, f.m, r, q,
                            min(kTile, f.n - s * kTile), kTile);
        else
            row_slice<T, C>(dst, M1, f.chain + (int64_t)s * kTile * kTile, kTile, r, q, kTile, kTile);
    };
    auto load_y = [&](int s, Xv (&v)[NR / kQ]) {
        const int ds = min(kTile, f.n - s * kTile);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            v[b] = (r < ds && j < a.nrhs) ? ldv_cg<T, C>(Part, (int64_t)(f.flag_base + s) * kPartialStride + j * kTile + r) : Xv{};
        }
    };
    // the product first: y_s, loaded at the end of the previous step (or
    // waited for now), arrives meanwhile
    auto step = [&](int s, Xv (&mt)[kE]) -> bool {
        const int r0 = s * kTile, ds = min(kTile, f.n - r0);
        Xv u[NR / kQ];
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) u[b] = Xv{};
        if (s > 0) {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<false, NR>(acc, mt, sx + ((s - 1) & 1) * kTile * NR, q);
            reduce_slices<NR>(acc, red, u, r, q);
        }
        Xv tv[NR / kQ];
        if (have_next) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] = nxt[b];
        } else {
            if (!wait_flag(&a.pflags[f.flag_base + s], a.epoch, a.status)) return false;
            load_y(s, tv);
        }
        Xv xv[NR / kQ];
        if (exact) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) sv[r * NR + q + kQ * b] = tv[b] - u[b];
            __syncthreads();
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<false, NR>(acc, dt, sv, q);
            reduce_slices<NR>(acc, red, xv, r, q);
            if (s + 1 < nT) row_slice<T, C>(dt, Dinv, f.dinv + (int64_t)(s + 1) * kTile * kTile, kTile, r, q, kTile, kTile);
        } else {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) xv[b] = tv[b] - u[b];
        }
        Xv* xs = sx + (s & 1) * kTile * NR;
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            const bool in = r < ds && j < a.nrhs;
            if (in) stv<T, C>(X, f.off + r0 + r + (int64_t)j * a.ldx, xv[b]);
            xs[r * NR + j] = in ? xv[b] : Xv{};
        }
        have_next = publish_and_test(&a.xprog[fi], s + 1, a.epoch, s + 1 < nT ? &a.pflags[f.flag_base + s + 1] : nullptr);
        if (have_next) load_y(s + 1, nxt);
        // the coupling tile for the step after next
        if (s + 2 < nT) load_m(s + 2, mt);
        return true;
    };
    Xv mA[kE], mB[kE];
    if (exact) row_slice<T, C>(dt, Dinv, f.dinv, kTile, r, q, kTile, kTile);
    if (nT > 1) load_m(1, mB);
    for (int s = 0; s < nT; s += 2) {
        if (!step(s, mA)) return;
        if (s + 1 < nT && !step(s + 1, mB)) return;
    }
}


// Forward sweep of a small front (at most two pivot blocks, kWholeLowerRows
// rows below) by one CTA: both blocks, then every 64-row tile below the
// pivots, with the solved blocks kept in shared memory (no flags).  The
// right-hand sides, the first inverse and the coupling tile are loaded up
// front; below the pivots the (tile, block) products stream with the next
// L tile and the tile's W_B entries in flight.
template <class T, bool C, int NR>
__device__ void fwd_whole(const SweepArgs& a, const FrontDev& f, int nT, int r, int q, V<T, C>* sx, V<T, C>* red, V<T, C>* sq) {
    using Xv = V<T, C>;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* Dinv = reinterpret_cast<const T*>(a.dinv);
    T* X = reinterpret_cast<T*>(a.X);
    Xv* st = sx;                     // right-hand side of the diagonal block
    Xv* xb = sq;                     // x_0, x_1
    Xv bv[2][NR / kQ];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int ds = min(kTile, f.n - s * kTile);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            bv[s][b] = (s < nT && r < ds && j < a.nrhs) ? ldv<T, C>(X, f.off + s * kTile + r + (int64_t)j * a.ldx) : Xv{};
        }
    }
    Xv la[kE], lb[kE];
    row_slice<T, C>(la, Dinv, f.dinv, kTile, r, q, kTile, kTile);
    if (nT > 1) row_slice<T, C>(lb, L, f.L + kTile, f.m, r, q, f.n - kTile, kTile);   // L_{1,0}
    // x_s = L_ss^{-1} t, t in st; result to X and xb[s]
    auto solve_block = [&](int s, const Xv (&dv)[kE], const Xv (&t)[NR / kQ]) {
        const int ds = min(kTile, f.n - s * kTile);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = t[b];
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
            if (in) stv<T, C>(X, f.off + s * kTile + r + (int64_t)j * a.ldx, xs[b]);
            xb[s * kTile * NR + r * NR + j] = in ? xs[b] : Xv{};
        }
        __syncthreads();
    };
    solve_block(0, la, bv[0]);
    if (nT > 1) {
        row_slice<T, C>(la, Dinv, f.dinv + (int64_t)kTile * kTile, kTile, r, q, kTile, kTile);
        Xv acc[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        slice_mac<false, NR>(acc, lb, xb, q);
        Xv u[NR / kQ];
        reduce_slices<NR>(acc, red, u, r, q);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) bv[1][b] -= u[b];
        solve_block(1, la, bv[1]);
    }
    // rows below the pivots: W_B -= L_B x_T, unit u = (tile u / nT, block u % nT)
    const int ntl = (f.m - f.n + kTile - 1) / kTile;
    const int units = ntl * nT;
    if (units == 0) return;
    T* wb = reinterpret_cast<T*>(f.pool == 0 ? a.w0 : a.w1);
    auto load_unit = [&](int u, Xv (&dst)[kE]) {
        const int i = u / nT, t = u % nT, R0 = f.n + kTile * i;
        row_slice<T, C>(dst, L, f.L + R0 + (int64_t)t * kTile * f.m, f.m, r, q, min(kTile, f.m - R0), min(kTile, f.n - t * kTile));
    };
    Xv acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = Xv{};
    Xv wv[NR / kQ];
    auto load_w = [&](int i) {
        const int R0 = f.n + kTile * i, nr = min(kTile, f.m - R0);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            wv[b] = (r < nr && j < a.nrhs) ? ldv<T, C>(wb, f.W * a.nrhs + (R0 - f.n + r) + (int64_t)j * f.u) : Xv{};
        }
    };
    auto unit = [&](int u, const Xv (&cur)[kE], Xv (&oth)[kE]) {
        const int i = u / nT, t = u % nT;
        if (u + 1 < units) load_unit(u + 1, oth);
        slice_mac<false, NR>(acc, cur, xb + t * kTile * NR, q);
        if (t == nT - 1) {
            Xv out[NR / kQ];
            reduce_slices<NR>(acc, red, out, r, q);
            const int R0 = f.n + kTile * i, nr = min(kTile, f.m - R0);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                if (r < nr && j < a.nrhs) stv<T, C>(wb, f.W * a.nrhs + (R0 - f.n + r) + (int64_t)j * f.u, wv[b] - out[b]);
            }
            if (i + 1 < ntl) load_w(i + 1);
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            __syncthreads();   // red is read before the next tile's reduction writes it
        }
    };
    load_w(0);
    load_unit(0, la);
    for (int u = 0; u < units; u += 2) {
        unit(u, la, lb);
        if (u + 1 < units) unit(u + 1, lb, la);
    }
}

// Forward worker: rows [R0, R0 + nr) of the front against the pivot blocks
// t < t_end.  Pivot-row worker of block s (t_end = s - 1):
//   y_s = L_ss^{-1} (b_s - sum_t L_st x_t)  -> partial store, flag;
// lower-row worker (t_end = nT): W_B -= sum_t L_Bt x_t.
// The L tile t + 1 is always in flight during tile t; the x tile t + 1 too
// once the chain's progress word shows it published.
template <class T, bool C, int NR>
__device__ void fwd_worker(const SweepArgs& a, const FrontDev& f, int fi, int nT, int kind, int blk, int r, int q, V<T, C>* sx,
                           V<T, C>* red) {
    using Xv = V<T, C>;
    using XS = XStage<NR>;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* X = reinterpret_cast<const T*>(a.X);
    const bool piv = kind == kItemPivotRows;
    const int R0 = piv ? kTile * blk : f.n + kTile * blk;
    const int nr = min(kTile, (piv ? f.n : f.m) - R0);
    const int t_end = piv ? blk - (kLag - 1) : nT;
    // right-hand side rows of a pivot block, read before the chain overwrites them
    Xv bv[NR / kQ];
    if (piv) {
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            bv[b] = (r < nr && j < a.nrhs) ? ldv<T, C>(X, f.off + R0 + r + (int64_t)j * a.ldx) : Xv{};
        }
    }
    Xv acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = Xv{};
    int known = 0;            // blocks the chain is known to have published
    Xv xr[XS::kN];
    // tile t (L in cur, x_t staged in sx[t & 1]); loads tile t + 1 into oth,
    // or the block inverse after the last tile of a pivot-row worker
    auto tile = [&](int t, Xv (&cur)[kE], Xv (&oth)[kE]) -> bool {
        const bool more = t + 1 < t_end;
        if (more)
            row_slice<T, C>(oth, L, f.L + R0 + (int64_t)(t + 1) * kTile * f.m, f.m, r, q, nr, min(kTile, f.n - (t + 1) * kTile));
        else if (piv)
            row_slice<T, C>(oth, reinterpret_cast<const T*>(a.dinv), f.dinv + (int64_t)blk * kTile * kTile, kTile, r, q, kTile, kTile);
        const bool pre = more && t + 1 < known;
        if (pre) stage_x<T, C, NR>(xr, X, f.off + (int64_t)(t + 1) * kTile, a.ldx, min(kTile, f.n - (t + 1) * kTile), a.nrhs);
        __syncthreads();   // x_t staged
        slice_mac<false, NR>(acc, cur, sx + (t & 1) * kTile * NR, q);
        if (more) {
            if (!pre) {
                const int c = wait_progress(&a.xprog[fi], t + 2, a.epoch, a.status);
                if (c < 0) return false;
                known = c;
                stage_x<T, C, NR>(xr, X, f.off + (int64_t)(t + 1) * kTile, a.ldx, min(kTile, f.n - (t + 1) * kTile), a.nrhs);
            }
            put_x<NR>(xr, sx + ((t + 1) & 1) * kTile * NR);
        }
        return true;
    };
    // y_s = L_ss^{-1} (b_s - acc) with the inverse in dv (substitution form:
    // t_s = b_s - acc, the chain applies the inverse)
    auto finish_pivot = [&](const Xv (&dv)[kE]) {
        Xv out[NR / kQ];
        reduce_slices<NR>(acc, red, out, r, q);
        if (a.exact) {
            T* Part = reinterpret_cast<T*>(a.partial);
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                if (j < a.nrhs) stv<T, C>(Part, (int64_t)(f.flag_base + blk) * kPartialStride + j * kTile + r, bv[b] - out[b]);
            }
            publish_flag(&a.pflags[f.flag_base + blk], a.epoch);
            return;
        }
        Xv* st = sx;   // every reader of sx passed the barrier in reduce_slices
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = bv[b] - out[b];
        __syncthreads();
        Xv acc2[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) acc2[j] = Xv{};
        slice_mac<false, NR>(acc2, dv, st, q);
        Xv y[NR / kQ];
        reduce_slices<NR>(acc2, red, y, r, q);
        T* Part = reinterpret_cast<T*>(a.partial);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) stv<T, C>(Part, (int64_t)(f.flag_base + blk) * kPartialStride + j * kTile + r, y[b]);
        }
        publish_flag(&a.pflags[f.flag_base + blk], a.epoch);
    };
    Xv la[kE], lb[kE];
    if (t_end <= 0) {   // pivot blocks 0 .. kLag-1: nothing to wait for
        row_slice<T, C>(la, reinterpret_cast<const T*>(a.dinv), f.dinv + (int64_t)blk * kTile * kTile, kTile, r, q, kTile, kTile);
        finish_pivot(la);
        return;
    }
    row_slice<T, C>(la, L, f.L + R0, f.m, r, q, nr, min(kTile, f.n));
    {
        const int c = wait_progress(&a.xprog[fi], 1, a.epoch, a.status);
        if (c < 0) return;
        known = c;
        stage_x<T, C, NR>(xr, X, f.off, a.ldx, min(kTile, f.n), a.nrhs);
        put_x<NR>(xr, sx);
    }
    for (int t = 0; t < t_end; t += 2) {
        if (!tile(t, la, lb)) return;
        if (t + 1 < t_end && !tile(t + 1, lb, la)) return;
    }
    if (piv) {
        if (t_end & 1) finish_pivot(lb);
        else finish_pivot(la);
        return;
    }
    Xv out[NR / kQ];
    reduce_slices<NR>(acc, red, out, r, q);
    if (r < nr) {
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

template <class T, bool C, int NR>
__global__ void __launch_bounds__(kSolveThreads, sweep_min_blocks<T, C, NR>()) fwd_sweep_kernel(SweepArgs a) {
    using Xv = V<T, C>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Xv* sx = reinterpret_cast<Xv*>(smem_raw);     // 2 x [64][NR]
    Xv* red = sx + 2 * kTile * NR;                // [kQ][NR][64]
    Xv* sq = red + kQ * NR * kTile;               // 2 x [64][NR]: solved blocks of a small front
    __shared__ int s_item, s_timed_out;
    if (threadIdx.x == 0) {
        s_item = atomicAdd(a.ticket, 1);
        s_timed_out = *reinterpret_cast<volatile int32_t*>(&a.status[1]) != 0;
    }
    __syncthreads();
    if (s_timed_out) return;   // an earlier wait gave up (one read for the whole CTA)
    const int4 it = a.items[s_item];
    const FrontDev f = a.F[it.x];
    const int r = threadIdx.x % kTile, q = threadIdx.x / kTile;
    const int nT = (f.n + kTile - 1) / kTile;
    if (it.y == kItemChain) fwd_chain<T, C, NR>(a, f, it.x, nT, r, q, sx, red, sq);
    else if (it.y == kItemWhole) fwd_whole<T, C, NR>(a, f, nT, r, q, sx, red, sq);
    else fwd_worker<T, C, NR>(a, f, it.x, nT, it.y, it.z, r, q, sx, red);
}

// Backward chain of front fi, last pivot block first: x_c = z_c - N_c x_{c+1}
// with z_c from the column worker; after each block the progress word counts
// the blocks solved from the end.
// Substitution form (a.exact): the worker publishes w_c (z_c before its
// inverse) and the step forms v = w_c - op(L_{c+1,c})^T x_{c+1} in shared
// memory (sv), then x_c = op(L_cc^{-1})^T v; the coupling tile is read
// transposed from the arena (each thread a contiguous run of one column).
template <class T, bool C, bool CJ, int NR>
__device__ void bwd_chain(const SweepArgs& a, const FrontDev& f, int fi, int nT, int r, int q, V<T, C>* sx, V<T, C>* red,
                          V<T, C>* sv) {
    using Xv = V<T, C>;
    const T* N1 = reinterpret_cast<const T*>(a.n1);
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* DinvT = reinterpret_cast<const T*>(a.dinvT);
    const T* Part = reinterpret_cast<const T*>(a.partial);
    T* X = reinterpret_cast<T*>(a.X);
    const bool exact = a.exact != 0;
    Xv nxt[NR / kQ];
    bool have_next = false;
    Xv dt[kE];   // exact form: op(L_cc^{-1})^T of the current step, as a row slice of the row-major inverse
    // coupling tile of block c <= nT - 2: N_c, or (exact) element (r, k) = L[(c+1)*64 + k, c*64 + r]
    // (op is applied in the product)
    auto load_n = [&](int c, Xv (&dst)[kE]) {
        if (exact) {
            const int dc = min(kTile, f.n - c * kTile), dn = min(kTile, f.n - (c + 1) * kTile);
            const int64_t a0 = f.L + (int64_t)(c + 1) * kTile + (int64_t)(c * kTile + r) * f.m;
#pragma unroll
            for (int k = 0; k < kE; ++k) {
                const int kk = q * kE + k;
                dst[k] = (r < dc && kk < dn) ? ldv<T, C>(L, a0 + kk) : Xv{};
            }
        } else {
            row_slice<T, C>(dst, N1, f.chain + (int64_t)c * kTile * kTile, kTile, r, q, kTile, kTile);
        }
    };
    auto load_z = [&](int c, Xv (&v)[NR / kQ]) {
        const int dc = min(kTile, f.n - c * kTile);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            v[b] = (r < dc && j < a.nrhs) ? ldv_cg<T, C>(Part, (int64_t)(f.flag_base + c) * kPartialStride + j * kTile + r) : Xv{};
        }
    };
    // i counts the chain's steps: block c = nT - 1 - i
    auto step = [&](int i, Xv (&nt)[kE]) -> bool {
        const int c = nT - 1 - i, c0 = c * kTile, dc = min(kTile, f.n - c0);
        Xv u[NR / kQ];
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) u[b] = Xv{};
        if (i > 0) {
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            if (exact) slice_mac<CJ, NR>(acc, nt, sx + ((i - 1) & 1) * kTile * NR, q);
            else slice_mac<false, NR>(acc, nt, sx + ((i - 1) & 1) * kTile * NR, q);
            reduce_slices<NR>(acc, red, u, r, q);
        }
        Xv tv[NR / kQ];
        if (have_next) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) tv[b] = nxt[b];
        } else {
            if (!wait_flag(&a.pflags[f.flag_base + c], a.epoch, a.status)) return false;
            load_z(c, tv);
        }
        Xv xv[NR / kQ];
        if (exact) {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) sv[r * NR + q + kQ * b] = tv[b] - u[b];
            __syncthreads();
            Xv acc[NR];
#pragma unroll
            for (int j = 0; j < NR; ++j) acc[j] = Xv{};
            slice_mac<CJ, NR>(acc, dt, sv, q);
            reduce_slices<NR>(acc, red, xv, r, q);
            if (c >= 1) row_slice<T, C>(dt, DinvT, f.dinv + (int64_t)(c - 1) * kTile * kTile, kTile, r, q, kTile, kTile);
        } else {
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) xv[b] = tv[b] - u[b];
        }
        Xv* xs = sx + (i & 1) * kTile * NR;
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            const bool in = r < dc && j < a.nrhs;
            if (in) stv<T, C>(X, f.off + c0 + r + (int64_t)j * a.ldx, xv[b]);
            xs[r * NR + j] = in ? xv[b] : Xv{};
        }
        have_next = publish_and_test(&a.xprog[fi], i + 1, a.epoch, c >= 1 ? &a.pflags[f.flag_base + c - 1] : nullptr);
        if (have_next) load_z(c - 1, nxt);
        // the coupling tile for the step after next
        if (c >= 2) load_n(c - 2, nt);
        return true;
    };
    Xv nA[kE], nB[kE];
    if (exact) row_slice<T, C>(dt, DinvT, f.dinv + (int64_t)(nT - 1) * kTile * kTile, kTile, r, q, kTile, kTile);
    if (nT > 1) load_n(nT - 2, nB);
    for (int i = 0; i < nT; i += 2) {
        if (!step(i, nA)) return;
        if (i + 1 < nT && !step(i + 1, nB)) return;
    }
}

// Backward sweep of a small front by one CTA: for each pivot block, last
// first, the transposed products with the later pivot block (x kept in
// shared memory) and with the rows below the pivots (x gathered at
// lowerStruct), then the transposed inverse.  The tiles of both blocks form
// one stream: the next tile's L and gathered x are in flight during the
// current one, staged through shared memory for the transposed product.
static_assert(kWholeLowerRows <= kLowerChunkTiles * kTile, "gather indices of a small front fit the index buffer");

template <class T, bool C, bool CJ, int NR>
__device__ void bwd_whole(const SweepArgs& a, const FrontDev& f, int nT, int r, int q, V<T, C>* sx, V<T, C>* red, V<T, C>* sL,
                          int32_t* sidx) {
    using Xv = V<T, C>;
    using XS = XStage<NR>;
    constexpr int ldl = kTile + 1;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* DinvT = reinterpret_cast<const T*>(a.dinvT);
    T* X = reinterpret_cast<T*>(a.X);
    Xv* st = sx;                     // right-hand side of the diagonal block
    Xv* xg = sx + kTile * NR;        // gathered x of one tile below the pivots
    Xv* xk = sx + 2 * kTile * NR;    // x of the later pivot block
    const int nlr = f.m - f.n, nl = (nlr + kTile - 1) / kTile;
    for (int i = threadIdx.x; i < nlr; i += kSolveThreads) sidx[i] = a.lower[f.lower + i];
    // y of both blocks, read before this CTA overwrites them
    Xv yv[2][NR / kQ];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int ds = min(kTile, f.n - s * kTile);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            yv[s][b] = (s < nT && r < ds && j < a.nrhs) ? ldv<T, C>(X, f.off + s * kTile + r + (int64_t)j * a.ldx) : Xv{};
        }
    }
    // units: block nT-1 has its nl lower tiles; block nT-2 (if any) the
    // pivot tile of block nT-1, then its nl lower tiles
    const int total = nl + (nT > 1 ? 1 + nl : 0);
    auto unit = [&](int u, int& c, int& R0, int& nr, bool& piv) {
        if (u < nl) { c = nT - 1; piv = false; R0 = f.n + kTile * u; }
        else { c = nT - 2; const int k = u - nl; piv = k == 0; R0 = piv ? (c + 1) * kTile : f.n + kTile * (k - 1); }
        nr = min(kTile, (piv ? f.n : f.m) - R0);
    };
    Xv pre[kE];
    Xv xr[XS::kN];
    auto fetch = [&](int u) {
        int c, R0, nr;
        bool piv;
        unit(u, c, R0, nr, piv);
        const int c0 = c * kTile, dc = min(kTile, f.n - c0);
#pragma unroll
        for (int p = 0; p < kE; ++p) {
            const int cc = q + kQ * p;
            pre[p] = (r < nr && cc < dc) ? ldv<T, C>(L, f.L + R0 + r + (int64_t)(c0 + cc) * f.m) : Xv{};
        }
        if (!piv) {
#pragma unroll
            for (int e = 0; e < XS::kN; ++e) {
                const int rr = XS::row(e), j = XS::rhs(e);
                xr[e] = (rr < nr && j < a.nrhs) ? ldv<T, C>(X, (int64_t)sidx[R0 - f.n + rr] + (int64_t)j * a.ldx) : Xv{};
            }
        }
    };
    Xv acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = Xv{};
    // x_c = op(L_cc^{-1})^T (y_c - acc): to X and xk
    auto finish = [&](int c) {
        const int dc = min(kTile, f.n - c * kTile);
        Xv dv[kE];
        row_slice<T, C>(dv, DinvT, f.dinv + (int64_t)c * kTile * kTile, kTile, r, q, kTile, kTile);
        Xv u[NR / kQ];
        reduce_slices<NR>(acc, red, u, r, q);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = (c == 1 ? yv[1][b] : yv[0][b]) - u[b];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        slice_mac<CJ, NR>(acc, dv, st, q);
        Xv xv[NR / kQ];
        reduce_slices<NR>(acc, red, xv, r, q);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            const bool in = r < dc && j < a.nrhs;
            if (in) stv<T, C>(X, f.off + c * kTile + r + (int64_t)j * a.ldx, xv[b]);
            xk[r * NR + j] = in ? xv[b] : Xv{};
        }
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] = Xv{};
        __syncthreads();
    };
    __syncthreads();   // gather indices
    if (total > 0) fetch(0);
    if (nl == 0) finish(nT - 1);
    for (int u = 0; u < total; ++u) {
        int c, R0, nr;
        bool piv;
        unit(u, c, R0, nr, piv);
        __syncthreads();   // the previous tile's readers are done with sL and xg
#pragma unroll
        for (int p = 0; p < kE; ++p) sL[(q + kQ * p) * ldl + r] = pre[p];
        if (!piv) put_x<NR>(xr, xg);
        if (u + 1 < total) fetch(u + 1);
        __syncthreads();
        Xv v[kE];
#pragma unroll
        for (int k = 0; k < kE; ++k) v[k] = sL[r * ldl + q * kE + k];
        slice_mac<CJ, NR>(acc, v, piv ? xk : xg, q);
        int cn = -1, R0n, nrn;
        bool pn;
        if (u + 1 < total) unit(u + 1, cn, R0n, nrn, pn);
        if (cn != c) finish(c);
    }
}

// Backward column worker of pivot block c (kItemColumns) or helper
// (kItemLowerChunk, chunk >= 1): op(L[R, c-block])^T x_R over its tiles of
// rows R below the pivots (x gathered at lowerStruct, final since the
// ancestors are solved).  The column worker then takes the pivot blocks
// nT-1 .. c+2 as the chain publishes them, adds its helpers' sums in chunk
// order and forms z_c = op(L_cc^{-1})^T (y_c - sum).  Tiles are staged
// through shared memory for the transposed product; the next tile's L and,
// when available, its x are in flight during the current one.
template <class T, bool C, bool CJ, int NR>
__device__ void bwd_worker(const SweepArgs& a, const FrontDev& f, int fi, int nT, int kind, int c, int chunk, int r, int q,
                           V<T, C>* sx, V<T, C>* red, V<T, C>* sL, int32_t* sidx) {
    using Xv = V<T, C>;
    using XS = XStage<NR>;
    constexpr int ldl = kTile + 1;
    const bool helper = kind == kItemLowerChunk;
    const T* L = reinterpret_cast<const T*>(a.L);
    const T* X = reinterpret_cast<const T*>(a.X);
    const int c0 = c * kTile, dc = min(kTile, f.n - c0);
    const int nlow = (f.m - f.n + kTile - 1) / kTile;
    const int low0 = helper ? chunk * kLowerChunkTiles : 0;
    const int low1 = min(nlow, low0 + kLowerChunkTiles);
    const int nl = max(0, low1 - low0);
    const int npiv = helper ? 0 : max(0, nT - 1 - c - (kLag - 1));
    const int ntiles = nl + npiv;
    // right-hand side of the block, read before the chain overwrites it
    Xv yv[NR / kQ];
    if (!helper) {
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            yv[b] = (r < dc && j < a.nrhs) ? ldv<T, C>(X, f.off + c0 + r + (int64_t)j * a.ldx) : Xv{};
        }
    }
    // gather indices of this item's rows below the pivots
    const int lrow0 = low0 * kTile, lrows = min(f.m - f.n - lrow0, nl * kTile);
    for (int i = threadIdx.x; i < lrows; i += kSolveThreads) sidx[i] = a.lower[f.lower + lrow0 + i];
    auto tile_of = [&](int i, int& R0, int& nr) {
        if (i < nl) { R0 = f.n + kTile * (low0 + i); nr = min(kTile, f.m - R0); }
        else { R0 = kTile * (nT - 1 - (i - nl)); nr = min(kTile, f.n - R0); }
    };
    // coalesced staging: element p of this thread is (row r, column q + kQ*p)
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
    int known = 0;   // blocks the chain is known to have published (from the last)
    Xv xr[XS::kN];
    auto stage = [&](int i) {   // x of tile i into xr (pivot tiles: published)
        int R0, nr;
        tile_of(i, R0, nr);
        if (i < nl) {
            const int base = (i * kTile);
#pragma unroll
            for (int e = 0; e < XS::kN; ++e) {
                const int rr = XS::row(e), j = XS::rhs(e);
                xr[e] = (rr < nr && j < a.nrhs) ? ldv<T, C>(X, (int64_t)sidx[base + rr] + (int64_t)j * a.ldx) : Xv{};
            }
        } else {
            stage_x<T, C, NR>(xr, X, f.off + R0, a.ldx, nr, a.nrhs);
        }
    };
    auto ready = [&](int i) { int R0, nr; tile_of(i, R0, nr); return i < nl || nT - R0 / kTile <= known; };
    Xv acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = Xv{};
    if (ntiles > 0) {
        fetch(0);
        __syncthreads();   // gather indices in shared memory
        if (!ready(0)) {
            int R0, nr;
            tile_of(0, R0, nr);
            const int cnt = wait_progress(&a.xprog[fi], nT - R0 / kTile, a.epoch, a.status);
            if (cnt < 0) return;
            known = cnt;
        }
        stage(0);
    }
    // sums of the helpers of this column block (issued before this CTA), in
    // chunk order; taken before the pivot tiles so that no wait on a helper
    // follows the chain's last block
    Xv hsum[NR / kQ];
#pragma unroll
    for (int b = 0; b < NR / kQ; ++b) hsum[b] = Xv{};
    auto add_helpers = [&]() -> bool {
        const T* HP = reinterpret_cast<const T*>(a.hpart);
        for (int ch = 1; ch < f.nch; ++ch) {
            const int64_t h = f.hbase + (int64_t)c * (f.nch - 1) + (ch - 1);
            if (!wait_flag(&a.hflags[h], a.epoch, a.status)) return false;
#pragma unroll
            for (int b = 0; b < NR / kQ; ++b) {
                const int j = q + kQ * b;
                if (j < a.nrhs) hsum[b] += ldv_cg<T, C>(HP, h * kPartialStride + j * kTile + r);
            }
        }
        return true;
    };
    if (!helper && nl == 0 && !add_helpers()) return;
    for (int i = 0; i < ntiles; ++i) {
        __syncthreads();   // the previous tile's readers are done with sL and sx
#pragma unroll
        for (int p = 0; p < kE; ++p) sL[(q + kQ * p) * ldl + r] = pre[p];
        put_x<NR>(xr, sx);
        const bool more = i + 1 < ntiles;
        if (more) fetch(i + 1);
        else if (!helper)   // pre is free: the block's transposed inverse, as a row slice
            row_slice<T, C>(pre, reinterpret_cast<const T*>(a.dinvT), f.dinv + (int64_t)c * kTile * kTile, kTile, r, q, kTile, kTile);
        const bool pre_x = more && ready(i + 1);
        if (pre_x) stage(i + 1);
        __syncthreads();
        Xv v[kE];
#pragma unroll
        for (int k = 0; k < kE; ++k) v[k] = sL[r * ldl + q * kE + k];
        slice_mac<CJ, NR>(acc, v, sx, q);
        if (more && !pre_x) {
            int R0, nr;
            tile_of(i + 1, R0, nr);
            const int cnt = wait_progress(&a.xprog[fi], nT - R0 / kTile, a.epoch, a.status);
            if (cnt < 0) return;
            known = cnt;
            stage(i + 1);
        }
        if (!helper && i + 1 == nl && !add_helpers()) return;
    }
    Xv out[NR / kQ];
    reduce_slices<NR>(acc, red, out, r, q);
    if (helper) {
        T* HP = reinterpret_cast<T*>(a.hpart);
        const int64_t h = f.hbase + (int64_t)c * (f.nch - 1) + (chunk - 1);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) stv<T, C>(HP, h * kPartialStride + j * kTile + r, out[b]);
        }
        publish_flag(&a.hflags[h], a.epoch);
        return;
    }
    if (ntiles == 0)
        row_slice<T, C>(pre, reinterpret_cast<const T*>(a.dinvT), f.dinv + (int64_t)c * kTile * kTile, kTile, r, q, kTile, kTile);
#pragma unroll
    for (int b = 0; b < NR / kQ; ++b) out[b] += hsum[b];
    if (a.exact) {   // substitution form: w_c = y_c - sum, the chain applies the inverse
        T* Part = reinterpret_cast<T*>(a.partial);
#pragma unroll
        for (int b = 0; b < NR / kQ; ++b) {
            const int j = q + kQ * b;
            if (j < a.nrhs) stv<T, C>(Part, (int64_t)(f.flag_base + c) * kPartialStride + j * kTile + r, yv[b] - out[b]);
        }
        publish_flag(&a.pflags[f.flag_base + c], a.epoch);
        return;
    }
    // z_c = op(L_cc^{-1})^T (y_c - sum); every reader of sx passed the
    // barrier in reduce_slices
    Xv* st = sx;
#pragma unroll
    for (int b = 0; b < NR / kQ; ++b) st[r * NR + q + kQ * b] = yv[b] - out[b];
    __syncthreads();
    Xv acc2[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc2[j] = Xv{};
    slice_mac<CJ, NR>(acc2, pre, st, q);
    Xv z[NR / kQ];
    reduce_slices<NR>(acc2, red, z, r, q);
    T* Part = reinterpret_cast<T*>(a.partial);
#pragma unroll
    for (int b = 0; b < NR / kQ; ++b) {
        const int j = q + kQ * b;
        if (j < a.nrhs) stv<T, C>(Part, (int64_t)(f.flag_base + c) * kPartialStride + j * kTile + r, z[b]);
    }
    publish_flag(&a.pflags[f.flag_base + c], a.epoch);
}

template <class T, bool C, bool CJ, int NR>
__global__ void __launch_bounds__(kSolveThreads, sweep_min_blocks<T, C, NR>()) bwd_sweep_kernel(SweepArgs a) {
    using Xv = V<T, C>;
    constexpr int ldl = kTile + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Xv* sx = reinterpret_cast<Xv*>(smem_raw);     // 3 x [64][NR]
    Xv* red = sx + 3 * kTile * NR;                // [kQ][NR][64]
    Xv* sL = red + kQ * NR * kTile;               // [64 columns][65]
    int32_t* sidx = reinterpret_cast<int32_t*>(sL + kTile * ldl);   // gather indices, kLowerChunkTiles x 64
    __shared__ int s_item, s_timed_out;
    if (threadIdx.x == 0) {
        s_item = atomicAdd(a.ticket, 1);
        s_timed_out = *reinterpret_cast<volatile int32_t*>(&a.status[1]) != 0;
    }
    __syncthreads();
    if (s_timed_out) return;   // an earlier wait gave up (one read for the whole CTA)
    const int4 it = a.items[s_item];
    const FrontDev f = a.F[it.x];
    const int r = threadIdx.x % kTile, q = threadIdx.x / kTile;
    const int nT = (f.n + kTile - 1) / kTile;
    if (it.y == kItemChain) bwd_chain<T, C, CJ, NR>(a, f, it.x, nT, r, q, sx, red, sx + 2 * kTile * NR);
    else if (it.y == kItemWhole) bwd_whole<T, C, CJ, NR>(a, f, nT, r, q, sx, red, sL, sidx);
    else bwd_worker<T, C, CJ, NR>(a, f, it.x, nT, it.y, it.z, it.w, r, q, sx, red, sL, sidx);
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
template <class T, bool C, bool CJ, int NR>
static int64_t run_sweeps(Plan& P, T* X, int nrhs) {
    using Xv = V<T, C>;
    const size_t smem_fwd = sizeof(Xv) * (4 + kQ) * kTile * NR;
    const size_t smem_bwd = sizeof(Xv) * ((3 + kQ) * kTile * NR + kTile * (kTile + 1)) + sizeof(int32_t) * kLowerChunkTiles * kTile;
    const size_t smem_tiny = sizeof(Xv) * kTinyWarps * kTile * NR;
    static bool attr_done = false;
    if (!attr_done) {
        cudaFuncSetAttribute(fwd_sweep_kernel<T, C, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fwd);
        cudaFuncSetAttribute(bwd_sweep_kernel<T, C, CJ, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bwd);
        cudaFuncSetAttribute(tiny_fwd_kernel<T, C, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tiny);
        cudaFuncSetAttribute(tiny_bwd_kernel<T, C, CJ, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tiny);
        attr_done = true;
    }
    const int4* items = reinterpret_cast<const int4*>(P.items);
    SweepArgs a{};
    a.F = P.fronts;
    a.xprog = P.xprog;
    a.pflags = P.flags;
    a.L = P.L;
    a.dinv = P.dinv;
    a.dinvT = P.dinvT;
    a.m1 = P.m1;
    a.n1 = P.n1;
    a.partial = P.partial;
    a.hpart = P.hpart;
    a.hflags = P.flags + P.flags_total;
    a.X = X;
    a.ldx = P.n;
    a.w0 = P.wpool[0];
    a.w1 = P.wpool[1];
    a.lower = P.lower;
    a.nrhs = nrhs;
    a.status = P.status;
    a.exact = P.solve_exact;
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
        if (lv.ntiny > 0) {
            tiny_fwd_kernel<T, C, NR><<<(lv.ntiny + kTinyWarps - 1) / kTinyWarps, 32 * kTinyWarps, smem_tiny, P.stream>>>(
                P.fronts, P.tiny_fronts + lv.tiny, lv.ntiny, X, P.n, w0, w1, reinterpret_cast<const T*>(P.L),
                reinterpret_cast<const T*>(P.dinv), nrhs);
            ++launches;
        }
        if (lv.nfwd > 0) {
            a.items = items + lv.fwd_items;
            a.ticket = P.tickets + 2 * d;
            a.epoch = ++P.epoch;
            fwd_sweep_kernel<T, C, NR><<<lv.nfwd, kSolveThreads, smem_fwd, P.stream>>>(a);
            ++launches;
        }
    }
    if (P.pivoted) launch_quasi_diag(P, X, P.n, nrhs);   // 1 x 1 and 2 x 2 blocks of D
    else diag_scale_kernel<T, C><<<1184, 256, 0, P.stream>>>(X, P.n, P.n, nrhs, P.D);
    ++launches;
    for (int d = 0; d <= P.max_depth; ++d) {
        const SolveLevel& lv = P.solve_levels[d];
        if (lv.ntiny > 0) {
            tiny_bwd_kernel<T, C, CJ, NR><<<(lv.ntiny + kTinyWarps - 1) / kTinyWarps, 32 * kTinyWarps, smem_tiny, P.stream>>>(
                P.fronts, P.tiny_fronts + lv.tiny, lv.ntiny, X, P.n, reinterpret_cast<const T*>(P.L),
                reinterpret_cast<const T*>(P.dinvT), P.lower, nrhs);
            ++launches;
        }
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

// Failure-detection check: one CTA waits on a flag for an epoch that is
// never published, through the same bounded wait as the sweeps, so the wait
// gives up after limit_ns and records a timeout (wait site 4).
__global__ void wait_selftest_kernel(const int32_t* __restrict__ flag, int32_t* __restrict__ status, uint64_t limit_ns) {
    wait_flag(flag, INT_MAX, status, limit_ns);
}

int launch_wait_selftest(Plan& P, uint64_t limit_ns) {
    wait_selftest_kernel<<<1, kSolveThreads, 0, P.stream>>>(P.flags, P.status, limit_ns);
    return check_cuda("wait self-test launch");
}

template <class T, bool C>
int run_solve_nodal(Plan& P, void* xn, int nrhs) {
    if (P.conjugate && C) return run_solve_impl<T, C, true>(P, reinterpret_cast<T*>(xn), nrhs);
    return run_solve_impl<T, C, false>(P, reinterpret_cast<T*>(xn), nrhs);
}

template <class T, bool C>
void launch_fwd_gather(Plan& P, const SolveLevel& lv, T* X, T* w0, T* w1, int nrhs) {
    fwd_gather_kernel<T, C><<<dim3(lv.nfronts, lv.gather_chunks), kSolveThreads, 0, P.stream>>>(
        P.fronts, P.level_fronts + lv.fronts, X, P.n, w0, w1, P.cmaps, nrhs);
}

template void launch_fwd_gather<float, false>(Plan&, const SolveLevel&, float*, float*, float*, int);
template void launch_fwd_gather<float, true>(Plan&, const SolveLevel&, float*, float*, float*, int);
template void launch_fwd_gather<double, false>(Plan&, const SolveLevel&, double*, double*, double*, int);
template void launch_fwd_gather<double, true>(Plan&, const SolveLevel&, double*, double*, double*, int);

template int run_solve_nodal<float, false>(Plan&, void*, int);
template int run_solve_nodal<float, true>(Plan&, void*, int);
template int run_solve_nodal<double, false>(Plan&, void*, int);
template int run_solve_nodal<double, true>(Plan&, void*, int);

}  // namespace cliqgpu
