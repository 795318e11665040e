// Block-LDL front type (BLOCK_LDL_1D / BLOCK_LDL_2D).
//
// Reference: FrontBlockLDL, include/clique/numeric/ldl/local_front_block.hpp:27-71
// (unpivoted branch): after FrontLDL the front keeps inv(A11) -- full,
// symmetric (Hermitian for LDL^H) -- in place of L11 / D, and the original
// A21 in place of L21; the solves (lower_solve/local_front_block.hpp:29-70,
// solve.hpp:48-53) are then products only, with no triangular solve and no
// diagonal solve:
//     forward   XT := inv(A11) XT,          XB -= A21 XT
//     backward  YT := op(A21)^T XB,         XT -= inv(A11) YT.
//
// Here the conversion runs after the standard factorization, for all fronts
// at once, with one batched GEMM kernel (CUDA cores, 64 x 64 tiles):
//   1. W = L11^{-1}: the 64 x 64 diagonal blocks of W are the inverse blocks
//      the factorization already formed; the rest by doubling, merging
//      adjacent groups of 2^r blocks: T = L21 W11, W21 = -W22 T.
//   2. A21 = L21 D op(L11)^T (op = conj for LDL^H), fronts in groups whose
//      results fit a bounded scratch, copied back over L21.
//   3. inv(A11) = op(W)^T D^{-1} W into the front's top n x n block.
// The block sweeps gather the children's / ancestors' entries as the
// standard ones do and run two GEMM launches per tree level.
//
// After a pivoted factorization (BLOCK_LDL_INTRAPIV_*, the intraPiv branch
// of FrontBlockLDL) the same three steps run with D's 2 x 2 blocks; the
// front then holds inv(P A11 P^T) and A21 P^T -- the reference's inv(A11)
// and A21 in the front's pivoted order, which the solves' maps already use.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "cliqgpu_internal.h"
#include "device_common.cuh"

namespace cliqgpu {
namespace blk {

constexpr int kBT = 64;          // output tile edge
constexpr int kThreads = 256;

// C = beta C + alpha op(A) diag op(B):  A M x K (op 0: A[i + k lda], 1: A[k + i lda],
// 2: conj of 1), B K x N (op 0: B[k + j ldb], 1: B[j + k ldb], 2: conj of 1),
// diag: scale k by D[dk + k] (1: times, 2: divided by), operands in the buffer
// table entries ba, bb, bc.
struct Prob {
    int64_t A, B, C, dk;
    int32_t M, N, K, lda, ldb, ldc;
    int8_t opA, opB, dmode, ba, bb, bc, beta1, neg;   // beta1: C += (else C =); neg: alpha = -1 (else 1)
    int8_t maskB;   // 1: B is op of a unit lower triangle (stored element (j, k): j > k kept, j == k one, else zero)
};

constexpr int kBufs = 7;   // 0 arena, 1 X (nodal), 2 scratch Y, 3 scratch G, 4 / 5 solve W pools, 6 partial sums
struct Bufs {
    void* p[kBufs];
};

// op(B)(k, j) of a problem, the unit-lower mask applied
template <class X>
__device__ __forceinline__ X bload(const Prob& pr, const X* B, int k, int j) {
    if (pr.maskB && j <= k) return j == k ? vone<X>() : X{};
    X v = pr.opB == 0 ? B[pr.B + k + (int64_t)j * pr.ldb] : B[pr.B + j + (int64_t)k * pr.ldb];
    return pr.opB == 2 ? conjv(v) : v;
}

// E (pivoted fronts, else null): D(k + 1, k) of each 2 x 2 block of D starting
// at k; D(k, k + 1) is E[k], conjugated when cj.  The diagonal scaling then
// mixes rows k and k +- 1 of op(B) within a block (dmode 1: D op(B), 2: D^{-1} op(B)).
template <class T, bool C>
__global__ void __launch_bounds__(kThreads) bgemm_kernel(const Prob* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                         const int32_t* __restrict__ bmap, Bufs bufs, const double* __restrict__ D,
                                                         const double* __restrict__ E, int cj) {
    using X = V<T, C>;
    using W = DV<C>;
    constexpr int BK = C ? 8 : 16;
    __shared__ X sA[BK][kBT + 1];
    __shared__ X sB[BK][kBT + 1];
    const int64_t bid = blockIdx.x;
    const int lo = bmap[bid];
    const Prob pr = probs[lo];
    const int64_t t = bid - prefix[lo];
    const int Nt = (pr.N + kBT - 1) / kBT;
    const int i0 = (int)(t / Nt) * kBT, j0 = (int)(t % Nt) * kBT;
    const X* A = reinterpret_cast<const X*>(bufs.p[pr.ba]);
    const X* B = reinterpret_cast<const X*>(bufs.p[pr.bb]);
    X* Cm = reinterpret_cast<X*>(bufs.p[pr.bc]);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    X acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = X{};
    for (int k0 = 0; k0 < pr.K; k0 += BK) {
#pragma unroll
        for (int q = 0; q < (kBT * BK) / kThreads; ++q) {
            const int idx = threadIdx.x + kThreads * q;
            const int r = idx % kBT, kk = idx / kBT;
            const int kg = k0 + kk;
            X av{}, bv{};
            if (kg < pr.K) {
                const int i = i0 + r, j = j0 + r;
                if (i < pr.M) {
                    av = pr.opA == 0 ? A[pr.A + i + (int64_t)kg * pr.lda] : A[pr.A + kg + (int64_t)i * pr.lda];
                    if (pr.opA == 2) av = conjv(av);
                }
                if (j < pr.N) {
                    bv = bload(pr, B, kg, j);
                    if (pr.dmode) {
                        const W* Dw = reinterpret_cast<const W*>(D) + pr.dk;
                        const W* Ew = E ? reinterpret_cast<const W*>(E) + pr.dk : nullptr;
                        const W d = Dw[kg];
                        const bool first = Ew && !is_zero(Ew[kg]);
                        const bool second = Ew && kg > 0 && !is_zero(Ew[kg - 1]);
                        auto oc = [&](W v) { return cj ? conjv(v) : v; };
                        if (!first && !second) {
                            bv = pr.dmode == 1 ? conv<X>(d * conv<W>(bv)) : conv<X>(conv<W>(bv) / d);
                        } else {
                            // the 2 x 2 block [[d11, op(e)], [e, d22]] holding k
                            const int k0 = first ? kg : kg - 1;
                            const W d11 = Dw[k0], d22 = Dw[k0 + 1], e = Ew[k0];
                            const W b0 = conv<W>(first ? bv : bload(pr, B, k0, j));
                            const W b1 = conv<W>(first ? bload(pr, B, k0 + 1, j) : bv);
                            W y;
                            if (pr.dmode == 1) y = first ? d11 * b0 + oc(e) * b1 : e * b0 + d22 * b1;
                            else {
                                const W det = d11 * d22 - e * oc(e);
                                y = first ? (d22 * b0 - oc(e) * b1) / det : (d11 * b1 - e * b0) / det;
                            }
                            bv = conv<X>(y);
                        }
                    }
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
    for (int a = 0; a < 4; ++a) {
        const int i = i0 + ty + 16 * a;
        if (i >= pr.M) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int j = j0 + tx + 16 * b;
            if (j >= pr.N) continue;
            const int64_t e = pr.C + i + (int64_t)j * pr.ldc;
            const X v = pr.neg ? X{} - acc[a][b] : acc[a][b];
            Cm[e] = pr.beta1 ? Cm[e] + v : v;
        }
    }
}

// ---------------------------------------------------------------------------
// skinny products of the block sweeps: C (M x N, N <= 16) (+)= (-) op(A) B.
// A (inv(A11) or A21) is streamed once from HBM; K is split over CTAs and the
// partial sums (buffer 6) are added in a fixed order by a second launch, so
// the result does not depend on scheduling.
// ---------------------------------------------------------------------------
struct SProb {
    int64_t A, B, C, part;           // part: partial sums of split s at part + s * M * N (when ks > 1)
    int32_t M, N, K, lda, ldb, ldc;
    int32_t kc, ks, rows;            // K per split, splits, rows per CTA
    int8_t opA, ba, bb, bc, beta1, neg, pad0, pad1;
};

constexpr int kSkRows = 64;        // opA 0: rows per CTA (one per thread of each k-group)
constexpr int kSkGroups = 4;       // opA 0: k-groups per CTA, reduced in shared memory at the end
constexpr int kSkK = 128;          // opA 0: rows of B staged per step (32 per k-group)
constexpr int kSkWarps = 8;        // opA 1 / 2: warps per CTA, two rows per warp
constexpr int kSkTRows = 2 * kSkWarps;
constexpr int kSkThreads = 256;

template <class X, int NR>
__device__ __forceinline__ void sk_store(const SProb& pr, X* Cm, X* part, int sp, int i, const X* acc) {
#pragma unroll
    for (int j = 0; j < NR; ++j) {
        if (j >= pr.N) break;
        if (pr.ks > 1) {
            part[pr.part + (int64_t)sp * pr.M * pr.N + i + (int64_t)j * pr.M] = acc[j];
        } else {
            const int64_t e = pr.C + i + (int64_t)j * pr.ldc;
            const X v = pr.neg ? X{} - acc[j] : acc[j];
            Cm[e] = pr.beta1 ? Cm[e] + v : v;
        }
    }
}

// opA 0: A column-major M x K.  64 rows x 4 k-groups per CTA: a warp reads
// 32 consecutive rows of one column (coalesced), each thread keeps 8 loads
// in flight, and the k-groups' sums are added in a fixed order at the end.
template <class T, bool C, int NR>
__global__ void __launch_bounds__(kSkThreads) skinny_kernel(const SProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                            const int32_t* __restrict__ bmap, Bufs bufs) {
    using X = V<T, C>;
    constexpr int U = 8;
    __shared__ X sbuf[kSkK * NR];   // staged B rows [k][j]; at the end the k-groups' sums [slot][j][row]
    const int lo = bmap[blockIdx.x];
    const SProb pr = probs[lo];
    const int64_t t = blockIdx.x - prefix[lo];
    const int rt = (int)(t / pr.ks), sp = (int)(t % pr.ks);
    const int k0 = sp * pr.kc, k1 = min(pr.K, k0 + pr.kc);
    const X* A = reinterpret_cast<const X*>(bufs.p[pr.ba]) + pr.A;
    const X* B = reinterpret_cast<const X*>(bufs.p[pr.bb]) + pr.B;
    const int r = threadIdx.x % kSkRows, g = threadIdx.x / kSkRows;
    const int i = rt * kSkRows + r;
    const bool row = i < pr.M;
    X acc[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc[j] = X{};
    for (int kb = k0; kb < k1; kb += kSkK) {
        const int kn = min(kSkK, k1 - kb);
        for (int e = threadIdx.x; e < kSkK * NR; e += kSkThreads) {
            const int kk = e % kSkK, j = e / kSkK;
            sbuf[kk * NR + j] = (kk < kn && j < pr.N) ? B[kb + kk + (int64_t)j * pr.ldb] : X{};
        }
        __syncthreads();
        if (row) {
            const X* a = A + i + (int64_t)kb * pr.lda;
#pragma unroll
            for (int h = 0; h < kSkK / kSkGroups; h += U) {
                const int kq = g * (kSkK / kSkGroups) + h;
                X av[U];
#pragma unroll
                for (int q = 0; q < U; ++q) av[q] = kq + q < kn ? a[(int64_t)(kq + q) * pr.lda] : X{};
#pragma unroll
                for (int q = 0; q < U; ++q)
#pragma unroll
                    for (int j = 0; j < NR; ++j) mac(acc[j], av[q], sbuf[(kq + q) * NR + j]);
            }
        }
        __syncthreads();
    }
    // k-groups 2, 3 -> shared; 0, 1 add them; 1 -> shared; 0 adds and stores
    X* red = sbuf;
    if (g >= 2)
#pragma unroll
        for (int j = 0; j < NR; ++j) red[((g - 2) * NR + j) * kSkRows + r] = acc[j];
    __syncthreads();
    if (g < 2)
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] += red[(g * NR + j) * kSkRows + r];
    __syncthreads();
    if (g == 1)
#pragma unroll
        for (int j = 0; j < NR; ++j) red[j * kSkRows + r] = acc[j];
    __syncthreads();
    if (g == 0 && row) {
#pragma unroll
        for (int j = 0; j < NR; ++j) acc[j] += red[j * kSkRows + r];
        sk_store<X, NR>(pr, reinterpret_cast<X*>(bufs.p[pr.bc]), reinterpret_cast<X*>(bufs.p[6]), sp, i, acc);
    }
}

// opA 1 / 2: C row i is column i of A (conjugated for 2).  Two rows per warp,
// lanes coalesced down the columns with 4-8 loads each in flight; B staged
// transposed so that lanes hit consecutive words.
template <class T, bool C, int NR, bool CJ>
__global__ void __launch_bounds__(kSkThreads) skinny_t_kernel(const SProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                              const int32_t* __restrict__ bmap, Bufs bufs) {
    using X = V<T, C>;
    constexpr int U = sizeof(X) >= 16 ? 4 : 8;
    constexpr int KT = 32 * U;
    __shared__ X sB[NR][KT + 1];
    const int lo = bmap[blockIdx.x];
    const SProb pr = probs[lo];
    const int64_t t = blockIdx.x - prefix[lo];
    const int rt = (int)(t / pr.ks), sp = (int)(t % pr.ks);
    const int k0 = sp * pr.kc, k1 = min(pr.K, k0 + pr.kc);
    const X* A = reinterpret_cast<const X*>(bufs.p[pr.ba]) + pr.A;
    const X* B = reinterpret_cast<const X*>(bufs.p[pr.bb]) + pr.B;
    const int lane = threadIdx.x % 32, w = threadIdx.x / 32;
    const int i0 = rt * kSkTRows + 2 * w;
    const bool row0 = i0 < pr.M, row1 = i0 + 1 < pr.M;
    X acc0[NR], acc1[NR];
#pragma unroll
    for (int j = 0; j < NR; ++j) acc0[j] = acc1[j] = X{};
    for (int kb = k0; kb < k1; kb += KT) {
        const int kn = min(KT, k1 - kb);
        for (int e = threadIdx.x; e < KT * NR; e += kSkThreads) {
            const int kk = e % KT, j = e / KT;
            sB[j][kk] = (kk < kn && j < pr.N) ? B[kb + kk + (int64_t)j * pr.ldb] : X{};
        }
        __syncthreads();
        if (row0) {
            const X* a0 = A + kb + (int64_t)i0 * pr.lda;
            const X* a1 = row1 ? a0 + pr.lda : a0;
            X v0[U], v1[U];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const int k = lane + 32 * q;
                v0[q] = k < kn ? opc<CJ>(a0[k]) : X{};
                v1[q] = (k < kn && row1) ? opc<CJ>(a1[k]) : X{};
            }
#pragma unroll
            for (int q = 0; q < U; ++q)
#pragma unroll
                for (int j = 0; j < NR; ++j) {
                    const X b = sB[j][lane + 32 * q];
                    mac(acc0[j], v0[q], b);
                    mac(acc1[j], v1[q], b);
                }
        }
        __syncthreads();
    }
    if (!row0) return;
#pragma unroll
    for (int j = 0; j < NR; ++j) {
#pragma unroll
        for (int o = 16; o > 0; o /= 2) {
            if constexpr (C) {
                acc0[j].r += __shfl_xor_sync(0xffffffffu, acc0[j].r, o);
                acc0[j].i += __shfl_xor_sync(0xffffffffu, acc0[j].i, o);
                acc1[j].r += __shfl_xor_sync(0xffffffffu, acc1[j].r, o);
                acc1[j].i += __shfl_xor_sync(0xffffffffu, acc1[j].i, o);
            } else {
                acc0[j] += __shfl_xor_sync(0xffffffffu, acc0[j], o);
                acc1[j] += __shfl_xor_sync(0xffffffffu, acc1[j], o);
            }
        }
    }
    X* Cm = reinterpret_cast<X*>(bufs.p[pr.bc]);
    X* part = reinterpret_cast<X*>(bufs.p[6]);
    if (lane == 0) sk_store<X, NR>(pr, Cm, part, sp, i0, acc0);
    if (lane == 1 && row1) sk_store<X, NR>(pr, Cm, part, sp, i0 + 1, acc1);
}

// C (+)= (-) sum over the splits of the partial sums, in split order
template <class T, bool C>
__global__ void skinny_reduce_kernel(const SProb* __restrict__ probs, const int64_t* __restrict__ prefix,
                                     const int32_t* __restrict__ bmap, Bufs bufs) {
    using X = V<T, C>;
    const int lo = bmap[blockIdx.x];
    const SProb pr = probs[lo];
    const int64_t e = (int64_t)(blockIdx.x - prefix[lo]) * 256 + threadIdx.x;
    const int64_t mn = (int64_t)pr.M * pr.N;
    if (e >= mn) return;
    const X* part = reinterpret_cast<const X*>(bufs.p[6]) + pr.part + e;
    X s{};
    for (int q = 0; q < pr.ks; ++q) s += part[q * mn];
    X* Cm = reinterpret_cast<X*>(bufs.p[pr.bc]);
    const int64_t c = pr.C + e % pr.M + (e / pr.M) * pr.ldc;
    const X v = pr.neg ? X{} - s : s;
    Cm[c] = pr.beta1 ? Cm[c] + v : v;
}

// dst[(rows, cols) of each job] = src, both column-major: job {src, dst, rows, cols, lds, ldd, bs, bd}
struct Copy {
    int64_t src, dst;
    int32_t rows, cols, lds, ldd;
    int8_t bs, bd, gather, pad;   // gather: src row r is lower[src_rows + r] (an ND index) of buffer bs (ld lds)
    int64_t gidx;
};

template <class T, bool C>
__global__ void copy_kernel(const Copy* __restrict__ jobs, const int64_t* __restrict__ prefix, const int32_t* __restrict__ bmap,
                            Bufs bufs, const int32_t* __restrict__ lower) {
    using X = V<T, C>;
    const int lo = bmap[blockIdx.x];
    const Copy cj = jobs[lo];
    const int64_t chunk = (int64_t)(blockIdx.x - prefix[lo]) * 4096;
    const int64_t total = (int64_t)cj.rows * cj.cols;
    const X* s = reinterpret_cast<const X*>(bufs.p[cj.bs]);
    X* d = reinterpret_cast<X*>(bufs.p[cj.bd]);
    for (int64_t e = chunk + threadIdx.x; e < min(total, chunk + 4096); e += blockDim.x) {
        const int r = (int)(e % cj.rows), c = (int)(e / cj.rows);
        const int64_t sr = cj.gather ? (int64_t)lower[cj.gidx + r] : (int64_t)r;
        d[cj.dst + r + (int64_t)c * cj.ldd] = s[cj.src + sr + (int64_t)c * cj.lds];
    }
}

// host-side launch lists: problems, per-problem first block, block -> problem
template <class J>
struct List {
    std::vector<J> jobs;
    std::vector<int64_t> prefix;
    std::vector<int32_t> bmap;
    int64_t nblocks = 0;
    void add(const J& j, int64_t blocks) {
        if (blocks <= 0) return;
        prefix.push_back(nblocks);
        for (int64_t b = 0; b < blocks; ++b) bmap.push_back((int32_t)jobs.size());
        jobs.push_back(j);
        nblocks += blocks;
    }
    bool empty() const { return jobs.empty(); }
};

static int64_t gemm_tiles(const Prob& p) { return (int64_t)((p.M + kBT - 1) / kBT) * ((p.N + kBT - 1) / kBT); }
static int64_t copy_blocks(const Copy& c) { return ((int64_t)c.rows * c.cols + 4095) / 4096; }

template <class J>
static int upload(const List<J>& L, std::vector<void*>& owned, const J** dj, const int64_t** dp, const int32_t** db) {
    const size_t bj = sizeof(J) * L.jobs.size(), bp = sizeof(int64_t) * L.prefix.size(), bb = sizeof(int32_t) * L.bmap.size();
    char* m = nullptr;
    if (cudaMalloc((void**)&m, bj + bp + bb + 64) != cudaSuccess) return check_cuda("block LDL: schedule");
    owned.push_back(m);
    const size_t ob = (bj + 7) / 8 * 8, oc = ob + (bp + 7) / 8 * 8;
    cudaMemcpy(m, L.jobs.data(), bj, cudaMemcpyHostToDevice);
    cudaMemcpy(m + ob, L.prefix.data(), bp, cudaMemcpyHostToDevice);
    cudaMemcpy(m + oc, L.bmap.data(), bb, cudaMemcpyHostToDevice);
    *dj = reinterpret_cast<const J*>(m);
    *dp = reinterpret_cast<const int64_t*>(m + ob);
    *db = reinterpret_cast<const int32_t*>(m + oc);
    return CLIQ_OK;
}

}  // namespace blk

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using blk::Bufs;
using blk::Copy;
using blk::List;
using blk::Prob;

template <class T, bool C>
static int run_gemms(Plan& P, const List<Prob>& L, const Bufs& b, std::vector<void*>& owned, cudaStream_t st) {
    if (L.empty()) return CLIQ_OK;
    const Prob* j; const int64_t* pf; const int32_t* bm;
    int rc = blk::upload(L, owned, &j, &pf, &bm);
    if (rc != CLIQ_OK) return rc;
    blk::bgemm_kernel<T, C><<<(unsigned)L.nblocks, blk::kThreads, 0, st>>>(j, pf, bm, b, P.D, P.pivoted ? P.E : nullptr,
                                                                         P.conjugate ? 1 : 0);
    P.total_launches += 1;
    P.last_launches += 1;
    return check_cuda("block LDL: gemm");
}

template <class T, bool C>
static int run_copies(Plan& P, const List<Copy>& L, const Bufs& b, std::vector<void*>& owned, cudaStream_t st) {
    if (L.empty()) return CLIQ_OK;
    const Copy* j; const int64_t* pf; const int32_t* bm;
    int rc = blk::upload(L, owned, &j, &pf, &bm);
    if (rc != CLIQ_OK) return rc;
    blk::copy_kernel<T, C><<<(unsigned)L.nblocks, 256, 0, st>>>(j, pf, bm, b, P.lower);
    P.total_launches += 1;
    P.last_launches += 1;
    return check_cuda("block LDL: copy");
}

static void free_owned(std::vector<void*>& owned) {
    for (void* m : owned) cudaFree(m);
    owned.clear();
}

static Prob mk_gemm(int64_t A, int64_t B, int64_t Cc, int M, int N, int K, int lda, int ldb, int ldc, int opA, int opB, int ba,
                 int bb, int bc, bool accumulate, bool negate, int dmode = 0, int64_t dk = 0, int maskB = 0) {
    Prob p{};
    p.A = A; p.B = B; p.C = Cc; p.dk = dk;
    p.M = M; p.N = N; p.K = K; p.lda = lda; p.ldb = ldb; p.ldc = ldc;
    p.opA = (int8_t)opA; p.opB = (int8_t)opB; p.dmode = (int8_t)dmode;
    p.ba = (int8_t)ba; p.bb = (int8_t)bb; p.bc = (int8_t)bc;
    p.beta1 = accumulate ? 1 : 0; p.neg = negate ? 1 : 0; p.maskB = (int8_t)maskB;
    return p;
}

static Copy mk_copy(int64_t src, int64_t dst, int rows, int cols, int lds, int ldd, int bs, int bd, int64_t gidx = -1) {
    Copy c{};
    c.src = src; c.dst = dst; c.rows = rows; c.cols = cols; c.lds = lds; c.ldd = ldd;
    c.bs = (int8_t)bs; c.bd = (int8_t)bd; c.gather = gidx >= 0 ? 1 : 0; c.gidx = gidx < 0 ? 0 : gidx;
    return c;
}

// Conversion of the factored fronts to the block form (see the file comment).
template <class T, bool C>
static int convert_t(Plan& P) {
    const bool cj = C && P.conjugate;
    const int opT = cj ? 2 : 1;   // op(X)^T read of a column-major X
    const int nf = P.num_fronts;
    const size_t eb = sizeof(T) * (C ? 2 : 1);
    std::vector<int64_t> sw(nf + 1, 0);
    for (int s = 0; s < nf; ++s) sw[s + 1] = sw[s] + (int64_t)P.hfronts[s].n * P.hfronts[s].n;
    std::vector<void*> owned;
    void *SW = nullptr, *ST = nullptr, *SA = nullptr;
    auto fail = [&](int rc) {
        free_owned(owned);
        if (SW) cudaFree(SW);
        if (ST) cudaFree(ST);
        if (SA) cudaFree(SA);
        return rc;
    };
    if (cudaMalloc(&SW, std::max<size_t>(1, (size_t)sw[nf] * eb)) != cudaSuccess ||
        cudaMalloc(&ST, std::max<size_t>(1, (size_t)sw[nf] * eb)) != cudaSuccess)
        return fail(check_cuda("block LDL: scratch"));
    cudaStream_t st = P.stream;
    cudaMemsetAsync(SW, 0, (size_t)sw[nf] * eb, st);
    Bufs b{};
    b.p[0] = P.L; b.p[1] = SW; b.p[2] = ST; b.p[4] = P.dinv;
    // 0. diagonal blocks of W = L11^{-1}: the factorization's inverse blocks
    {
        List<Copy> L;
        for (int s = 0; s < nf; ++s) {
            const FrontDev& f = P.hfronts[s];
            for (int k = 0; k < f.n; k += kTile) {
                const int kb = std::min(kTile, f.n - k);
                const Copy c = mk_copy(f.dinv + (int64_t)(k / kTile) * kTile * kTile, sw[s] + k + (int64_t)k * f.n, kb, kb, kTile, f.n, 4, 1);
                L.add(c, blk::copy_blocks(c));
            }
        }
        int rc = run_copies<T, C>(P, L, b, owned, st);
        if (rc != CLIQ_OK) return fail(rc);
    }
    // 1. W by doubling: T = L(a1:a2, a0:a1) W(a0:a1, a0:a1); W(a1:a2, a0:a1) = -W(a1:a2, a1:a2) T
    int maxT = 0;
    for (int s = 0; s < nf; ++s) maxT = std::max(maxT, (P.hfronts[s].n + kTile - 1) / kTile);
    for (int g = 1; g < maxT; g *= 2) {
        List<Prob> L1, L2;
        for (int s = 0; s < nf; ++s) {
            const FrontDev& f = P.hfronts[s];
            const int nT = (f.n + kTile - 1) / kTile;
            for (int a0b = 0; a0b + g < nT; a0b += 2 * g) {
                const int a0 = a0b * kTile, a1 = std::min(f.n, (a0b + g) * kTile), a2 = std::min(f.n, (a0b + 2 * g) * kTile);
                const Prob p1 = mk_gemm(f.L + a1 + (int64_t)a0 * f.m, sw[s] + a0 + (int64_t)a0 * f.n, sw[s] + a1 + (int64_t)a0 * f.n,
                                     a2 - a1, a1 - a0, a1 - a0, f.m, f.n, f.n, 0, 0, 0, 1, 2, false, false);
                const Prob p2 = mk_gemm(sw[s] + a1 + (int64_t)a1 * f.n, sw[s] + a1 + (int64_t)a0 * f.n, sw[s] + a1 + (int64_t)a0 * f.n,
                                     a2 - a1, a1 - a0, a2 - a1, f.n, f.n, f.n, 0, 0, 1, 2, 1, false, true);
                L1.add(p1, blk::gemm_tiles(p1));
                L2.add(p2, blk::gemm_tiles(p2));
            }
        }
        int rc = run_gemms<T, C>(P, L1, b, owned, st);
        if (rc == CLIQ_OK) rc = run_gemms<T, C>(P, L2, b, owned, st);
        if (rc != CLIQ_OK) return fail(rc);
    }
    // 2. A21 = L21 D op(L11)^T, in groups of fronts whose results fit the scratch, copied back over L21
    {
        int64_t cap = 1 << 26;
        for (int s = 0; s < nf; ++s) cap = std::max(cap, (int64_t)P.hfronts[s].u * P.hfronts[s].n);
        if (cudaMalloc(&SA, (size_t)cap * eb) != cudaSuccess) return fail(check_cuda("block LDL: scratch"));
        b.p[3] = SA;
        int s0 = 0;
        while (s0 < nf) {
            List<Prob> G;
            List<Copy> K;
            int64_t used = 0;
            int s = s0;
            for (; s < nf; ++s) {
                const FrontDev& f = P.hfronts[s];
                const int64_t need = (int64_t)f.u * f.n;
                if (used + need > cap && s > s0) break;
                if (need > 0) {
                    const Prob p = mk_gemm(f.L + f.n, f.L, used, f.u, f.n, f.n, f.m, f.m, f.u, 0, opT, 0, 0, 3, false, false, 1, f.off, 1);
                    G.add(p, blk::gemm_tiles(p));
                    const Copy c = mk_copy(used, f.L + f.n, f.u, f.n, f.u, f.m, 3, 0);
                    K.add(c, blk::copy_blocks(c));
                    used += need;
                }
            }
            int rc = run_gemms<T, C>(P, G, b, owned, st);
            if (rc == CLIQ_OK) rc = run_copies<T, C>(P, K, b, owned, st);
            if (rc != CLIQ_OK) return fail(rc);
            s0 = s;
        }
    }
    // 3. inv(A11) = op(W)^T D^{-1} W over the top n x n block of every front
    {
        List<Prob> L;
        for (int s = 0; s < nf; ++s) {
            const FrontDev& f = P.hfronts[s];
            const Prob p = mk_gemm(sw[s], sw[s], f.L, f.n, f.n, f.n, f.n, f.n, f.m, opT, 0, 1, 1, 0, false, false, 2, f.off);
            L.add(p, blk::gemm_tiles(p));
        }
        int rc = run_gemms<T, C>(P, L, b, owned, st);
        if (rc != CLIQ_OK) return fail(rc);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(check_cuda("block LDL: convert"));
    return fail(CLIQ_OK);
}

// ---------------------------------------------------------------------------
// block sweeps: the launch records for one right-hand-side count are built on
// the first solve with that count and kept, so later solves launch without
// host work or synchronization (and can be captured into a graph)
// ---------------------------------------------------------------------------
struct Rec {
    int kind;   // 0 GEMM list, 1 copy list, 2 forward gather of one level, 3 / 4 / 5 skinny products
                // with op(A) = A / A^T / A^H, 6 reduction of split products
    int level;
    int64_t jobs, prefix, bmap, nblocks;   // byte offsets into the uploaded buffer
};

struct SolveSched {
    int nrhs = 0;
    char* mem = nullptr;
    int64_t part_elems = 0;   // partial sums the split products need at once
    std::vector<Rec> recs;
};

struct BlockState {
    std::vector<SolveSched> scheds;
    void* y = nullptr;      // inv(A11) operands: the level's XT (or YT), sum of n x 16
    void* g = nullptr;      // backward: the level's gathered X[lowerStruct], sum of u x 16
    void* part = nullptr;   // split products' partial sums
    int64_t part_elems = 0;
};

using blk::SProb;

// one skinny product (its K split is chosen per launch list)
static SProb mk_sprob(int64_t A, int64_t B, int64_t Cc, int M, int N, int K, int lda, int ldb, int ldc, int opA, int ba, int bb,
                      int bc, bool accumulate, bool negate) {
    SProb p{};
    p.A = A; p.B = B; p.C = Cc; p.part = -1;
    p.M = M; p.N = N; p.K = K; p.lda = lda; p.ldb = ldb; p.ldc = ldc;
    p.opA = (int8_t)opA; p.ba = (int8_t)ba; p.bb = (int8_t)bb; p.bc = (int8_t)bc;
    p.beta1 = accumulate ? 1 : 0; p.neg = negate ? 1 : 0;
    p.rows = opA == 0 ? blk::kSkRows : blk::kSkTRows;
    p.kc = std::max(1, K);
    p.ks = 1;
    return p;
}

struct Packer {
    std::vector<char> bytes;
    std::vector<Rec> recs;
    template <class V>
    int64_t put(const std::vector<V>& v) {
        const int64_t o = (int64_t)bytes.size();
        bytes.resize(o + (sizeof(V) * v.size() + 15) / 16 * 16);
        if (!v.empty()) std::memcpy(bytes.data() + o, v.data(), sizeof(V) * v.size());
        return o;
    }
    int64_t part_max = 0;
    // a list of skinny products of one kind (opA 0, 1 or 2) and, for the split
    // ones, the reduction of their partial sums
    void add_skinny(std::vector<SProb> v) {
        if (v.empty()) return;
        List<SProb> L, R;
        int64_t part = 0;
        // split K until the list has about 16 CTAs per SM, a split keeping at
        // least 256 (opA 0) or 512 (opA 1 / 2) columns of K and at most 32 splits
        int64_t base = 0;
        for (const SProb& p : v) base += (p.M + p.rows - 1) / p.rows;
        const int64_t f = std::max<int64_t>(1, (16 * 148 + std::max<int64_t>(base, 1) - 1) / std::max<int64_t>(base, 1));
        for (SProb& p : v) {
            if (p.M <= 0 || p.N <= 0 || p.K <= 0) continue;
            const int kmin = p.opA == 0 ? 256 : 512;
            const int ks = (int)std::max<int64_t>(1, std::min<int64_t>({f, (int64_t)(p.K / kmin), 32}));
            p.kc = ((p.K + ks - 1) / ks + 31) / 32 * 32;
            p.ks = (p.K + p.kc - 1) / p.kc;
            if (p.ks > 1) {
                p.part = part;
                part += (int64_t)p.ks * p.M * p.N;
                R.add(p, ((int64_t)p.M * p.N + 255) / 256);
            }
            L.add(p, (int64_t)((p.M + p.rows - 1) / p.rows) * p.ks);
        }
        part_max = std::max(part_max, part);
        add(v[0].opA == 0 ? 3 : (v[0].opA == 1 ? 4 : 5), L);
        add(6, R);
    }
    template <class J>
    void add(int kind, const List<J>& L) {
        if (L.empty()) return;
        Rec r{kind, -1, 0, 0, 0, L.nblocks};
        r.jobs = put(L.jobs);
        r.prefix = put(L.prefix);
        r.bmap = put(L.bmap);
        recs.push_back(r);
    }
};

static int build_sched(Plan& P, int nrhs, SolveSched& S) {
    const bool cj = P.cplx() && P.conjugate;
    const int opT = cj ? 2 : 1;
    const int ldx = (int)P.n;
    Packer pk;
    for (int d = P.max_depth; d >= 0; --d) {   // forward: XT := inv(A11) XT, XB -= A21 XT
        if (P.solve_levels[d].nfronts == 0) continue;
        pk.recs.push_back(Rec{2, d, 0, 0, 0, 0});
        List<Copy> K;
        std::vector<SProb> G1, G2;
        int64_t y = 0;
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n <= 0) continue;
            const Copy c = mk_copy(f.off, y, f.n, nrhs, ldx, f.n, 1, 2);
            K.add(c, blk::copy_blocks(c));
            G1.push_back(mk_sprob(f.L, y, f.off, f.n, nrhs, f.n, f.m, f.n, ldx, 0, 0, 2, 1, false, false));
            if (f.u > 0)
                G2.push_back(mk_sprob(f.L + f.n, f.off, f.W * nrhs, f.u, nrhs, f.n, f.m, ldx, f.u, 0, 0, 1, 4 + f.pool, true, true));
            y += (int64_t)f.n * nrhs;
        }
        pk.add(1, K);
        pk.add_skinny(G1);
        pk.add_skinny(G2);
    }
    for (int d = 0; d <= P.max_depth; ++d) {   // backward: YT := op(A21)^T XB, XT -= inv(A11) YT
        List<Copy> K;
        std::vector<SProb> G1, G2;
        int64_t y = 0, g = 0;
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n <= 0 || f.u <= 0) continue;
            const Copy c = mk_copy(0, g, f.u, nrhs, ldx, f.u, 1, 3, f.lower);
            K.add(c, blk::copy_blocks(c));
            G1.push_back(mk_sprob(f.L + f.n, g, y, f.n, nrhs, f.u, f.m, f.u, f.n, opT, 0, 3, 2, false, false));
            G2.push_back(mk_sprob(f.L, y, f.off, f.n, nrhs, f.n, f.m, f.n, ldx, 0, 0, 2, 1, true, true));
            y += (int64_t)f.n * nrhs;
            g += (int64_t)f.u * nrhs;
        }
        pk.add(1, K);
        pk.add_skinny(G1);
        pk.add_skinny(G2);
    }
    S.nrhs = nrhs;
    S.recs = pk.recs;
    S.part_elems = pk.part_max;
    if (cudaMalloc((void**)&S.mem, std::max<size_t>(16, pk.bytes.size())) != cudaSuccess) return check_cuda("block solve: schedule");
    if (cudaMemcpy(S.mem, pk.bytes.data(), pk.bytes.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return check_cuda("block solve: schedule");
    return CLIQ_OK;
}

template <class T, bool C, int NR>
static void launch_skinny(const Rec& r, const char* mem, const Bufs& b, cudaStream_t st) {
    const SProb* j = reinterpret_cast<const SProb*>(mem + r.jobs);
    const int64_t* pf = reinterpret_cast<const int64_t*>(mem + r.prefix);
    const int32_t* bm = reinterpret_cast<const int32_t*>(mem + r.bmap);
    const unsigned g = (unsigned)r.nblocks;
    if (r.kind == 3) blk::skinny_kernel<T, C, NR><<<g, blk::kSkThreads, 0, st>>>(j, pf, bm, b);
    else if (r.kind == 4) blk::skinny_t_kernel<T, C, NR, false><<<g, blk::kSkThreads, 0, st>>>(j, pf, bm, b);
    else if constexpr (C) blk::skinny_t_kernel<T, C, NR, true><<<g, blk::kSkThreads, 0, st>>>(j, pf, bm, b);
}

template <class T, bool C>
static int64_t run_sched(Plan& P, const SolveSched& S, BlockState& B, T* xn) {
    cudaStream_t st = P.stream;
    Bufs b{};
    b.p[0] = P.L; b.p[1] = xn; b.p[2] = B.y; b.p[3] = B.g; b.p[4] = P.wpool[0]; b.p[5] = P.wpool[1]; b.p[6] = B.part;
    int64_t launches = 0;
    for (const Rec& r : S.recs) {
        if (r.kind >= 3 && r.kind <= 5) {
            if (S.nrhs <= 4) launch_skinny<T, C, 4>(r, S.mem, b, st);
            else if (S.nrhs <= 8) launch_skinny<T, C, 8>(r, S.mem, b, st);
            else launch_skinny<T, C, 16>(r, S.mem, b, st);
        } else if (r.kind == 6) {
            blk::skinny_reduce_kernel<T, C><<<(unsigned)r.nblocks, 256, 0, st>>>(
                reinterpret_cast<const SProb*>(S.mem + r.jobs), reinterpret_cast<const int64_t*>(S.mem + r.prefix),
                reinterpret_cast<const int32_t*>(S.mem + r.bmap), b);
        } else if (r.kind == 2) {
            launch_fwd_gather<T, C>(P, P.solve_levels[r.level], xn, reinterpret_cast<T*>(P.wpool[0]),
                                    reinterpret_cast<T*>(P.wpool[1]), S.nrhs);
        } else if (r.kind == 0) {
            blk::bgemm_kernel<T, C><<<(unsigned)r.nblocks, blk::kThreads, 0, st>>>(
                reinterpret_cast<const Prob*>(S.mem + r.jobs), reinterpret_cast<const int64_t*>(S.mem + r.prefix),
                reinterpret_cast<const int32_t*>(S.mem + r.bmap), b, P.D, nullptr, 0);
        } else {
            blk::copy_kernel<T, C><<<(unsigned)r.nblocks, 256, 0, st>>>(
                reinterpret_cast<const Copy*>(S.mem + r.jobs), reinterpret_cast<const int64_t*>(S.mem + r.prefix),
                reinterpret_cast<const int32_t*>(S.mem + r.bmap), b, P.lower);
        }
        ++launches;
    }
    return launches;
}

template <class T, bool C>
static int block_solve_t(Plan& P, T* xn, int nrhs_total) {
    BlockState& B = *reinterpret_cast<BlockState*>(P.block_state);
    if (!B.y) {
        // scratch: the largest level's sum of n (and of u) times 16 columns
        int64_t ny = 1, ng = 1;
        for (int d = 0; d <= P.max_depth; ++d) {
            int64_t a = 0, c = 0;
            for (int s : P.level_list[d]) { a += P.hfronts[s].n; c += P.hfronts[s].u; }
            ny = std::max(ny, a);
            ng = std::max(ng, c);
        }
        const size_t eb = sizeof(T) * (C ? 2 : 1);
        if (cudaMalloc(&B.y, (size_t)ny * kSolveRhsChunk * eb) != cudaSuccess ||
            cudaMalloc(&B.g, (size_t)ng * kSolveRhsChunk * eb) != cudaSuccess)
            return check_cuda("block solve: scratch");
        P.device_bytes += (int64_t)(ny + ng) * kSolveRhsChunk * eb;
    }
    int64_t launches = 0;
    for (int j0 = 0; j0 < nrhs_total; j0 += kSolveRhsChunk) {
        const int nrhs = std::min(kSolveRhsChunk, nrhs_total - j0);
        SolveSched* S = nullptr;
        for (SolveSched& q : B.scheds)
            if (q.nrhs == nrhs) S = &q;
        if (!S) {
            B.scheds.emplace_back();
            S = &B.scheds.back();
            const int rc = build_sched(P, nrhs, *S);
            if (rc != CLIQ_OK) return rc;
            if (S->part_elems > B.part_elems) {   // grow the partial-sum buffer (no launch of this plan uses it now)
                if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("block solve");
                if (B.part) cudaFree(B.part);
                B.part = nullptr;
                if (cudaMalloc(&B.part, (size_t)S->part_elems * sizeof(T) * (C ? 2 : 1)) != cudaSuccess)
                    return check_cuda("block solve: partial sums");
                P.device_bytes += (S->part_elems - B.part_elems) * (int64_t)sizeof(T) * (C ? 2 : 1);
                B.part_elems = S->part_elems;
            }
        }
        launches += run_sched<T, C>(P, *S, B, xn + (C ? 2 : 1) * (int64_t)j0 * P.n);
    }
    P.last_launches += launches;
    P.total_launches += launches;
    return check_cuda("block solve launch");
}

int run_block_solve(Plan& P, void* xn, int nrhs) {
    if (!P.block_state) return CLIQ_ERR_STATE;
    if (P.precision == CLIQ_FP64)
        return P.cplx() ? block_solve_t<double, true>(P, (double*)xn, nrhs) : block_solve_t<double, false>(P, (double*)xn, nrhs);
    return P.cplx() ? block_solve_t<float, true>(P, (float*)xn, nrhs) : block_solve_t<float, false>(P, (float*)xn, nrhs);
}

void free_block_state(Plan& P) {
    BlockState* B = reinterpret_cast<BlockState*>(P.block_state);
    if (!B) return;
    for (SolveSched& q : B->scheds)
        if (q.mem) cudaFree(q.mem);
    if (B->y) cudaFree(B->y);
    if (B->g) cudaFree(B->g);
    if (B->part) cudaFree(B->part);
    delete B;
    P.block_state = nullptr;
}

int convert_to_block(Plan& P) {
    int rc;
    if (P.precision == CLIQ_FP64) rc = P.cplx() ? convert_t<double, true>(P) : convert_t<double, false>(P);
    else rc = P.cplx() ? convert_t<float, true>(P) : convert_t<float, false>(P);
    if (rc != CLIQ_OK) return rc;
    if (!P.block_state) P.block_state = new BlockState();
    return CLIQ_OK;
}

}  // namespace cliqgpu
