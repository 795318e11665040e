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

constexpr int kBufs = 6;   // 0 arena, 1 X (nodal), 2 scratch Y, 3 scratch G, 4 / 5 solve W pools
struct Bufs {
    void* p[kBufs];
};

template <class T, bool C>
__global__ void __launch_bounds__(kThreads) bgemm_kernel(const Prob* __restrict__ probs, const int64_t* __restrict__ prefix,
                                                         const int32_t* __restrict__ bmap, Bufs bufs, const double* __restrict__ D) {
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
                    if (pr.maskB && j <= kg) bv = j == kg ? vone<X>() : X{};
                    else {
                        bv = pr.opB == 0 ? B[pr.B + kg + (int64_t)j * pr.ldb] : B[pr.B + j + (int64_t)kg * pr.ldb];
                        if (pr.opB == 2) bv = conjv(bv);
                    }
                    if (pr.dmode) {
                        const W d = reinterpret_cast<const W*>(D)[pr.dk + kg];
                        bv = pr.dmode == 1 ? conv<X>(d * conv<W>(bv)) : conv<X>(conv<W>(bv) / d);
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
    blk::bgemm_kernel<T, C><<<(unsigned)L.nblocks, blk::kThreads, 0, st>>>(j, pf, bm, b, P.D);
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
    int kind;   // 0 GEMM list, 1 copy list, 2 forward gather of one level
    int level;
    int64_t jobs, prefix, bmap, nblocks;   // byte offsets into the uploaded buffer
};

struct SolveSched {
    int nrhs = 0;
    char* mem = nullptr;
    std::vector<Rec> recs;
};

struct BlockState {
    std::vector<SolveSched> scheds;
    void* y = nullptr;   // inv(A11) operands: the level's XT (or YT), sum of n x 16
    void* g = nullptr;   // backward: the level's gathered X[lowerStruct], sum of u x 16
};

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
        List<Prob> G1, G2;
        int64_t y = 0;
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n <= 0) continue;
            const Copy c = mk_copy(f.off, y, f.n, nrhs, ldx, f.n, 1, 2);
            K.add(c, blk::copy_blocks(c));
            const Prob p1 = mk_gemm(f.L, y, f.off, f.n, nrhs, f.n, f.m, f.n, ldx, 0, 0, 0, 2, 1, false, false);
            G1.add(p1, blk::gemm_tiles(p1));
            if (f.u > 0) {
                const Prob p2 =
                    mk_gemm(f.L + f.n, f.off, f.W * nrhs, f.u, nrhs, f.n, f.m, ldx, f.u, 0, 0, 0, 1, 4 + f.pool, true, true);
                G2.add(p2, blk::gemm_tiles(p2));
            }
            y += (int64_t)f.n * nrhs;
        }
        pk.add(1, K);
        pk.add(0, G1);
        pk.add(0, G2);
    }
    for (int d = 0; d <= P.max_depth; ++d) {   // backward: YT := op(A21)^T XB, XT -= inv(A11) YT
        List<Copy> K;
        List<Prob> G1, G2;
        int64_t y = 0, g = 0;
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n <= 0 || f.u <= 0) continue;
            const Copy c = mk_copy(0, g, f.u, nrhs, ldx, f.u, 1, 3, f.lower);
            K.add(c, blk::copy_blocks(c));
            const Prob p1 = mk_gemm(f.L + f.n, g, y, f.n, nrhs, f.u, f.m, f.u, f.n, opT, 0, 0, 3, 2, false, false);
            G1.add(p1, blk::gemm_tiles(p1));
            const Prob p2 = mk_gemm(f.L, y, f.off, f.n, nrhs, f.n, f.m, f.n, ldx, 0, 0, 0, 2, 1, true, true);
            G2.add(p2, blk::gemm_tiles(p2));
            y += (int64_t)f.n * nrhs;
            g += (int64_t)f.u * nrhs;
        }
        pk.add(1, K);
        pk.add(0, G1);
        pk.add(0, G2);
    }
    S.nrhs = nrhs;
    S.recs = pk.recs;
    if (cudaMalloc((void**)&S.mem, std::max<size_t>(16, pk.bytes.size())) != cudaSuccess) return check_cuda("block solve: schedule");
    if (cudaMemcpy(S.mem, pk.bytes.data(), pk.bytes.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return check_cuda("block solve: schedule");
    return CLIQ_OK;
}

template <class T, bool C>
static int64_t run_sched(Plan& P, const SolveSched& S, BlockState& B, T* xn) {
    cudaStream_t st = P.stream;
    Bufs b{};
    b.p[0] = P.L; b.p[1] = xn; b.p[2] = B.y; b.p[3] = B.g; b.p[4] = P.wpool[0]; b.p[5] = P.wpool[1];
    int64_t launches = 0;
    for (const Rec& r : S.recs) {
        if (r.kind == 2) {
            launch_fwd_gather<T, C>(P, P.solve_levels[r.level], xn, reinterpret_cast<T*>(P.wpool[0]),
                                    reinterpret_cast<T*>(P.wpool[1]), S.nrhs);
        } else if (r.kind == 0) {
            blk::bgemm_kernel<T, C><<<(unsigned)r.nblocks, blk::kThreads, 0, st>>>(
                reinterpret_cast<const Prob*>(S.mem + r.jobs), reinterpret_cast<const int64_t*>(S.mem + r.prefix),
                reinterpret_cast<const int32_t*>(S.mem + r.bmap), b, P.D);
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
