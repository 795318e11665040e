// Plan construction (front layout, level schedule, work lists, assembly map)
// and the numeric entry points of the C ABI.
//
// Memory layout in HBM (one allocation per buffer, sized once per plan):
//   factor arena  all frontL blocks, column-major m x n, ld m, 128-byte aligned,
//                 in the storage precision (FP64 plain, FP32 mixed).
//   D             pivots in FP64 (complex interleaved), ND order, length n.
//   update pools  two stacks indexed by depth parity: the updates of depth d
//                 live in pool[d % 2] and are consumed by depth d-1, which
//                 writes pool[(d-1) % 2]; the reference frees each child
//                 update right after its extend-add (ldl/local.hpp:80,102).
//   tinv          one nb x nb inverse diagonal block per front of a step.
//   work lists    int4 items, GEMM problems and tile prefix sums for every
//                 launch of the schedule, built here once.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <complex>
#include <cstring>
#include <mutex>
#include <string>

#include "cliqgpu_internal.h"


namespace cliqgpu {

static std::mutex g_err_mu;
static std::string g_last_error;

void set_last_error(const std::string& msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_error = msg;
}

int check_cuda(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string(where) + ": " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? CLIQ_ERR_OOM : CLIQ_ERR_CUDA;
    }
    return CLIQ_OK;
}

static int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

template <class T>
static int dev_upload(Plan& P, T** dst, const std::vector<T>& src) {
    const size_t bytes = sizeof(T) * std::max<size_t>(src.size(), 1);
    if (cudaMalloc((void**)dst, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("cudaMalloc failed for " + std::to_string(bytes) + " bytes");
        return CLIQ_ERR_OOM;
    }
    P.device_bytes += bytes;
    if (!src.empty() && cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return check_cuda("upload");
    return CLIQ_OK;
}

static int dev_alloc(Plan& P, void** dst, size_t bytes) {
    bytes = std::max<size_t>(bytes, 256);
    if (cudaMalloc(dst, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_last_error("cudaMalloc failed for " + std::to_string(bytes) + " bytes");
        *dst = nullptr;
        return CLIQ_ERR_OOM;
    }
    P.device_bytes += bytes;
    return CLIQ_OK;
}

void free_plan(Plan& P) {
    void* ptrs[] = {P.L, P.D, P.pool[0], P.pool[1], P.tinv, P.dinv, P.dinvT, P.m1, P.n1, P.chain_items, P.xprog, P.hpart, P.partial, P.eblk, P.erow, P.fronts, P.cmaps, P.lower, P.items, P.probs, P.packjobs, P.pack,
                    P.prefix, P.bmap, P.dest, P.asm_src, P.asm_dst,
                    P.perm, P.level_fronts, P.tiny_fronts, P.flags, P.tickets, P.status, P.rowptr, P.colind, P.aval, P.wpool[0], P.pack2,
                    P.wpool[1], P.xnodal, P.xwork, P.norms, P.krylov, P.pack3, P.E, P.pivg, P.qpos, P.perm_piv,
                    P.cmaps_orig, P.lower_orig, P.pstate, P.pvec, P.pivot_items};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (cudaEvent_t e : P.events) cudaEventDestroy(e);
    P.events.clear();
    for (cudaEvent_t e : P.sync_events) cudaEventDestroy(e);
    P.sync_events.clear();
    if (P.factor_exec) cudaGraphExecDestroy(P.factor_exec);
    if (P.batch_exec) cudaGraphExecDestroy(P.batch_exec);
    if (P.seg) cudaFree(P.seg);
    if (P.segnorm) cudaFree(P.segnorm);
    if (P.hsegnorm) cudaFreeHost(P.hsegnorm);
    if (P.stream1) cudaStreamDestroy(P.stream1);
    if (P.stream2) cudaStreamDestroy(P.stream2);
    if (P.stream3) cudaStreamDestroy(P.stream3);
    if (P.own_stream && P.stream) cudaStreamDestroy(P.stream);
    free_block_state(P);
}

#define TRY(x)                      \
    do {                            \
        int _st = (x);              \
        if (_st != CLIQ_OK) return _st; \
    } while (0)

// ---------------------------------------------------------------------------
int build_plan(Plan& P, const cliq_symm_info* info, int64_t n, const int32_t* map, const int64_t* rowptr,
                      const int32_t* colind) {
    const int nn = info->num_nodes;
    if (nn <= 0 || !info->size || !info->off || !info->parent || !info->children || !info->lower_ptr ||
        (!info->lower && info->lower_ptr[nn] > 0)) {
        set_last_error("plan_create: incomplete symbolic info");
        return CLIQ_ERR_ARG;
    }
    P.n = n;
    P.nnz = rowptr[n];
    P.num_fronts = nn;
    const int nb = P.nb;
    // ---- depths (post-order: parents have larger indices) ----
    P.depth.assign(nn, 0);
    int64_t total_size = 0;
    for (int s = nn - 1; s >= 0; --s) {
        const int par = info->parent[s];
        if (par >= 0 && par < nn && par > s) P.depth[s] = P.depth[par] + 1;
        else if (par >= 0 && par < nn) { set_last_error("plan_create: parent index not after child"); return CLIQ_ERR_ARG; }
        total_size += info->size[s];
        if (info->size[s] < 0) return CLIQ_ERR_ARG;
    }
    if (total_size != n) { set_last_error("plan_create: front sizes do not sum to n"); return CLIQ_ERR_ARG; }
    P.max_depth = *std::max_element(P.depth.begin(), P.depth.end());
    P.level_list.assign(P.max_depth + 1, {});
    for (int s = 0; s < nn; ++s) P.level_list[P.depth[s]].push_back(s);

    // ---- front layout ----
    P.hfronts.assign(nn, FrontDev{});
    const int64_t align_elems = std::max<int64_t>(1, 128 / P.elem_bytes());
    int64_t arena = 0;
    std::vector<int64_t> level_pool(P.max_depth + 1, 0), level_w(P.max_depth + 1, 0);
    P.factor_flops = P.solve_flops = P.factor_entries = 0;
    P.dinv_elems = 0;
    P.chain_elems = 0;
    P.eblk_total = P.erow_total = 0;
    for (int s = 0; s < nn; ++s) {
        FrontDev& f = P.hfronts[s];
        const int64_t nlow = info->lower_ptr[s + 1] - info->lower_ptr[s];
        f.n = info->size[s];
        f.m = (int32_t)(f.n + nlow);
        f.u = (int32_t)nlow;
        f.off = info->off[s];
        f.L = arena;
        arena = align_up(arena + (int64_t)f.m * f.n, align_elems);
        const int d = P.depth[s];
        f.pool = d & 1;
        f.U = level_pool[d];
        level_pool[d] = align_up(level_pool[d] + (int64_t)f.u * f.u, align_elems);
        f.W = level_w[d];
        level_w[d] += f.u;
        f.lower = info->lower_ptr[s];
        f.dinv = P.dinv_elems;
        P.dinv_elems += (int64_t)((f.n + kTile - 1) / kTile) * kTile * kTile;
        f.eblk = P.eblk_total;
        P.eblk_total += (int64_t)f.m * ((f.n + kTile - 1) / kTile);
        f.erow = P.erow_total;
        P.erow_total += f.m;
        f.cmap = -1;
        f.chain = -1;
        f.CU[0] = f.CU[1] = -1;
        f.CW[0] = f.CW[1] = 0;
        f.cu[0] = f.cu[1] = 0;
        const double m = f.m, nd = f.n;
        P.factor_flops += nd * nd * nd / 3.0 + (m - nd) * nd * nd + (m - nd) * (m - nd) * nd;
        P.solve_flops += nd * nd + 2.0 * (m - nd) * nd;
        P.factor_entries += m * nd;
    }
    if (P.cplx()) { P.factor_flops *= 4; P.solve_flops *= 4; }
    P.arena_elems = std::max<int64_t>(arena, 1);
    P.pool_elems[0] = P.pool_elems[1] = 1;
    P.wpool_elems[0] = P.wpool_elems[1] = 1;
    for (int d = 0; d <= P.max_depth; ++d) {
        P.pool_elems[d & 1] = std::max(P.pool_elems[d & 1], level_pool[d]);
        P.wpool_elems[d & 1] = std::max(P.wpool_elems[d & 1], level_w[d]);
    }

    // ---- children maps (inverse relative indices) ----
    std::vector<int32_t> cmaps;
    static const int32_t kNoLower = 0;
    const int32_t* low = info->lower ? info->lower : &kNoLower;
    for (int s = 0; s < nn; ++s) {
        const int l = info->children[2 * s], r = info->children[2 * s + 1];
        if (l < 0 && r < 0) continue;
        if (l < 0 || r < 0 || l >= s || r >= s) { set_last_error("plan_create: bad children"); return CLIQ_ERR_ARG; }
        FrontDev& f = P.hfronts[s];
        f.cmap = (int64_t)cmaps.size();
        cmaps.resize(cmaps.size() + 2 * (size_t)f.m, -1);
        const int32_t* plow = low + info->lower_ptr[s];
        const int64_t pnl = info->lower_ptr[s + 1] - info->lower_ptr[s];
        for (int c = 0; c < 2; ++c) {
            const int ch = c == 0 ? l : r;
            const FrontDev& cf = P.hfronts[ch];
            f.CU[c] = cf.U;
            f.CW[c] = cf.W;
            f.cu[c] = cf.u;
            const int32_t* clow = low + info->lower_ptr[ch];
            for (int ci = 0; ci < cf.u; ++ci) {
                const int g = clow[ci];
                int rel;
                if (g >= f.off && g < f.off + f.n) rel = g - f.off;
                else {
                    const int32_t* it = std::lower_bound(plow, plow + pnl, g);
                    if (it == plow + pnl || *it != g) { set_last_error("plan_create: child structure not contained in parent"); return CLIQ_ERR_ARG; }
                    rel = f.n + (int)(it - plow);
                }
                cmaps[f.cmap + (int64_t)c * f.m + rel] = ci;
            }
        }
    }

    // ---- factor schedule ----
    std::vector<int32_t> items;   // int4 quads
    std::vector<GemmProb> probs;
    std::vector<int64_t> prefix;
    std::vector<int32_t> bmap;   // block -> job / problem, per launch
    auto push_item = [&](int a, int b, int c, int d) { items.push_back(a); items.push_back(b); items.push_back(c); items.push_back(d); };
    P.launches.clear();
    int64_t max_slots = 1;
    // update tiles over the lower trapezoid i >= j: 64 x 64 on the CUDA cores,
    // kTcBM x kTcBN (row tile ti needed when ti >= (kTcBN / kTcBM) tj) on the
    // tensor cores
    const bool tcp = P.tensor_path();
    auto tiles_of = [](bool tc, int M, int N) -> int64_t {
        if (tc) {
            const int64_t R = kTcBN / kTcBM;
            const int64_t Mt = (M + kTcBM - 1) / kTcBM, Nt = (N + kTcBN - 1) / kTcBN;
            return Nt * Mt - R * Nt * (Nt - 1) / 2;
        }
        const int64_t Mt = (M + kTile - 1) / kTile, Nt = (N + kTile - 1) / kTile;
        return Nt * Mt - Nt * (Nt - 1) / 2;
    };
    std::vector<PackJob> packjobs;
    const int planes = P.cplx() ? 4 : 2;
    const int64_t blkA = (int64_t)planes * kTcBM * 8, blkB = (int64_t)planes * kTcBN * 8;   // floats per packed block
    int64_t pack_max = 1;
    int nbulk = 0;   // lookahead launches (both kinds)
    int nschur_chunks = 0;
    const bool chunked = tcp && P.lookahead && P.schur_chunk > 0;
    const int schur_chunk = std::max(kTile, P.schur_chunk / kTile * kTile);
    // in-panel updates on the tensor path with the 2xFP16 split: the panel
    // writes their packed operands itself
    const bool prepack = tcp && P.split_f16 && P.inpanel_tc;
    auto add_gemm = [&](std::vector<GemmProb>& lst, int depth, int schur, bool inpanel) {
        if (lst.empty()) return;
        Launch ln{};
        ln.kind = Launch::GEMM;
        ln.schur = schur;
        const bool tc = tcp && !(inpanel && !P.inpanel_tc);
        ln.simt = tcp && !tc;
        for (auto& pr : lst) {
            const double M = pr.M, N = pr.N;
            ln.work += (N * M - N * (N - 1) / 2) * pr.K * (P.cplx() ? 8.0 : 2.0);
        }
        ln.items = (int64_t)probs.size();
        ln.nitems = (int32_t)lst.size();
        if (tc) {
            // pack jobs: A (128-row tiles) and S = d op(B) (256-row tiles) of every problem
            int64_t off = 0, blocks = 0;
            ln.pack_items = (int64_t)packjobs.size();
            ln.pack_prefix = (int64_t)prefix.size();
            // 3xTF32: one pack CTA per (row tile, 8-wide k step); 2xFP16: one
            // pack CTA per row tile (16-wide k steps, same bytes per block),
            // followed by the tile's inverse row scales
            const bool f16 = P.split_f16 != 0;
            const int kstep = f16 ? 16 : 8;
            for (auto& pr : lst) {
                const int64_t nk = (pr.K + kstep - 1) / kstep;
                const int64_t tA = (pr.M + kTcBM - 1) / kTcBM, tB = (pr.N + kTcBN - 1) / kTcBN;
                const FrontDev& fr = P.hfronts[pr.front];
                const int nT = (fr.n + kTile - 1) / kTile;
                PackJob a{pr.A, off, -1, pr.M, pr.K, pr.lda, kTcBM, 0, 0, nT, pr.nkb, 0, 0, 0, -1, 0};
                a.emax = pr.nkb > 0 ? fr.eblk + (int64_t)pr.row0 * nT + pr.kb0 : fr.erow + pr.row0;
                pr.packA = off;
                off += tA * nk * blkA;
                a.dst_scale = pr.scaleA = off;
                if (f16) off += tA * kTcBM;
                PackJob b = a;
                b.src = pr.B;
                b.dst = off;
                b.d = pr.d;
                b.R = pr.N;
                b.tile_rows = kTcBN;
                b.emax += pr.nkb > 0 ? P.eblk_total : P.erow_total;   // the D op(L) half
                pr.packB = off;
                off += tB * nk * blkB;
                b.dst_scale = pr.scaleB = off;
                if (f16) off += tB * kTcBN;
                if (inpanel && prepack) {
                    // written by the panel kernel at the same offsets
                } else if (f16 && pr.B == pr.A && pr.N <= pr.M && kTcBN == kTcBM) {
                    // one job: the B rows are the first N rows of A, read once
                    a.dS = pr.d;
                    a.dstS = b.dst;
                    a.dst_scaleS = b.dst_scale;
                    a.emaxS = b.emax;
                    a.RS = pr.N;
                    prefix.push_back(blocks);
                    blocks += (int64_t)((a.R + a.tile_rows - 1) / a.tile_rows) * nk;
                    packjobs.push_back(a);
                } else {
                    for (const PackJob& j : {a, b}) {
                        prefix.push_back(blocks);
                        blocks += (int64_t)((j.R + j.tile_rows - 1) / j.tile_rows) * nk;
                        packjobs.push_back(j);
                    }
                }
            }
            ln.pack_njobs = (int32_t)(packjobs.size() - ln.pack_items);
            ln.pack_blocks = blocks;
            ln.pack_map = (int64_t)bmap.size();
            for (int32_t j = 0; j < ln.pack_njobs; ++j) {
                const int64_t b0 = prefix[ln.pack_prefix + j];
                const int64_t b1 = j + 1 < ln.pack_njobs ? prefix[ln.pack_prefix + j + 1] : blocks;
                for (int64_t b = b0; b < b1; ++b) bmap.push_back(j);
            }
            ln.prepacked = inpanel && prepack ? 1 : 0;
            pack_max = std::max(pack_max, off);
        }
        ln.prefix = (int64_t)prefix.size();
        ln.gemm_map = (int64_t)bmap.size();
        int64_t tot = 0;
        for (size_t q = 0; q < lst.size(); ++q) {
            const GemmProb& pr = lst[q];
            prefix.push_back(tot);
            const int64_t nt = tiles_of(tc, pr.M, pr.N);
            for (int64_t t = 0; t < nt; ++t) bmap.push_back((int32_t)q);
            tot += nt;
            ln.maxM = std::max(ln.maxM, pr.M);
            ln.maxN = std::max(ln.maxN, pr.N);
            ln.maxK = std::max(ln.maxK, pr.K);
        }
        ln.nblocks = tot;
        if (tc) {   // the CUDA-core kernel's 64 x 64 tiling of the same problems
            ln.alt_prefix = (int64_t)prefix.size();
            ln.alt_gemm_map = (int64_t)bmap.size();
            int64_t alt = 0;
            for (size_t q = 0; q < lst.size(); ++q) {
                prefix.push_back(alt);
                const int64_t nt = tiles_of(false, lst[q].M, lst[q].N);
                for (int64_t t = 0; t < nt; ++t) bmap.push_back((int32_t)q);
                alt += nt;
            }
            ln.alt_nblocks = alt;
        }
        ln.switchable = tc || !tcp ? 1 : 0;
        for (auto& pr : lst) probs.push_back(pr);
        ln.depth = depth;
        P.launches.push_back(ln);
    };
    for (int d = P.max_depth; d >= 0; --d) {
        const auto& lv = P.level_list[d];
        // extend-add
        {
            Launch ln{};
            ln.kind = Launch::EXTEND_ADD;
            ln.items = (int64_t)items.size() / 4;
            for (int s : lv) {
                const FrontDev& f = P.hfronts[s];
                // every front, leaves included: the extend-add writes each lower
                // entry (the fronts are not cleared beforehand)
                for (int j0 = 0; j0 < f.m; j0 += kEACols)
                    for (int i0 = j0 / kEARows * kEARows; i0 < f.m; i0 += kEARows) push_item(s, j0, i0, 0);
            }
            ln.nitems = (int32_t)(items.size() / 4 - ln.items);
            ln.nblocks = ln.nitems;
            ln.depth = d;
            for (int s : lv) {
                const FrontDev& f = P.hfronts[s];
                const double m = f.m, nn2 = f.n, u = f.u, eb = P.elem_bytes();
                double b = u * (u + 1) / 2 * eb;                                  // ABR written
                b += (m * nn2 - nn2 * (nn2 - 1) / 2) * eb;                        // frontL written (lower part)
                if (f.cmap >= 0)
                    for (int c = 0; c < 2; ++c) b += (double)f.cu[c] * (f.cu[c] + 1) / 2 * eb;   // children read
                ln.work += b;
            }
            if (ln.nitems) P.launches.push_back(ln);
        }
        int maxn = 0;
        for (int s : lv) maxn = std::max(maxn, P.hfronts[s].n);
        // Two-level blocking: inside an outer block of width nbo the nb-wide
        // steps update only the outer block's own columns (all rows below);
        // the columns right of the block receive the whole block's update
        // at once (K = nbo), which the reference spreads over nbo/nb Gemm
        // calls (ldl/local_front.hpp:67).
        const int nbo = std::max(nb, P.outer_nb / nb * nb);
        int schur_done = 0;   // pivot columns whose Schur-complement update is issued
        for (int K0 = 0; K0 < maxn; K0 += nbo) {
            for (int k = K0; k < std::min(K0 + nbo, maxn); k += nb) {
                Launch dg{};
                dg.kind = Launch::DIAG;
                dg.k = k;
                dg.depth = d;
                dg.items = (int64_t)items.size() / 4;
                std::vector<std::pair<int, int>> active;
                for (int s : lv)
                    if (P.hfronts[s].n > k) {
                        push_item(s, (int)active.size(), 0, 0);
                        active.push_back({s, (int)active.size()});
                    }
                dg.nitems = (int32_t)active.size();
                dg.nblocks = dg.nitems;
                max_slots = std::max<int64_t>(max_slots, dg.nitems);
                P.launches.push_back(dg);
                Launch pn{};
                pn.kind = Launch::PANEL;
                pn.k = k;
                pn.depth = d;
                pn.items = (int64_t)items.size() / 4;
                std::vector<GemmProb> trail;
                for (auto& a : active) {
                    const FrontDev& f = P.hfronts[a.first];
                    const int kb = std::min(nb, f.n - k);
                    const int rows = f.m - k - kb;
                    const int prows = P.f16_scales() ? 128 : kTile;   // tensor-core panel: 128-row tiles
                    const int N = std::min(K0 + nbo, f.n) - k - kb;
                    const int w = N > 0 ? (int)trail.size() : -1;   // this front's in-panel problem
                    for (int rb = 0; rb * prows < rows; ++rb) push_item(a.first, a.second, rb, w);
                    if (N > 0) {
                        GemmProb pr{};
                        pr.front = a.first;
                        pr.row0 = k + kb;
                        pr.kb0 = k / kTile;
                        pr.nkb = 1;
                        pr.A = f.L + (k + kb) + (int64_t)k * f.m;
                        pr.B = pr.A;
                        pr.C = f.L + (k + kb) + (int64_t)(k + kb) * f.m;
                        pr.d = f.off + k;
                        pr.lda = f.m;
                        pr.ldc = f.m;
                        pr.M = rows;
                        pr.N = N;
                        pr.K = kb;
                        pr.cpool = -1;
                        trail.push_back(pr);
                    }
                }
                pn.nitems = (int32_t)(items.size() / 4 - pn.items);
                pn.nblocks = pn.nitems;
                pn.pk_probs = prepack && !trail.empty() ? (int64_t)probs.size() : -1;
                if (pn.nitems) P.launches.push_back(pn);
                add_gemm(trail, d, 0, true);
            }
            // the outer block's update of the columns to its right: with
            // lookahead, the next outer block's columns [c1, c2) on the main
            // stream and the columns from c2 on the second stream (tensor
            // path: the GEMM epilogue adds atomically, so both may overlap
            // other updates of the same columns)
            const bool la = tcp && P.lookahead;
            std::vector<GemmProb> outer, bulk;
            for (int s : lv) {
                const FrontDev& f = P.hfronts[s];
                const int c1 = K0 + nbo;
                if (f.n <= c1) continue;
                const int c2 = la ? std::min(f.n, c1 + nbo) : f.n;
                for (int part = 0; part < 2; ++part) {
                    const int r0 = part == 0 ? c1 : c2;
                    const int N = part == 0 ? c2 - c1 : f.n - c2;
                    if (N <= 0) continue;
                    GemmProb pr{};
                    pr.front = s;
                    pr.row0 = r0;
                    pr.kb0 = K0 / kTile;
                    pr.nkb = nbo / kTile;
                    pr.A = f.L + r0 + (int64_t)K0 * f.m;
                    pr.B = pr.A;
                    pr.C = f.L + r0 + (int64_t)r0 * f.m;
                    pr.d = f.off + K0;
                    pr.lda = f.m;
                    pr.ldc = f.m;
                    pr.M = f.m - r0;
                    pr.N = N;
                    pr.K = nbo;
                    pr.cpool = -1;
                    (part == 0 ? outer : bulk).push_back(pr);
                }
            }
            add_gemm(outer, d, 0, false);
            if (!bulk.empty()) {
                add_gemm(bulk, d, 0, false);
                P.launches.back().bulk = 1;
                P.launches.back().k = K0;
                ++nbulk;
            }
            // the Schur-complement update of the chunk of pivot columns that
            // just became final (all panels of the chunk done), on stream3
            const int kc1 = K0 + nbo;
            if (chunked && (kc1 - schur_done >= schur_chunk || kc1 >= maxn)) {
                const int kc0 = schur_done;
                schur_done = kc1;
                std::vector<GemmProb> sc;
                for (int s : lv) {
                    const FrontDev& f = P.hfronts[s];
                    if (f.u <= 0 || f.n <= kc0) continue;
                    const int ke = std::min(kc1, f.n);
                    GemmProb pr{};
                    pr.front = s;
                    pr.row0 = f.n;
                    pr.kb0 = kc0 / kTile;
                    pr.nkb = (ke - kc0 + kTile - 1) / kTile;
                    pr.A = f.L + f.n + (int64_t)kc0 * f.m;
                    pr.B = pr.A;
                    pr.C = f.U;
                    pr.d = f.off + kc0;
                    pr.lda = f.m;
                    pr.ldc = f.u;
                    pr.M = f.u;
                    pr.N = f.u;
                    pr.K = ke - kc0;
                    pr.cpool = f.pool;
                    sc.push_back(pr);
                }
                if (!sc.empty()) {
                    add_gemm(sc, d, 1, false);
                    P.launches.back().bulk = 2;
                    P.launches.back().k = -1;
                    ++nbulk;
                    ++nschur_chunks;
                }
            }
        }
        std::vector<GemmProb> schur;
        for (int s : lv) {
            const FrontDev& f = P.hfronts[s];
            if (f.u <= 0 || f.n <= 0 || chunked) continue;
            GemmProb pr{};
            pr.front = s;
            pr.row0 = f.n;
            pr.kb0 = 0;
            pr.nkb = 0;
            pr.A = f.L + f.n;
            pr.B = pr.A;
            pr.C = f.U;
            pr.d = f.off;
            pr.lda = f.m;
            pr.ldc = f.u;
            pr.M = f.u;
            pr.N = f.u;
            pr.K = f.n;
            pr.cpool = f.pool;
            schur.push_back(pr);
        }
        add_gemm(schur, d, 1, false);
    }
    apply_tuned_choices(P);   // kernel choices an earlier autotuning made for launches of the same size bucket
    P.tinv_slots = max_slots;
    P.pack_floats = tcp ? pack_max : 0;

    // ---- solve schedule ----
    P.solve_levels.assign(P.max_depth + 1, SolveLevel{});
    P.helpers_total = 0;
    std::vector<int32_t> level_fronts, tiny_fronts;
    std::vector<int32_t> chain_items;   // int4 {front, block, 0, 0}: chain tiles to form after the factorization
    int flag = 0;
    for (int d = 0; d <= P.max_depth; ++d) {
        SolveLevel& sl = P.solve_levels[d];
        sl.depth = d;
        sl.fronts = (int64_t)level_fronts.size();
        for (int s : P.level_list[d]) level_fronts.push_back(s);
        sl.nfronts = (int32_t)P.level_list[d].size();
        sl.gather_chunks = 1;
        for (int s : P.level_list[d]) sl.gather_chunks = std::max(sl.gather_chunks, (P.hfronts[s].m + 1023) / 1024);
        // forward: each front's chain followed by its pivot-row workers in the
        // order the chain consumes their results, then the workers for the
        // rows below the pivots (they only wait on chains, all issued before)
        // Small fronts (whole()) get one CTA that solves the front alone, last.
        auto whole = [](const FrontDev& f) { return f.n <= 2 * kTile && f.m - f.n <= kWholeLowerRows; };
        // one pivot block and few rows below: one warp per front (a subset of whole())
        auto tiny = [](const FrontDev& f) { return f.n <= kTile && f.m - f.n <= kTinyLowerRows; };
        sl.tiny = (int64_t)tiny_fronts.size();
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n > 0 && f.m > 0 && tiny(f)) tiny_fronts.push_back(s);
        }
        sl.ntiny = (int32_t)(tiny_fronts.size() - sl.tiny);
        sl.fwd_items = (int64_t)items.size() / 4;
        for (int s : P.level_list[d]) {
            FrontDev& f = P.hfronts[s];
            if (f.n <= 0 || f.m <= 0) continue;
            const int nT = (f.n + kTile - 1) / kTile;
            f.flag_base = flag;
            flag += nT;
            if (whole(f)) continue;
            if (!P.solve_exact) {   // chain tiles: only fronts whose sweeps run a chain in the product form
                f.chain = P.chain_elems;
                P.chain_elems += (int64_t)nT * kTile * kTile;
            }
            push_item(s, kItemChain, 0, 0);
            for (int rb = 0; rb < nT; ++rb) push_item(s, kItemPivotRows, rb, 0);
            for (int b = 1; b < nT; ++b) {
                chain_items.push_back(s); chain_items.push_back(b); chain_items.push_back(0); chain_items.push_back(0);
            }
        }
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n <= 0 || f.m <= 0 || whole(f)) continue;
            for (int i = 0; f.n + i * kTile < f.m; ++i) push_item(s, kItemLowerRows, i, 0);
        }
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n > 0 && f.m > 0 && whole(f) && !tiny(f)) push_item(s, kItemWhole, 0, 0);
        }
        sl.nfwd = (int32_t)(items.size() / 4 - sl.fwd_items);
        // backward: first the helpers (rows below the pivots beyond the first
        // 16-tile chunk, no waits), then each front's chain followed by its
        // column workers, last block first
        sl.bwd_items = (int64_t)items.size() / 4;
        for (int s : P.level_list[d]) {
            FrontDev& f = P.hfronts[s];
            if (f.n <= 0 || f.m <= 0) continue;
            const int nT = (f.n + kTile - 1) / kTile;
            const int low_tiles = (f.m - f.n + kTile - 1) / kTile;
            f.nch = std::max(1, (low_tiles + kLowerChunkTiles - 1) / kLowerChunkTiles);
            f.hbase = (int32_t)P.helpers_total;
            if (whole(f)) { f.nch = 1; continue; }
            P.helpers_total += (int64_t)nT * (f.nch - 1);
            for (int c = nT - 1; c >= 0; --c)
                for (int ch = 1; ch < f.nch; ++ch) push_item(s, kItemLowerChunk, c, ch);
        }
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n <= 0 || f.m <= 0 || whole(f)) continue;
            const int nT = (f.n + kTile - 1) / kTile;
            push_item(s, kItemChain, 0, 0);
            for (int c = nT - 1; c >= 0; --c) push_item(s, kItemColumns, c, 0);
        }
        for (int s : P.level_list[d]) {
            const FrontDev& f = P.hfronts[s];
            if (f.n > 0 && f.m > 0 && whole(f) && !tiny(f)) push_item(s, kItemWhole, 0, 0);
        }
        sl.nbwd = (int32_t)(items.size() / 4 - sl.bwd_items);
    }
    P.flags_total = std::max(flag, 1);

    // ---- assembly map (DistSymmFrontTree::Initialize, impl.hpp:244-297) ----
    std::vector<int32_t> node_of(n), inv(n);
    for (int s = 0; s < nn; ++s)
        for (int t = 0; t < info->size[s]; ++t) node_of[info->off[s] + t] = s;
    for (int64_t i = 0; i < n; ++i) {
        if (map[i] < 0 || map[i] >= n) { set_last_error("plan_create: map out of range"); return CLIQ_ERR_ARG; }
        inv[map[i]] = (int32_t)i;
    }
    std::vector<int64_t> dest(P.nnz, -1);
    for (int64_t i = 0; i < n; ++i) {
        const int p = map[i];
        const int s = node_of[p];
        const FrontDev& f = P.hfronts[s];
        const int t = p - f.off;
        const int32_t* plow = low + info->lower_ptr[s];
        const int64_t pnl = info->lower_ptr[s + 1] - info->lower_ptr[s];
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            const int c = colind[e];
            if (c < 0 || c >= n) { set_last_error("plan_create: column index out of range"); return CLIQ_ERR_ARG; }
            const int target = map[c];
            if (target < f.off + t) continue;
            if (target < f.off + f.n) dest[e] = f.L + (target - f.off) + (int64_t)t * f.m;
            else {
                const int32_t* it = std::lower_bound(plow, plow + pnl, target);
                if (it == plow + pnl || *it != target) { set_last_error("plan_create: entry outside the front structure"); return CLIQ_ERR_ARG; }
                dest[e] = f.L + f.n + (it - plow) + (int64_t)t * f.m;
            }
        }
    }

    // ---- assembly by level (kept entries grouped by their front's depth) ----
    {
        std::vector<int64_t> cnt(P.max_depth + 2, 0);
        for (int64_t i = 0; i < n; ++i) {
            const int d = P.depth[node_of[map[i]]];
            for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
                if (dest[e] >= 0) ++cnt[d + 1];
        }
        P.asm_level.assign(P.max_depth + 2, 0);
        for (int d = 0; d <= P.max_depth; ++d) P.asm_level[d + 1] = P.asm_level[d] + cnt[d + 1];
        std::vector<int64_t> src(std::max<int64_t>(P.asm_level.back(), 1)), dst(src.size());
        std::vector<int64_t> pos(P.asm_level.begin(), P.asm_level.end() - 1);
        for (int64_t i = 0; i < n; ++i) {
            const int d = P.depth[node_of[map[i]]];
            for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e)
                if (dest[e] >= 0) { src[pos[d]] = e; dst[pos[d]] = dest[e]; ++pos[d]; }
        }
        TRY(dev_upload(P, &P.asm_src, src));
        TRY(dev_upload(P, &P.asm_dst, dst));
    }

    // ---- device allocations ----
    const int eb = P.elem_bytes();
    TRY(dev_alloc(P, &P.L, (size_t)P.arena_elems * eb));
    TRY(dev_alloc(P, (void**)&P.D, sizeof(double) * (P.cplx() ? 2 : 1) * (size_t)n));
    TRY(dev_alloc(P, &P.pool[0], (size_t)P.pool_elems[0] * eb));
    TRY(dev_alloc(P, &P.pool[1], (size_t)P.pool_elems[1] * eb));
    TRY(dev_alloc(P, &P.tinv, (size_t)P.tinv_slots * nb * nb * eb));
    TRY(dev_alloc(P, &P.dinv, (size_t)std::max<int64_t>(P.dinv_elems, 1) * eb));
    TRY(dev_alloc(P, &P.dinvT, (size_t)std::max<int64_t>(P.dinv_elems, 1) * eb));
    // chain tiles only for the product form of the sweeps
    const int64_t chain_elems = std::max<int64_t>(P.chain_elems, 1);
    TRY(dev_alloc(P, &P.m1, (size_t)chain_elems * eb));
    TRY(dev_alloc(P, &P.n1, (size_t)chain_elems * eb));
    TRY(dev_alloc(P, &P.hpart, (size_t)std::max<int64_t>(P.helpers_total, 1) * kTile * kSolveRhsChunk * eb));
    TRY(dev_alloc(P, &P.partial, (size_t)P.flags_total * kTile * kSolveRhsChunk * eb));
    if (P.f16_scales()) {
        TRY(dev_alloc(P, (void**)&P.eblk, sizeof(uint32_t) * 2 * (size_t)std::max<int64_t>(P.eblk_total, 1)));
        TRY(dev_alloc(P, (void**)&P.erow, sizeof(uint32_t) * 2 * (size_t)std::max<int64_t>(P.erow_total, 1)));
    }
    TRY(dev_upload(P, &P.fronts, P.hfronts));
    TRY(dev_upload(P, &P.cmaps, cmaps));
    std::vector<int32_t> lowv(low, low + info->lower_ptr[nn]);
    TRY(dev_upload(P, &P.lower, lowv));
    P.cmaps_len = (int64_t)cmaps.size();
    P.lower_len = (int64_t)lowv.size();
    TRY(dev_upload(P, &P.items, items));
    TRY(dev_upload(P, &P.probs, probs));
    TRY(dev_upload(P, &P.packjobs, packjobs));
    if (P.pack_floats > 0) TRY(dev_alloc(P, &P.pack, (size_t)P.pack_floats * sizeof(float)));
    if (nbulk > 0) {
        TRY(dev_alloc(P, &P.pack2, (size_t)P.pack_floats * sizeof(float)));
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (cudaStreamCreateWithPriority(&P.stream1, cudaStreamNonBlocking, greatest) != cudaSuccess ||
            cudaStreamCreateWithPriority(&P.stream2, cudaStreamNonBlocking, least) != cudaSuccess ||
            cudaStreamCreateWithPriority(&P.stream3, cudaStreamNonBlocking, least) != cudaSuccess)
            return check_cuda("lookahead streams");
        if (nschur_chunks > 0) TRY(dev_alloc(P, &P.pack3, (size_t)P.pack_floats * sizeof(float)));
        P.sync_events.resize(2 * (size_t)nbulk + 4, nullptr);
        for (cudaEvent_t& e : P.sync_events)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return check_cuda("lookahead events");
    }
    TRY(dev_upload(P, &P.prefix, prefix));
    TRY(dev_upload(P, &P.bmap, bmap));
    TRY(dev_upload(P, &P.dest, dest));
    TRY(dev_upload(P, &P.perm, inv));
    TRY(dev_upload(P, &P.level_fronts, level_fronts));
    if (tiny_fronts.empty()) tiny_fronts.push_back(0);
    TRY(dev_upload(P, &P.tiny_fronts, tiny_fronts));
    std::vector<int32_t> zeros_flags(P.flags_total + P.helpers_total, 0);
    TRY(dev_upload(P, &P.flags, zeros_flags));
    P.nchain_items = (int32_t)(chain_items.size() / 4);
    if (chain_items.empty()) chain_items.assign(4, 0);
    TRY(dev_upload(P, &P.chain_items, chain_items));
    std::vector<unsigned long long> zprog(std::max(nn, 1), 0ull);
    TRY(dev_upload(P, &P.xprog, zprog));
    std::vector<int32_t> zt(2 * (P.max_depth + 1) + 2, 0);
    TRY(dev_upload(P, &P.tickets, zt));
    std::vector<int32_t> st = {INT_MAX, 0, 0, 0};
    TRY(dev_upload(P, &P.status, st));
    // A's values stay on the device (the factorization assembles from them)
    TRY(dev_alloc(P, (void**)&P.aval, sizeof(double) * (P.cplx() ? 2 : 1) * (size_t)std::max<int64_t>(P.nnz, 1)));
    if (P.keep_matrix) {
        std::vector<int64_t> rp(rowptr, rowptr + n + 1);
        std::vector<int32_t> ci(colind, colind + P.nnz);
        TRY(dev_upload(P, &P.rowptr, rp));
        TRY(dev_upload(P, &P.colind, ci));
    }
    return CLIQ_OK;
}

int ensure_workspace(Plan& P, int nrhs) {
    if (nrhs <= P.ws_nrhs) return CLIQ_OK;
    void* old[] = {P.wpool[0], P.wpool[1], P.xnodal, P.xwork, P.norms};
    for (void* p : old)
        if (p) cudaFree(p);
    P.wpool[0] = P.wpool[1] = P.xnodal = nullptr;
    P.xwork = P.norms = nullptr;
    const int eb = P.elem_bytes();
    const int chunk = std::min(nrhs, 16);
    TRY(dev_alloc(P, &P.wpool[0], (size_t)P.wpool_elems[0] * chunk * eb));
    TRY(dev_alloc(P, &P.wpool[1], (size_t)P.wpool_elems[1] * chunk * eb));
    TRY(dev_alloc(P, &P.xnodal, (size_t)P.n * nrhs * eb));
    TRY(dev_alloc(P, (void**)&P.xwork, sizeof(double) * (P.cplx() ? 2 : 1) * 3 * (size_t)P.n * nrhs));
    TRY(dev_alloc(P, (void**)&P.norms, sizeof(double) * (2 + 128) * nrhs));   // two norm vectors + partial sums
    P.ws_nrhs = nrhs;
    return CLIQ_OK;
}

int solve_nodal_dispatch(Plan& P, void* xn, int nrhs) {
    if (P.block) return run_block_solve(P, xn, nrhs);
    if (P.precision == CLIQ_FP64)
        return P.cplx() ? run_solve_nodal<double, true>(P, xn, nrhs) : run_solve_nodal<double, false>(P, xn, nrhs);
    return P.cplx() ? run_solve_nodal<float, true>(P, xn, nrhs) : run_solve_nodal<float, false>(P, xn, nrhs);
}

// Row order of the solves' nodal vectors: ND order, or after a pivoted
// factorization each front's pivot rows in pivoted order.  The map takes a
// natural-order (nodal = false) or ND-order (nodal = true) vector there.
const int32_t* solve_perm(const Plan& P, bool nodal) {
    if (P.pivoted) return nodal ? P.pivg : P.perm_piv;
    return nodal ? nullptr : P.perm;
}

int read_status(Plan& P, int64_t* zero_pivot) {
    int32_t st[4];
    if (cudaMemcpyAsync(st, P.status, sizeof(st), cudaMemcpyDeviceToHost, P.stream) != cudaSuccess) return check_cuda("status");
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("sync");
    if (zero_pivot) *zero_pivot = st[0] == INT_MAX ? -1 : (int64_t)st[0] - 1;
    if (st[1]) {
        static const char* sites[] = {"?", "update: stage full", "update: stage empty", "update: accumulator", "solve: block flag",
                                      "update: tile outside the schedule", "panel: tensor-core products"};
        set_last_error(std::string("a device-side wait timed out at ") + sites[(st[2] >= 0 && st[2] <= 6) ? st[2] : 0]);
        return CLIQ_ERR_TIMEOUT;
    }
    if (st[0] == INT_MAX) return CLIQ_OK;
    set_last_error("zero pivot at ND index " + std::to_string((int64_t)st[0] - 1));
    return CLIQ_ERR_ZERO_PIVOT;
}

}  // namespace cliqgpu

using namespace cliqgpu;

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int cliqgpu_plan_create(const cliq_symm_info* info, int64_t n, const int32_t* map, const int64_t* rowptr,
                        const int32_t* colind, const cliqgpu_options* options, void* stream, cliqgpu_plan* out) {
    if (!info || !map || !rowptr || !colind || !out || n <= 0) return CLIQ_ERR_ARG;
    *out = nullptr;
    cliqgpu_plan h = new (std::nothrow) cliqgpu_plan_s;
    if (!h) return CLIQ_ERR_OOM;
    Plan& P = h->p;
    if (options) {
        P.field = options->field == CLIQ_COMPLEX ? CLIQ_COMPLEX : CLIQ_REAL;
        P.precision = options->precision == CLIQ_FP32 ? CLIQ_FP32 : CLIQ_FP64;
        P.conjugate = options->conjugate ? 1 : 0;
        P.keep_matrix = options->keep_matrix ? 1 : 0;
        if (options->block_size != 0 && options->block_size != kTile) {
            delete h;
            set_last_error("plan_create: only block_size 64 is supported");
            return CLIQ_ERR_ARG;
        }
    }
    P.nb = kTile;
    if (const char* e = getenv("CLIQGPU_TENSOR_CORES")) P.use_tc = atoi(e) != 0;
    if (const char* e = getenv("CLIQGPU_OUTER_BLOCK")) P.outer_nb = std::max(kTile, atoi(e));
    if (const char* e = getenv("CLIQGPU_DIAG_FP64")) P.diag_fp64 = atoi(e) != 0;
    if (const char* e = getenv("CLIQGPU_FP64_DMMA")) P.fp64_dmma = atoi(e) != 0;
    P.solve_exact = P.precision == CLIQ_FP64 ? 1 : 0;
    if (const char* e = getenv("CLIQGPU_SOLVE_FORM")) P.solve_exact = strcmp(e, "tiles") != 0;
    if (const char* e = getenv("CLIQGPU_SPLIT")) P.split_f16 = strcmp(e, "tf32") != 0;
    if (const char* e = getenv("CLIQGPU_INPANEL_TC")) P.inpanel_tc = atoi(e) != 0;
    if (const char* e = getenv("CLIQGPU_REFINE")) P.refine_gmres = strcmp(e, "ir") != 0;
    if (const char* e = getenv("CLIQGPU_LOOKAHEAD")) P.lookahead = atoi(e) != 0;
    if (const char* e = getenv("CLIQGPU_GRAPH")) P.use_graph = atoi(e) != 0;
    if (const char* e = getenv("CLIQGPU_SCHUR_CHUNK")) P.schur_chunk = std::max(0, atoi(e));
    if (const char* e = getenv("CLIQGPU_BATCH_GRAPH")) P.batch_graph = atoi(e) != 0;
    if (stream) P.stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return check_cuda("stream"); }
        P.own_stream = true;
    }
    int st = build_plan(P, info, n, map, rowptr, colind);
    if (st != CLIQ_OK) {
        free_plan(P);
        delete h;
        return st;
    }
    *out = h;
    return CLIQ_OK;
}

int cliqgpu_assemble(cliqgpu_plan h, const void* values, int32_t values_on_device) {
    if (!h || !values) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    const size_t bytes = sizeof(double) * (P.cplx() ? 2 : 1) * (size_t)P.nnz;
    // the values go to the plan's device copy; the factorization adds them to
    // the fronts level by level, right after each level's extend-add
    if (cudaMemcpyAsync(P.aval, values, bytes, values_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        P.stream) != cudaSuccess)
        return check_cuda("copy A");
    int st = launch_assemble(P, P.aval);
    if (st != CLIQ_OK) return st;
    if (!values_on_device && cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("assemble sync");
    P.assembled = true;
    P.factored = false;
    return CLIQ_OK;
}

}  // extern "C"

namespace cliqgpu {
int run_factor_dispatch(Plan& P) {
    if (P.precision == CLIQ_FP64) return P.cplx() ? run_factor<double, true>(P) : run_factor<double, false>(P);
    return P.cplx() ? run_factor<float, true>(P) : run_factor<float, false>(P);
}
}  // namespace cliqgpu

extern "C" {

static int factor_common(cliqgpu_plan h, int64_t* zero_pivot, bool pivoted) {
    if (!h) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (!P.assembled) { set_last_error("factor: fronts were not assembled"); return CLIQ_ERR_STATE; }
    if (P.factored) { set_last_error("Matrix is already factored"); return CLIQ_ERR_STATE; }
    int32_t st0[4] = {INT_MAX, 0, 0, 0};
    cudaMemcpyAsync(P.status, st0, sizeof(st0), cudaMemcpyHostToDevice, P.stream);
    P.block = false;
    P.pivoted = pivoted;
    const int st = run_factor_dispatch(P);
    if (st != CLIQ_OK) return st;
    P.factored = true;
    return read_status(P, zero_pivot);
}

int cliqgpu_factor(cliqgpu_plan h, int64_t* zero_pivot) { return factor_common(h, zero_pivot, false); }

int cliqgpu_factor_intrapiv(cliqgpu_plan h, int64_t* zero_pivot) { return factor_common(h, zero_pivot, true); }

int cliqgpu_get_front_pivots(cliqgpu_plan h, int32_t s, double* sub, int32_t* piv) {
    if (!h) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (s < 0 || s >= P.num_fronts) return CLIQ_ERR_ARG;
    const FrontDev& f = P.hfronts[s];
    const int w = P.cplx() ? 2 : 1;
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("sync");
    if (!P.pivoted || !P.factored) {   // unpivoted fronts: no 2 x 2 blocks, identity order
        if (sub) for (int64_t i = 0; i < (int64_t)w * f.n; ++i) sub[i] = 0.0;
        if (piv) for (int i = 0; i < f.n; ++i) piv[i] = i;
        return CLIQ_OK;
    }
    if (sub && f.n > 0 &&
        cudaMemcpy(sub, P.E + (size_t)w * f.off, sizeof(double) * w * f.n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return check_cuda("get pivots");
    if (piv && f.n > 0) {
        if (cudaMemcpy(piv, P.pivg + f.off, sizeof(int32_t) * f.n, cudaMemcpyDeviceToHost) != cudaSuccess)
            return check_cuda("get pivots");
        for (int i = 0; i < f.n; ++i) piv[i] -= f.off;
    }
    return CLIQ_OK;
}

int cliqgpu_block_ldl(cliqgpu_plan h) {
    if (!h) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (!P.factored) { set_last_error("block LDL: the front tree is not factored"); return CLIQ_ERR_STATE; }
    if (P.block) return CLIQ_OK;
    const int st = convert_to_block(P);
    if (st != CLIQ_OK) return st;
    P.block = true;
    return CLIQ_OK;
}

int cliqgpu_solve(cliqgpu_plan h, void* X, int64_t ldx, int32_t nrhs, int32_t x_on_device, int32_t nodal) {
    if (!h || !X || nrhs <= 0) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (ldx < P.n) return CLIQ_ERR_ARG;
    if (!P.factored) { set_last_error("solve: the front tree is not factored"); return CLIQ_ERR_STATE; }
    TRY(ensure_workspace(P, nrhs));
    P.last_launches = 0;
    const int w = P.cplx() ? 2 : 1;
    const size_t colbytes = sizeof(double) * w * (size_t)P.n;
    double* xd = (double*)X;
    double* stage = nullptr;
    if (!x_on_device) {
        stage = P.xwork;   // FP64 staging, ld n
        for (int j = 0; j < nrhs; ++j)
            if (cudaMemcpyAsync(stage + (size_t)w * j * P.n, (const double*)X + (size_t)w * j * ldx, colbytes,
                                cudaMemcpyHostToDevice, P.stream) != cudaSuccess)
                return check_cuda("copy X");
        xd = stage;
        ldx = P.n;
    }
    int32_t st0[4] = {INT_MAX, 0, 0, 0};
    cudaMemcpyAsync(P.status, st0, sizeof(st0), cudaMemcpyHostToDevice, P.stream);
    const int32_t* perm = solve_perm(P, nodal != 0);
    TRY(launch_pull(P, perm, xd, ldx, nrhs, P.xnodal, 1.0));
    TRY(solve_nodal_dispatch(P, P.xnodal, nrhs));
    TRY(launch_push(P, perm, P.xnodal, xd, ldx, nrhs, 1.0, 0));
    P.last_launches += 2;
    if (!x_on_device) {
        for (int j = 0; j < nrhs; ++j)
            if (cudaMemcpyAsync((double*)X + (size_t)w * j * ldx, stage + (size_t)w * j * P.n, colbytes,
                                cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
                return check_cuda("copy X back");
    }
    int64_t zp;
    int st = read_status(P, &zp);
    if (st == CLIQ_ERR_ZERO_PIVOT) st = CLIQ_OK;   // pivots were reported by factor
    return st;
}

int cliqgpu_multiply(cliqgpu_plan h, const double* alpha, const void* X, const double* beta, void* Y, int64_t ld, int32_t nrhs) {
    if (!h || !alpha || !beta || !X || !Y || nrhs <= 0) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (!P.keep_matrix || !P.assembled) { set_last_error("multiply: plan holds no FP64 matrix"); return CLIQ_ERR_STATE; }
    const bool c = P.cplx();
    return launch_spmv(P, alpha[0], c ? alpha[1] : 0.0, (const double*)X, beta[0], c ? beta[1] : 0.0, (double*)Y, ld, nrhs);
}

int cliqgpu_grad_A_pattern(cliqgpu_plan h, const void* Xbar, const void* X, int64_t ld, int32_t nrhs, int32_t conj_x,
                           void* out) {
    if (!h || !Xbar || !X || !out || nrhs <= 0) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (ld < P.n) return CLIQ_ERR_ARG;
    if (!P.keep_matrix) { set_last_error("grad_A_pattern: the plan holds no matrix pattern (keep_matrix = 0)"); return CLIQ_ERR_STATE; }
    return launch_grad_pattern(P, (const double*)Xbar, (const double*)X, ld, nrhs, conj_x ? 1 : 0, (double*)out);
}

// ---------------------------------------------------------------------------
// Krylov refinement: right-preconditioned FGMRES (restart length up to
// kKrylovMax) with the stored factorization as the preconditioner, FP64
// residuals and basis.  x_k minimises ||b - A x|| over x0 + span(Z), which
// contains the classical refinement iterate after the same number of
// solves, so it never needs more solves than classical refinement.  Each
// right-hand side runs its own Arnoldi process (complex Givens rotations on
// the host); the basis vectors of all right-hand sides are processed
// together (one solve per step).  Orthogonalisation: classical Gram-Schmidt,
// applied twice.  The relative residual returned is recomputed from x.
// ---------------------------------------------------------------------------
constexpr int kKrylovMax = 8;

static int ensure_krylov(Plan& P, int nrhs) {
    const int w = P.cplx() ? 2 : 1;
    const int64_t vec = (int64_t)w * P.n * nrhs;
    const int64_t need = (2 * kKrylovMax + 2) * vec + 2 * (int64_t)(kKrylovMax + 1) * nrhs * (128 + 4) + 8 * nrhs;
    if (need <= P.krylov_doubles) return CLIQ_OK;
    if (P.krylov) cudaFree(P.krylov);
    P.krylov = nullptr;
    P.krylov_doubles = 0;
    TRY(dev_alloc(P, (void**)&P.krylov, sizeof(double) * (size_t)need));
    P.krylov_doubles = need;
    return CLIQ_OK;
}

static int refine_fgmres(Plan& P, const double* b, double* x, double* r, int nrhs, double tol, int max_iter, int* iters,
                         double* relres) {
    using cd = std::complex<double>;
    const bool cplx = P.cplx();
    const int w = cplx ? 2 : 1;
    const int64_t n = P.n;
    const int64_t vec = (int64_t)w * n * nrhs;
    TRY(ensure_krylov(P, nrhs));
    double* V = P.krylov;                              // kKrylovMax + 1 basis block vectors
    double* Z = V + (kKrylovMax + 1) * vec;             // kKrylovMax preconditioned block vectors
    double* wv = Z + kKrylovMax * vec;                  // work block vector
    double* part = wv + vec;                            // dot partial sums
    double* hdev = part + 2 * (int64_t)(kKrylovMax + 1) * nrhs * 128;   // (k+1) x nrhs complex coefficients
    double* sdev = hdev + 2 * (int64_t)(kKrylovMax + 1) * nrhs * 2;     // per-column scales / solution coefficients
    std::vector<double> bn(nrhs), hn(2 * nrhs);
    // ||b_j|| (norms[nrhs..] were filled by the caller)
    if (cudaMemcpyAsync(hn.data(), P.norms, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
        return check_cuda("norms");
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("refine sync");
    for (int j = 0; j < nrhs; ++j) bn[j] = std::sqrt(hn[nrhs + j]);
    int it = 0;
    double rel = 0;
    std::vector<double> hbuf(2 * (kKrylovMax + 1) * nrhs), h2(2 * (kKrylovMax + 1) * nrhs), sc(2 * nrhs);
    auto residual = [&](double* relp, std::vector<double>& beta) -> int {
        cudaMemcpyAsync(r, b, sizeof(double) * vec, cudaMemcpyDeviceToDevice, P.stream);
        TRY(launch_spmv(P, -1.0, 0.0, x, 1.0, 0.0, r, n, nrhs));
        TRY(launch_col_norms(P, r, n, nrhs, P.norms));
        if (cudaMemcpyAsync(hn.data(), P.norms, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
            return check_cuda("norms");
        if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("refine sync");
        double rl = 0;
        for (int j = 0; j < nrhs; ++j) {
            beta[j] = std::sqrt(hn[j]);
            rl = std::max(rl, bn[j] > 0 ? beta[j] / bn[j] : beta[j]);
        }
        *relp = rl;
        return CLIQ_OK;
    };
    std::vector<double> beta(nrhs);
    TRY(residual(&rel, beta));
    while (rel > tol && it < max_iter && rel == rel) {
        // v_0 = r / beta
        for (int j = 0; j < nrhs; ++j) sc[j] = beta[j] > 0 ? 1.0 / beta[j] : 0.0;
        cudaMemcpyAsync(sdev, sc.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, P.stream);
        TRY(launch_col_scale(P, r, V, nrhs, sdev));
        // per right-hand side: rotated Hessenberg R, rotations, right-hand side g
        std::vector<std::vector<cd>> R(nrhs, std::vector<cd>((kKrylovMax + 1) * kKrylovMax)), g(nrhs, std::vector<cd>(kKrylovMax + 1));
        std::vector<std::vector<double>> cs(nrhs, std::vector<double>(kKrylovMax));
        std::vector<std::vector<cd>> sn(nrhs, std::vector<cd>(kKrylovMax));
        for (int j = 0; j < nrhs; ++j) g[j][0] = beta[j];
        int k = 0;
        double est = rel;
        for (; k < kKrylovMax && it < max_iter; ++k) {
            // z_k = M^{-1} v_k (natural order FP64 -> nodal storage precision -> solve -> back)
            TRY(launch_pull(P, solve_perm(P, false), V + k * vec, n, nrhs, P.xnodal, 1.0));
            TRY(solve_nodal_dispatch(P, P.xnodal, nrhs));
            TRY(launch_push(P, solve_perm(P, false), P.xnodal, Z + k * vec, n, nrhs, 1.0, 0));
            ++it;
            // w = A z_k, orthogonalised twice against v_0 .. v_k
            TRY(launch_spmv(P, 1.0, 0.0, Z + k * vec, 0.0, 0.0, wv, n, nrhs));
            TRY(launch_multi_dot(P, V, vec, k + 1, wv, nrhs, part, hdev));
            TRY(launch_multi_axpy(P, V, vec, k + 1, hdev, wv, nrhs, -1.0));
            if (cudaMemcpyAsync(hbuf.data(), hdev, sizeof(double) * 2 * (k + 1) * nrhs, cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
                return check_cuda("dots");
            TRY(launch_multi_dot(P, V, vec, k + 1, wv, nrhs, part, hdev));
            TRY(launch_multi_axpy(P, V, vec, k + 1, hdev, wv, nrhs, -1.0));
            if (cudaMemcpyAsync(h2.data(), hdev, sizeof(double) * 2 * (k + 1) * nrhs, cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
                return check_cuda("dots");
            TRY(launch_col_norms(P, wv, n, nrhs, P.norms));
            if (cudaMemcpyAsync(hn.data(), P.norms, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
                return check_cuda("norms");
            if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("refine sync");
            for (int j = 0; j < nrhs; ++j) sc[j] = hn[j] > 0 ? 1.0 / std::sqrt(hn[j]) : 0.0;
            cudaMemcpyAsync(sdev, sc.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, P.stream);
            TRY(launch_col_scale(P, wv, V + (k + 1) * vec, nrhs, sdev));
            est = 0;
            for (int j = 0; j < nrhs; ++j) {
                cd* col = &R[j][(kKrylovMax + 1) * k];
                for (int i = 0; i <= k; ++i)
                    col[i] = cd(hbuf[2 * (i * nrhs + j)] + h2[2 * (i * nrhs + j)],
                                cplx ? hbuf[2 * (i * nrhs + j) + 1] + h2[2 * (i * nrhs + j) + 1] : 0.0);
                col[k + 1] = std::sqrt(hn[j]);
                for (int i = 0; i < k; ++i) {   // earlier rotations
                    const cd a = col[i], bb = col[i + 1];
                    col[i] = cs[j][i] * a + sn[j][i] * bb;
                    col[i + 1] = -std::conj(sn[j][i]) * a + cs[j][i] * bb;
                }
                const double ha = std::abs(col[k]), hb = std::abs(col[k + 1]), rr = std::hypot(ha, hb);
                if (rr == 0) { cs[j][k] = 1; sn[j][k] = 0; }
                else if (ha == 0) { cs[j][k] = 0; sn[j][k] = std::conj(col[k + 1]) / hb; }
                else {
                    const cd al = col[k] / ha;
                    cs[j][k] = ha / rr;
                    sn[j][k] = al * std::conj(col[k + 1]) / rr;
                }
                col[k] = cs[j][k] * col[k] + sn[j][k] * col[k + 1];
                col[k + 1] = 0;
                g[j][k + 1] = -std::conj(sn[j][k]) * g[j][k];
                g[j][k] = cs[j][k] * g[j][k];
                est = std::max(est, bn[j] > 0 ? std::abs(g[j][k + 1]) / bn[j] : std::abs(g[j][k + 1]));
            }
            if (est <= tol) { ++k; break; }
        }
        // x += Z y, R y = g (back substitution per right-hand side)
        std::vector<double> ycoef(2 * kKrylovMax * nrhs, 0.0);
        for (int j = 0; j < nrhs; ++j) {
            std::vector<cd> y(k);
            for (int i = k - 1; i >= 0; --i) {
                cd t = g[j][i];
                for (int l = i + 1; l < k; ++l) t -= R[j][(kKrylovMax + 1) * l + i] * y[l];
                const cd d = R[j][(kKrylovMax + 1) * i + i];
                y[i] = d != cd(0) ? t / d : cd(0);
            }
            for (int i = 0; i < k; ++i) { ycoef[2 * (i * nrhs + j)] = y[i].real(); ycoef[2 * (i * nrhs + j) + 1] = y[i].imag(); }
        }
        cudaMemcpyAsync(hdev, ycoef.data(), sizeof(double) * 2 * k * nrhs, cudaMemcpyHostToDevice, P.stream);
        TRY(launch_multi_axpy(P, Z, vec, k, hdev, x, nrhs, 1.0));
        TRY(residual(&rel, beta));
    }
    *iters = it;
    *relres = rel;
    return CLIQ_OK;
}

int cliqgpu_refine(cliqgpu_plan h, const void* B, void* X, int64_t ld, int32_t nrhs, int32_t on_device, double tol,
                   int32_t max_iter, int32_t* iters, double* relres) {
    if (!h || !B || !X || nrhs <= 0 || ld <= 0) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (ld < P.n) return CLIQ_ERR_ARG;
    if (!P.factored) { set_last_error("refine: the front tree is not factored"); return CLIQ_ERR_STATE; }
    if (!P.keep_matrix) { set_last_error("refine: plan was created without keep_matrix"); return CLIQ_ERR_STATE; }
    TRY(ensure_workspace(P, nrhs));
    P.last_launches = 0;
    const int w = P.cplx() ? 2 : 1;
    const int64_t n = P.n;
    const size_t colbytes = sizeof(double) * w * (size_t)n;
    double* b = P.xwork;
    double* x = b + (size_t)w * n * nrhs;
    double* r = x + (size_t)w * n * nrhs;
    const cudaMemcpyKind kin = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int j = 0; j < nrhs; ++j)
        if (cudaMemcpyAsync(b + (size_t)w * j * n, (const double*)B + (size_t)w * j * ld, colbytes, kin, P.stream) != cudaSuccess)
            return check_cuda("copy B");
    cudaMemsetAsync(x, 0, colbytes * nrhs, P.stream);
    cudaMemcpyAsync(r, b, colbytes * nrhs, cudaMemcpyDeviceToDevice, P.stream);
    std::vector<double> hn(2 * nrhs);
    TRY(launch_col_norms(P, b, n, nrhs, P.norms + nrhs));
    int it = 0;
    double rel = 0;
    int32_t st0[4] = {INT_MAX, 0, 0, 0};
    cudaMemcpyAsync(P.status, st0, sizeof(st0), cudaMemcpyHostToDevice, P.stream);
    if (P.refine_gmres) {
        TRY(refine_fgmres(P, b, x, r, nrhs, tol, max_iter, &it, &rel));
        goto done;
    }
    for (;;) {
        TRY(launch_col_norms(P, r, n, nrhs, P.norms));
        if (cudaMemcpyAsync(hn.data(), P.norms, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, P.stream) != cudaSuccess)
            return check_cuda("norms");
        if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("refine sync");
        rel = 0;
        double rmax = 0;
        for (int j = 0; j < nrhs; ++j) {
            const double bn = std::sqrt(hn[nrhs + j]), rn = std::sqrt(hn[j]);
            rel = std::max(rel, bn > 0 ? rn / bn : rn);
            rmax = std::max(rmax, rn);
        }
        if (rel <= tol || it >= max_iter || !(rel == rel)) break;
        const double scale = rmax > 0 ? 1.0 / rmax : 1.0;
        TRY(launch_pull(P, solve_perm(P, false), r, n, nrhs, P.xnodal, scale));
        TRY(solve_nodal_dispatch(P, P.xnodal, nrhs));
        TRY(launch_push(P, solve_perm(P, false), P.xnodal, x, n, nrhs, 1.0 / scale, 1));
        cudaMemcpyAsync(r, b, colbytes * nrhs, cudaMemcpyDeviceToDevice, P.stream);
        TRY(launch_spmv(P, -1.0, 0.0, x, 1.0, 0.0, r, n, nrhs));
        ++it;
    }
done:
    const cudaMemcpyKind kout = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (int j = 0; j < nrhs; ++j)
        if (cudaMemcpyAsync((double*)X + (size_t)w * j * ld, x + (size_t)w * j * n, colbytes, kout, P.stream) != cudaSuccess)
            return check_cuda("copy X");
    int32_t dst[2];
    cudaMemcpyAsync(dst, P.status, sizeof(dst), cudaMemcpyDeviceToHost, P.stream);
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("refine end");
    if (iters) *iters = it;
    if (relres) *relres = rel;
    if (dst[1]) { set_last_error("a device-side wait timed out"); return CLIQ_ERR_TIMEOUT; }
    return rel <= tol ? CLIQ_OK : CLIQ_ERR_NOCONV;
}

int cliqgpu_get_front(cliqgpu_plan h, int32_t s, double* Lout, double* Dout, int32_t dims[2]) {
    if (!h) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (s < 0 || s >= P.num_fronts) return CLIQ_ERR_ARG;
    const FrontDev& f = P.hfronts[s];
    if (dims) { dims[0] = f.m; dims[1] = f.n; }
    if (!Lout && !Dout) return CLIQ_OK;
    if (P.assembled && !P.factored) TRY(launch_materialize_assembly(P));   // the fronts as Initialize leaves them
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("sync");
    const int w = P.cplx() ? 2 : 1;
    if (Lout) {
        const size_t cnt = (size_t)w * f.m * f.n;
        if (P.precision == CLIQ_FP64) {
            if (cudaMemcpy(Lout, (const double*)P.L + (size_t)w * f.L, sizeof(double) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
                return check_cuda("get front");
        } else {
            std::vector<float> tmp(cnt);
            if (cudaMemcpy(tmp.data(), (const float*)P.L + (size_t)w * f.L, sizeof(float) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
                return check_cuda("get front");
            for (size_t i = 0; i < cnt; ++i) Lout[i] = tmp[i];
        }
        // strictly upper part of the pivot block: zero (the kernels never write it);
        // the block-LDL form keeps the full inv(A11) there
        for (int j = 0; j < (P.block ? 0 : f.n); ++j)
            for (int i = 0; i < j && i < f.m; ++i)
                for (int c = 0; c < w; ++c) Lout[(size_t)w * (i + (size_t)j * f.m) + c] = 0.0;
    }
    if (Dout && f.n > 0) {
        if (cudaMemcpy(Dout, P.D + (size_t)w * f.off, sizeof(double) * w * f.n, cudaMemcpyDeviceToHost) != cudaSuccess)
            return check_cuda("get diag");
    }
    return CLIQ_OK;
}

int cliqgpu_plan_query(cliqgpu_plan h, int32_t key, double* value) {
    if (!h || !value) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    switch (key) {
        case 0: *value = P.factor_flops; break;
        case 1: *value = P.solve_flops; break;
        case 2: *value = P.factor_entries; break;
        case 3: *value = (double)P.device_bytes; break;
        case 4: *value = (double)P.last_launches; break;
        case 5: *value = P.num_fronts; break;
        case 6: *value = P.max_depth; break;
        case 7: *value = (double)P.arena_elems * P.elem_bytes(); break;
        case 8: *value = (double)P.total_launches; break;
        default: return CLIQ_ERR_ARG;
    }
    return CLIQ_OK;
}

int cliqgpu_set_profiling(cliqgpu_plan h, int32_t enable) {
    if (!h) return CLIQ_ERR_ARG;
    h->p.profile = enable ? 1 : 0;
    return CLIQ_OK;
}

int cliqgpu_profile_read(cliqgpu_plan h, double* out, int32_t nout) {
    if (!h || !out || nout <= 0) return CLIQ_ERR_ARG;
    Plan& P = h->p;
    if (P.prof_pending) {
        if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("profile sync");
        for (double& v : P.prof) v = 0;
        int first = -1, last = -1;
        for (size_t li = 0; li < P.launches.size(); ++li) {
            const Launch& ln = P.launches[li];
            if (ln.nblocks <= 0) continue;
            float ms = 0;
            cudaEventElapsedTime(&ms, P.events[3 * li], P.events[3 * li + 1]);
            if (ln.kind == Launch::GEMM && P.tensor_path() && !ln.simt) {
                float pk = 0;
                cudaEventElapsedTime(&pk, P.events[3 * li], P.events[3 * li + 2]);
                P.prof[PROF_PACK_MS] += pk;
                ms -= pk;
            }
            if (first < 0) first = (int)li;
            last = (int)li;
            switch (ln.kind) {
                case Launch::EXTEND_ADD: P.prof[PROF_EA_MS] += ms; P.prof[PROF_EA_BYTES] += ln.work; break;
                case Launch::DIAG: P.prof[PROF_DIAG_MS] += ms; break;
                case Launch::PANEL: P.prof[PROF_PANEL_MS] += ms; break;
                case Launch::GEMM:
                    if (ln.schur) { P.prof[PROF_SCHUR_MS] += ms; P.prof[PROF_SCHUR_FLOPS] += ln.work; P.prof[PROF_SCHUR_LAUNCHES] += 1; }
                    else { P.prof[PROF_TRAIL_MS] += ms; P.prof[PROF_TRAIL_FLOPS] += ln.work; P.prof[PROF_TRAIL_LAUNCHES] += 1; }
                    break;
            }
        }
        if (first >= 0) {
            float ms = 0;
            cudaEventElapsedTime(&ms, P.events[3 * first], P.events[3 * last + 1]);
            P.prof[PROF_FACTOR_MS] = ms;
        }
        cudaGetLastError();
        P.prof_pending = false;
    }
    for (int i = 0; i < nout && i < PROF_SLOTS; ++i) out[i] = P.prof[i];
    return CLIQ_OK;
}

int cliqgpu_wait_selftest(cliqgpu_plan h, int64_t limit_ns) {
    if (!h || limit_ns <= 0 || limit_ns > 2000000000ll) {
        set_last_error("wait_selftest: limit_ns must be in (0, 2e9]");
        return CLIQ_ERR_ARG;
    }
    Plan& P = h->p;
    if (cudaStreamSynchronize(P.stream) != cudaSuccess) return check_cuda("wait_selftest sync");
    // the zero-pivot record of an earlier factorization survives the test
    int32_t saved[4];
    if (cudaMemcpy(saved, P.status, sizeof(saved), cudaMemcpyDeviceToHost) != cudaSuccess)
        return check_cuda("wait_selftest save");
    const int32_t clean[4] = {INT_MAX, 0, 0, 0};
    if (cudaMemcpy(P.status, clean, sizeof(clean), cudaMemcpyHostToDevice) != cudaSuccess)
        return check_cuda("wait_selftest clear");
    int st = launch_wait_selftest(P, (uint64_t)limit_ns);
    if (st == CLIQ_OK) {
        st = read_status(P, nullptr);
        if (st == CLIQ_ERR_ZERO_PIVOT) st = CLIQ_OK;   // not possible here: the word was clean
    }
    // clear the recorded timeout (status[1..3]) and put back status[0]: the plan stays usable
    const int32_t st0[4] = {saved[0], 0, 0, 0};
    if (cudaMemcpyAsync(P.status, st0, sizeof(st0), cudaMemcpyHostToDevice, P.stream) != cudaSuccess ||
        cudaStreamSynchronize(P.stream) != cudaSuccess)
        return check_cuda("wait_selftest reset");
    return st;
}

int cliqgpu_synchronize(cliqgpu_plan h) {
    if (!h) return CLIQ_ERR_ARG;
    if (cudaStreamSynchronize(h->p.stream) != cudaSuccess) return check_cuda("sync");
    return CLIQ_OK;
}

void cliqgpu_plan_destroy(cliqgpu_plan h) {
    if (!h) return;
    cudaStreamSynchronize(h->p.stream);
    free_plan(h->p);
    delete h;
}

const char* cliqgpu_status_string(int32_t status) {
    switch (status) {
        case CLIQ_OK: return "ok";
        case CLIQ_ERR_ARG: return "invalid argument";
        case CLIQ_ERR_OOM: return "out of memory";
        case CLIQ_ERR_ZERO_PIVOT: return "zero pivot";
        case CLIQ_ERR_CUDA: return "CUDA error";
        case CLIQ_ERR_TIMEOUT: return "device wait timed out";
        case CLIQ_ERR_STATE: return "call out of order";
        case CLIQ_ERR_NOCONV: return "refinement did not converge";
        default: return "unknown status";
    }
}

const char* cliqgpu_last_error(void) {
    static thread_local std::string copy;
    std::lock_guard<std::mutex> lk(g_err_mu);
    copy = g_last_error;
    return copy.c_str();
}

}  // extern "C"
