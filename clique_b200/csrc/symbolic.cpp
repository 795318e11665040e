// Host-side symbolic phase: natural nested dissection and symbolic analysis
// for a single process.  This is the product's own implementation (the CPU
// oracle under oracle/ is a separate restatement used only to check it).
//
// Behaviour follows the reference:
//   NaturalNestedDissection   include/clique/symbolic/natural_nested_dissection.hpp:447-488
//   NaturalBisect             include/clique/symbolic/natural_nested_dissection.hpp:490-619
//   recursion / node order    include/clique/symbolic/natural_nested_dissection.hpp:60-189, 313-445
//   ReverseOrder              include/clique/symbolic/nested_dissection.hpp:817-886
//   BuildMap (P=1)            include/clique/symbolic/nested_dissection.hpp:1206-1363
//   LocalSymmetricAnalysis    src/symbolic/LocalSymmetricAnalysis.cpp:15-114
//   NestedDissection (general graphs, P=1)
//                             include/clique/symbolic/nested_dissection.hpp:115-230
//                             (the tree and numbering; the bisection is this
//                             file's own, see graph_nested_dissection)
//
// Design: instead of materialising a child graph at every bisection (the
// reference copies the graph into left/right children), the recursion here
// works on index boxes only.  Every vertex of a box sub-problem is adjacent
// only to vertices of the same box or of ancestor separators, so a node's
// original lower structure is recovered afterwards from the global graph as
// { ND(target) : target adjacent to the node's vertices, ND(target) >= end of
// the node's subtree range }.  That is the same set the reference collects
// from its child graphs (targets numbered >= numSources), computed in
// O(nnz log) once instead of once per tree level.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "cliqgpu_internal.h"

namespace cliqgpu {

namespace {

struct Box { int x0, y0, z0, nx, ny, nz; };

struct PreNode {
    int size = 0, off = 0, parent = -1, sep_parent = -1;
    int nchild = 0, child[2] = {-1, -1};
    std::vector<int> inds;      // natural indices in the node's local order
    int subtree_end = 0;        // one past the last ND index of the node's subtree
};

struct NDBuilder {
    int NX, NY, NZ, cutoff;
    std::vector<PreNode> nodes;

    int gidx(int x, int y, int z) const { return x + y * NX + z * NX * NY; }

    // Natural order of a box (x fastest, then y, then z) -- the order in which
    // NaturalBisect fills each child, so it is also each child's local order.
    void box_inds(const Box& b, std::vector<int>& out) const {
        out.clear();
        out.reserve((size_t)b.nx * b.ny * b.nz);
        for (int z = 0; z < b.nz; ++z)
            for (int y = 0; y < b.ny; ++y)
                for (int x = 0; x < b.nx; ++x) out.push_back(gidx(b.x0 + x, b.y0 + y, b.z0 + z));
    }

    void recurse(const Box& b, int parent, int off) {
        const int n = b.nx * b.ny * b.nz;
        const int id = (int)nodes.size();
        nodes.emplace_back();
        if (n <= cutoff) {
            PreNode& nd = nodes[id];
            nd.size = n; nd.off = off; nd.parent = parent; nd.sep_parent = parent;
            box_inds(b, nd.inds);
            nd.subtree_end = off + n;
            return;
        }
        Box L = b, R = b;
        std::vector<int> sep;
        // longest axis, ties broken x > y > z (NaturalBisect)
        if (b.nx >= b.ny && b.nx >= b.nz) {
            const int l = (b.nx - 1) / 2;
            L.nx = l; R.x0 = b.x0 + l + 1; R.nx = b.nx - 1 - l;
            for (int z = 0; z < b.nz; ++z)
                for (int y = 0; y < b.ny; ++y) sep.push_back(gidx(b.x0 + l, b.y0 + y, b.z0 + z));
        } else if (b.ny >= b.nx && b.ny >= b.nz) {
            const int l = (b.ny - 1) / 2;
            L.ny = l; R.y0 = b.y0 + l + 1; R.ny = b.ny - 1 - l;
            for (int z = 0; z < b.nz; ++z)
                for (int x = 0; x < b.nx; ++x) sep.push_back(gidx(b.x0 + x, b.y0 + l, b.z0 + z));
        } else {
            const int l = (b.nz - 1) / 2;
            L.nz = l; R.z0 = b.z0 + l + 1; R.nz = b.nz - 1 - l;
            for (int y = 0; y < b.ny; ++y)
                for (int x = 0; x < b.nx; ++x) sep.push_back(gidx(b.x0 + x, b.y0 + y, b.z0 + l));
        }
        const int nl = L.nx * L.ny * L.nz, nr = R.nx * R.ny * R.nz;
        {
            PreNode& nd = nodes[id];
            nd.size = (int)sep.size();
            nd.off = off + nl + nr;
            nd.parent = parent; nd.sep_parent = parent;
            nd.nchild = 2;
            nd.inds = std::move(sep);
            nd.subtree_end = off + n;
        }
        nodes[id].child[1] = (int)nodes.size();
        recurse(R, id, off + nl);
        nodes[id].child[0] = (int)nodes.size();
        recurse(L, id, off);
    }
};

// std::set_union of two sorted vectors
static void sorted_union(const std::vector<int>& a, const std::vector<int>& b, std::vector<int>& out) {
    out.resize(a.size() + b.size());
    out.resize(std::set_union(a.begin(), a.end(), b.begin(), b.end(), out.begin()) - out.begin());
}

static void relative_indices(const std::vector<int>& sub, const std::vector<int>& full, std::vector<int>& rel) {
    rel.resize(sub.size());
    auto it = full.begin();
    for (size_t i = 0; i < sub.size(); ++i) {
        it = std::lower_bound(it, full.end(), sub[i]);
        rel[i] = (int)(it - full.begin());
    }
}

}  // namespace

// ReverseOrder, BuildMap, the original lower structures and
// LocalSymmetricAnalysis for a separator tree in pre-order (each separator
// before its right then left subtree, as the recursions above build it)
static int finish_symbolic(std::vector<PreNode>& pre, int64_t n, const int64_t* rowptr, const int32_t* colind, Symbolic& S) {
    struct Holder { std::vector<PreNode>& nodes; } B{pre};
    // ReverseOrder: new index = last - old; the root keeps parent -1 unless it is the only node.
    const int nn = (int)B.nodes.size(), last = nn - 1;
    S.num_nodes = nn;
    S.n = n;
    S.size.assign(nn, 0); S.off.assign(nn, 0); S.my_off.assign(nn, 0); S.parent.assign(nn, -1);
    S.sep_parent.assign(nn, -1); S.children.assign(2 * (size_t)nn, -1); S.on_left.assign(nn, 0);
    S.lower.assign(nn, {}); S.orig_lower.assign(nn, {}); S.orig_rel.assign(nn, {});
    S.left_rel.assign(nn, {}); S.right_rel.assign(nn, {}); S.inds.assign(nn, {});
    std::vector<int> subtree_end(nn);
    for (int old = 0; old < nn; ++old) {
        PreNode& p = B.nodes[old];
        const int s = last - old;
        S.size[s] = p.size; S.off[s] = p.off;
        if (nn == 1) { S.parent[s] = last - p.parent; S.sep_parent[s] = last - p.sep_parent; }
        else if (old == 0) { S.parent[s] = -1; S.sep_parent[s] = -1; }
        else { S.parent[s] = last - p.parent; S.sep_parent[s] = last - p.sep_parent; }
        if (p.nchild == 2) { S.children[2 * s] = last - p.child[0]; S.children[2 * s + 1] = last - p.child[1]; }
        S.inds[s] = std::move(p.inds);
        subtree_end[s] = p.subtree_end;
    }
    B.nodes.clear();

    // BuildMap at P=1
    S.map.assign(n, 0); S.inv_map.assign(n, 0);
    for (int s = 0; s < nn; ++s)
        for (size_t t = 0; t < S.inds[s].size(); ++t) S.map[S.inds[s][t]] = S.off[s] + (int)t;
    for (int64_t i = 0; i < n; ++i) S.inv_map[S.map[i]] = (int)i;

    // original lower structure from the global graph
    for (int s = 0; s < nn; ++s) {
        std::vector<int>& o = S.orig_lower[s];
        const int end = subtree_end[s];
        for (int v : S.inds[s])
            for (int64_t e = rowptr[v]; e < rowptr[v + 1]; ++e) {
                const int c = colind[e];
                if (c < 0 || c >= n) continue;
                const int t = S.map[c];
                if (t >= end) o.push_back(t);
            }
        std::sort(o.begin(), o.end());
        o.erase(std::unique(o.begin(), o.end()), o.end());
    }

    // LocalSymmetricAnalysis
    int my_off = 0;
    std::vector<int> cs, ps, fs, own;
    for (int s = 0; s < nn; ++s) {
        S.my_off[s] = my_off;
        const int l = S.children[2 * s], r = S.children[2 * s + 1];
        if (l >= 0) {
            S.on_left[l] = 1; S.on_left[r] = 0;
            sorted_union(S.lower[l], S.lower[r], cs);
            sorted_union(S.orig_lower[s], cs, ps);
            own.resize(S.size[s]);
            for (int i = 0; i < S.size[s]; ++i) own[i] = S.off[s] + i;
            sorted_union(ps, own, fs);
            relative_indices(S.orig_lower[s], fs, S.orig_rel[s]);
            relative_indices(S.lower[l], fs, S.left_rel[s]);
            relative_indices(S.lower[r], fs, S.right_rel[s]);
            S.lower[s].assign(fs.begin() + S.size[s], fs.end());
        } else {
            S.lower[s] = S.orig_lower[s];
            S.orig_rel[s].resize(S.orig_lower[s].size());
            for (size_t i = 0; i < S.orig_rel[s].size(); ++i) S.orig_rel[s][i] = (int)i + S.size[s];
        }
        my_off += S.size[s];
    }
    S.finalize_views();
    return CLIQ_OK;
}

int natural_nested_dissection(int nx, int ny, int nz, int64_t n, const int64_t* rowptr, const int32_t* colind,
                              int cutoff, Symbolic& S) {
    if (nx < 0 || ny < 0 || nz < 0 || (int64_t)nx * ny * nz != n || n <= 0 || !rowptr || !colind) return CLIQ_ERR_ARG;
    if (n > INT32_MAX / 2) return CLIQ_ERR_ARG;
    NDBuilder B{nx, ny, nz, cutoff, {}};
    B.recurse(Box{0, 0, 0, nx, ny, nz}, -1, 0);
    return finish_symbolic(B.nodes, n, rowptr, colind, S);
}

// ---------------------------------------------------------------------------
// NestedDissection for a general (structurally symmetric) graph at P=1.
// The recursion, node numbering and the rest of the analysis follow the
// reference (nested_dissection.hpp:115-230: a sub-graph of at most cutoff
// vertices is a leaf; otherwise a vertex separator splits it, the separator
// becomes the node, the right part is recursed on, then the left).  The
// reference bisects with METIS; this bisection is its own:
//   * a pseudo-peripheral start vertex (repeated breadth-first searches,
//     George & Liu) and its level structure; the level at which the count
//     of vertices reaches half is a vertex separator (edges join only equal
//     or adjacent levels);
//   * separator vertices with no neighbour on one side move to the other
//     (to the smaller side when they touch neither), which keeps the split
//     a separation and shrinks the separator;
//   * num_seps start vertices are tried (the reference's numSeqSeps) and the
//     smallest separator whose smaller side holds at least a fifth of the
//     vertices is kept;
//   * a disconnected sub-graph is split between its components (each whole
//     component to the side with fewer vertices so far) with an empty
//     separator;
//     a sub-graph with no useful separator (fewer than three levels, as in
//     a dense block) becomes a leaf.
// Vertices keep the order of the input within leaves, and breadth-first
// order within separators.
// ---------------------------------------------------------------------------
namespace {

struct GraphND {
    int64_t n;
    const int64_t* rp;
    const int32_t* ci;
    int cutoff, num_seps;
    std::vector<int> stamp_of, level, part, seen;
    int stamp = 0, visit = 0;
    std::vector<PreNode> nodes;

    // breadth-first level structure of the current sub-graph (stamp) from s:
    // order of visit; level[] set for the visited vertices
    int bfs(int s, std::vector<int>& order) {
        order.clear();
        order.push_back(s);
        level[s] = 0;
        seen[s] = ++visit;
        int depth = 0;
        for (size_t h = 0; h < order.size(); ++h) {
            const int v = order[h];
            depth = level[v];
            for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {
                const int t = ci[e];
                if (t < 0 || t >= n || stamp_of[t] != stamp || seen[t] == visit) continue;
                seen[t] = visit;
                level[t] = level[v] + 1;
                order.push_back(t);
            }
        }
        return depth;
    }

    // a disconnected sub-graph: its components (in the order of their first
    // vertex) assigned whole, each to the side holding fewer vertices so far;
    // no separator.  Returns false for a connected one.
    bool split_components(const std::vector<int>& verts, std::vector<int>& L, std::vector<int>& R) {
        std::vector<int> order;
        bfs(verts[0], order);
        if (order.size() == verts.size()) return false;
        const int first = visit;   // searches from here on label components
        for (int v : verts) {
            if (seen[v] >= first && seen[v] <= visit) continue;
            bfs(v, order);
        }
        // component sizes by their search number, then the assignment
        std::vector<int> size(visit - first + 1, 0);
        for (int v : verts) ++size[seen[v] - first];
        std::vector<char> left(size.size(), 0);
        int64_t nl = 0, nr = 0;
        for (size_t c = 0; c < size.size(); ++c) {   // each component to the smaller side so far
            if (nl <= nr) { left[c] = 1; nl += size[c]; }
            else nr += size[c];
        }
        for (int v : verts) (left[seen[v] - first] ? L : R).push_back(v);
        return !L.empty() && !R.empty();
    }

    int degree_in(int v) const {
        int d = 0;
        for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {
            const int t = ci[e];
            if (t >= 0 && t < n && stamp_of[t] == stamp && t != v) ++d;
        }
        return d;
    }

    // one separator attempt from start vertex s0; returns false when no
    // useful split exists.  part[] = 0 left, 1 right, 2 separator
    bool attempt(const std::vector<int>& verts, int s0, std::vector<int>& order, int& sep_size, int& small) {
        int s = s0, ecc = bfs(s, order);
        for (int it = 0; it < 8; ++it) {   // pseudo-peripheral vertex
            int best = -1, bd = INT32_MAX;
            for (size_t h = order.size(); h-- > 0;) {
                const int v = order[h];
                if (level[v] != ecc) break;
                const int d = degree_in(v);
                if (d < bd) { bd = d; best = v; }
            }
            std::vector<int> o2;
            const int e2 = bfs(best, o2);
            if (e2 <= ecc) { bfs(s, order); break; }
            s = best; ecc = e2; order.swap(o2);
        }
        const int cnt = (int)verts.size();
        std::vector<int> per(ecc + 1, 0);
        for (int v : order) ++per[level[v]];
        int lsep = 0, acc = 0;
        while (lsep <= ecc && acc + per[lsep] < cnt / 2) acc += per[lsep++];
        if (lsep == 0 && ecc > 0) lsep = 1;
        if (lsep >= ecc) lsep = ecc - 1;
        if (lsep <= 0) return false;   // no level strictly inside the structure
        int nl = 0, nr = 0;
        std::vector<int> sep;
        for (int v : order) {
            if (level[v] < lsep) { part[v] = 0; ++nl; }
            else if (level[v] > lsep) { part[v] = 1; ++nr; }
            else { part[v] = 2; sep.push_back(v); }
        }
        if (nl == 0 || nr == 0) return false;
        for (int v : sep) {   // shrink: a vertex touching one side only joins it
            bool hl = false, hr = false;
            for (int64_t e = rp[v]; e < rp[v + 1]; ++e) {
                const int t = ci[e];
                if (t < 0 || t >= n || stamp_of[t] != stamp || t == v) continue;
                if (part[t] == 0) hl = true;
                else if (part[t] == 1) hr = true;
            }
            if (!hr && (!hl || nl <= nr)) { part[v] = 0; ++nl; }
            else if (!hl) { part[v] = 1; ++nr; }
        }
        sep_size = cnt - nl - nr;
        small = std::min(nl, nr);
        return true;
    }

    void leaf(std::vector<int>& verts, int parent, int off, int id) {
        PreNode& nd = nodes[id];
        nd.size = (int)verts.size(); nd.off = off; nd.parent = parent; nd.sep_parent = parent;
        nd.inds = std::move(verts);
        nd.subtree_end = off + nd.size;
    }

    void recurse(std::vector<int>& verts, int parent, int off) {
        const int cnt = (int)verts.size();
        const int id = (int)nodes.size();
        nodes.emplace_back();
        if (cnt <= cutoff) { leaf(verts, parent, off, id); return; }
        ++stamp;
        for (int v : verts) stamp_of[v] = stamp;
        {
            std::vector<int> L, R;
            if (split_components(verts, L, R)) {   // empty separator
                verts.clear();
                verts.shrink_to_fit();
                const int nl = (int)L.size(), nr = (int)R.size();
                PreNode& nd = nodes[id];
                nd.size = 0; nd.off = off + nl + nr; nd.parent = parent; nd.sep_parent = parent;
                nd.nchild = 2; nd.subtree_end = off + cnt;
                nodes[id].child[1] = (int)nodes.size();
                recurse(R, id, off + nl);
                nodes[id].child[0] = (int)nodes.size();
                recurse(L, id, off);
                return;
            }
        }
        // tries: the first vertex, then vertices spread over the input order
        std::vector<int> order, best_part;
        int best_sep = INT32_MAX, best_small = -1;
        for (int t = 0; t < std::max(1, num_seps); ++t) {
            const int s0 = verts[(size_t)((int64_t)t * cnt / std::max(1, num_seps))];
            int sep_size = 0, small = 0;
            if (!attempt(verts, s0, order, sep_size, small)) continue;
            const bool balanced = 5 * small >= cnt, best_balanced = 5 * best_small >= cnt;
            if (best_small < 0 || (balanced && !best_balanced) ||
                (balanced == best_balanced && (sep_size < best_sep || (sep_size == best_sep && small > best_small)))) {
                best_sep = sep_size; best_small = small;
                best_part.resize(cnt);
                for (int i = 0; i < cnt; ++i) best_part[i] = part[verts[i]];
            }
        }
        if (best_small <= 0) { leaf(verts, parent, off, id); return; }   // no useful split
        std::vector<int> L, R, sep;
        for (int i = 0; i < cnt; ++i) (best_part[i] == 0 ? L : best_part[i] == 1 ? R : sep).push_back(verts[i]);
        if (L.empty() || R.empty()) { leaf(verts, parent, off, id); return; }
        verts.clear();
        verts.shrink_to_fit();
        const int nl = (int)L.size(), nr = (int)R.size();
        {
            PreNode& nd = nodes[id];
            nd.size = (int)sep.size();
            nd.off = off + nl + nr;
            nd.parent = parent; nd.sep_parent = parent;
            nd.nchild = 2;
            nd.inds = std::move(sep);
            nd.subtree_end = off + cnt;
        }
        nodes[id].child[1] = (int)nodes.size();
        recurse(R, id, off + nl);
        nodes[id].child[0] = (int)nodes.size();
        recurse(L, id, off);
    }
};

}  // namespace

int graph_nested_dissection(int64_t n, const int64_t* rowptr, const int32_t* colind, int cutoff, int num_seps, Symbolic& S) {
    if (n <= 0 || !rowptr || !colind || n > INT32_MAX / 2) return CLIQ_ERR_ARG;
    GraphND G{n, rowptr, colind, std::max(1, cutoff), std::max(1, num_seps), {}, {}, {}, {}, 0, 0, {}};
    G.stamp_of.assign(n, 0);
    G.level.assign(n, 0);
    G.part.assign(n, 0);
    G.seen.assign(n, 0);
    std::vector<int> all(n);
    for (int64_t i = 0; i < n; ++i) all[i] = (int)i;
    G.recurse(all, -1, 0);
    return finish_symbolic(G.nodes, n, rowptr, colind, S);
}

// Forest of independent grid problems: the block-diagonal matrix whose
// diagonal block p is problem p (rows rowoff_p .. rowoff_p + n_p - 1, natural
// order within the block).  Each block gets its own natural nested
// dissection; the union numbers problem p's nodes after those of problems
// 0 .. p-1 and its ND indices after theirs (ND block p = natural block p), so
// the forest is in post-order with every root's parent -1.  No reference
// counterpart (Clique factors one matrix per tree).
int batch_nested_dissection(int count, const int32_t* dims, int64_t n, const int64_t* rowptr, const int32_t* colind,
                            int cutoff, Symbolic& S) {
    if (count <= 0 || !dims || !rowptr || !colind || n <= 0 || n > INT32_MAX / 2) return CLIQ_ERR_ARG;
    S = Symbolic{};
    S.n = n;
    S.map.assign(n, 0);
    S.inv_map.assign(n, 0);
    int64_t r0 = 0;
    for (int p = 0; p < count; ++p) {
        const int nx = dims[3 * p], ny = dims[3 * p + 1], nz = dims[3 * p + 2];
        const int64_t np = (int64_t)nx * ny * nz;
        if (nx <= 0 || ny <= 0 || nz <= 0 || r0 + np > n) {
            set_last_error("batch_nested_dissection: problem sizes do not match the matrix");
            return CLIQ_ERR_ARG;
        }
        // the diagonal block of problem p, with block-local column indices
        std::vector<int64_t> rp(np + 1);
        std::vector<int32_t> ci(rowptr[r0 + np] - rowptr[r0]);
        for (int64_t i = 0; i <= np; ++i) rp[i] = rowptr[r0 + i] - rowptr[r0];
        for (size_t e = 0; e < ci.size(); ++e) {
            const int64_t c = colind[rowptr[r0] + (int64_t)e] - r0;
            if (c < 0 || c >= np) {
                set_last_error("batch_nested_dissection: the matrix is not block diagonal in the problems' rows");
                return CLIQ_ERR_ARG;
            }
            ci[e] = (int32_t)c;
        }
        Symbolic Q;
        const int st = natural_nested_dissection(nx, ny, nz, np, rp.data(), ci.data(), cutoff, Q);
        if (st != CLIQ_OK) return st;
        const int n0 = S.num_nodes, nq = Q.num_nodes, off = (int)r0;
        auto node = [&](int t) { return (t >= 0 && t < nq) ? t + n0 : -1; };   // parents outside the problem: none
        auto shift = [&](std::vector<int>& v) { for (int& x : v) x += off; };
        for (int t = 0; t < nq; ++t) {
            S.size.push_back(Q.size[t]);
            S.off.push_back(Q.off[t] + off);
            S.my_off.push_back(Q.my_off[t] + off);
            S.parent.push_back(node(Q.parent[t]));
            S.sep_parent.push_back(node(Q.sep_parent[t]));
            S.children.push_back(node(Q.children[2 * t]));
            S.children.push_back(node(Q.children[2 * t + 1]));
            S.on_left.push_back(Q.on_left[t]);
            shift(Q.lower[t]);
            shift(Q.orig_lower[t]);
            shift(Q.inds[t]);
            S.lower.push_back(std::move(Q.lower[t]));
            S.orig_lower.push_back(std::move(Q.orig_lower[t]));
            S.orig_rel.push_back(std::move(Q.orig_rel[t]));
            S.left_rel.push_back(std::move(Q.left_rel[t]));
            S.right_rel.push_back(std::move(Q.right_rel[t]));
            S.inds.push_back(std::move(Q.inds[t]));
        }
        for (int64_t i = 0; i < np; ++i) {
            S.map[r0 + i] = Q.map[i] + off;
            S.inv_map[r0 + i] = Q.inv_map[i] + off;
        }
        S.num_nodes += nq;
        r0 += np;
    }
    if (r0 != n) {
        set_last_error("batch_nested_dissection: the problems do not cover the matrix");
        return CLIQ_ERR_ARG;
    }
    S.finalize_views();
    return CLIQ_OK;
}

void Symbolic::finalize_views() {
    lower_ptr.assign(num_nodes + 1, 0);
    orig_ptr.assign(num_nodes + 1, 0);
    for (int s = 0; s < num_nodes; ++s) {
        lower_ptr[s + 1] = lower_ptr[s] + (int64_t)lower[s].size();
        orig_ptr[s + 1] = orig_ptr[s] + (int64_t)orig_lower[s].size();
    }
    lower_flat.resize(lower_ptr[num_nodes]);
    orig_flat.resize(orig_ptr[num_nodes]);
    for (int s = 0; s < num_nodes; ++s) {
        std::copy(lower[s].begin(), lower[s].end(), lower_flat.begin() + lower_ptr[s]);
        std::copy(orig_lower[s].begin(), orig_lower[s].end(), orig_flat.begin() + orig_ptr[s]);
    }
}

}  // namespace cliqgpu
