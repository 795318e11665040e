/*
 * CPU oracle for the multifrontal LDL^T hot path of Clique (poulson/Clique).
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the reference's
 * single-process algorithm so that the GPU product can be checked against it
 * and so that the reference's CPU path can be timed.  Only tests/, the smoke
 * check and bench.py's cpu_baseline / reference arm may load it.  The product
 * (clique_b200/) never links or calls it.
 *
 * Parity status: the reference's numeric path is header-only C++ over the
 * Elemental library, whose submodule is empty in the reference checkout, so
 * the reference itself cannot be compiled here.  This restatement is pinned
 * against mathematics instead: dense unpivoted LDL^T of the permuted matrix
 * (L and D entry by entry), dense solves, and hand-derived orderings of tiny
 * grids (tests/golden/).  The reference's own tests assert no values.
 *
 * What is restated, with the reference file each part follows:
 *   natural nested dissection ... include/clique/symbolic/natural_nested_dissection.hpp:60-189,313-445,447-488,490-619
 *   child graphs ................ include/clique/symbolic/nested_dissection.hpp:888-963 (BuildChildrenFromPerm)
 *   post-order reversal ......... include/clique/symbolic/nested_dissection.hpp:817-886 (ReverseOrder)
 *   ordering map ................ include/clique/symbolic/nested_dissection.hpp:1206-1363 (BuildMap, P=1)
 *   symbolic analysis ........... src/symbolic/LocalSymmetricAnalysis.cpp:15-114
 *   set helpers ................. include/clique/core/environment/impl.hpp:95-162 (Union, RelativeIndices, Find)
 *   front assembly .............. include/clique/numeric/dist_symm_front_tree/impl.hpp:244-297
 *   multifrontal factor ......... include/clique/numeric/ldl/local.hpp:25-122 (LocalLDL)
 *   dense partial front LDL^T ... include/clique/numeric/ldl/local_front.hpp:30-71 (FrontLDL)
 *   pivoted front LDL^T ......... include/clique/numeric/ldl/local_front.hpp:74-94 (FrontLDLIntraPiv;
 *                                 Bunch-Kaufman partial pivoting restated from its publication)
 *   pivoted block front ......... include/clique/numeric/ldl/local_front_block.hpp:36-58
 *   pivoted front solves ........ include/clique/numeric/lower_solve/local_front.hpp:53-93,
 *                                 include/clique/numeric/diagonal_solve.hpp:53-59 (QuasiDiagonalSolve)
 *   forward / backward sweeps ... include/clique/numeric/lower_solve/local.hpp:42-119,203-277
 *   front triangular solves ..... include/clique/numeric/lower_solve/local_front.hpp:36-82
 *   root backward solve (P=1) ... include/clique/numeric/lower_solve/dist.hpp:374-387
 *   diagonal solve .............. include/clique/numeric/diagonal_solve.hpp:49-69
 *   solve driver ................ include/clique/numeric/solve.hpp:41-65
 *   nodal pull / push ........... include/clique/numeric/dist_nodal_multi_vec/impl.hpp:67-219 (P=1)
 *   sparse multiply ............. include/clique/numeric/multiply.hpp:28-166
 *
 * Dense kernels (Elemental's LDL, Trsm, Gemm, Trrk, DiagonalSolve) are
 * restated from their definitions.  When a CBLAS library is registered with
 * orc_set_blas() (the OpenBLAS bundled with numpy, ILP64 symbol names
 * scipy_cblas_*64_), GEMM / TRSM / GEMMT go through it, as Elemental's do;
 * otherwise plain loops are used.  Both are exercised by the tests.
 */
#include <complex.h>
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;
typedef double complex zd;

#define XMALLOC(T, n) ((T*)xmalloc(sizeof(T) * (size_t)((n) > 0 ? (n) : 1)))
static void* xmalloc(size_t b) {
    void* p = malloc(b);
    if (!p) { fprintf(stderr, "oracle: out of memory (%zu bytes)\n", b); abort(); }
    return p;
}
static void* xcalloc(size_t n, size_t sz) {
    void* p = calloc(n ? n : 1, sz);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}

/* ------------------------------------------------------------------------ */
/* Growable int vector                                                       */
/* ------------------------------------------------------------------------ */
typedef struct { int* a; i64 n, cap; } ivec;
static void iv_push(ivec* v, int x) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 16; v->a = (int*)realloc(v->a, sizeof(int) * v->cap); }
    v->a[v->n++] = x;
}
static int cmp_int(const void* a, const void* b) { int x = *(const int*)a, y = *(const int*)b; return (x > y) - (x < y); }
/* sort + unique, the effect of inserting into a std::set */
static void iv_sort_unique(ivec* v) {
    if (v->n == 0) return;
    qsort(v->a, v->n, sizeof(int), cmp_int);
    i64 w = 0;
    for (i64 r = 1; r < v->n; ++r) if (v->a[r] != v->a[w]) v->a[++w] = v->a[r];
    v->n = w + 1;
}

/* Union of two sorted vectors (std::set_union), environment/impl.hpp:95-104 */
static ivec set_union(const int* a, i64 na, const int* b, i64 nb) {
    ivec r = {0, 0, 0};
    i64 i = 0, j = 0;
    while (i < na || j < nb) {
        if (j >= nb || (i < na && a[i] < b[j])) iv_push(&r, a[i++]);
        else if (i >= na || b[j] < a[i]) iv_push(&r, b[j++]);
        else { iv_push(&r, a[i]); ++i; ++j; }
    }
    return r;
}
/* RelativeIndices (lower_bound walk), environment/impl.hpp:114-131 */
static int* relative_indices(const int* sub, i64 nsub, const int* full, i64 nfull) {
    int* rel = XMALLOC(int, nsub);
    i64 it = 0;
    for (i64 i = 0; i < nsub; ++i) {
        i64 lo = it, hi = nfull;
        while (lo < hi) { i64 mid = (lo + hi) / 2; if (full[mid] < sub[i]) lo = mid + 1; else hi = mid; }
        it = lo;
        rel[i] = (int)it;
    }
    return rel;
}
/* Find (lower_bound), environment/impl.hpp:150-162 */
static i64 find_sorted(const int* a, i64 n, int x) {
    i64 lo = 0, hi = n;
    while (lo < hi) { i64 mid = (lo + hi) / 2; if (a[mid] < x) lo = mid + 1; else hi = mid; }
    return lo;
}

/* ------------------------------------------------------------------------ */
/* Sequential graph in CSR form (the reference's Graph after StopAssembly:   */
/* sorted, duplicate-free edges, targets may exceed numSources)              */
/* ------------------------------------------------------------------------ */
typedef struct { int n; i64* ptr; int* tgt; } graph_t;
static void graph_free(graph_t* g) { free(g->ptr); free(g->tgt); g->ptr = 0; g->tgt = 0; }

/* ------------------------------------------------------------------------ */
/* Symbolic structures                                                       */
/* ------------------------------------------------------------------------ */
typedef struct {
    int size, off, parent;
    int nchild, child[2];
    ivec lower;        /* SymmNode::lowerStruct as built by ND (original structure) */
    ivec inds;         /* SepOrLeaf::inds (natural indices) */
    int sep_parent;    /* SepOrLeaf::parent */
} pnode;              /* pre-order node */

typedef struct {
    int num_nodes;
    i64 N;
    int* size; int* off; int* my_off; int* parent; int* nchild; int* child; /* child: 2 per node */
    int* on_left;
    ivec* lower;       /* analysed lowerStruct */
    ivec* orig;        /* origLowerStruct */
    int** orig_rel; int** left_rel; int** right_rel;
    i64* n_left_rel; i64* n_right_rel;
    ivec* inds;        /* separator / leaf natural indices */
    int* sep_parent;
    int* map;          /* natural -> ND */
    int* inv_map;      /* ND -> natural */
} oracle_symb;

typedef struct { pnode* a; int n, cap; } pnode_list;
static int pl_push(pnode_list* l) {
    if (l->n == l->cap) { l->cap = l->cap ? 2 * l->cap : 64; l->a = (pnode*)realloc(l->a, sizeof(pnode) * l->cap); }
    memset(&l->a[l->n], 0, sizeof(pnode));
    return l->n++;
}

/* BuildChildrenFromPerm, nested_dissection.hpp:888-963 */
static void build_children(const graph_t* g, const int* perm, int nl, graph_t* L, int nr, graph_t* R) {
    const int n = g->n;
    int* inv = XMALLOC(int, n);
    for (int i = 0; i < n; ++i) inv[perm[i]] = i;
    graph_t* out[2] = {L, R};
    int sizes[2] = {nl, nr}, base[2] = {0, nl};
    for (int c = 0; c < 2; ++c) {
        graph_t* G = out[c];
        G->n = sizes[c];
        G->ptr = XMALLOC(i64, sizes[c] + 1);
        i64 cap = 0;
        for (int s = 0; s < sizes[c]; ++s) cap += g->ptr[inv[s + base[c]] + 1] - g->ptr[inv[s + base[c]]];
        G->tgt = XMALLOC(int, cap);
        i64 e = 0;
        G->ptr[0] = 0;
        for (int s = 0; s < sizes[c]; ++s) {
            const int src = inv[s + base[c]];
            i64 start = e;
            for (i64 k = g->ptr[src]; k < g->ptr[src + 1]; ++k) {
                int it = g->tgt[k];
                int t = (it < n ? perm[it] : it) - base[c];
                G->tgt[e++] = t;
            }
            /* Graph::StopAssembly sorts and compresses duplicates */
            qsort(G->tgt + start, e - start, sizeof(int), cmp_int);
            i64 w = start;
            for (i64 r = start; r < e; ++r) if (r == start || G->tgt[r] != G->tgt[w - 1]) G->tgt[w++] = G->tgt[r];
            e = w;
            G->ptr[s + 1] = e;
        }
    }
    free(inv);
}

/* NaturalBisect, natural_nested_dissection.hpp:490-619 */
static int natural_bisect(int nx, int ny, int nz, const graph_t* g,
                          int* nxL, int* nyL, int* nzL, graph_t* L,
                          int* nxR, int* nyR, int* nzR, graph_t* R, int* perm) {
    int nl, nr, sep, off;
    if (nx >= ny && nx >= nz) {
        *nxL = (nx - 1) / 2; *nyL = ny; *nzL = nz; nl = (*nxL) * ny * nz;
        *nxR = nx - 1 - *nxL; *nyR = ny; *nzR = nz; nr = (*nxR) * ny * nz;
        sep = ny * nz;
        off = 0;
        for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < *nxL; ++x) perm[x + y * nx + z * nx * ny] = off++;
        off = nl;
        for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = *nxL + 1; x < nx; ++x) perm[x + y * nx + z * nx * ny] = off++;
        off = nl + nr;
        for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) perm[*nxL + y * nx + z * nx * ny] = off++;
    } else if (ny >= nx && ny >= nz) {
        *nxL = nx; *nyL = (ny - 1) / 2; *nzL = nz; nl = nx * (*nyL) * nz;
        *nxR = nx; *nyR = ny - 1 - *nyL; *nzR = nz; nr = nx * (*nyR) * nz;
        sep = nx * nz;
        off = 0;
        for (int z = 0; z < nz; ++z) for (int y = 0; y < *nyL; ++y) for (int x = 0; x < nx; ++x) perm[x + y * nx + z * nx * ny] = off++;
        off = nl;
        for (int z = 0; z < nz; ++z) for (int y = *nyL + 1; y < ny; ++y) for (int x = 0; x < nx; ++x) perm[x + y * nx + z * nx * ny] = off++;
        off = nl + nr;
        for (int z = 0; z < nz; ++z) for (int x = 0; x < nx; ++x) perm[x + (*nyL) * nx + z * nx * ny] = off++;
    } else {
        *nxL = nx; *nyL = ny; *nzL = (nz - 1) / 2; nl = nx * ny * (*nzL);
        *nxR = nx; *nyR = ny; *nzR = nz - 1 - *nzL; nr = nx * ny * (*nzR);
        sep = nx * ny;
        off = 0;
        for (int z = 0; z < *nzL; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) perm[x + y * nx + z * nx * ny] = off++;
        off = nl;
        for (int z = *nzL + 1; z < nz; ++z) for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) perm[x + y * nx + z * nx * ny] = off++;
        off = nl + nr;
        for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) perm[x + y * nx + (*nzL) * nx * ny] = off++;
    }
    build_children(g, perm, nl, L, nr, R);
    return sep;
}

/* connectedAncestors of a set of local sources (targets >= numSources) */
static void connected_ancestors(const graph_t* g, const int* srcs, int nsrc, int off, ivec* out) {
    out->n = 0;
    for (int s = 0; s < nsrc; ++s) {
        int src = srcs ? srcs[s] : s;
        for (i64 k = g->ptr[src]; k < g->ptr[src + 1]; ++k)
            if (g->tgt[k] >= g->n) iv_push(out, off + g->tgt[k]);
    }
    iv_sort_unique(out);
}

/* NaturalNestedDissectionRecursion (sequential graph), natural_nested_dissection.hpp:60-189.
 * The P=1 top level (the DistGraph overload, :313-445) differs only in that
 * the root's parent is -1 and its children are recursed with parent 0; the
 * sequential overload produces the same values when called with parent=-1
 * at the root, because the root is node 0. */
static void nd_recursion(int nx, int ny, int nz, graph_t* g, int* perm, pnode_list* nodes, int parent, int off, int cutoff) {
    if (g->n <= cutoff) {
        int id = pl_push(nodes);
        pnode* nd = &nodes->a[id];
        nd->sep_parent = parent;
        nd->off = off;
        for (int s = 0; s < g->n; ++s) iv_push(&nd->inds, perm[s]);
        nd->size = g->n;
        nd->parent = parent;
        nd->nchild = 0;
        connected_ancestors(g, NULL, g->n, off, &nd->lower);
        return;
    }
    int nxL, nyL, nzL, nxR, nyR, nzR;
    graph_t L = {0, 0, 0}, R = {0, 0, 0};
    int* map = XMALLOC(int, g->n);
    const int sep = natural_bisect(nx, ny, nz, g, &nxL, &nyL, &nzL, &L, &nxR, &nyR, &nzR, &R, map);
    const int n = g->n;
    int* inv = XMALLOC(int, n);
    for (int s = 0; s < n; ++s) inv[map[s]] = s;

    int id = pl_push(nodes);
    {
        pnode* nd = &nodes->a[id];
        nd->sep_parent = parent;
        nd->off = off + (n - sep);
        int* sepinds = XMALLOC(int, sep);
        for (int s = 0; s < sep; ++s) sepinds[s] = inv[s + (n - sep)];
        nd->size = sep;
        nd->parent = parent;
        nd->nchild = 2;
        connected_ancestors(g, sepinds, sep, off, &nd->lower);
        for (int s = 0; s < sep; ++s) iv_push(&nd->inds, perm[sepinds[s]]);
        free(sepinds);
    }
    const int nl = L.n, nr = R.n;
    int* lperm = XMALLOC(int, nl);
    int* rperm = XMALLOC(int, nr);
    for (int s = 0; s < nl; ++s) lperm[s] = perm[inv[s]];
    for (int s = 0; s < nr; ++s) rperm[s] = perm[inv[s + nl]];
    free(map); free(inv);
    graph_free(g);   /* the parent graph is no longer needed */

    /* right first, then left, so that after reversal the left comes first */
    nodes->a[id].child[1] = nodes->n;
    nd_recursion(nxR, nyR, nzR, &R, rperm, nodes, id, off + nl, cutoff);
    nodes->a[id].child[0] = nodes->n;
    nd_recursion(nxL, nyL, nzL, &L, lperm, nodes, id, off, cutoff);
    graph_free(&L); graph_free(&R);
    free(lperm); free(rperm);
}

void orc_symb_free(oracle_symb* S);

oracle_symb* orc_natural_nd(int nx, int ny, int nz, i64 N, const i64* rowptr, const int* colind, int cutoff) {
    if ((i64)nx * ny * nz != N) return NULL;
    graph_t g;
    g.n = (int)N;
    g.ptr = XMALLOC(i64, N + 1);
    memcpy(g.ptr, rowptr, sizeof(i64) * (N + 1));
    g.tgt = XMALLOC(int, rowptr[N]);
    memcpy(g.tgt, colind, sizeof(int) * rowptr[N]);
    for (i64 i = 0; i < N; ++i) {           /* sorted, unique per row */
        qsort(g.tgt + g.ptr[i], g.ptr[i + 1] - g.ptr[i], sizeof(int), cmp_int);
    }
    int* perm = XMALLOC(int, N);
    for (i64 i = 0; i < N; ++i) perm[i] = (int)i;
    pnode_list nodes = {0, 0, 0};
    nd_recursion(nx, ny, nz, &g, perm, &nodes, -1, 0, cutoff);
    free(perm);
    graph_free(&g);

    /* ReverseOrder, nested_dissection.hpp:817-886: new index = last - old.
     * Every parent index is mapped the same way except the root's (-1),
     * which is only kept when there is more than one node. */
    const int nn = nodes.n, last = nn - 1;
    oracle_symb* S = (oracle_symb*)xcalloc(1, sizeof(oracle_symb));
    S->num_nodes = nn; S->N = N;
    S->size = XMALLOC(int, nn); S->off = XMALLOC(int, nn); S->my_off = XMALLOC(int, nn);
    S->parent = XMALLOC(int, nn); S->nchild = XMALLOC(int, nn); S->child = XMALLOC(int, 2 * nn);
    S->on_left = (int*)xcalloc(nn, sizeof(int));
    S->lower = (ivec*)xcalloc(nn, sizeof(ivec)); S->orig = (ivec*)xcalloc(nn, sizeof(ivec));
    S->orig_rel = (int**)xcalloc(nn, sizeof(int*)); S->left_rel = (int**)xcalloc(nn, sizeof(int*));
    S->right_rel = (int**)xcalloc(nn, sizeof(int*));
    S->n_left_rel = (i64*)xcalloc(nn, sizeof(i64)); S->n_right_rel = (i64*)xcalloc(nn, sizeof(i64));
    S->inds = (ivec*)xcalloc(nn, sizeof(ivec)); S->sep_parent = XMALLOC(int, nn);
    for (int old = 0; old < nn; ++old) {
        pnode* p = &nodes.a[old];
        const int s = last - old;
        S->size[s] = p->size; S->off[s] = p->off;
        if (nn == 1) { S->parent[s] = last - p->parent; S->sep_parent[s] = last - p->sep_parent; }
        else if (old == 0) { S->parent[s] = p->parent; S->sep_parent[s] = p->sep_parent; }
        else { S->parent[s] = last - p->parent; S->sep_parent[s] = last - p->sep_parent; }
        S->nchild[s] = p->nchild;
        S->child[2 * s] = p->nchild ? last - p->child[0] : -1;
        S->child[2 * s + 1] = p->nchild ? last - p->child[1] : -1;
        S->orig[s] = p->lower;   /* take ownership */
        S->inds[s] = p->inds;
    }
    free(nodes.a);

    /* BuildMap (P=1): map[inds[t]] = off + t */
    S->map = XMALLOC(int, N);
    S->inv_map = XMALLOC(int, N);
    for (int s = 0; s < nn; ++s)
        for (i64 t = 0; t < S->inds[s].n; ++t) S->map[S->inds[s].a[t]] = S->off[s] + (int)t;
    for (i64 i = 0; i < N; ++i) S->inv_map[S->map[i]] = (int)i;

    /* LocalSymmetricAnalysis, LocalSymmetricAnalysis.cpp:15-114 */
    int my_off = 0;
    for (int s = 0; s < nn; ++s) {
        S->my_off[s] = my_off;
        if (S->nchild[s] == 2) {
            const int l = S->child[2 * s], r = S->child[2 * s + 1];
            S->on_left[l] = 1; S->on_left[r] = 0;
            ivec cs = set_union(S->lower[l].a, S->lower[l].n, S->lower[r].a, S->lower[r].n);
            ivec ps = set_union(S->orig[s].a, S->orig[s].n, cs.a, cs.n);
            int* own = XMALLOC(int, S->size[s]);
            for (int i = 0; i < S->size[s]; ++i) own[i] = S->off[s] + i;
            ivec fs = set_union(ps.a, ps.n, own, S->size[s]);
            free(own); free(cs.a); free(ps.a);
            S->orig_rel[s] = relative_indices(S->orig[s].a, S->orig[s].n, fs.a, fs.n);
            S->left_rel[s] = relative_indices(S->lower[l].a, S->lower[l].n, fs.a, fs.n);
            S->n_left_rel[s] = S->lower[l].n;
            S->right_rel[s] = relative_indices(S->lower[r].a, S->lower[r].n, fs.a, fs.n);
            S->n_right_rel[s] = S->lower[r].n;
            ivec low = {0, 0, 0};
            for (i64 i = S->size[s]; i < fs.n; ++i) iv_push(&low, fs.a[i]);
            S->lower[s] = low;
            free(fs.a);
        } else {
            ivec low = {0, 0, 0};
            for (i64 i = 0; i < S->orig[s].n; ++i) iv_push(&low, S->orig[s].a[i]);
            S->lower[s] = low;
            S->orig_rel[s] = XMALLOC(int, S->orig[s].n);
            for (i64 i = 0; i < S->orig[s].n; ++i) S->orig_rel[s][i] = (int)i + S->size[s];
        }
        my_off += S->size[s];
    }
    return S;
}

void orc_symb_free(oracle_symb* S) {
    if (!S) return;
    for (int s = 0; s < S->num_nodes; ++s) {
        free(S->lower[s].a); free(S->orig[s].a); free(S->orig_rel[s]);
        free(S->left_rel[s]); free(S->right_rel[s]); free(S->inds[s].a);
    }
    free(S->size); free(S->off); free(S->my_off); free(S->parent); free(S->nchild); free(S->child);
    free(S->on_left); free(S->lower); free(S->orig); free(S->orig_rel); free(S->left_rel);
    free(S->right_rel); free(S->n_left_rel); free(S->n_right_rel); free(S->inds); free(S->sep_parent);
    free(S->map); free(S->inv_map); free(S);
}

int orc_num_nodes(const oracle_symb* S) { return S->num_nodes; }
/* out[0..9] = size, off, myOff, parent, child0, child1, onLeft, |lowerStruct|, |origLowerStruct|, sepParent */
void orc_node_info(const oracle_symb* S, int s, int* out) {
    out[0] = S->size[s]; out[1] = S->off[s]; out[2] = S->my_off[s]; out[3] = S->parent[s];
    out[4] = S->child[2 * s]; out[5] = S->child[2 * s + 1]; out[6] = S->on_left[s];
    out[7] = (int)S->lower[s].n; out[8] = (int)S->orig[s].n; out[9] = S->sep_parent[s];
}
/* which: 0 lowerStruct, 1 origLowerStruct, 2 origLowerRelInds, 3 leftRelInds, 4 rightRelInds, 5 inds.
 * Returns the length; copies into out when out != NULL. */
i64 orc_node_array(const oracle_symb* S, int s, int which, int* out) {
    const int* src = NULL; i64 n = 0;
    switch (which) {
        case 0: src = S->lower[s].a; n = S->lower[s].n; break;
        case 1: src = S->orig[s].a; n = S->orig[s].n; break;
        case 2: src = S->orig_rel[s]; n = S->orig[s].n; break;
        case 3: src = S->left_rel[s]; n = S->nchild[s] ? S->n_left_rel[s] : 0; break;
        case 4: src = S->right_rel[s]; n = S->nchild[s] ? S->n_right_rel[s] : 0; break;
        case 5: src = S->inds[s].a; n = S->inds[s].n; break;
        default: return -1;
    }
    if (out && n) memcpy(out, src, sizeof(int) * n);
    return n;
}
void orc_map(const oracle_symb* S, int* map_out, int* inv_out) {
    if (map_out) memcpy(map_out, S->map, sizeof(int) * S->N);
    if (inv_out) memcpy(inv_out, S->inv_map, sizeof(int) * S->N);
}

/* ------------------------------------------------------------------------ */
/* Optional CBLAS (ILP64 OpenBLAS bundled with numpy)                        */
/* ------------------------------------------------------------------------ */
enum { CB_COL = 102, CB_N = 111, CB_T = 112, CB_C = 113, CB_UP = 121, CB_LO = 122, CB_NU = 131, CB_U = 132, CB_L = 141, CB_R = 142 };
typedef void (*gemm_d_t)(int, int, int, i64, i64, i64, double, const double*, i64, const double*, i64, double, double*, i64);
typedef void (*gemmt_d_t)(int, int, int, int, i64, i64, double, const double*, i64, const double*, i64, double, double*, i64);
typedef void (*trsm_d_t)(int, int, int, int, int, i64, i64, double, const double*, i64, double*, i64);
typedef void (*gemm_z_t)(int, int, int, i64, i64, i64, const void*, const void*, i64, const void*, i64, const void*, void*, i64);
typedef void (*gemmt_z_t)(int, int, int, int, i64, i64, const void*, const void*, i64, const void*, i64, const void*, void*, i64);
typedef void (*trsm_z_t)(int, int, int, int, int, i64, i64, const void*, const void*, i64, void*, i64);
typedef void (*setthr_t)(int);
static struct {
    void* h; gemm_d_t dgemm; gemmt_d_t dgemmt; trsm_d_t dtrsm; gemm_z_t zgemm; gemmt_z_t zgemmt; trsm_z_t ztrsm;
} blas;

/* Register (or with path=NULL, unregister) a CBLAS library; nthreads>0 sets its thread count. */
int orc_set_blas(const char* path, int nthreads) {
    if (!path) { memset(&blas, 0, sizeof(blas)); return 0; }
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return -1;
    blas.h = h;
    blas.dgemm = (gemm_d_t)dlsym(h, "scipy_cblas_dgemm64_");
    blas.dgemmt = (gemmt_d_t)dlsym(h, "scipy_cblas_dgemmt64_");
    blas.dtrsm = (trsm_d_t)dlsym(h, "scipy_cblas_dtrsm64_");
    blas.zgemm = (gemm_z_t)dlsym(h, "scipy_cblas_zgemm64_");
    blas.zgemmt = (gemmt_z_t)dlsym(h, "scipy_cblas_zgemmt64_");
    blas.ztrsm = (trsm_z_t)dlsym(h, "scipy_cblas_ztrsm64_");
    setthr_t st = (setthr_t)dlsym(h, "scipy_openblas_set_num_threads64_");
    if (!(blas.dgemm && blas.dgemmt && blas.dtrsm && blas.zgemm && blas.zgemmt && blas.ztrsm)) {
        memset(&blas, 0, sizeof(blas));
        return -2;
    }
    if (st && nthreads > 0) st(nthreads);
    return 0;
}
int orc_blas_active(void) { return blas.h != NULL; }

/* ------------------------------------------------------------------------ */
/* Numeric part, instantiated for real double (d) and complex double (z)     */
/* ------------------------------------------------------------------------ */
#define F double
#define SUF(x) x##_d
#define IS_COMPLEX 0
#include "cliq_oracle_numeric.inc"
#undef F
#undef SUF
#undef IS_COMPLEX

#define F zd
#define SUF(x) x##_z
#define IS_COMPLEX 1
#include "cliq_oracle_numeric.inc"
#undef F
#undef SUF
#undef IS_COMPLEX

/* ------------------------------------------------------------------------ */
/* Type-dispatching entry points (values are interleaved doubles for complex) */
/* ------------------------------------------------------------------------ */
typedef struct { int is_complex; void* impl; } orc_fronts;

orc_fronts* orc_fronts_create(const oracle_symb* S, const i64* rowptr, const int* colind, const double* values,
                              int is_complex, int conjugate) {
    orc_fronts* f = (orc_fronts*)xcalloc(1, sizeof(orc_fronts));
    f->is_complex = is_complex;
    f->impl = is_complex ? (void*)fronts_init_z(S, rowptr, colind, (const zd*)values, conjugate)
                         : (void*)fronts_init_d(S, rowptr, colind, values, conjugate);
    return f;
}
void orc_fronts_free(orc_fronts* f) {
    if (!f) return;
    if (f->is_complex) fronts_free_z(f->impl); else fronts_free_d(f->impl);
    free(f);
}
/* LocalLDL with blocksize nb; returns 0, or 1 + (ND index) of the first zero pivot. */
i64 orc_ldl(orc_fronts* f, int nb) { return f->is_complex ? local_ldl_z(f->impl, nb) : local_ldl_d(f->impl, nb); }
/* LocalLDL with the front type chosen: kind = 1 for BLOCK_LDL_2D (FrontBlockLDL,
 * block solves), 2 for LDL_INTRAPIV_2D (FrontLDLIntraPiv, pivoted solves),
 * 3 for BLOCK_LDL_INTRAPIV_2D (FrontBlockLDL's intraPiv branch) */
i64 orc_ldl_ex(orc_fronts* f, int nb, int kind) {
    const int block = kind == 1 || kind == 3, pivot = kind == 2 || kind == 3;
    if (f->is_complex) { set_block_z(f->impl, block); set_pivot_z(f->impl, pivot); }
    else { set_block_d(f->impl, block); set_pivot_d(f->impl, pivot); }
    return orc_ldl(f, nb);
}
/* pivoted fronts: D[k + 1, k] of the 2 x 2 blocks (n) and the pivot rows (n) of node s */
void orc_front_pivots(const orc_fronts* f, int s, double* sub_out, int* piv_out) {
    if (f->is_complex) front_pivots_z(f->impl, s, (zd*)sub_out, piv_out); else front_pivots_d(f->impl, s, sub_out, piv_out);
}
/* FrontLDLIntraPiv on one dense front: AL (m x n, ld lda), ABR ((m-n)^2, ld
 * ldb); diag, sub, piv get n entries (AL's diagonal keeps D) */
i64 orc_front_ldl_intrapiv(int is_complex, int m, int n, double* AL, i64 lda, double* ABR, i64 ldb, double* diag, double* sub,
                           int* piv, int conjugate) {
    return is_complex ? front_ldl_intrapiv_z(m, n, (zd*)AL, lda, (zd*)ABR, ldb, (zd*)diag, (zd*)sub, piv, conjugate)
                      : front_ldl_intrapiv_d(m, n, AL, lda, ABR, ldb, diag, sub, piv, conjugate);
}
/* copy frontL (m x n, column-major) or diag (n) of node s */
void orc_front_get(const orc_fronts* f, int s, double* L_out, double* d_out) {
    if (f->is_complex) front_get_z(f->impl, s, (zd*)L_out, (zd*)d_out); else front_get_d(f->impl, s, L_out, d_out);
}
void orc_front_dims(const orc_fronts* f, int s, int* m, int* n) {
    if (f->is_complex) front_dims_z(f->impl, s, m, n); else front_dims_d(f->impl, s, m, n);
}
/* overwrite frontL of node s (used to factor externally prepared fronts) */
void orc_front_set(orc_fronts* f, int s, const double* L_in) {
    if (f->is_complex) front_set_z(f->impl, s, (const zd*)L_in); else front_set_d(f->impl, s, L_in);
}
/* install frontL and D of node s factored elsewhere (then orc_solve uses them) */
void orc_front_set_factored(orc_fronts* f, int s, const double* L_in, const double* d_in) {
    if (f->is_complex) front_set_factored_z(f->impl, s, (const zd*)L_in, (const zd*)d_in);
    else front_set_factored_d(f->impl, s, L_in, d_in);
}
/* Solve on a nodal multivector in ND order (N x nrhs, column-major, ld = N). */
i64 orc_solve(orc_fronts* f, double* X, int nrhs) {
    return f->is_complex ? solve_z(f->impl, (zd*)X, nrhs) : solve_d(f->impl, X, nrhs);
}
/* FrontLDL on one dense front: AL (m x n, ld lda) and ABR ((m-n)^2, ld ldb). */
i64 orc_front_ldl(int is_complex, int m, int n, double* AL, i64 lda, double* ABR, i64 ldb, int conjugate, int nb) {
    return is_complex ? front_ldl_z(m, n, (zd*)AL, lda, (zd*)ABR, ldb, conjugate, nb)
                      : front_ldl_d(m, n, AL, lda, ABR, ldb, conjugate, nb);
}
/* Multiply: Y := alpha A X + beta Y (CSR, natural order) */
void orc_multiply(int is_complex, i64 N, const i64* rowptr, const int* colind, const double* vals,
                  const double* alpha, const double* X, const double* beta, double* Y, int nrhs) {
    if (is_complex) multiply_z(N, rowptr, colind, (const zd*)vals, *(const zd*)alpha, (const zd*)X, *(const zd*)beta, (zd*)Y, nrhs);
    else multiply_d(N, rowptr, colind, vals, *alpha, X, *beta, Y, nrhs);
}
/* Pull / Push at P=1: nodal[p] = X[inv_map[p]] and back. */
void orc_pull(const oracle_symb* S, int is_complex, const double* X, double* Xn, int nrhs) {
    const int w = is_complex ? 2 : 1;
    for (int j = 0; j < nrhs; ++j)
        for (i64 p = 0; p < S->N; ++p)
            for (int c = 0; c < w; ++c) Xn[(j * S->N + p) * w + c] = X[(j * S->N + S->inv_map[p]) * w + c];
}
void orc_push(const oracle_symb* S, int is_complex, const double* Xn, double* X, int nrhs) {
    const int w = is_complex ? 2 : 1;
    for (int j = 0; j < nrhs; ++j)
        for (i64 p = 0; p < S->N; ++p)
            for (int c = 0; c < w; ++c) X[(j * S->N + S->inv_map[p]) * w + c] = Xn[(j * S->N + p) * w + c];
}
