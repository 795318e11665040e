"""Nested dissection of general graphs (cliq.NestedDissection, the
reference's NestedDissection at one process with this library's own
bisection in place of METIS): structural checks on irregular, disconnected
and grid graphs.  The GPU factorizations over these orderings are checked in
tests/test_gpu_graph_nd.py."""
import numpy as np
import pytest

import clique_b200 as cliq
from clique_b200 import operators as ops


def knn_graph(npts, k, seed, dim=2, shift=0.3, components=1, isolated=0):
    """Graph Laplacian (+ shift) of the symmetrized k-nearest-neighbour graph
    of random points, optionally as several separate point clouds plus
    isolated vertices."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    base = 0
    for c in range(components):
        pts = rng.random((npts, dim))
        _, nb = cKDTree(pts).query(pts, k + 1)
        for i in range(npts):
            for j in nb[i, 1:]:
                rows += [base + i, base + int(j)]
                cols += [base + int(j), base + i]
        base += npts
    n = base + isolated
    rows, cols = np.array(rows), np.array(cols)
    key = np.unique(rows.astype(np.int64) * n + cols)
    r, c = key // n, key % n
    w = -np.ones(len(r))
    deg = np.bincount(r, minlength=n).astype(float)
    rr = np.concatenate([r, np.arange(n)])
    cc = np.concatenate([c, np.arange(n)])
    vv = np.concatenate([w, deg + shift])
    return ops.from_triplets(n, rr, cc, vv)


def check_tree(A, info, map_, cutoff):
    n = A.n
    m = np.asarray(map_.array)
    assert sorted(m.tolist()) == list(range(n))
    nodes = info.localNodes
    # subtree ND ranges
    lo = {}
    for s, nd in enumerate(nodes):
        lo[s] = min([nd.off] + [lo[c] for c in nd.children])
    inv = np.empty(n, np.int64)
    inv[m] = np.arange(n)
    rows = np.repeat(np.arange(n), np.diff(A.rowptr))
    cols = A.colind
    nd_r, nd_c = m[rows], m[cols]
    for s, nd in enumerate(nodes):
        if nd.children:
            l, r = nd.children
            L0, L1 = lo[l], nodes[l].off + nodes[l].size
            R0, R1 = lo[r], nodes[r].off + nodes[r].size
            assert L1 <= R0 and R1 == nd.off
            cross = ((nd_r >= L0) & (nd_r < L1) & (nd_c >= R0) & (nd_c < R1))
            assert not cross.any(), s          # the separator separates
        # the update rows are ancestors' pivots, and cover A's couplings
        anc, p = set(), nd.parent
        while 0 <= p < len(nodes) and p != s:   # (a one-node tree's root keeps ReverseOrder's parent 1)
            anc.update(range(nodes[p].off, nodes[p].off + nodes[p].size))
            p = nodes[p].parent
        assert set(np.asarray(nd.lowerStruct).tolist()) <= anc, s
        own = (nd_r >= nd.off) & (nd_r < nd.off + nd.size) & (nd_c >= nd.off + nd.size)
        assert set(nd_c[own].tolist()) <= set(np.asarray(nd.lowerStruct).tolist()), s
    return sum(nd.size * (nd.size + len(nd.lowerStruct)) for nd in nodes)


@pytest.mark.parametrize("npts,k,dim,cutoff", [(400, 6, 2, 16), (2000, 8, 2, 64), (1500, 10, 3, 64)])
def test_graph_nd_knn(npts, k, dim, cutoff):
    A = knn_graph(npts, k, seed=npts, dim=dim)
    map_, _, info = cliq.NestedDissection(A, cutoff)
    check_tree(A, info, map_, cutoff)
    assert info.num_nodes > 3


def test_graph_nd_disconnected_and_isolated():
    """Several components and 3000 isolated vertices: split between
    components with empty separators (balanced, so the recursion stays
    shallow)."""
    A = knn_graph(300, 6, seed=3, components=4, isolated=3000)
    map_, _, info = cliq.NestedDissection(A, 32)
    check_tree(A, info, map_, 32)
    sizes = [nd.size for nd in info.localNodes]
    assert 0 in sizes                      # empty separators between components
    depth = 0
    for s, nd in enumerate(info.localNodes):
        d, p = 0, nd.parent
        while 0 <= p < len(info.localNodes):
            d, p = d + 1, info.localNodes[p].parent
        depth = max(depth, d)
    assert depth <= 40, depth


@pytest.mark.parametrize("dims,cutoff", [((20, 20, 20), 64), ((60, 60, 1), 64), ((12, 9, 30), 32)])
def test_graph_nd_on_grids(dims, cutoff):
    """On grid graphs the factor entries stay within 2x of natural nested
    dissection's (whose separators are the grid's planes)."""
    A = ops.laplacian_3d(*dims, 6.1)
    map_, _, info = cliq.NestedDissection(A, cutoff, numSeqSeps=2)
    ent = check_tree(A, info, map_, cutoff)
    _, _, info_nat = cliq.NaturalNestedDissection(*dims, A, cutoff)
    ent_nat = sum(nd.size * (nd.size + len(nd.lowerStruct)) for nd in info_nat.localNodes)
    print(f"factor entries: graph ND {ent}, natural ND {ent_nat} ({ent / ent_nat:.2f}x)")
    assert ent <= 2.0 * ent_nat


def test_graph_nd_dense_block_is_a_leaf():
    """A dense block has no vertex separator: it stays one front."""
    n = 200
    r, c = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    A = ops.from_triplets(n, r.ravel(), c.ravel(), np.ones(n * n) + n * np.eye(n).ravel())
    map_, _, info = cliq.NestedDissection(A, 16)
    check_tree(A, info, map_, 16)
    assert info.num_nodes == 1 and info.localNodes[0].size == n


def _pattern(n, edges):
    e = np.asarray(edges, np.int64).reshape(-1, 2)
    r = np.concatenate([e[:, 0], e[:, 1], np.arange(n)])
    c = np.concatenate([e[:, 1], e[:, 0], np.arange(n)])
    v = np.concatenate([-np.ones(2 * len(e)), np.full(n, 10.0)])
    return ops.from_triplets(n, r, c, v)


def _shapes(rng):
    n = 700
    yield "star", _pattern(n, [(0, i) for i in range(1, n)])
    yield "path", _pattern(n, [(i, i + 1) for i in range(n - 1)])
    yield "tree", _pattern(n, [(i, int(rng.integers(0, i))) for i in range(1, n)])
    a, b = 40, 30
    yield "bipartite", _pattern(a + b, [(i, a + j) for i in range(a) for j in range(b)])
    yield "random", _pattern(n, rng.integers(0, n, size=(3 * n, 2)))
    g1 = [(i, i + 1) for i in range(299)]
    g2 = [(300 + i, 300 + int(rng.integers(0, i + 1))) for i in range(1, 300)]
    yield "union", _pattern(700, g1 + g2)   # a path, a tree and 100 isolated vertices


@pytest.mark.parametrize("seps", [1, 3])
def test_graph_nd_shapes(seps):
    rng = np.random.default_rng(7)
    for name, A in _shapes(rng):
        for cutoff in (1, 8, 64):
            map_, _, info = cliq.NestedDissection(A, cutoff, numSeqSeps=seps)
            check_tree(A, info, map_, cutoff)
