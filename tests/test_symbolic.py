"""Host symbolic phase of the product (natural nested dissection + analysis,
compiled into libcliqgpu.so) against the CPU oracle and the hand-derived
known answers: integer outputs must match exactly."""
import json
import os

import numpy as np
import pytest

import clique_b200 as cliq
from clique_b200 import operators as ops

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _check_against(info, map_, ref_sym):
    assert info.num_nodes == ref_sym.num_nodes
    assert np.array_equal(map_.array, ref_sym.map)
    nodes = info.localNodes
    for s, nd in enumerate(nodes):
        assert nd.size == ref_sym.size[s]
        assert nd.off == ref_sym.off[s]
        assert nd.myOff == ref_sym.my_off[s]
        assert nd.parent == ref_sym.parent[s]
        assert nd.sepParent == ref_sym.sep_parent[s]
        exp_children = [ref_sym.child0[s], ref_sym.child1[s]] if ref_sym.child0[s] >= 0 else []
        assert nd.children == exp_children
        assert nd.onLeft == bool(ref_sym.on_left[s])
        assert np.array_equal(nd.lowerStruct, ref_sym.array(s, "lower"))
        assert np.array_equal(nd.origLowerStruct, ref_sym.array(s, "orig"))
        assert np.array_equal(nd.origLowerRelInds, ref_sym.array(s, "orig_rel"))
        assert np.array_equal(nd.leftRelInds, ref_sym.array(s, "left_rel"))
        assert np.array_equal(nd.rightRelInds, ref_sym.array(s, "right_rel"))


@pytest.mark.parametrize("dims,cutoff", [((3, 1, 1), 1), ((3, 3, 1), 2), ((2, 2, 2), 100), ((6, 5, 4), 8),
                                         ((7, 3, 2), 5), ((9, 9, 9), 16), ((12, 10, 7), 30), ((30, 30, 30), 128),
                                         ((1, 1, 1), 1), ((5, 1, 1), 1), ((17, 3, 1), 4), ((40, 40, 1), 64)])
def test_product_symbolic_matches_oracle(oracle, dims, cutoff):
    A = ops.laplacian_3d(*dims, 6.1)
    map_, sep, info = cliq.NaturalNestedDissection(*dims, A, cutoff)
    ref = oracle.Symbolic(*dims, A.rowptr, A.colind, cutoff=cutoff)
    _check_against(info, map_, ref)
    for s in range(info.num_nodes):
        assert np.array_equal(sep.inds(s), ref.array(s, "inds"))


def test_product_symbolic_known_answers():
    cases = json.load(open(os.path.join(GOLD, "nd_known_answers.json")))["cases"]
    for c in cases:
        A = ops.laplacian_3d(*c["grid"], 6.1)
        map_, _, info = cliq.NaturalNestedDissection(*c["grid"], A, c["cutoff"])
        assert list(map_.array) == c["map"]
        nodes = info.localNodes
        assert [n.size for n in nodes] == c["size"]
        assert [n.parent for n in nodes] == c["parent"]
        assert [list(n.lowerStruct) for n in nodes] == c["lowerStruct"]


def test_symbolic_bad_grid_raises():
    A = ops.laplacian_3d(3, 3, 3)
    with pytest.raises(cliq.LogicError):
        cliq.NaturalNestedDissection(3, 3, 2, A, 8)


def test_symbolic_100cubed_shape():
    """The 100^3 workload's tree: the root separator is the 100x100 mid plane."""
    A = ops.laplacian_3d(100, 100, 100)
    map_, _, info = cliq.NaturalNestedDissection(100, 100, 100, A, 128)
    nodes = info.localNodes
    assert nodes[-1].size == 100 * 100
    assert sum(n.size for n in nodes) == A.n
    assert sorted(map_.array.tolist()) == list(range(A.n))


def test_batch_forest_is_the_union_of_the_problems():
    """cliq_batch_nested_dissection on a block-diagonal matrix equals the
    per-problem analyses shifted by each problem's node and row offsets."""
    import ctypes as C
    import clique_b200 as cliq
    from clique_b200 import _capi, operators as ops
    from clique_b200.batch import block_diagonal
    rng = np.random.default_rng(1)
    mats, dims = [], []
    for i in range(7):
        s = int(rng.integers(1, 24))
        mats.append(ops.helmholtz_workload_2d(s, seed=i)[0] if s > 1 else ops.laplacian_2d(1, 1))
        dims.append((s, s, 1))
    mats.append(ops.laplacian_3d(5, 4, 3, 6.1))
    dims.append((5, 4, 3))
    A = block_diagonal([ops.CSR(M.n, M.rowptr, M.colind, M.values.astype(np.complex128)) for M in mats])
    d = np.array([list(t) for t in dims], np.int32).reshape(-1)
    lib = _capi.load()
    h = C.c_void_p()
    assert lib.cliq_batch_nested_dissection(len(mats), d.ctypes.data_as(C.c_void_p), A.n,
                                            A.rowptr.ctypes.data_as(C.c_void_p), A.colind.ctypes.data_as(C.c_void_p),
                                            16, C.byref(h)) == 0
    info = cliq.DistSymmInfo(h.value, A.n)
    m = np.zeros(A.n, np.int32)
    lib.cliq_symbolic_map(h.value, m.ctypes.data_as(C.c_void_p), None)
    r0 = n0 = 0
    for B, dd in zip(mats, dims):
        m1, _, i1 = cliq.NaturalNestedDissection(*dd, B, 16)
        assert np.array_equal(m[r0:r0 + B.n], m1.array + r0)
        for t in range(i1.num_nodes):
            a, b = i1.localNodes[t], info.localNodes[n0 + t]
            assert (a.size, a.off + r0) == (b.size, b.off)
            assert (a.parent + n0 if 0 <= a.parent < i1.num_nodes else -1) == b.parent
            assert np.array_equal(a.lowerStruct + r0, b.lowerStruct)
            assert np.array_equal(a.leftRelInds, b.leftRelInds) and np.array_equal(a.rightRelInds, b.rightRelInds)
        r0 += B.n
        n0 += i1.num_nodes
    assert info.num_nodes == n0
    # a matrix that is not block diagonal in the given problems is rejected
    bad = np.array([3, 3, 1, 3, 3, 1], np.int32)
    Ab = ops.laplacian_2d(3, 6)
    assert lib.cliq_batch_nested_dissection(2, bad.ctypes.data_as(C.c_void_p), Ab.n, Ab.rowptr.ctypes.data_as(C.c_void_p),
                                            Ab.colind.ctypes.data_as(C.c_void_p), 16, C.byref(h)) == _capi.CLIQ_ERR_ARG
