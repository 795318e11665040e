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
