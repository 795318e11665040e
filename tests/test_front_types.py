"""Front-type helpers and ChangeFrontType (dist_symm_front_tree/decl.hpp:27-165,
change_front_type.hpp:27-107) at one process: pure host logic."""
import pytest

import clique_b200 as cliq

T = cliq.SymmFrontType


class _Tree:
    def __init__(self, t):
        self.frontType = t


def test_helpers_match_the_reference_tables():
    fam = [(T.SYMM_1D, T.SYMM_2D), (T.LDL_1D, T.LDL_2D), (T.LDL_SELINV_1D, T.LDL_SELINV_2D),
           (T.LDL_INTRAPIV_1D, T.LDL_INTRAPIV_2D), (T.LDL_INTRAPIV_SELINV_1D, T.LDL_INTRAPIV_SELINV_2D),
           (T.BLOCK_LDL_1D, T.BLOCK_LDL_2D), (T.BLOCK_LDL_INTRAPIV_1D, T.BLOCK_LDL_INTRAPIV_2D)]
    for one, two in fam:
        assert cliq.ConvertTo2d(one) == two and cliq.ConvertTo2d(two) == two
        assert cliq.ConvertTo1d(two) == one and cliq.ConvertTo1d(one) == one
        assert cliq.FrontsAre1d(one) and not cliq.FrontsAre1d(two)
    assert cliq.AppendSelInv(T.LDL_2D) == T.LDL_SELINV_2D
    assert cliq.AppendSelInv(T.LDL_INTRAPIV_1D) == T.LDL_INTRAPIV_SELINV_1D
    assert cliq.RemoveSelInv(T.LDL_INTRAPIV_SELINV_2D) == T.LDL_INTRAPIV_2D
    with pytest.raises(cliq.LogicError):
        cliq.AppendSelInv(T.BLOCK_LDL_2D)
    assert cliq.PivotedFactorization(T.BLOCK_LDL_INTRAPIV_1D) and not cliq.PivotedFactorization(T.LDL_2D)
    assert cliq.SelInvFactorization(T.LDL_INTRAPIV_SELINV_2D) and not cliq.SelInvFactorization(T.LDL_INTRAPIV_2D)
    assert cliq.BlockFactorization(T.BLOCK_LDL_1D) and cliq.Unfactored(T.SYMM_1D)


def test_change_front_type():
    L = _Tree(T.LDL_2D)
    cliq.ChangeFrontType(L, T.LDL_1D)
    assert L.frontType == T.LDL_1D
    cliq.ChangeFrontType(L, T.LDL_SELINV_2D)          # selective inversion: distributed fronts only
    assert L.frontType == T.LDL_SELINV_2D
    L = _Tree(T.LDL_INTRAPIV_2D)
    cliq.ChangeFrontType(L, T.LDL_INTRAPIV_SELINV_1D)
    assert L.frontType == T.LDL_INTRAPIV_SELINV_1D
    for old, new in [(T.LDL_2D, T.BLOCK_LDL_2D), (T.LDL_2D, T.LDL_INTRAPIV_2D), (T.BLOCK_LDL_2D, T.LDL_SELINV_2D),
                     (T.LDL_SELINV_2D, T.LDL_2D)]:
        with pytest.raises(cliq.LogicError):
            cliq.ChangeFrontType(_Tree(old), new)
