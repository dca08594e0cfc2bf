"""The final order of the nested dissection: hierarchical constrained minimum degree
over the separator forest (hierarchical_camd.cc:165-333; cut depth 4 by default,
MFS_ND_CAMD_CUT_DEPTH overrides it like the reference's CHOLMOD_NESDIS_CAMD_CUT_DEPTH).
Analysis-only handles, no GPU."""
import os

import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, fem


def analyse(H, pins, cut):
    old = os.environ.get("MFS_ND_CAMD_CUT_DEPTH")
    os.environ["MFS_ND_CAMD_CUT_DEPTH"] = str(cut)
    try:
        f = B200Factorizer(True, refine=True, device=-1)
        f.factorizeSymbolic(H, pins)
    finally:
        if old is None:
            os.environ.pop("MFS_ND_CAMD_CUT_DEPTH", None)
        else:
            os.environ["MFS_ND_CAMD_CUT_DEPTH"] = old
    return f


def cube(k, seed=1):
    nodes, tets = fem.tet_cube(k, jitter=0.1, seed=seed)
    return SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets), fem.bottom_pins(nodes), nodes.shape[0]


@pytest.mark.parametrize("k", [8, 14])
def test_constrained_order_keeps_the_fill_and_is_deterministic(k):
    H, pins, _ = cube(k)
    plain = analyse(H, pins, -1)          # the dissection's own order
    f4 = analyse(H, pins, 4)
    assert f4.getFactorNNZ() <= 1.01 * plain.getFactorNNZ()
    assert f4.getFlopEstimate() <= 1.02 * plain.getFlopEstimate()
    p = f4.getInversePermutation()
    assert np.array_equal(np.sort(p), np.arange(p.size))
    assert np.array_equal(analyse(H, pins, 4).getInversePermutation(), p)
    # the separator forest itself is the dissection's (only the order inside changes)
    a, b = plain.ndOrdering(), f4.ndOrdering()
    assert np.array_equal(a.CParent, b.CParent) and np.array_equal(a.CMember, b.CMember)


@pytest.mark.parametrize("cut", [0, 1, 2, 3, 4, 30])
def test_every_cut_depth_gives_a_valid_order(cut):
    """Depth 0: one problem per tree; a depth beyond the forest is clamped to it."""
    H, pins, _ = cube(10, seed=3)
    ref = analyse(H, pins, -1).getFactorNNZ()
    f = analyse(H, pins, cut)
    p = f.getInversePermutation()
    assert np.array_equal(np.sort(p), np.arange(p.size))
    assert f.getFactorNNZ() <= 1.05 * ref


def test_forest_of_two_bodies():
    """Two separate cubes: two trees, one subproblem per subtree at the cut in each."""
    nodes, tets = fem.tet_cube(7, seed=4)
    nn = nodes.shape[0]
    H = SystemAssembler(2 * nn).blockSparsityPattern(np.vstack([tets, tets + nn]))
    plain = analyse(H, [], -1)
    f = analyse(H, [], 4)
    assert f.getFactorNNZ() <= 1.03 * plain.getFactorNNZ()      # measured +1.8% on these small trees
    one = analyse(SystemAssembler(nn).blockSparsityPattern(tets), [], 4)
    assert f.getFactorNNZ() <= 2 * one.getFactorNNZ() * 1.03
