"""Adaptive ordering selection (Solvers/AdaptiveOrderingSelection.hh; the factorizer's
OrderingMethod::Adaptive): the heuristic on synthetic timing histories, and the
factorizer's analysis-only path switching between nested dissection and minimum degree.
Host only."""
import numpy as np

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, fem
from meshfemsparse_b200.adaptive_ordering import AdaptiveOrderingSelection
from meshfemsparse_b200.factorizer import CholeskyProvider, OrderingMethod, make_cholesky_factorizer

ND, MD = "nd", "md"


def run(sel, sym, num, sol, numerics, nnz=1000):
    """One symbolic analysis with the selected method, then `numerics` factorizations
    each followed by one solve; times per method from the dicts."""
    m = sel.update_selection()
    sel.record_symbolic(sym[m], nnz)
    for _ in range(numerics):
        sel.record_numeric(num[m])
        sel.record_solve(sol[m])
    return m


def test_frequent_analyses_switch_to_the_cheap_ordering_and_back():
    sel = AdaptiveOrderingSelection(ND, MD)
    sym = {ND: 1.0, MD: 0.1}
    num = {ND: 0.1, MD: 0.135}
    sol = {ND: 0.01, MD: 0.0135}
    # warm-up: the first two analyses use the primary method whatever the history says
    assert run(sel, sym, num, sol, 1) == ND
    assert run(sel, sym, num, sol, 1) == ND
    # one factorization per analysis: the symbolic time dominates, minimum degree pays
    assert run(sel, sym, num, sol, 1) == MD
    seen = [run(sel, sym, num, sol, 1) for _ in range(3)]
    assert seen == [MD, MD, MD]
    # many factorizations per analysis: nested dissection's faster factor pays again
    methods = [run(sel, sym, num, sol, 200) for _ in range(6)]
    assert methods[-1] == ND and MD in methods[:2]


def test_many_factorizations_keep_the_primary_ordering():
    sel = AdaptiveOrderingSelection(ND, MD)
    sym, num, sol = {ND: 1.0, MD: 0.1}, {ND: 0.1, MD: 0.135}, {ND: 0.01, MD: 0.0135}
    assert [run(sel, sym, num, sol, 100) for _ in range(8)] == [ND] * 8


def test_early_recompute_needs_a_known_faster_method_and_25_factorizations():
    sel = AdaptiveOrderingSelection(ND, MD)
    sym, num, sol = {ND: 1.0, MD: 0.1}, {ND: 0.1, MD: 0.135}, {ND: 0.01, MD: 0.0135}
    for _ in range(3):
        run(sel, sym, num, sol, 1)
    assert sel.current_method() == MD
    # on minimum degree with many factorizations: nested dissection is known to factor faster
    sel.update_selection()
    sel.record_symbolic(sym[MD], 1000)
    # the window's estimate favours nested dissection by 10 % only after about 145
    # factorizations on this analysis (4 analyses at 1.0 vs 0.1 s against 0.11 vs
    # 0.1485 s per factorization and solve)
    for k in range(300):
        sel.record_numeric(num[MD])
        sel.record_solve(sol[MD])
        if k + 1 <= 25:
            assert not sel.should_trigger_recompute()
    assert sel.should_trigger_recompute()


def test_factor_shrinking_resets_the_inactive_history():
    sel = AdaptiveOrderingSelection(ND, MD)
    sel.record_symbolic(1.0, 1000)
    sel.times[1].numeric.add(0.5)
    sel.record_symbolic(1.0, 800)          # -20 %: the other method's data is stale
    assert not sel.times[1].numeric.known()


def test_factorizer_adaptive_provider_and_analyses():
    nodes, tets = fem.tet_cube(5, seed=2)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    f = make_cholesky_factorizer(CholeskyProvider.CatamariAdaptive, device=-1)
    assert f.orderingMethod == OrderingMethod.Adaptive and f.provider() == CholeskyProvider.CatamariAdaptive
    f.factorizeSymbolic(H, [])
    assert f.ndOrdering() is not None                        # nested dissection first
    nd_nnz = f.getFactorNNZ()
    # a history in which analyses dominate sends the next analysis to minimum degree
    sel = f.adaptiveOrdering
    for _ in range(3):
        sel.record_numeric(0.01)
        sel.record_solve(0.001)
        sel.record_symbolic(10.0, nd_nnz)
    f.factorizeSymbolic(H, [])
    assert sel.current_method() == OrderingMethod.AMD and f.ndOrdering() is None
    p = f.getInversePermutation()
    assert np.array_equal(np.sort(p), np.arange(p.size))
    assert not f.wantsSymbolicFactorizationRecompute()
