"""The temporal nested-dissection reuse rule and its history against the reference's known answers
(tests/test_hierarchical_camd.cc:670-725, "temporal ND detects minimal disjoint invalid
subtrees", and :1178-1230, "temporal ND repairs forest roots independently"): the same
15-component tree (two vertices per component), the same base graph, the same added
edges, the same expected dirty roots and full-rebuild decisions. Host only."""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, ScalarCSC, SystemAssembler, _lib
from meshfemsparse_b200.hessian import BlockCSCHessian

# the reference's test tree: parent of each of the 15 components, member[v] = v / 2
TREE_PARENT = [2, 2, 6, 5, 5, 6, 14, 9, 9, 13, 12, 12, 13, 14, -1]


def base_edges(trees=1):
    """Each component's first vertex with itself, and both vertices of a component to
    the first vertex of its parent (tests/test_hierarchical_camd.cc:678-693)."""
    edges = []
    for t in range(trees):
        o = 30 * t
        for c in range(15):
            edges.append((o + 2 * c, o + 2 * c))
            p = TREE_PARENT[c]
            if p >= 0:
                edges.append((o + 2 * c, o + 2 * p))
                edges.append((o + 2 * c + 1, o + 2 * p))
    return edges


def csr(n, edges):
    adj = [set() for _ in range(n)]
    for a, b in edges:
        adj[a].add(b)
        adj[b].add(a)
    xadj = np.zeros(n + 1, dtype=np.int64)
    for v in range(n):
        xadj[v + 1] = xadj[v] + len(adj[v])
    return xadj, np.array([u for v in range(n) for u in sorted(adj[v])], dtype=np.int64)


def forest(trees):
    parent = []
    for t in range(trees):
        parent += [p if p < 0 else p + 15 * t for p in TREE_PARENT]
    member = np.arange(30 * trees) // 2
    return np.array(parent, dtype=np.int64), member


def dirty(n, edges, trees=1):
    xadj, adj = csr(n, edges)
    parent, member = forest(trees)
    return _lib.debug_dirty_subtrees(xadj, adj, parent, member)


SINGLE_TREE = {
    "unchanged": ([], [], False),
    "deletion": (None, [], False),
    "within node": ([(0, 1)], [], False),
    "separator to descendant": ([(13, 0)], [], False),
    "siblings": ([(0, 2)], [2], False),
    "duplicate violations": ([(0, 2), (1, 3)], [2], False),
    "disjoint": ([(0, 2), (14, 16)], [2, 9], False),
    "nested": ([(0, 2), (0, 6)], [6], False),
    "root": ([(0, 14)], [], True),
}


@pytest.mark.parametrize("case", list(SINGLE_TREE))
def test_single_tree_dirty_subtrees(case):
    extra, expected, full = SINGLE_TREE[case]
    edges = [] if extra is None else base_edges() + extra
    assert dirty(30, edges) == (full, expected)


FOREST = {
    "first root": ([(0, 14)], [14], False),
    "middle root": ([(30, 44)], [29], False),
    "last root": ([(60, 74)], [44], False),
    "two roots": ([(0, 14), (60, 74)], [14, 44], False),
    "root and subtree in another tree": ([(0, 14), (30, 32)], [14, 17], False),
    "root subsumes descendant": ([(0, 2), (0, 14)], [14], False),
    "cross-tree edge still forces full ND": ([(0, 30)], [], True),
}


@pytest.mark.parametrize("case", list(FOREST))
def test_forest_roots_dirty_subtrees(case):
    """With three trees a violated root is repaired alone; only an edge between two trees
    forces a full dissection."""
    extra, expected, full = FOREST[case]
    assert dirty(90, base_edges(3) + extra, trees=3) == (full, expected)


def test_root_splits_into_multiple_roots():
    """The first tree's own edges removed, then a root-crossing edge inside it: that root
    is the only dirty subtree (its region is disconnected afterwards)."""
    edges = [e for e in base_edges(3) if e[0] >= 30] + [(0, 14)]
    assert dirty(90, edges, trees=3) == (False, [14])


def test_invalid_forest_is_rejected():
    xadj, adj = csr(30, base_edges())
    parent, member = forest(1)
    bad = parent.copy()
    bad[3] = 1                      # a parent numbered before its child
    with pytest.raises(ValueError):
        _lib.debug_dirty_subtrees(xadj, adj, bad, member)


# ----------------------------------------------------------------- reuse history


def scalar_matrix(n, edges, diag):
    cols = [[] for _ in range(n)]
    for a, b in edges:
        a, b = min(a, b), max(a, b)
        cols[b].append(a)
    Ap, Ai = [0], []
    for j in range(n):
        Ai += sorted(set(cols[j])) + [j]
        Ap.append(len(Ai))
    Ax = np.where(np.array(Ai) == np.repeat(np.arange(n), np.diff(Ap)), diag, -1.0)
    S = ScalarCSC(n, np.array(Ap), np.array(Ai), Ax)
    return BlockCSCHessian(n, S.Ap, S.Ai, 1, S.Ax)


def analyse(f, A, pins):
    f.factorizeSymbolic(A, pins)
    st = f.stats()
    return st["nd_reused"] == 0, st["nd_rebuilt_vertices"]


def test_reuse_period_counts_incremental_analyses():
    """tests/test_catamari_factorizer.cc:232-258: period 32 on an unchanged 16-vertex path:
    analyses 0 and 33 are full, 1-32 incremental with nothing re-dissected."""
    A = scalar_matrix(16, [(v, v + 1) for v in range(15)], 4.0)
    f = B200Factorizer(device=-1, nd_reuse_period=32)
    for call in range(34):
        full, rebuilt = analyse(f, A, [])
        assert full == (call in (0, 33))
        assert rebuilt == (16 if full else 0)


def test_reuse_history_resets_for_pin_changes():
    """tests/test_hierarchical_camd.cc:1024-1061: period 2 on a 16 x 16 grid; a new edge at
    step 4; pins {0} from step 5 and {1} from step 7. Full at steps 0, 3, 5 and 7 (the
    first, the period, and each pin change); incremental with nothing re-dissected at 1, 2,
    6 and 8."""
    n, side = 256, 16
    edges = [(v, v + 1) for v in range(n) if v % side + 1 < side] + [(v, v + side) for v in range(n - side)]
    f = B200Factorizer(device=-1, nd_reuse_period=2)
    for step in range(9):
        if step == 4:
            edges.append((0, n - 1))
        pins = [] if step < 5 else [0 if step <= 6 else 1]
        full, rebuilt = analyse(f, scalar_matrix(n, edges, 10.0), pins)
        if step in (0, 3, 5, 7):
            assert full
        if step in (1, 2, 6, 8):
            assert not full and rebuilt == 0


def test_reuse_history_follows_the_scalar_fallback():
    """tests/test_catamari_factorizer.cc:270-297: a 32-node chain of 3 x 3 blocks; a
    partial-block pin analyses 95 scalar variables, whole-block pins 31 blocks, and each
    switch starts a new history (full first, then incremental)."""
    H = SystemAssembler(32).blockSparsityPattern(np.array([[i, i + 1] for i in range(31)]))
    f = B200Factorizer(device=-1, nd_reuse_period=2)
    for pins, nv in (([1], 95), ([0, 1, 2], 31)):
        for repeat in range(2):
            full, rebuilt = analyse(f, H, pins)
            assert full == (repeat == 0)
            assert f.ndOrdering().CMember.size == nv
            if repeat:
                assert rebuilt == 0
