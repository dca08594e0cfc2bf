"""The temporal nested-dissection reuse rule against the reference's known answers
(tests/test_hierarchical_camd.cc:670-725, "temporal ND detects minimal disjoint invalid
subtrees", and :1178-1230, "temporal ND repairs forest roots independently"): the same
15-component tree (two vertices per component), the same base graph, the same added
edges, the same expected dirty roots and full-rebuild decisions. Host only."""
import numpy as np
import pytest

from meshfemsparse_b200 import _lib

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
