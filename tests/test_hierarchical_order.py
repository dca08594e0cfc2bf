"""The hierarchical constrained-minimum-degree final order on small forests, mirroring the
reference's structural tests of hierarchical CAMD (tests/test_hierarchical_camd.cc:126-238):
constraints (every descendant component before its ancestors, each component
contiguous), determinism, the clamped cut depth, one boundary clique per connected part of
a subtree, a star's boundary as one element, and empty / invalid forests. Host only."""
import numpy as np
import pytest

from meshfemsparse_b200 import _lib


def csr(n, edges):
    adj = [set() for _ in range(n)]
    for a, b in edges:
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    xadj = np.zeros(n + 1, dtype=np.int64)
    for v in range(n):
        xadj[v + 1] = xadj[v] + len(adj[v])
    return xadj, np.array([u for v in range(n) for u in sorted(adj[v])], dtype=np.int64)


def order(n, edges, parent, member, cut):
    xadj, adj = csr(n, edges)
    return _lib.debug_hierarchical_order(xadj, adj, np.array(parent), np.array(member), cut)


def is_ancestor(parent, a, b):
    while b >= 0:
        if a == b:
            return True
        b = parent[b]
    return False


def check_constraints(perm, parent, member):
    n = len(member)
    assert np.array_equal(np.sort(perm), np.arange(n))
    pos = np.empty(n, dtype=np.int64)
    pos[perm] = np.arange(n)
    nc = len(parent)
    first = [min((pos[v] for v in range(n) if member[v] == c), default=n) for c in range(nc)]
    last = [max((pos[v] for v in range(n) if member[v] == c), default=-1) for c in range(nc)]
    for c in range(nc):
        if last[c] >= 0:
            assert last[c] - first[c] + 1 == sum(1 for v in range(n) if member[v] == c)   # contiguous
        a = parent[c]
        while a >= 0:
            if last[c] >= 0 and last[a] >= 0:
                assert last[c] < first[a]                # descendants before ancestors
            a = parent[a]


def test_random_forests_every_cut_depth():
    """64 vertices in 8 components of the forest {2,2,6,5,5,6,-1,-1}, random edges between
    ancestor-related components (tests/test_hierarchical_camd.cc:126-176)."""
    parent = [2, 2, 6, 5, 5, 6, -1, -1]
    rng = np.random.default_rng(19)
    for trial in range(12):
        member = [v % len(parent) for v in range(64)]
        edges = [(a, b) for a in range(64) for b in range(a + 1, 64)
                 if (is_ancestor(parent, member[a], member[b]) or is_ancestor(parent, member[b], member[a]))
                 and rng.integers(7) == 0]
        for cut in range(5):
            perm, st = order(64, edges, parent, member, cut)
            check_constraints(perm, parent, member)
            assert st["cut"] == min(cut, 2)
            again, _ = order(64, edges, parent, member, cut)
            assert np.array_equal(perm, again)


def test_disconnected_parts_of_a_subtree_give_separate_boundary_cliques():
    """Vertices 0 and 1 of the lower component are not connected: their boundaries {2,3}
    and {3,4} are two elements, not one clique {2,3,4} (tests/test_hierarchical_camd.cc:178-200);
    the default depth clamps to the forest's height and gives the same order."""
    edges = [(0, 2), (0, 3), (1, 3), (1, 4)]
    parent, member = [1, -1], [0, 0, 1, 1, 1]
    perm, st = order(5, edges, parent, member, 1)
    check_constraints(perm, parent, member)
    assert st == dict(cut=1, tasks=1, upper_vertices=3, upper_elements=2)
    clamped, st4 = order(5, edges, parent, member, 4)
    assert np.array_equal(clamped, perm) and st4["tasks"] == st["tasks"]


def test_star_boundary_is_one_element():
    """A star: centre 0 in the lower component, its 50 neighbours above; the boundary enters
    the upper problem as one element of 50 (tests/test_hierarchical_camd.cc:202-220)."""
    edges = [(0, v) for v in range(1, 51)]
    member = [0] + [1] * 50
    perm, st = order(51, edges, [1, -1], member, 1)
    check_constraints(perm, [1, -1], member)
    assert st == dict(cut=1, tasks=1, upper_vertices=50, upper_elements=1)
    assert perm[0] == 0


def test_empty_and_invalid_forests():
    """tests/test_hierarchical_camd.cc:222-238: an empty graph; two roots (depth 0: two
    problems, nothing above); an edge between two root components is rejected."""
    perm, st = order(0, [], [], [], 4)
    assert perm.size == 0
    perm, st = order(4, [(0, 1), (2, 3)], [-1, -1], [0, 0, 1, 1], 4)
    assert st["tasks"] == 2 and st["upper_vertices"] == 0
    check_constraints(perm, [-1, -1], [0, 0, 1, 1])
    with pytest.raises(ValueError):
        order(2, [(0, 1)], [-1, -1], [0, 1], 0)
