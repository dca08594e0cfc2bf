"""Temporal reuse of the nested dissection (separator tree replayed, only the
subtrees a new edge violates re-dissected), on analysis-only handles (no GPU)."""
import numpy as np

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, fem


def tet_edges(tets):
    pairs = [(a, b) for a in range(4) for b in range(a + 1, 4)]
    return np.vstack([tets[:, [a, b]] for a, b in pairs])


def pattern(nn, edges):
    return SystemAssembler(nn).blockSparsityPattern(edges)


def analyse(f, H):
    f.factorizeSymbolic(H, [])
    st = f.stats()
    return st["nd_reused"], st["nd_rebuilt_vertices"]


def subtree_vertices(cparent, cmember, c):
    first = np.arange(len(cparent))
    for k in range(len(cparent)):
        p = cparent[k]
        if p >= 0:
            first[p] = min(first[p], first[k])
    return np.nonzero((cmember >= first[c]) & (cmember <= c))[0], first


def test_reuse_same_pattern_keeps_the_ordering():
    nodes, tets = fem.tet_cube(7, seed=1)
    H = pattern(nodes.shape[0], tet_edges(tets))
    f = B200Factorizer(device=-1, nd_reuse_period=4)
    assert analyse(f, H) == (0, nodes.shape[0])
    p0 = f.getInversePermutation()
    assert analyse(f, H) == (1, 0)
    assert np.array_equal(f.getInversePermutation(), p0)


def test_new_edge_rebuilds_only_the_violated_subtree_and_period():
    nodes, tets = fem.tet_cube(8, seed=2)
    nn = nodes.shape[0]
    edges = tet_edges(tets)
    H = pattern(nn, edges)
    f = B200Factorizer(device=-1, nd_reuse_period=2)
    analyse(f, H)
    nd = f.ndOrdering()
    cparent, cmember = nd.CParent, nd.CMember
    # a separator component below the root with two child subtrees: join them
    kids = {}
    for c, p in enumerate(cparent):
        if p >= 0:
            kids.setdefault(p, []).append(c)
    root = int(np.nonzero(cparent < 0)[0][0])
    cand = [c for c, ch in kids.items() if len(ch) >= 2 and c != root]
    c = max(cand, key=lambda c: len(subtree_vertices(cparent, cmember, c)[0]))
    a_verts, _ = subtree_vertices(cparent, cmember, kids[c][0])
    b_verts, _ = subtree_vertices(cparent, cmember, kids[c][1])
    u, v = int(a_verts[0]), int(b_verts[-1])
    H2 = pattern(nn, np.vstack([edges, [[u, v]]]))
    reused, rebuilt = analyse(f, H2)
    n_sub = len(subtree_vertices(cparent, cmember, c)[0])
    assert reused == 1 and 0 < rebuilt <= n_sub < nn
    nnz_reuse = f.getFactorNNZ()
    fresh = B200Factorizer(device=-1)
    fresh.factorizeSymbolic(H2, [])
    assert nnz_reuse <= 1.5 * fresh.getFactorNNZ()
    # the period: two reuses, then a full dissection
    assert analyse(f, H2)[0] == 1
    assert analyse(f, H2) == (0, nn)
