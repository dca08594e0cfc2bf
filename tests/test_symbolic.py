"""Host symbolic stage (pattern, pins, ordering, supernodes, relative indices,
conversion plan) checked against the reference's known answers and the
independent CPU oracle. No GPU needed: analysis-only handles (device -1)."""
import json
from pathlib import Path

import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, OrderingMethod, SystemAssembler, fem
from oracle import pyoracle

from helpers import cube_problem, grid_forest, path_hessian, random_stencil_hessian

GOLDEN = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())


def analyze(H, pins=(), ordering=OrderingMethod.CholmodNesdisParallel, relax=True, **kw):
    f = B200Factorizer(device=-1, orderingMethod=ordering, relax=relax)
    f.factorizeSymbolic(H, pins, **kw)
    return f


def reduced_analysis_pattern(H, pins, vb):
    """Pin-reduced upper pattern at analysis granularity (numpy restatement)."""
    if vb == H.bs:
        Ap, Ai, nv = H.Ap, H.Ai, H.numBlocks
        fixed = np.zeros(nv, dtype=bool)
        for p in pins:
            fixed[p // H.bs] = True
    else:
        S = H.toScalar(sparsityOnly=True)
        Ap, Ai, nv = S.Ap, S.Ai, S.n
        fixed = np.zeros(nv, dtype=bool)
        fixed[list(pins)] = True
    rr = np.full(nv, -1, dtype=np.int64)
    rr[~fixed] = np.arange(int((~fixed).sum()))
    nAp, nAi = [0], []
    for j in range(nv):
        if fixed[j]:
            continue
        for k in range(Ap[j], Ap[j + 1]):
            if not fixed[Ai[k]]:
                nAi.append(rr[Ai[k]])
        nAp.append(len(nAi))
    return np.array(nAp, dtype=np.int64), np.array(nAi, dtype=np.int64)


def check_against_oracle(f, H, pins, relax=True):
    sn = f.supernodes()
    vb = sn["vb"]
    iperm_s = f.getInversePermutation()
    assert np.array_equal(np.sort(iperm_s), np.arange(f.n_reduced()))
    iperm_v = iperm_s[::vb] // vb
    Ap, Ai = reduced_analysis_pattern(H, pins, vb)
    o = pyoracle.symbolic(Ap, Ai, iperm_v, vb, relax=relax)
    # supernode partition: bit-exact
    assert np.array_equal(o["sn_start"], sn["sn_start"])
    nsn = len(sn["sn_start"]) - 1
    start = sn["sn_start"]
    sn_of = np.repeat(np.arange(nsn), np.diff(start))
    for s in range(nsn):
        last = start[s + 1] - 1
        # assembly-tree parent
        p = o["parent"][last]
        assert sn["parent"][s] == (-1 if p < 0 else sn_of[p])
        # structure = union of column structures below the supernode
        rows = set()
        for j in range(start[s], start[s + 1]):
            rows.update(int(r) for r in o["L_rows"][o["L_ptr"][j]:o["L_ptr"][j + 1]] if r > last)
        mine = sn["struct_rows"][sn["struct_ptr"][s]:sn["struct_ptr"][s + 1]]
        assert list(mine) == sorted(rows)
    # relative indices (child_rel_indices): restated position in the parent's front
    for c in range(nsn):
        p = sn["parent"][c]
        if p < 0:
            continue
        wp = vb * (start[p + 1] - start[p])
        prow = list(sn["struct_rows"][sn["struct_ptr"][p]:sn["struct_ptr"][p + 1]])
        for t in range(sn["struct_ptr"][c], sn["struct_ptr"][c + 1]):
            r = sn["struct_rows"][t]
            exp = vb * (r - start[p]) if start[p] <= r < start[p + 1] else wp + vb * prow.index(r)
            assert sn["rel"][t] == exp
    return sn, iperm_s


def check_plan(f, H, pins, sn, iperm_s):
    """Injected panels reproduce the lower triangle of the permuted reduced matrix exactly."""
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    vals = pyoracle.inject(plan["entries"], sn["vb"], H.bs, H.Ax, int(pan[-1]))
    L = pyoracle.panels_to_dense(sn, vals, f.n_reduced())
    A = pyoracle.reduced_permuted_dense(H, pins, iperm_s)
    assert np.array_equal(L, np.tril(A))


def test_known_answer_native_relaxation():
    g = GOLDEN["native_relaxed_example"]
    H = SystemAssembler(g["num_blocks"], g["block_size"]).blockSparsityPattern(g["edges"])
    assert analyze(H, ordering=OrderingMethod.Native).getFactorNNZ() == g["factor_nnz_relaxed"]
    assert analyze(H, ordering=OrderingMethod.Native, relax=False).getFactorNNZ() == g["factor_nnz_fundamental"]
    # native ordering keeps the identity (removeFixedEntries(permute) == plain)
    f = analyze(H, ordering=OrderingMethod.Native)
    assert np.array_equal(f.getInversePermutation(), np.arange(10))
    # the oracle agrees on both counts
    Ap, Ai = reduced_analysis_pattern(H, [], 2)
    for relax, key in ((True, "factor_nnz_relaxed"), (False, "factor_nnz_fundamental")):
        o = pyoracle.symbolic(Ap, Ai, np.arange(5), 2, relax=relax)
        sizes = np.diff(o["sn_start"]) * 2
        degs = []
        for s in range(len(sizes)):
            rows = set()
            for j in range(o["sn_start"][s], o["sn_start"][s + 1]):
                rows.update(int(r) for r in o["L_rows"][o["L_ptr"][j]:o["L_ptr"][j + 1]] if r >= o["sn_start"][s + 1])
            degs.append(2 * len(rows))
        nnz = sum(wv * (wv + 1) // 2 + wv * dv for wv, dv in zip(sizes, degs))
        assert nnz == g[key]


@pytest.mark.parametrize("case", GOLDEN["child_rel_indices"]["cases"], ids=lambda c: f"d{c['d']}")
def test_known_answer_child_rel_indices(case):
    d = case["d"]
    # block pattern whose analysis (native order, supplied partition [1,2,1] blocks)
    # gives supernode structures {block 1, block 3} and {block 3}
    H = SystemAssembler(4, d).blockSparsityPattern([[0, 1], [0, 3], [1, 2], [2, 3]])
    f = analyze(H, ordering=OrderingMethod.Native, supernode_sizes=[1, 2, 1])
    sn = f.supernodes()
    assert list(np.diff(sn["sn_start"]) * d) == case["sizes"]
    assert list(np.diff(sn["struct_ptr"]) * d) == case["degrees"]
    struct = [list(sn["struct_rows"][sn["struct_ptr"][s]:sn["struct_ptr"][s + 1]] * d) for s in range(3)]
    assert struct == case["structure"]
    assert list(sn["parent"]) == case["parents"]
    assert list(sn["rel"]) == case["child_rel_indices"]


def test_supplied_partition_must_be_etree_chain():
    H = SystemAssembler(5, 2).blockSparsityPattern([[0, 3], [1, 2], [2, 4], [3, 4]])
    with pytest.raises(ValueError):
        analyze(H, ordering=OrderingMethod.Native, supernode_sizes=[2, 3])


@pytest.mark.parametrize("bs", [1, 2, 3])
@pytest.mark.parametrize("pinmode", [0, 1, 2])
@pytest.mark.parametrize("ordering", [OrderingMethod.Native, OrderingMethod.AMD,
                                      OrderingMethod.CholmodNesdisParallel])
def test_path_matrices_against_oracle(bs, pinmode, ordering):
    H = path_hessian(20, bs)
    pins = [] if pinmode == 0 else (list(range(bs)) if pinmode == 1 else [1])
    f = analyze(H, pins, ordering)
    sn, ip = check_against_oracle(f, H, pins)
    check_plan(f, H, pins, sn, ip)
    if pinmode == 2 and bs > 1:
        assert sn["vb"] == 1          # partial-block pin: scalar analysis
    assert f.n_reduced() == H.n - len(set(pins))


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("relax", [True, False])
def test_random_stencils_against_oracle(seed, relax):
    H = random_stencil_hessian(seed, bs=3)
    rng = np.random.default_rng(seed)
    pinned_blocks = rng.choice(H.numBlocks, size=2, replace=False)
    pins = [3 * b + c for b in pinned_blocks for c in range(3)]
    f = analyze(H, pins, relax=relax)
    sn, ip = check_against_oracle(f, H, pins, relax=relax)
    check_plan(f, H, pins, sn, ip)


@pytest.mark.parametrize("k", [3, 5])
def test_cube_against_oracle(k):
    H, tets, Ke, pins, nodes = cube_problem(k)
    f = analyze(H, pins)
    sn, ip = check_against_oracle(f, H, pins)
    check_plan(f, H, pins, sn, ip)


def test_forest_components():
    H = grid_forest(13, 3)
    f = analyze(H)
    sn, ip = check_against_oracle(f, H, [])
    assert (sn["parent"] == -1).sum() >= 2        # one root per disconnected grid


def test_nested_dissection_separator_tree():
    nodes, tets = fem.tet_cube(8, jitter=0.1, seed=2)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    pins = fem.bottom_pins(nodes)
    f = analyze(H, pins)
    nd = f.ndOrdering()
    assert nd is not None and nd.blockSize == 3
    nv = f.n_reduced() // 3
    cp, cm = nd.CParent, nd.CMember
    assert cm.size == nv
    assert all(p == -1 or p > c for c, p in enumerate(cp))     # postordered
    # separator property: adjacent vertices lie on one root path of the separator tree
    anc = [set() for _ in cp]
    for c in range(len(cp)):
        p, chain = c, set()
        while p != -1:
            chain.add(p)
            p = cp[p]
        anc[c] = chain
    Ap, Ai = reduced_analysis_pattern(H, pins, 3)
    for j in range(nv):
        for k in range(Ap[j], Ap[j + 1]):
            a, b = cm[Ai[k]], cm[j]
            assert a in anc[b] or b in anc[a]


def test_invalid_inputs_raise():
    H = path_hessian(5, 3)
    f = B200Factorizer(device=-1)
    with pytest.raises(RuntimeError):
        f.factorizeSymbolic(H, [100])          # "Fixed variable index out of range"
    bad = H.copy()
    bad.Ai = bad.Ai[::-1].copy()
    with pytest.raises(ValueError):
        f.factorizeSymbolic(bad, [])
    with pytest.raises(RuntimeError):
        f.getFactorNNZ()


def test_pattern_matches_oracle_restatement():
    for k in (2, 4):
        nodes, tets = fem.tet_cube(k)
        H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
        Ap, Ai = pyoracle.build_pattern(nodes.shape[0], tets)
        assert np.array_equal(H.Ap, Ap) and np.array_equal(H.Ai, Ai)
    for seed in range(3):
        rng = np.random.default_rng(seed)
        n = 30
        el = np.array([rng.choice(n, 4, replace=False) for _ in range(40)])
        H = SystemAssembler(n, 2).blockSparsityPattern(el)
        Ap, Ai = pyoracle.build_pattern(n, el)
        assert np.array_equal(H.Ap, Ap) and np.array_equal(H.Ai, Ai)
