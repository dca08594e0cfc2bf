"""FP64 re-factor of FP32 diagonal blocks that meet a non-positive or tiny pivot.

Under refinement the FP32 factorization of a large front's diagonal block whose
pivot falls to at most 1e-5 of the injected diagonal is redone in FP64 from the
block's stored values, instead of perturbing the pivot. The case: one dense front
of 210 scalars (a 70-node stencil, native order, so the panel kernel factors it
in 128 + 82 column blocks) with two nearly dependent columns, so that pivot 5 is
about 3e-6 of its diagonal: FP32 loses it to cancellation, FP64 keeps it.
Checked: the block is counted as re-factored, no pivot is perturbed, the stored
factor's first column block matches the FP64 oracle factor to FP32 precision,
and FP64 refinement reaches 1e-10.
The reference's own loss-of-definiteness case (tests/test_catamari_factorizer.cc:
197-211: an FP32 factorization of [[1, 1], [1, 1 + 1e-8]] throws) keeps its
semantics without refinement.
"""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, OrderingMethod, SystemAssembler
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def dense_front_hessian(nn=70, eps=1e-4, seed=3):
    n = 3 * nn
    rng = np.random.default_rng(seed)
    M = rng.normal(size=(n, n))
    M[5] = M[4] + eps * rng.normal(size=n)             # rows 4 and 5 nearly dependent
    A = M @ M.T + 3e-4 * np.eye(n)                       # pivot 5: about 3e-6 of its diagonal
    H = SystemAssembler(nn).blockSparsityPattern([list(range(nn))])
    H.setZero()
    for j in range(n):
        for i in range(j + 1):
            H.addNZScalar(i, j, A[i, j])
    return H, A


def test_tiny_fp32_pivot_is_refactored_in_fp64():
    H, A = dense_front_hessian()
    f = B200Factorizer(True, refine=True, tensor_cores=2, orderingMethod=OrderingMethod.Native)
    f.factorizeSymbolic(H, [])
    f.factorizeNumeric(H)
    st = f.stats()
    assert st["num_large"] >= 1
    assert st["refactored_blocks"] >= 1
    assert st["perturbed_pivots"] == 0
    sn = f.supernodes()
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    ref = pyoracle.inject(plan["entries"], sn["vb"], 3, H.Ax, int(pan[-1]))
    assert pyoracle.mf_factor(sn, ref, 0) == -1
    got = f.factorValues()
    n = A.shape[0]
    L = pyoracle.panels_to_csc(sn, got, n).toarray()
    Lref = pyoracle.panels_to_csc(sn, ref, n).toarray()
    # the re-factored first column block matches FP64 up to the FP32 rounding of the
    # block's inputs (about 1e-7 of the diagonal), which the small pivot 5 amplifies
    # in the columns from 5 on to about 1e-4 of the largest entry
    blk = slice(0, 128)
    assert np.max(np.abs(L[blk, blk] - Lref[blk, blk])) <= 2e-4 * np.max(np.abs(Lref[blk, blk]))
    assert np.max(np.abs(L[blk, :5] - Lref[blk, :5])) <= 1e-6 * np.max(np.abs(Lref[blk, blk]))
    assert abs(L[5, 5] - Lref[5, 5]) <= 5e-2 * abs(Lref[5, 5])
    b = np.random.default_rng(1).normal(size=n)
    x = f.solve(b)
    assert np.linalg.norm(A @ x - b) <= 1e-10 * np.linalg.norm(b)


def test_reference_loss_of_definiteness_without_refinement():
    from meshfemsparse_b200 import ScalarCSC
    Ap = np.array([0, 1, 3], dtype=np.int64)
    Ai = np.array([0, 0, 1], dtype=np.int64)
    Ax = np.array([1.0, 1.0, 1.0 + 1e-8])
    S = ScalarCSC(2, Ap, Ai, Ax)
    dbl = B200Factorizer(False, orderingMethod=OrderingMethod.AMD)
    dbl.factorize(S)
    single = B200Factorizer(True, orderingMethod=OrderingMethod.AMD)
    with pytest.raises(RuntimeError):
        single.factorize(S)
    assert not single.hasNumericFactorization()
