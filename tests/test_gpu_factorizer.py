"""Factorizer lifecycle on the GPU, mirroring tests/test_catamari_factorizer.cc and
tests/test_native_ordering.cc (tolerances as there: 1e-11 FP64, 2e-5 FP32)."""
import numpy as np
import pytest

from meshfemsparse_b200 import (B200Factorizer, BlockCSCHessian, CholeskyProvider, OrderingMethod, ScalarCSC,
                                SystemAssembler, make_cholesky_factorizer)

from helpers import grid_forest, path_hessian, plain_scalar_path

pytestmark = pytest.mark.gpu


def check_solves(A, single, ordering, pins, **kw):
    """Restatement of checkSolves (tests/test_catamari_factorizer.cc:13-98)."""
    f = B200Factorizer(single, orderingMethod=ordering, **kw)
    n = A.n
    expected = np.array([[np.sin(0.2 * (i + 1) * (j + 1)) for j in range(3)] for i in range(n)])
    expected[list(pins)] = 0
    rhs = np.stack([A.apply(expected[:, j]) for j in range(3)], axis=1)
    tol = 2e-5 if single else 1e-11

    def verify(b):
        x = f.solveMultiRHS(b)
        assert np.linalg.norm(x - expected) < tol * np.linalg.norm(expected)
        b0 = b[:, 0]
        x0 = f.solve(b0)
        assert np.linalg.norm(x0 - expected[:, 0]) < tol * np.linalg.norm(expected[:, 0])
        for permuted in (False, True):
            red = f.removeFixedEntries(b0, permuted)
            xr = f.solveRawReduced(red, alreadyPermuted=permuted)
            full = f.extractFullSolution(xr, permuted)
            assert np.linalg.norm(full - expected[:, 0]) < tol * np.linalg.norm(expected[:, 0])
            f.solveRawReducedInPlace(red, alreadyPermuted=permuted)
            full = f.extractFullSolution(red, permuted)
            assert np.linalg.norm(full - expected[:, 0]) < tol * np.linalg.norm(expected[:, 0])

    for _ in range(2):
        f.factorizeSymbolic(A, pins)
        assert f.getFactorNNZ() > 0 and f.getFlopEstimate() > 0
        f.factorizeNumeric(A)
        verify(rhs)
        f.stashFactorization()
        assert f.hasStashedFactorization()
        for sigma in (0.75, 0.25):
            f.factorizeNumericWithShift(A, sigma)
            verify(rhs + sigma * expected)
        f.factorizeNumericWithShift(A, 0.5, A)
        verify(1.5 * rhs)
        f.swapStashedFactorization()
        verify(rhs)
        f.swapStashedFactorization()
        verify(1.5 * rhs)
        f.clearStashedFactorization()
        assert not f.hasStashedFactorization()
        A.Ax *= 2.0
        f.factorizeNumeric(A)
        verify(2.0 * rhs)
        A.Ax *= 0.5
    f.clearFactors()
    assert not f.hasNumericFactorization()
    f.factorizeSymbolic(A, pins)
    f.factorizeNumeric(A)
    verify(rhs)
    # failure invalidates the numeric factor and allows recovery
    A.Ax *= -1.0
    with pytest.raises(RuntimeError):
        f.factorizeNumeric(A)
    assert not f.hasNumericFactorization()
    A.Ax *= -1.0
    f.factorizeNumeric(A)
    verify(rhs)
    f.stashFactorization()
    f.clearFactors()
    f.swapStashedFactorization()
    verify(rhs)
    f.factorizeNumeric(A)
    verify(rhs)
    f.clearStashedFactorization()


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("ordering", [OrderingMethod.Native, OrderingMethod.AMD, OrderingMethod.CholmodNesdisParallel])
@pytest.mark.parametrize("pinmode", [0, 1, 2])
@pytest.mark.parametrize("bs", [1, 2, 3])
def test_precision_preserves_block_solver_behavior(single, ordering, pinmode, bs):
    A = path_hessian(20, bs)
    pins = [] if pinmode == 0 else (list(range(bs)) if pinmode == 1 else [1])
    check_solves(A, single, ordering, pins)


@pytest.mark.parametrize("single", [False, True])
def test_plain_scalar_matrix(single):
    S = plain_scalar_path(20)
    A = BlockCSCHessian(S.n, S.Ap, S.Ai, 1, S.Ax)
    check_solves(A, single, OrderingMethod.CholmodNesdisParallel, [1])


@pytest.mark.parametrize("single", [False, True])
def test_tiled_large_front_path(single):
    """small_front_max = 8 sends every front through the tiled POTRF/TRSM/GEMM kernels."""
    A = grid_forest(13, 3)
    check_solves(A, single, OrderingMethod.CholmodNesdisParallel, [], small_front_max=8)


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("bs", [2, 3])
def test_block_forest(single, bs):
    check_solves(grid_forest(13, bs), single, OrderingMethod.CholmodNesdisParallel, [])


def test_separator_forest_changes():
    side, comp = 17, 17 * 17
    n = 2 * comp
    f = B200Factorizer()
    rng = np.random.default_rng(0)
    for connect in (False, True, False):
        Ap, Ai, Ax = [0], [], []
        for j in range(n):
            rows = []
            if j % side > 0:
                rows.append((j - 1, -0.5))
            if j % comp >= side:
                rows.append((j - side, -0.5))
            if connect and j == comp:
                rows.append((comp - 1, -0.5))
            rows.sort()
            for i, v in rows:
                Ai.append(i); Ax.append(v)
            Ai.append(j); Ax.append(5.0)
            Ap.append(len(Ai))
        S = ScalarCSC(n, np.array(Ap), np.array(Ai), np.array(Ax))
        A = BlockCSCHessian(n, S.Ap, S.Ai, 1, S.Ax)
        f.factorizeSymbolic(A, [])
        f.factorizeNumeric(A)
        expected = rng.uniform(-1, 1, size=(n, 3))
        rhs = S.apply(expected)
        for _ in range(2):
            x = f.solveMultiRHS(rhs)
            assert np.linalg.norm(x - expected) < 1e-11 * np.linalg.norm(expected)
            assert np.linalg.norm(f.solve(rhs[:, 0]) - expected[:, 0]) < 1e-11 * np.linalg.norm(expected[:, 0])


def test_rounding_induced_loss_of_positive_definiteness():
    S = ScalarCSC(2, np.array([0, 1, 3]), np.array([0, 0, 1]), np.array([1.0, 1.0, 1.0 + 1e-8]))
    A = BlockCSCHessian(2, S.Ap, S.Ai, 1, S.Ax)
    single = B200Factorizer(True, orderingMethod=OrderingMethod.AMD)
    dbl = B200Factorizer(False, orderingMethod=OrderingMethod.AMD)
    dbl.factorize(A)
    with pytest.raises(RuntimeError):
        single.factorize(A)
    assert not single.hasNumericFactorization()
    with pytest.raises(RuntimeError):
        single.solveRawReduced(np.ones(2))
    with pytest.raises(RuntimeError):
        single.solveMultiRHS(np.ones((2, 1)))


def test_refined_fp32_perturbs_instead_of_failing():
    """Under FP64 refinement the FP32 factor is a preconditioner: a pivot lost to
    rounding is perturbed (and counted) and the refined solve still reaches 1e-10."""
    S = ScalarCSC(2, np.array([0, 1, 3]), np.array([0, 0, 1]), np.array([1.0, 1.0, 1.0 + 1e-8]))
    A = BlockCSCHessian(2, S.Ap, S.Ai, 1, S.Ax)
    f = B200Factorizer(True, refine=True, orderingMethod=OrderingMethod.AMD, refine_maxit=20)
    f.factorize(A)
    assert f.stats()["perturbed_pivots"] >= 1
    b = np.array([1.0, 2.0])
    x = f.solve(b)
    r = S.apply(x) - b
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b)


@pytest.mark.parametrize("single", [False, True])
def test_symbolic_reuse_resets_scalar_fallback(single):
    S = plain_scalar_path(6)
    block = BlockCSCHessian.fromScalar(S, 2)
    f = B200Factorizer(single, orderingMethod=OrderingMethod.AMD)
    f.factorizeSymbolic(block, [1])
    f.factorizeNumeric(block)
    A = BlockCSCHessian(6, S.Ap, S.Ai, 1, S.Ax)
    f.factorize(A)
    expected = np.linspace(0.1, 0.9, 6)
    b = S.apply(expected)
    assert np.linalg.norm(f.solve(b) - expected) < (1e-5 if single else 1e-12)


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("blocks", [False, True])
@pytest.mark.parametrize("pins", [[], [2, 3], [3]])
def test_native_ordering_preserves_reduced_input_order(single, blocks, pins):
    """tests/test_native_ordering.cc:8-60."""
    H = SystemAssembler(12, 2).blockSparsityPattern([[0, e + 1] for e in range(11)])
    H.setZero()
    for i, j in H.toScalar(sparsityOnly=True).entries():
        H.addNZScalar(i, j, 30.0 if i == j else -0.1 * (1 + (i + j) % 7))
    S = H.toScalar()
    A = H if blocks else BlockCSCHessian(S.n, S.Ap, S.Ai, 1, S.Ax)
    f = make_cholesky_factorizer(CholeskyProvider.B200Native, single)
    assert f.provider() == CholeskyProvider.B200Native
    expected = np.linspace(-0.7, 1.3, 24)
    expected[pins] = 0
    f.factorizeSymbolic(A, pins)
    tol = 1e-5 if single else 1e-12
    for shift in (0.0, 0.25):
        if shift == 0:
            f.factorizeNumeric(A)
        else:
            f.factorizeNumericWithShift(A, shift)
        rhs = S.apply(expected) + shift * expected
        assert np.linalg.norm(f.solve(rhs) - expected) < tol * np.linalg.norm(expected)
        reduced = f.removeFixedEntries(rhs, False)
        res = f.solveRawReduced(reduced, alreadyPermuted=True)
        full = f.extractFullSolution(res, False)
        assert np.linalg.norm(full - expected) < tol * np.linalg.norm(expected)
        permuted = f.removeFixedEntries(rhs, True)
        assert np.array_equal(permuted, reduced)


def test_native_ordering_changes_take_effect_at_symbolic_analysis():
    n = 12
    Ap, Ai, Ax = [0], [], []
    for j in range(n):
        if j:
            Ai.append(0); Ax.append(-0.2 * j)
        Ai.append(j); Ax.append(20.0)
        Ap.append(len(Ai))
    S = ScalarCSC(n, np.array(Ap), np.array(Ai), np.array(Ax))
    A = BlockCSCHessian(n, S.Ap, S.Ai, 1, S.Ax)
    expected = np.linspace(-1, 2, n)
    rhs = S.apply(expected)
    f = B200Factorizer()
    for native in (True, False, True):
        f.orderingMethod = OrderingMethod.Native if native else OrderingMethod.AMD
        f.factorize(A)
        assert np.linalg.norm(f.solve(rhs) - expected) < 1e-12
        f.orderingMethod = OrderingMethod.AMD if native else OrderingMethod.Native
        assert np.linalg.norm(f.solve(rhs) - expected) < 1e-12


@pytest.mark.parametrize("single", [False, True])
def test_native_amalgamation_known_answer(single):
    """tests/test_native_ordering.cc:123-153: nnz 43, identity permutation, solves."""
    H = SystemAssembler(5, 2).blockSparsityPattern([[0, 3], [1, 2], [2, 4], [3, 4]])
    H.setZero()
    for i, j in H.toScalar(sparsityOnly=True).entries():
        H.addNZScalar(i, j, 20.0 + i if i == j else 0.2)
    S = H.toScalar()
    expected = np.linspace(1, 10, 10)
    rhs = S.apply(expected)
    f = make_cholesky_factorizer(CholeskyProvider.CatamariNative, single)
    f.factorizeSymbolic(H, [])
    assert f.getFactorNNZ() == 43
    f.factorizeNumeric(H)
    tol = 1e-5 if single else 1e-12
    assert np.linalg.norm(f.solve(rhs) - expected) < tol * np.linalg.norm(expected)
    res = f.solveRawReduced(rhs, alreadyPermuted=True)
    assert np.linalg.norm(res - expected) < tol * np.linalg.norm(expected)
    assert np.array_equal(f.removeFixedEntries(rhs, True), rhs)


def test_padding_rows_untouched():
    """mfs_solve with ldb > rows leaves the padding of every column untouched
    (the padded-RHS behaviour of tests/test_catamari_solve_kernels.cc:33-51)."""
    import ctypes as C
    from meshfemsparse_b200 import _lib
    A = path_hessian(6, 3)
    f = B200Factorizer()
    f.factorize(A)
    n = A.n
    ld = n + 3
    X = np.zeros((3, ld))
    X[:, n:] = 99.0
    expected = np.random.default_rng(1).normal(size=(3, n))
    for r in range(3):
        X[r, :n] = A.apply(expected[r])
    flat = np.ascontiguousarray(X)
    _lib.check(f._lib.mfs_solve(f._h, _lib.dptr(flat), _lib.dptr(flat), 3, ld, _lib.MFS_SOLVE_FULL), f._h)
    assert np.all(flat[:, n:] == 99.0)
    assert np.linalg.norm(flat[:, :n] - expected) < 1e-11 * np.linalg.norm(expected)
