"""Bordered Hessians (dense border + low-rank term) reduced through the sparse
factorization, checked against a dense solve (CPU; the factorizer here is a dense
stand-in with the same interface as B200Factorizer)."""
import numpy as np
import pytest

from meshfemsparse_b200.bordered import BorderedSparseFactorization, BorderedSparseHessian

from helpers import random_stencil_hessian


class DenseFactorizer:
    def factorizeSymbolic(self, H, pins):
        self.pins = np.asarray(pins, dtype=np.int64)

    def factorizeNumeric(self, H):
        self.A = H.to_scipy_full().toarray()
        self.keep = np.ones(self.A.shape[0], dtype=bool)
        self.keep[self.pins] = False

    def solveMultiRHS(self, B):
        X = np.zeros_like(B)
        k = self.keep
        X[k] = np.linalg.solve(self.A[np.ix_(k, k)], B[k])
        return X

    def solve(self, b):
        return self.solveMultiRHS(b[:, None])[:, 0]


def bordered(seed, nd=3, rank=2, hdd_scale=50.0):
    rng = np.random.default_rng(seed)
    Hs = random_stencil_hessian(seed)
    ns = Hs.n
    H_sd = rng.normal(size=(ns, nd)) * 0.3
    H_dd = np.diag(rng.uniform(1, 2, nd)) * hdd_scale
    H = BorderedSparseHessian(Hs, H_sd, H_dd)
    if rank:
        H.addLowRank(rng.normal(size=(ns + nd, rank)), 0.5)
    return H


def dense(H):
    ns, nd = H.numSparseVars(), H.numDenseVars()
    M = np.zeros((ns + nd, ns + nd))
    M[:ns, :ns] = H.H_ss.to_scipy_full().toarray()
    M[:ns, ns:] = H.H_sd
    M[ns:, :ns] = H.H_sd.T
    M[ns:, ns:] = H.H_dd
    V = np.vstack([H.V_s, H.V_d])
    return M + V @ V.T


@pytest.mark.parametrize("rank", [0, 2])
def test_bordered_solve_matches_dense(rank):
    H = bordered(4, rank=rank)
    M = dense(H)
    x = np.random.default_rng(1).normal(size=H.numVars())
    assert np.allclose(H.apply(x), M @ x)
    pins = np.array([0, 1, 2])
    F = BorderedSparseFactorization(H, DenseFactorizer(), pins)
    assert not F.indefinite
    b = M @ x
    keep = np.ones(H.numVars(), dtype=bool)
    keep[pins] = False
    xr = np.zeros_like(x)
    xr[keep] = np.linalg.solve(M[np.ix_(keep, keep)], b[keep])
    got = F.solve(b)
    assert np.allclose(got, xr, rtol=1e-9, atol=1e-9 * np.abs(xr).max())
    assert np.all(got[pins] == 0.0)


def test_indefinite_dense_block_is_projected():
    H = bordered(6, rank=0, hdd_scale=-5.0)
    F = BorderedSparseFactorization(H, DenseFactorizer(), [])
    assert F.indefinite
    nd = H.numDenseVars()
    assert np.linalg.eigvalsh(F.S[:nd, :nd]).min() > 0
    assert np.all(np.isfinite(F.solve(np.ones(H.numVars()))))


def test_no_border_is_the_sparse_solve():
    H = BorderedSparseHessian(random_stencil_hessian(2))
    f = DenseFactorizer()
    F = BorderedSparseFactorization(H, f, [])
    b = np.arange(H.numVars(), dtype=float)
    assert np.allclose(F.solve(b), f.solve(b))


def test_equality_constraints_match_dense_kkt():
    H = bordered(8, nd=2, rank=1)
    rng = np.random.default_rng(3)
    m = 3
    C = rng.normal(size=(m, H.numVars()))
    H.setConstraints(C)
    F = BorderedSparseFactorization(H, DenseFactorizer(), [])
    b = rng.normal(size=H.numVars())
    r = rng.normal(size=m)
    x, lam = F.solve(b, r, return_multipliers=True)
    M = dense(H)
    K = np.block([[M, C.T], [C, np.zeros((m, m))]])
    ref = np.linalg.solve(K, np.concatenate([b, r]))
    assert np.allclose(x, ref[:H.numVars()], rtol=1e-8, atol=1e-9)
    assert np.allclose(lam, ref[H.numVars():], rtol=1e-8, atol=1e-9)
    assert np.allclose(C @ x, r)
