"""Bordered Hessians: a sparse block H_ss plus dense rows/columns and a low-rank term,
solved through the supernodal factorization of H_ss (BorderedSparseHessian.hh:1-100,
BorderedSparseHessian.cc:60-206).

    H = [H_ss  H_sd] + [V_s][V_s]^T        (sparse variables first, dense last)
        [H_ds  H_dd]   [V_d][V_d]

With B = [H_sd V_s] and D = [[H_dd, V_d], [V_d^T, -I_r]] the system [H_ss B; B^T D]
is reduced by block elimination: Y = H_ss^{-1} B (one multi-RHS solve on the GPU
with n_d + r right-hand sides), S = D - B^T Y; then for a right-hand side b,
y = S^{-1} (c - Y^T b_s) with c = [b_d; 0] (dense QR, since S is indefinite
once a low-rank term is present) and x_s = H_ss^{-1} (b_s - B y). As in the
reference, the dense-variable block of S is projected positive definite
(|eigenvalues| floored at 1e-10) when it is indefinite, and `indefinite` says so.
The reference's equality-constraint fields have no solve path there either and
are not carried here.
"""
from __future__ import annotations

import numpy as np

from .hessian import BlockCSCHessian


class BorderedSparseHessian:
    def __init__(self, H_ss: BlockCSCHessian, H_sd=None, H_dd=None):
        self.H_ss = H_ss
        ns = H_ss.n
        self.H_sd = np.zeros((ns, 0)) if H_sd is None else np.asarray(H_sd, dtype=float)
        nd = self.H_sd.shape[1]
        self.H_dd = np.zeros((nd, nd)) if H_dd is None else np.asarray(H_dd, dtype=float)
        self.V_s = np.zeros((ns, 0))
        self.V_d = np.zeros((nd, 0))
        if self.H_sd.shape[0] != ns or self.H_dd.shape != (nd, nd):
            raise ValueError("dense blocks do not match the sparse block's size")

    def numSparseVars(self) -> int:
        return self.H_ss.n

    def numDenseVars(self) -> int:
        return self.H_sd.shape[1]

    def numVars(self) -> int:
        return self.numSparseVars() + self.numDenseVars()

    def low_rank_rank(self) -> int:
        return self.V_s.shape[1]

    def addLowRank(self, V, w: float = 1.0) -> None:
        """Add w V V^T (V has numVars rows; w >= 0)."""
        V = np.asarray(V, dtype=float).reshape(self.numVars(), -1)
        if w < 0:
            raise ValueError("low-rank weight must be nonnegative")
        V = np.sqrt(w) * V
        ns = self.numSparseVars()
        self.V_s = np.hstack([self.V_s, V[:ns]])
        self.V_d = np.hstack([self.V_d, V[ns:]])

    def apply(self, x) -> np.ndarray:
        """([H_ss H_sd; H_ds H_dd] + V V^T) x."""
        x = np.asarray(x, dtype=float)
        ns = self.numSparseVars()
        xs, xd = x[:ns], x[ns:]
        ys = self.H_ss.apply(xs) + self.H_sd @ xd
        yd = self.H_sd.T @ xs + self.H_dd @ xd
        if self.low_rank_rank():
            t = self.V_s.T @ xs + self.V_d.T @ xd
            ys = ys + self.V_s @ t
            yd = yd + self.V_d @ t
        return np.concatenate([ys, yd])


class BorderedSparseFactorization:
    """Factorization of a BorderedSparseHessian over a sparse factorizer (B200Factorizer)."""

    def __init__(self, H: BorderedSparseHessian, factorizer, fixedVars=()):
        self.solver = factorizer
        self.fixed = np.asarray(fixedVars, dtype=np.int64)
        self.solver.factorizeSymbolic(H.H_ss, self.fixed)
        self.updateNumericFactorization(H)

    def updateNumericFactorization(self, H: BorderedSparseHessian) -> bool:
        self.solver.factorizeNumeric(H.H_ss)
        nd, r = H.numDenseVars(), H.low_rank_rank()
        self.ndv, self.r = nd, r
        self.B = np.hstack([H.H_sd, H.V_s])
        self.indefinite = False
        if self.B.shape[1] == 0:
            self.S = np.zeros((0, 0))
            self.Y = np.zeros((H.numSparseVars(), 0))
            return False
        Bp = self.B.copy()
        Bp[self.fixed] = 0.0
        self.Y = self.solver.solveMultiRHS(Bp)
        D = np.zeros((nd + r, nd + r))
        D[:nd, :nd] = H.H_dd
        D[:nd, nd:] = H.V_d
        D[nd:, :nd] = H.V_d.T
        D[nd:, nd:] = -np.eye(r)
        self.S = D - Bp.T @ self.Y
        if nd:
            S_dd = 0.5 * (self.S[:nd, :nd] + self.S[:nd, :nd].T)
            lam, Q = np.linalg.eigh(S_dd)
            self.indefinite = bool((lam < 0).any())
            lam = np.maximum(np.abs(lam), 1e-10)
            self.S[:nd, :nd] = (Q * lam) @ Q.T
        return self.indefinite

    def solve(self, b) -> np.ndarray:
        b = np.asarray(b, dtype=float)
        ns = self.Y.shape[0]
        bs = b[:ns].copy()
        bs[self.fixed] = 0.0
        if self.B.shape[1] == 0:
            return self.solver.solve(bs)
        c = np.concatenate([b[ns:], np.zeros(self.r)])
        q, rr = np.linalg.qr(self.S)
        y = np.linalg.solve(rr, q.T @ (c - self.Y.T @ bs))
        rhs = bs - self.B @ y
        rhs[self.fixed] = 0.0
        xs = self.solver.solve(rhs)
        return np.concatenate([xs, y[:self.ndv]])
