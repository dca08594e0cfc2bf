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
Equality constraints C x = r (C = [C_s C_d], m rows) add Lagrange multipliers
(BorderedSparseHessian.hh:56-75 derives the elimination; the reference's
factorization does not solve with them). With W = H_ss^{-1} C_s^T (m more
right-hand sides in the same multi-RHS solve) and C_2' = [C_d 0] - C_s Y, the
dense system becomes
    [S     C_2'^T      ] [y]   [c - Y^T b_s]
    [C_2'  -C_s W      ] [l] = [r - C_s z  ],   z = H_ss^{-1} b_s,
and x_s = z - Y y - W l. The multiplier block is negative definite and is not
projected (a saddle point is sought).
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
        self.C_s = np.zeros((0, ns))
        self.C_d = np.zeros((0, nd))
        if self.H_sd.shape[0] != ns or self.H_dd.shape != (nd, nd):
            raise ValueError("dense blocks do not match the sparse block's size")

    def setConstraints(self, C) -> None:
        """Equality constraints C x = r (C has numVars columns); r is given to solve()."""
        C = np.atleast_2d(np.asarray(C, dtype=float))
        if C.shape[1] != self.numVars():
            raise ValueError("constraint matrix must have numVars columns")
        ns = self.numSparseVars()
        self.C_s, self.C_d = C[:, :ns], C[:, ns:]

    def numConstraints(self) -> int:
        return self.C_s.shape[0]

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
        nd, r, m = H.numDenseVars(), H.low_rank_rank(), H.numConstraints()
        self.ndv, self.r, self.m = nd, r, m
        self.B = np.hstack([H.H_sd, H.V_s])
        self.C_s = H.C_s.copy()
        self.C_s[:, self.fixed] = 0.0
        self.indefinite = False
        k = self.B.shape[1]
        if k + m == 0:
            self.S = np.zeros((0, 0))
            self.Y = np.zeros((H.numSparseVars(), 0))
            return False
        Bp = np.hstack([self.B, self.C_s.T])
        Bp[self.fixed] = 0.0
        YW = self.solver.solveMultiRHS(Bp)
        self.Y, self.W = YW[:, :k], YW[:, k:]
        self.B[self.fixed] = 0.0
        D = np.zeros((nd + r, nd + r))
        D[:nd, :nd] = H.H_dd
        D[:nd, nd:] = H.V_d
        D[nd:, :nd] = H.V_d.T
        D[nd:, nd:] = -np.eye(r)
        self.S = D - self.B.T @ self.Y
        if nd:
            S_dd = 0.5 * (self.S[:nd, :nd] + self.S[:nd, :nd].T)
            lam, Q = np.linalg.eigh(S_dd)
            self.indefinite = bool((lam < 0).any())
            lam = np.maximum(np.abs(lam), 1e-10)
            self.S[:nd, :nd] = (Q * lam) @ Q.T
        if m:
            C2 = np.hstack([H.C_d, np.zeros((m, r))]) - self.C_s @ self.Y
            K = np.zeros((k + m, k + m))
            K[:k, :k] = self.S
            K[:k, k:] = C2.T
            K[k:, :k] = C2
            K[k:, k:] = -self.C_s @ self.W
            self.S = K
        return self.indefinite

    def solve(self, b, r=None, return_multipliers: bool = False):
        """x for right-hand side b (numVars); with constraints, C x = r (zero when r is None)."""
        b = np.asarray(b, dtype=float)
        ns = self.Y.shape[0]
        bs = b[:ns].copy()
        bs[self.fixed] = 0.0
        k = self.B.shape[1]
        if k + self.m == 0:
            x = self.solver.solve(bs)
            return (x, np.zeros(0)) if return_multipliers else x
        c = np.concatenate([b[ns:], np.zeros(self.r)])
        z = self.solver.solve(bs) if self.m else None
        rhs_d = c - self.Y.T @ bs
        if self.m:
            rv = np.zeros(self.m) if r is None else np.asarray(r, dtype=float)
            rhs_d = np.concatenate([rhs_d, rv - self.C_s @ z])
        q, rr = np.linalg.qr(self.S)
        sol = np.linalg.solve(rr, q.T @ rhs_d)
        y, lam = sol[:k], sol[k:]
        if self.m:
            xs = z - self.Y @ y - self.W @ lam
        else:
            rhs = bs - self.B @ y
            rhs[self.fixed] = 0.0
            xs = self.solver.solve(rhs)
        x = np.concatenate([xs, y[:self.ndv]])
        return (x, lam) if return_multipliers else x
