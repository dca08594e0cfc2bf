"""`solve_system` driver and SPSD system over the GPU factorizer.

The reference's CLI (tests/solve_system.cc:9-41) reads a triplet matrix in the
TripletMatrix binary format (SparseMatrices.hh:642-686: uint64 N, N uint64 row
indices, N uint64 column indices, N doubles; the sizes are the largest indices
plus one) and a text file of right-hand-side values, solves with SPSDSystem
(Solvers/SPSDSystem.hh: only the upper triangle is referenced, duplicates sum,
fixed variables may carry values) and prints the solution with 19 significant
digits. Here the factorization is B200Factorizer (FP64 plain by default):

    python -m meshfemsparse_b200.solve_system tmat.bin rhs.txt
"""
from __future__ import annotations

import struct
import sys

import numpy as np

from .hessian import BlockCSCHessian, ScalarCSC


def read_triplet_binary(path):
    """(m, n, rows, cols, values) of a TripletMatrix binary file."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < 8:
        raise RuntimeError(f"Failed to read triplet matrix {path}")
    (N,) = struct.unpack("<Q", raw[:8])
    if len(raw) < 8 + 24 * N:
        raise RuntimeError(f"truncated triplet matrix {path}")
    I = np.frombuffer(raw[8:8 + 8 * N], dtype="<u8").astype(np.int64)
    J = np.frombuffer(raw[8 + 8 * N:8 + 16 * N], dtype="<u8").astype(np.int64)
    V = np.frombuffer(raw[8 + 16 * N:8 + 24 * N], dtype="<f8").astype(np.float64)
    m = int(I.max()) + 1 if N else 0
    n = int(J.max()) + 1 if N else 0
    return m, n, I, J, V


def write_triplet_binary(path, rows, cols, values) -> None:
    rows = np.asarray(rows, dtype="<u8")
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", rows.size))
        f.write(rows.tobytes())
        f.write(np.asarray(cols, dtype="<u8").tobytes())
        f.write(np.asarray(values, dtype="<f8").tobytes())


def upper_csc(n, I, J, V) -> ScalarCSC:
    """Upper-triangle scalar CSC (i <= j entries, duplicates summed, diagonal ensured)."""
    keep = I <= J
    I, J, V = I[keep], J[keep], V[keep]
    diag = np.arange(n, dtype=np.int64)
    I = np.concatenate([I, diag])
    J = np.concatenate([J, diag])
    V = np.concatenate([V, np.zeros(n)])
    key = J * n + I
    uk, inv = np.unique(key, return_inverse=True)
    vals = np.zeros(uk.size)
    np.add.at(vals, inv, V)
    cols, rows = uk // n, uk % n
    Ap = np.zeros(n + 1, dtype=np.int64)
    np.add.at(Ap, cols + 1, 1)
    return ScalarCSC(n, np.cumsum(Ap), rows, vals)


class SPSDSystem:
    """Symmetric positive (semi)definite system K u = f with optional fixed variables,
    solved by a sparse Cholesky factorizer (SPSDSystem.hh: the SPD path)."""

    def __init__(self, n, rows, cols, values, factorizer=None):
        self.S = upper_csc(int(n), np.asarray(rows, dtype=np.int64), np.asarray(cols, dtype=np.int64),
                           np.asarray(values, dtype=float))
        self.H = BlockCSCHessian(self.S.n, self.S.Ap, self.S.Ai, 1, self.S.Ax)
        if factorizer is None:
            from .factorizer import B200Factorizer
            factorizer = B200Factorizer()
        self.fac = factorizer
        self.fixed = np.zeros(0, dtype=np.int64)
        self.fixed_values = np.zeros(0)
        self._factored = False

    def fixVariables(self, fixedVars, fixedVarValues=()) -> None:
        fv = np.asarray(fixedVars, dtype=np.int64)
        vals = np.asarray(fixedVarValues, dtype=float)
        if vals.size not in (0, fv.size):
            raise RuntimeError("Incorrect number of fixedVarValues")
        self.fixed = fv
        self.fixed_values = vals if vals.size else np.zeros(fv.size)
        self._factored = False

    def solve(self, f) -> np.ndarray:
        f = np.asarray(f, dtype=float)
        if f.shape[0] != self.S.n:
            raise RuntimeError("Bad RHS")
        if not self._factored:
            self.fac.factorizeSymbolic(self.H, self.fixed)
            self.fac.factorizeNumeric(self.H)
            self._factored = True
        b = f.copy()
        if self.fixed.size and np.any(self.fixed_values != 0):
            u0 = np.zeros(self.S.n)
            u0[self.fixed] = self.fixed_values
            b = b - self.S.apply(u0)               # move the fixed values to the right-hand side
        b[self.fixed] = 0.0
        u = self.fac.solve(b)
        u[self.fixed] = self.fixed_values
        return u


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2:
        print("usage: solve_system tmat.bin rhs.txt", file=sys.stderr)
        return 255
    m, n, I, J, V = read_triplet_binary(argv[0])
    try:
        rhs = np.loadtxt(argv[1], dtype=float, ndmin=1)
    except OSError:
        raise RuntimeError(f"Couldn't open input file {argv[1]}")
    if rhs.size != m:
        raise RuntimeError(f"System size mismatch ({rhs.size} vs {m})")
    u = SPSDSystem(max(m, n), I, J, V).solve(rhs)
    sys.stdout.write("".join(f"{v:.19g}\n" for v in u))
    return 0


if __name__ == "__main__":
    sys.exit(main())
