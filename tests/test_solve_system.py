"""solve_system driver: triplet binary format, the SPSD system's upper-triangle
and fixed-variable handling (CPU, dense stand-in factorizer), and the CLI on the GPU."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from meshfemsparse_b200.solve_system import SPSDSystem, read_triplet_binary, upper_csc, write_triplet_binary

ROOT = Path(__file__).resolve().parents[1]


class DenseFactorizer:
    def factorizeSymbolic(self, H, pins):
        self.pins = np.asarray(pins, dtype=np.int64)

    def factorizeNumeric(self, H):
        self.A = H.to_scipy_full().toarray()

    def solve(self, b):
        k = np.ones(self.A.shape[0], dtype=bool)
        k[self.pins] = False
        x = np.zeros_like(b)
        x[k] = np.linalg.solve(self.A[np.ix_(k, k)], b[k])
        return x


def spd_triplets(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.normal(size=(n, n)) * 0.2
    K = M @ M.T + n * np.eye(n)
    K[np.abs(K) < 0.5] = 0.0
    K = 0.5 * (K + K.T) + np.eye(n)
    I, J = np.nonzero(K)
    return K, I, J, K[I, J]


def test_triplet_round_trip_and_upper_triangle(tmp_path):
    K, I, J, V = spd_triplets(12, 0)
    p = tmp_path / "t.bin"
    write_triplet_binary(p, I, J, V)
    m, n, I2, J2, V2 = read_triplet_binary(p)
    assert (m, n) == (12, 12) and np.array_equal(I2, I) and np.array_equal(V2, V)
    S = upper_csc(12, I2, J2, V2)
    assert np.allclose(S.to_dense(), K)
    # duplicates sum; lower entries are ignored
    S2 = upper_csc(3, np.array([0, 0, 1, 2, 1]), np.array([0, 0, 1, 2, 0]), np.array([1.0, 2.0, 5.0, 6.0, 9.0]))
    assert np.allclose(S2.to_dense(), np.diag([3.0, 5.0, 6.0]))


def test_spsd_system_with_fixed_values():
    K, I, J, V = spd_triplets(15, 1)
    sysm = SPSDSystem(15, I, J, V, factorizer=DenseFactorizer())
    f = np.arange(15, dtype=float)
    assert np.allclose(K @ sysm.solve(f), f)
    fixed, vals = np.array([2, 7]), np.array([0.5, -1.25])
    sysm.fixVariables(fixed, vals)
    u = sysm.solve(f)
    assert np.allclose(u[fixed], vals)
    free = np.setdiff1d(np.arange(15), fixed)
    assert np.allclose((K @ u)[free], f[free])
