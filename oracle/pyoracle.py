"""ctypes wrapper of the C oracle -- test infrastructure only (tests/, smoke(), bench CPU legs).

Also holds the small numpy restatements used to cross-check the C oracle
(dense permuted matrices, residuals).
"""
from __future__ import annotations

import ctypes as C
import glob
import os
from pathlib import Path

import numpy as np

from .build import build_oracle

_lib = None


def _i64(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int64))


def _d(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def load():
    global _lib
    if _lib is not None:
        return _lib
    path = build_oracle()
    lib = C.CDLL(str(path))
    i64p = C.POINTER(C.c_int64)
    dp = C.POINTER(C.c_double)
    lib.orc_blas_load.argtypes = [C.c_char_p]
    lib.orc_blas_load.restype = C.c_int
    lib.orc_blas_loaded.restype = C.c_int
    lib.orc_max_threads.restype = C.c_int
    lib.orc_build_pattern.argtypes = [C.c_int64, C.c_int64, C.c_int, i64p, i64p, i64p]
    lib.orc_build_pattern.restype = C.c_int64
    lib.orc_assemble.argtypes = [C.c_int64, i64p, i64p, C.c_int64, i64p, dp, dp]
    lib.orc_assemble.restype = C.c_int
    lib.orc_symbolic.argtypes = [C.c_int64, i64p, i64p, i64p, C.c_int, C.c_int, C.c_int64, C.c_double, i64p, i64p,
                                 i64p, i64p, i64p, C.c_int64]
    lib.orc_symbolic.restype = C.c_int64
    lib.orc_inject.argtypes = [C.c_int64, i64p, C.c_int, C.c_int, dp, dp, C.c_double, dp, C.c_int64]
    lib.orc_mf_factor.argtypes = [C.c_int64, C.c_int, i64p, i64p, i64p, i64p, dp, C.c_int]
    lib.orc_mf_factor.restype = C.c_int64
    lib.orc_mf_solve.argtypes = [C.c_int64, C.c_int, i64p, i64p, i64p, i64p, dp, dp, C.c_int64, C.c_int, C.c_int]
    lib.orc_set_range.argtypes = [C.c_int64, C.c_int64]
    _lib = lib
    return lib


def load_blas() -> bool:
    """Load the OpenBLAS copy bundled with scipy for the timed CPU baseline."""
    lib = load()
    if lib.orc_blas_loaded():
        return True
    import scipy
    cands = glob.glob(os.path.join(os.path.dirname(scipy.__file__) + ".libs", "libscipy_openblas*.so"))
    for c in cands:
        if lib.orc_blas_load(c.encode()):
            return True
    return False


def build_pattern(nvars: int, conn: np.ndarray):
    lib = load()
    conn = np.ascontiguousarray(conn, dtype=np.int64)
    Ap = np.zeros(nvars + 1, dtype=np.int64)
    nnz = lib.orc_build_pattern(nvars, conn.shape[0], conn.shape[1], _i64(conn), _i64(Ap), None)
    Ai = np.zeros(nnz, dtype=np.int64)
    lib.orc_build_pattern(nvars, conn.shape[0], conn.shape[1], _i64(conn), _i64(Ap), _i64(Ai))
    return Ap, Ai


def assemble(nb: int, Ap, Ai, conn, Ke) -> np.ndarray:
    lib = load()
    conn = np.ascontiguousarray(conn, dtype=np.int64)
    Ke = np.ascontiguousarray(Ke, dtype=np.float64)
    Ax = np.zeros(int(Ap[-1]) * 9)
    if lib.orc_assemble(nb, _i64(Ap), _i64(Ai), conn.shape[0], _i64(conn), _d(Ke), _d(Ax)) != 0:
        raise ValueError("element block missing from the pattern")
    return Ax


def symbolic(Ap, Ai, iperm, vb: int, relax: bool = True, relax_zeros: int = 128, relax_ratio: float = 0.01):
    """Explicit-elimination symbolic analysis: returns dict(parent, cc, sn_start, L_ptr, L_rows)."""
    lib = load()
    nv = len(Ap) - 1
    Ap = np.ascontiguousarray(Ap, dtype=np.int64)
    Ai = np.ascontiguousarray(Ai, dtype=np.int64)
    iperm = np.ascontiguousarray(iperm, dtype=np.int64)
    parent = np.zeros(nv, dtype=np.int64)
    cc = np.zeros(nv, dtype=np.int64)
    sn = np.zeros(nv + 1, dtype=np.int64)
    Lp = np.zeros(nv + 1, dtype=np.int64)
    nsn = lib.orc_symbolic(nv, _i64(Ap), _i64(Ai), _i64(iperm), vb, int(relax), relax_zeros, relax_ratio,
                           _i64(parent), _i64(cc), _i64(sn), _i64(Lp), None, 0)
    Lr = np.zeros(max(int(Lp[-1]), 1), dtype=np.int64)
    lib.orc_symbolic(nv, _i64(Ap), _i64(Ai), _i64(iperm), vb, int(relax), relax_zeros, relax_ratio, _i64(parent),
                     _i64(cc), _i64(sn), _i64(Lp), _i64(Lr), Lr.size)
    return dict(parent=parent, cc=cc, sn_start=sn[:nsn + 1].copy(), L_ptr=Lp, L_rows=Lr[:Lp[-1]])


def inject(entries: np.ndarray, vb: int, src_ld: int, Ax, factor_size: int, Bx=None, sigma_b: float = 0.0):
    lib = load()
    ent = np.ascontiguousarray(entries, dtype=np.int64).reshape(-1)
    out = np.zeros(factor_size)
    Ax = np.ascontiguousarray(Ax, dtype=np.float64)
    Bx = None if Bx is None else np.ascontiguousarray(Bx, dtype=np.float64)
    lib.orc_inject(ent.size // 4, _i64(ent), vb, src_ld, _d(Ax), _d(Bx), sigma_b, _d(out), factor_size)
    return out


def mf_factor(sn: dict, factor: np.ndarray, threads: int = 0) -> int:
    """In-place multifrontal factorization of injected panels; returns -1 or the failing column."""
    lib = load()
    return int(lib.orc_mf_factor(len(sn["parent"]), sn["vb"], _i64(sn["sn_start"]), _i64(sn["parent"]),
                                 _i64(sn["struct_ptr"]), _i64(sn["struct_rows"]), _d(factor), threads))


def set_range(lo: int = 0, hi: int = -1):
    """Restrict mf_factor / mf_solve to the supernodes [lo, hi] (a postordered subtree)."""
    load().orc_set_range(lo, hi)


def mf_solve(sn: dict, factor: np.ndarray, B: np.ndarray, threads: int = 0) -> np.ndarray:
    lib = load()
    X = np.asfortranarray(np.array(B, dtype=np.float64, copy=True).reshape(B.shape[0], -1))
    lib.orc_mf_solve(len(sn["parent"]), sn["vb"], _i64(sn["sn_start"]), _i64(sn["parent"]), _i64(sn["struct_ptr"]),
                     _i64(sn["struct_rows"]), _d(factor), _d(X), X.shape[0], X.shape[1], threads)
    return X if B.ndim == 2 else X[:, 0]


def panel_layout(sn: dict):
    """(w, d, f, pan_off, col0) in scalar units for a supernode dict."""
    vb = sn["vb"]
    w = np.diff(sn["sn_start"]) * vb
    d = np.diff(sn["struct_ptr"]) * vb
    f = w + d
    pan = np.concatenate([[0], np.cumsum(f * w)])
    return w, d, f, pan, sn["sn_start"][:-1] * vb


def panels_to_dense(sn: dict, factor: np.ndarray, n: int) -> np.ndarray:
    """Scatter factor panels into a dense lower-triangular n x n matrix (lower part only)."""
    vb = sn["vb"]
    w, d, f, pan, col0 = panel_layout(sn)
    L = np.zeros((n, n))
    for s in range(len(w)):
        P = factor[pan[s]:pan[s + 1]].reshape(w[s], f[s]).T      # f x w
        rows = np.concatenate([col0[s] + np.arange(w[s]),
                               (sn["struct_rows"][sn["struct_ptr"][s]:sn["struct_ptr"][s + 1]][:, None] * vb
                                + np.arange(vb)[None, :]).reshape(-1)])
        cols = col0[s] + np.arange(w[s])
        for jj in range(w[s]):
            r = rows[jj:]
            L[r, cols[jj]] = P[jj:, jj]
    return L


def reduced_permuted_dense(H, pins, iperm_scalar) -> np.ndarray:
    """Dense A[p][:, p] of the pin-reduced scalar matrix under the scalar inverse permutation."""
    A = H.to_scipy_full().toarray()
    keep = np.ones(A.shape[0], dtype=bool)
    keep[np.asarray(pins, dtype=np.int64)] = False
    Ar = A[np.ix_(keep, keep)]
    return Ar[np.ix_(iperm_scalar, iperm_scalar)]


def scalar_perm_map(n_full: int, pins, iperm_scalar):
    """Full scalar index -> permuted reduced index (-1 for pins)."""
    keep = np.ones(n_full, dtype=bool)
    keep[np.asarray(pins, dtype=np.int64)] = False
    rr = np.full(n_full, -1, dtype=np.int64)
    rr[keep] = np.arange(int(keep.sum()))
    perm = np.empty_like(iperm_scalar)
    perm[iperm_scalar] = np.arange(iperm_scalar.size)
    return np.where(rr >= 0, perm[np.maximum(rr, 0)], -1)


def panels_to_csc(sn: dict, factor: np.ndarray, n: int):
    """The lower-triangular factor (or injected lower triangle) stored in catamari panels
    as an n x n scipy CSC matrix in the permuted reduced order."""
    import scipy.sparse as sp
    vb = sn["vb"]
    w, d, f, pan, col0 = panel_layout(sn)
    rows_all, cols_all, vals_all = [], [], []
    for s in range(len(w)):
        P = factor[pan[s]:pan[s + 1]].reshape(w[s], f[s]).T      # f x w, column-major panel
        srows = sn["struct_rows"][sn["struct_ptr"][s]:sn["struct_ptr"][s + 1]]
        rows = np.concatenate([col0[s] + np.arange(w[s]), (srows[:, None] * vb + np.arange(vb)[None, :]).reshape(-1)])
        ii, jj = np.nonzero(np.arange(f[s])[:, None] >= np.arange(w[s])[None, :])
        rows_all.append(rows[ii])
        cols_all.append(col0[s] + jj)
        vals_all.append(P[ii, jj])
    r = np.concatenate(rows_all)
    c = np.concatenate(cols_all)
    v = np.concatenate(vals_all)
    return sp.csc_matrix((v, (r, c)), shape=(n, n))
