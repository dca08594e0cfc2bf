"""mfs_apply_noalloc through the C ABI: y = H x without any device allocation.

Some callers cannot allocate device memory where they apply the operator: a
process whose caching allocator has already reserved the GPU, or a loop that
cannot afford the device-wide synchronisation of cudaMalloc / cudaFree. The
entry point keeps its temporaries in one fixed device array instead. Its
result must equal the host product H x (restricted to the free rows, in the
caller's vector order) and mfs_apply's on the same inputs, call after call (the
array keeps the previous call's contents). This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from meshfemsparse_b200 import B200Factorizer, _lib

from helpers import cube_problem, path_hessian

pytestmark = pytest.mark.gpu

D = _lib.MFS_DEVICE_POINTERS
MAX_ENTRIES = 1 << 20


def _ptr(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


def _factorized_cube():
    H, tets, Ke, pins, nodes = cube_problem(4)
    f = B200Factorizer()
    f.factorize(H, pins)
    return H, f


def _host_product(H, f, X: np.ndarray, mode: int) -> np.ndarray:
    """H x on the host in the vector order of `mode` (X: rows x nrhs)."""
    if mode == _lib.MFS_SOLVE_FULL:
        xf = X.copy()
        xf[f.getFixedVars()] = 0.0
        y = H.apply(xf)
        y[f.getFixedVars()] = 0.0
        return y
    permute = mode == _lib.MFS_SOLVE_REDUCED_PERMUTED
    xf = f.extractFullSolution(X, permute=permute)
    return f.removeFixedEntries(H.apply(xf), permute=permute)


@pytest.mark.parametrize("mode", [_lib.MFS_SOLVE_FULL, _lib.MFS_SOLVE_REDUCED, _lib.MFS_SOLVE_REDUCED_PERMUTED])
def test_apply_noalloc_matches_host_and_apply_on_two_calls(mode):
    H, f = _factorized_cube()
    lib = _lib.load()
    rows = H.n if mode == _lib.MFS_SOLVE_FULL else f.n_reduced()
    rng = np.random.default_rng(5)
    for nrhs in (3, 1):   # the second, smaller call runs over the first call's leftovers
        Xh = rng.normal(size=(nrhs, rows))
        X = torch.from_numpy(Xh).cuda()                               # column-major rows x nrhs
        Y_ref = torch.empty_like(X)
        Y = torch.full_like(X, float("nan"))
        _lib.check(lib.mfs_apply(f._h, _ptr(X), _ptr(Y_ref), nrhs, rows, mode | D), f._h, "apply")
        _lib.check(lib.mfs_apply_noalloc(f._h, _ptr(X), _ptr(Y), nrhs, rows, mode | D), f._h, "apply_noalloc")
        torch.cuda.synchronize()
        assert bool(torch.isfinite(Y).all())
        host = _host_product(H, f, Xh.T, mode).T
        Yh = Y.cpu().numpy()
        assert np.linalg.norm(Yh - host) <= 1e-13 * np.linalg.norm(host)
        assert float((Y - Y_ref).norm()) <= 1e-13 * float(Y_ref.norm())


def test_apply_noalloc_accepts_exactly_the_limit():
    """free variables x right-hand sides == 1,048,576 is accepted (1,024 x 1,024)."""
    H = path_hessian(1025, 1)
    f = B200Factorizer()
    f.factorize(H, [0])
    assert f.n_reduced() == 1024
    nrhs = MAX_ENTRIES // 1024
    lib = _lib.load()
    Xh = np.random.default_rng(9).normal(size=(nrhs, H.n))
    X = torch.from_numpy(Xh).cuda()
    Y = torch.full_like(X, float("nan"))
    _lib.check(lib.mfs_apply_noalloc(f._h, _ptr(X), _ptr(Y), nrhs, H.n, _lib.MFS_SOLVE_FULL | D), f._h,
               "apply_noalloc")
    torch.cuda.synchronize()
    host = _host_product(H, f, Xh.T, _lib.MFS_SOLVE_FULL).T
    assert np.linalg.norm(Y.cpu().numpy() - host) <= 1e-13 * np.linalg.norm(host)
    X1 = torch.zeros((nrhs + 1, H.n), dtype=torch.float64, device="cuda")
    st = lib.mfs_apply_noalloc(f._h, _ptr(X1), _ptr(X1), nrhs + 1, H.n, _lib.MFS_SOLVE_FULL | D)
    assert st == _lib.MFS_SIZE_MISMATCH


def test_apply_noalloc_rejects_oversize_and_host_vectors():
    H, f = _factorized_cube()
    lib = _lib.load()
    nrhs = MAX_ENTRIES // f.n_reduced() + 1
    X = torch.zeros((nrhs, H.n), dtype=torch.float64, device="cuda")
    st = lib.mfs_apply_noalloc(f._h, _ptr(X), _ptr(X), nrhs, H.n, _lib.MFS_SOLVE_FULL | D)
    assert st == _lib.MFS_SIZE_MISMATCH
    x = np.zeros(H.n)
    st = lib.mfs_apply_noalloc(f._h, _lib.dptr(x), _lib.dptr(x), 1, H.n, _lib.MFS_SOLVE_FULL)
    assert st == _lib.MFS_INVALID_ARG
