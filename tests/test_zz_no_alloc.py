"""mfs_apply_noalloc through the C ABI: y = H x without any device allocation.

Some callers cannot allocate device memory where they apply the operator: a
process whose caching allocator has already reserved the GPU, or a loop that
cannot afford the device-wide synchronisation of cudaMalloc / cudaFree. The
entry point keeps its temporaries in one fixed device array instead. Its
result must equal mfs_apply's on the same inputs, call after call (the array
keeps the previous call's contents). This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from meshfemsparse_b200 import B200Factorizer, _lib

from helpers import cube_problem

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


@pytest.mark.parametrize("mode", [_lib.MFS_SOLVE_FULL, _lib.MFS_SOLVE_REDUCED_PERMUTED])
def test_apply_noalloc_matches_apply_on_two_calls(mode):
    H, f = _factorized_cube()
    lib = _lib.load()
    rows = H.n if mode == _lib.MFS_SOLVE_FULL else f.n_reduced()
    rng = np.random.default_rng(5)
    for nrhs in (3, 1):   # the second, smaller call runs over the first call's leftovers
        X = torch.from_numpy(rng.normal(size=(nrhs, rows))).cuda()   # column-major rows x nrhs
        Y_ref = torch.empty_like(X)
        Y = torch.full_like(X, float("nan"))
        _lib.check(lib.mfs_apply(f._h, _ptr(X), _ptr(Y_ref), nrhs, rows, mode | D), f._h, "apply")
        _lib.check(lib.mfs_apply_noalloc(f._h, _ptr(X), _ptr(Y), nrhs, rows, mode | D), f._h, "apply_noalloc")
        torch.cuda.synchronize()
        assert bool(torch.isfinite(Y).all())
        assert float((Y - Y_ref).norm()) <= 1e-13 * float(Y_ref.norm())


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
