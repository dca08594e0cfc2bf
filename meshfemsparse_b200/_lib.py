"""ctypes binding of the in-tree C ABI (include/mfs_b200.h).

The shared library is required: importing a GPU entry point without it raises
immediately instead of silently falling back to CPU code.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libmfs_b200.so"

MFS_OK, MFS_NOT_POSDEF, MFS_INVALID_ARG, MFS_SIZE_MISMATCH, MFS_NO_FACTOR, MFS_OOM, MFS_TIMEOUT, \
    MFS_CUDA_ERROR, MFS_INTERNAL = range(9)
MFS_PREC_FP64, MFS_PREC_FP32 = 0, 1
MFS_ORDER_ND, MFS_ORDER_NATIVE, MFS_ORDER_MD, MFS_ORDER_USER = 0, 1, 2, 3
MFS_SOLVE_FULL, MFS_SOLVE_REDUCED, MFS_SOLVE_REDUCED_PERMUTED = 0, 1, 2
MFS_DEVICE_POINTERS = 16

EXPORTED = [
    "mfs_default_options", "mfs_create", "mfs_destroy", "mfs_last_error", "mfs_build_pattern", "mfs_symbolic",
    "mfs_numeric", "mfs_solve", "mfs_assembly_setup", "mfs_assemble", "mfs_apply", "mfs_info",
    "mfs_inverse_permutation", "mfs_nd_ordering", "mfs_supernodes", "mfs_conversion_plan", "mfs_factor_values",
    "mfs_stash", "mfs_swap_stash", "mfs_clear_stash", "mfs_has_stash", "mfs_clear_factors", "mfs_get_stats",
    "mfs_set_options", "mfs_apply_noalloc", "mfs_lpc_param_count", "mfs_lpc_create", "mfs_lpc_destroy",
    "mfs_lpc_get_weights", "mfs_lpc_set_weights", "mfs_lpc_loss_grad", "mfs_lpc_train_step", "mfs_pcg_solve",
    "mfs_debug_gemm", "mfs_build_pattern_device", "mfs_conversion_plan_device", "mfs_debug_gemm_launches",
    "mfs_debug_dirty_subtrees", "mfs_debug_hierarchical_order",
]
GEMM_TASK_FIELDS = 12


class Options(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("ordering", C.c_int32), ("relax", C.c_int32), ("device", C.c_int32),
        ("relax_zeros", C.c_int64), ("relax_ratio", C.c_double), ("nd_leaf_size", C.c_int64),
        ("seed", C.c_uint64), ("stream", C.c_void_p), ("small_front_max", C.c_int32), ("refine", C.c_int32),
        ("refine_tol", C.c_double), ("refine_maxit", C.c_int32), ("use_graphs", C.c_int32),
        ("tensor_cores", C.c_int32), ("time_kernels", C.c_int32), ("nd_reuse_period", C.c_int32),
        ("solve_chain", C.c_int32), ("factor_group", C.c_int32),
        ("solve_subtrees", C.c_int32), ("reserved", C.c_int32 * 2),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("factor_ms", C.c_double), ("solve_ms", C.c_double), ("assemble_ms", C.c_double),
        ("refine_iterations", C.c_int32), ("failed_column", C.c_int32), ("residual", C.c_double),
        ("device_bytes", C.c_int64), ("num_levels", C.c_int32), ("num_large", C.c_int32),
        ("kernel_launches", C.c_int64), ("perturbed_pivots", C.c_int32), ("pcg_iterations", C.c_int32),
        ("pcg_fallback", C.c_int32), ("nd_reused", C.c_int32), ("pcg_ms", C.c_double),
        ("gemm_ms", C.c_double), ("gemm_flops", C.c_double), ("gemm_launches", C.c_int64),
        ("nd_rebuilt_vertices", C.c_int64), ("refactored_blocks", C.c_int32), ("split_escalations", C.c_int32),
    ]


_lib = None


def load() -> C.CDLL:
    """Load libmfs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m meshfemsparse_b200.build` first")
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    i64p = C.POINTER(C.c_int64)
    lib.mfs_default_options.argtypes = [C.POINTER(Options)]
    lib.mfs_create.argtypes = [C.POINTER(P), C.POINTER(Options)]
    lib.mfs_set_options.argtypes = [P, C.POINTER(Options)]
    lib.mfs_destroy.argtypes = [P]
    lib.mfs_last_error.argtypes = [P, C.c_char_p, C.c_size_t]
    lib.mfs_build_pattern.argtypes = [C.c_int64, C.c_int64, C.c_int32, i64p, i64p, i64p, i64p]
    lib.mfs_symbolic.argtypes = [P, C.c_int64, i64p, i64p, C.c_int32, i64p, C.c_int64, i64p, i64p, C.c_int64]
    lib.mfs_numeric.argtypes = [P, P, P, C.c_double, C.c_int32]
    lib.mfs_solve.argtypes = [P, P, P, C.c_int64, C.c_int64, C.c_int32]
    lib.mfs_assembly_setup.argtypes = [P, C.c_int64, i64p]
    lib.mfs_assemble.argtypes = [P, P, P, C.c_int32]
    lib.mfs_apply.argtypes = [P, P, P, C.c_int64, C.c_int64, C.c_int32]
    lib.mfs_apply_noalloc.argtypes = [P, P, P, C.c_int64, C.c_int64, C.c_int32]
    lib.mfs_info.argtypes = [P, i64p, i64p, i64p, C.POINTER(C.c_double), i64p, C.POINTER(C.c_int32)]
    lib.mfs_inverse_permutation.argtypes = [P, i64p]
    lib.mfs_nd_ordering.argtypes = [P, i64p, i64p, i64p, i64p]
    lib.mfs_supernodes.argtypes = [P, i64p, i64p, C.POINTER(C.c_int32), i64p, i64p, i64p, i64p, i64p]
    lib.mfs_conversion_plan.argtypes = [P, i64p, i64p, i64p, i64p]
    lib.mfs_conversion_plan_device.argtypes = [P, i64p, i64p, i64p, i64p]
    lib.mfs_build_pattern_device.argtypes = [C.c_int32, C.c_int64, C.c_int64, C.c_int32, P, P, P, i64p, P]
    lib.mfs_factor_values.argtypes = [P, i64p, P]
    for name in ("mfs_stash", "mfs_swap_stash", "mfs_clear_stash", "mfs_clear_factors"):
        getattr(lib, name).argtypes = [P]
    lib.mfs_has_stash.argtypes = [P, C.POINTER(C.c_int32)]
    lib.mfs_get_stats.argtypes = [P, C.POINTER(Stats)]
    f32p = C.POINTER(C.c_float)
    lib.mfs_lpc_param_count.argtypes = [i64p]
    lib.mfs_lpc_create.argtypes = [C.POINTER(P), C.c_int32, C.c_uint64]
    lib.mfs_lpc_destroy.argtypes = [P]
    lib.mfs_lpc_get_weights.argtypes = [P, f32p, C.c_int64]
    lib.mfs_lpc_set_weights.argtypes = [P, f32p, C.c_int64]
    lib.mfs_lpc_loss_grad.argtypes = [P, P, P, P, P, C.c_int64, C.c_int64, C.c_int32, C.POINTER(C.c_double), f32p]
    lib.mfs_lpc_train_step.argtypes = [P, P, P, P, P, C.c_int64, C.c_int64, C.c_int32, C.c_float,
                                       C.POINTER(C.c_double)]
    lib.mfs_pcg_solve.argtypes = [P, P, P, P, P, C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_double,
                                  C.POINTER(C.c_int32)]
    lib.mfs_debug_gemm.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, i64p, P, C.c_int64, P, C.c_int64,
                                   P, C.c_int64, C.c_char_p, C.c_size_t]
    lib.mfs_debug_gemm_launches.argtypes = [P, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    lib.mfs_debug_hierarchical_order.argtypes = [C.c_int64, i64p, i64p, C.c_int64, i64p, i64p, C.c_int32, i64p,
                                                 i64p]
    lib.mfs_debug_dirty_subtrees.argtypes = [C.c_int64, i64p, i64p, C.c_int64, i64p, i64p, C.POINTER(C.c_int32),
                                             i64p, C.POINTER(C.c_int64)]
    for name in EXPORTED:
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def i64ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64
    return C.c_void_p(a.ctypes.data)


class MFSError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


def check(status: int, handle=None, what: str = ""):
    """Raise like the reference: invalid_argument -> ValueError, everything else RuntimeError."""
    if status == MFS_OK:
        return
    msg = what
    if handle is not None:
        buf = C.create_string_buffer(1024)
        load().mfs_last_error(handle, buf, 1024)
        if buf.value:
            msg = buf.value.decode(errors="replace")
    if status == MFS_INVALID_ARG:
        raise ValueError(msg or "invalid argument")
    raise MFSError(status, msg or f"mfs status {status}")


def default_options(**kw) -> Options:
    o = Options()
    load().mfs_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def build_pattern(nvars: int, conn: np.ndarray):
    """SystemAssembler::blockSparsityPattern through the C ABI: returns (Ap, Ai)."""
    lib = load()
    conn = np.ascontiguousarray(conn, dtype=np.int64)
    nelem, npe = conn.shape
    Ap = np.zeros(nvars + 1, dtype=np.int64)
    nnz = C.c_int64(0)
    check(lib.mfs_build_pattern(nvars, nelem, npe, i64ptr(conn), i64ptr(Ap), None, C.byref(nnz)), what="pattern")
    Ai = np.zeros(nnz.value, dtype=np.int64)
    check(lib.mfs_build_pattern(nvars, nelem, npe, i64ptr(conn), i64ptr(Ap), i64ptr(Ai), C.byref(nnz)),
          what="pattern")
    return Ap, Ai


def debug_gemm(device: int, precision: int, kernel: int, tasks: np.ndarray, A: int, a_len: int, B: int,
               b_len: int, Cp: int, c_len: int):
    """Test hook: one launch of the factorization's GEMM kernel over `tasks`
    (ntasks x GEMM_TASK_FIELDS int64) on device arrays given by address."""
    tasks = np.ascontiguousarray(tasks, dtype=np.int64).reshape(-1, GEMM_TASK_FIELDS)
    buf = C.create_string_buffer(512)
    st = load().mfs_debug_gemm(device, precision, kernel, tasks.shape[0], i64ptr(tasks), C.c_void_p(A), a_len,
                               C.c_void_p(B), b_len, C.c_void_p(Cp), c_len, buf, 512)
    if st != MFS_OK:
        msg = buf.value.decode(errors="replace") or f"mfs status {st}"
        if st == MFS_INVALID_ARG:
            raise ValueError(msg)
        raise MFSError(st, msg)


def build_pattern_device(nvars: int, conn_ptr: int, nelem: int, npe: int, Ap_ptr: int, Ai_ptr: int | None,
                         device: int = 0, stream: int | None = None) -> int:
    """SystemAssembler::blockSparsityPattern on the GPU (device pointers by address);
    returns nnz (fills Ai when given)."""
    nnz = C.c_int64(0)
    st = load().mfs_build_pattern_device(device, nvars, nelem, npe, C.c_void_p(conn_ptr), C.c_void_p(Ap_ptr),
                                         C.c_void_p(Ai_ptr) if Ai_ptr else None, C.byref(nnz),
                                         C.c_void_p(stream) if stream else None)
    check(st, what="GPU pattern")
    return nnz.value


def library_present() -> bool:
    return LIB_PATH.exists() and os.access(LIB_PATH, os.R_OK)


def debug_gemm_launches(handle) -> np.ndarray:
    """Per tensor-core GEMM launch of the handle's last numeric factorization run with
    time_kernels on: rows of (ms, flops, tiles, tasks, kind); kind 0 left-looking group
    update, 1 row solve, 2 next-group update, 3 trailing update, 4 level SYRK."""
    lib = load()
    cnt = C.c_int64(0)
    check(lib.mfs_debug_gemm_launches(handle, 0, None, C.byref(cnt)), None, "mfs_debug_gemm_launches")
    out = np.zeros((max(cnt.value, 1), 5), dtype=np.float64)
    check(lib.mfs_debug_gemm_launches(handle, cnt.value, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(cnt)),
          None, "mfs_debug_gemm_launches")
    return out[:cnt.value]


def debug_dirty_subtrees(xadj: np.ndarray, adj: np.ndarray, cparent: np.ndarray, cmember: np.ndarray):
    """(full_rebuild, roots) of the temporal nested-dissection reuse rule for a previous
    separator forest and a new graph in CSR form (host only)."""
    xadj = np.ascontiguousarray(xadj, dtype=np.int64)
    adj = np.ascontiguousarray(adj, dtype=np.int64)
    cparent = np.ascontiguousarray(cparent, dtype=np.int64)
    cmember = np.ascontiguousarray(cmember, dtype=np.int64)
    roots = np.zeros(max(cparent.size, 1), dtype=np.int64)
    full, nroots = C.c_int32(0), C.c_int64(0)
    check(load().mfs_debug_dirty_subtrees(xadj.size - 1, i64ptr(xadj), i64ptr(adj if adj.size else np.zeros(1, np.int64)),
                                          cparent.size, i64ptr(cparent), i64ptr(cmember), C.byref(full),
                                          i64ptr(roots), C.byref(nroots)), None, "mfs_debug_dirty_subtrees")
    return bool(full.value), roots[:nroots.value].tolist()


def debug_hierarchical_order(xadj: np.ndarray, adj: np.ndarray, cparent: np.ndarray, cmember: np.ndarray,
                             cut_depth: int):
    """(perm new -> old, stats {cut, tasks, upper vertices, upper elements}) of the
    hierarchical constrained-minimum-degree final order (host only)."""
    xadj = np.ascontiguousarray(xadj, dtype=np.int64)
    adj = np.ascontiguousarray(adj, dtype=np.int64)
    cparent = np.ascontiguousarray(cparent, dtype=np.int64)
    cmember = np.ascontiguousarray(cmember, dtype=np.int64)
    n = xadj.size - 1
    perm = np.zeros(max(n, 1), dtype=np.int64)
    stats = np.zeros(4, dtype=np.int64)
    one = np.zeros(1, dtype=np.int64)
    check(load().mfs_debug_hierarchical_order(n, i64ptr(xadj), i64ptr(adj if adj.size else one), cparent.size,
                                              i64ptr(cparent if cparent.size else one),
                                              i64ptr(cmember if cmember.size else one), int(cut_depth),
                                              i64ptr(perm), i64ptr(stats)), None, "mfs_debug_hierarchical_order")
    return perm[:n], dict(cut=int(stats[0]), tasks=int(stats[1]), upper_vertices=int(stats[2]),
                          upper_elements=int(stats[3]))
