"""Learned preconditioner for PCG on Newton sequences (no reference counterpart).

A 4-layer message-passing network (hidden 64, BF16 weights, FP32 accumulation)
reads the Jacobi-scaled Hessian blocks and emits a lower block-triangular G on
H's pattern; PCG runs with M^{-1} = D^{-1/2} G^T G D^{-1/2} and falls back to
the supernodal Cholesky factor when it misses the tolerance within the cap.
Training, inference and PCG run in the library's own CUDA kernels
(csrc/kernels_learned.cu); this module only holds the handle and the weights.
"""
from __future__ import annotations

import ctypes as C
import struct
from pathlib import Path

import numpy as np

from . import _lib

_MAGIC = b"MFSLPC01"


def param_count() -> int:
    n = C.c_int64()
    _lib.check(_lib.load().mfs_lpc_param_count(C.byref(n)), None, "param count")
    return int(n.value)


def _f32ptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _vectors(B: np.ndarray):
    B = np.asarray(B, dtype=np.float64)
    return np.asfortranarray(B.reshape(B.shape[0], -1))


class LearnedPreconditioner:
    """Network weights (FP32 master + BF16 copy) and Adam state on one GPU."""

    def __init__(self, device: int = 0, seed: int = 0):
        self._lib = _lib.load()
        self._p = C.c_void_p()
        _lib.check(self._lib.mfs_lpc_create(C.byref(self._p), int(device), int(seed)), None, "mfs_lpc_create failed")
        self.device = device
        self.n = param_count()

    def __del__(self):
        p = getattr(self, "_p", None)
        if p is not None and p.value:
            try:
                self._lib.mfs_lpc_destroy(p)
            except Exception:
                pass
            self._p = None

    def get_weights(self) -> np.ndarray:
        w = np.zeros(self.n, dtype=np.float32)
        _lib.check(self._lib.mfs_lpc_get_weights(self._p, _f32ptr(w), self.n), None, "get weights")
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != self.n:
            raise ValueError(f"expected {self.n} weights, got {w.size}")
        _lib.check(self._lib.mfs_lpc_set_weights(self._p, _f32ptr(w), self.n), None, "set weights")

    def save(self, path) -> None:
        """Weights with a versioned header: magic, parameter count, float32 data."""
        w = self.get_weights()
        Path(path).write_bytes(_MAGIC + struct.pack("<q", w.size) + w.tobytes())

    def load(self, path) -> None:
        raw = Path(path).read_bytes()
        if raw[:8] != _MAGIC:
            raise ValueError("not a learned-preconditioner weight file")
        (n,) = struct.unpack("<q", raw[8:16])
        if n != self.n:
            raise ValueError(f"weight file holds {n} parameters, this network has {self.n}")
        self.set_weights(np.frombuffer(raw[16:16 + 4 * n], dtype=np.float32))

    def loss_grad(self, fac, B, X, Ax=None, mode: int = _lib.MFS_SOLVE_FULL):
        """Loss and gradient (float32, host) for pairs (B, X) on fac's pattern."""
        Bm, Xm = _vectors(B), _vectors(X)
        loss = C.c_double()
        g = np.zeros(self.n, dtype=np.float32)
        ax = None if Ax is None else np.ascontiguousarray(Ax, dtype=np.float64)
        _lib.check(self._lib.mfs_lpc_loss_grad(fac._h, self._p, _lib.dptr(ax), _lib.dptr(Bm), _lib.dptr(Xm),
                                               Bm.shape[1], Bm.shape[0], mode, C.byref(loss), _f32ptr(g)),
                   fac._h, "loss/gradient failed")
        return float(loss.value), g

    def train_step(self, fac, B, X, lr: float = 1e-3, Ax=None, mode: int = _lib.MFS_SOLVE_FULL,
                   device_pointers: bool = False, nrhs: int | None = None, ld: int | None = None) -> float:
        """One Adam step on pairs (B, X = H^{-1} B). With device_pointers, B / X / Ax are
        device addresses (ints) and nrhs / ld must be given."""
        loss = C.c_double()
        if device_pointers:
            flags = mode | _lib.MFS_DEVICE_POINTERS
            _lib.check(self._lib.mfs_lpc_train_step(fac._h, self._p, C.c_void_p(Ax), C.c_void_p(B), C.c_void_p(X),
                                                    nrhs, ld, flags, float(lr), C.byref(loss)), fac._h,
                       "train step failed")
            return float(loss.value)
        Bm, Xm = _vectors(B), _vectors(X)
        ax = None if Ax is None else np.ascontiguousarray(Ax, dtype=np.float64)
        _lib.check(self._lib.mfs_lpc_train_step(fac._h, self._p, _lib.dptr(ax), _lib.dptr(Bm), _lib.dptr(Xm),
                                                Bm.shape[1], Bm.shape[0], mode, float(lr), C.byref(loss)),
                   fac._h, "train step failed")
        return float(loss.value)


def pcg_solve(fac, B, net: LearnedPreconditioner | None = None, Ax=None, maxit: int = 200, tol: float = 1e-10,
              mode: int = _lib.MFS_SOLVE_FULL):
    """PCG on fac's pattern with the learned preconditioner (Jacobi when net is None);
    falls back to fac's Cholesky factor when PCG misses tol within maxit.
    Returns (X, iterations, fallback_used)."""
    lib = _lib.load()
    Bm = _vectors(B)
    X = np.zeros_like(Bm, order="F")
    it = C.c_int32()
    ax = None if Ax is None else np.ascontiguousarray(Ax, dtype=np.float64)
    _lib.check(lib.mfs_pcg_solve(fac._h, net._p if net is not None else None, _lib.dptr(ax), _lib.dptr(Bm),
                                 _lib.dptr(X), Bm.shape[1], Bm.shape[0], mode, int(maxit), float(tol), C.byref(it)),
               fac._h, "PCG solve failed")
    st = fac.stats()
    out = X[:, 0].copy() if np.asarray(B).ndim == 1 else np.ascontiguousarray(X)
    return out, int(it.value), bool(st["pcg_fallback"])
