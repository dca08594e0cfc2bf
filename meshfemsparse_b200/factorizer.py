"""``CholeskyFactorizerBase``-compatible factorizer over the B200 C ABI.

Method names, argument meaning and error behaviour follow the reference's
``Solvers/CholeskyFactorizerBase.hh:50-443`` and ``Solvers/CatamariFactorizer.hh``
so code written against the catamari provider ports line by line:

* ``factorizeSymbolic(H, pinnedVars)`` / ``factorizeNumeric(H)`` /
  ``factorizeNumericWithShift(H, sigma[, B])`` / ``factorize(H, fixedVars)``
* ``solve(b)``, ``solveMultiRHS(B)``, ``solveRawReduced(b, alreadyPermuted)``,
  ``solveRawReducedInPlace(bx, alreadyPermuted)``
* ``removeFixedEntries(x, permute)`` / ``extractFullSolution(xr, permute)``
* stash/swap/clear, ``clearFactors``, ``getFactorNNZ``, ``getFlopEstimate``,
  ``getInversePermutation``, ``ndOrdering``, ``provider``.

Failures raise ``RuntimeError`` (``ValueError`` for invalid arguments, like the
reference's ``std::invalid_argument``). A non-positive pivot invalidates the
numeric factor (CatamariFactorizer.cc:701-705).
"""
from __future__ import annotations

import ctypes as C
import enum
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .adaptive_ordering import AdaptiveOrderingSelection
from .hessian import BlockCSCHessian, ScalarCSC


class CholeskyProvider(enum.Enum):
    CHOLMOD = 0
    Catamari = 1
    CatamariNesdis = 2
    CatamariNesdisParallel = 3
    CatamariMetis = 4
    CatamariLegacy = 5
    CatamariAMD = 6
    CatamariScotch = 7
    CatamariAdaptive = 8
    PARDISO = 9
    Accelerate = 10
    CatamariNesdisReuse = 11
    CatamariNative = 12
    CHOLMODNative = 13
    B200 = 14            # this library, nested-dissection ordering
    B200Native = 15      # this library, input order kept


class CholeskySys(enum.Enum):
    A = 0
    L = 1
    Lt = 2
    P = 3
    Pt = 4


class OrderingMethod(enum.IntEnum):
    CholmodNesdisParallel = _lib.MFS_ORDER_ND
    Native = _lib.MFS_ORDER_NATIVE
    AMD = _lib.MFS_ORDER_MD
    User = _lib.MFS_ORDER_USER
    # nested dissection or minimum degree, chosen per analysis from the timing history
    # (CatamariFactorizer::OrderingMethod::Adaptive); host-side only
    Adaptive = 100


class FactorizationType(enum.IntEnum):
    None_ = 0
    Symbolic = 1
    Numeric = 2


@dataclass
class NDOrdering:
    CParent: np.ndarray
    CMember: np.ndarray
    blockSize: int


def _as_hessian(mat) -> BlockCSCHessian:
    if isinstance(mat, BlockCSCHessian):
        return mat
    if isinstance(mat, ScalarCSC):
        return BlockCSCHessian(mat.n, mat.Ap, mat.Ai, 1, mat.Ax)
    raise TypeError("expected a BlockCSCHessian or ScalarCSC")


class B200Factorizer:
    """Supernodal Cholesky on one B200 (FP64 plain, or FP32 factor + FP64 refinement)."""

    def __init__(self, singlePrecision: bool = False, *, refine: bool = False, device: int = 0,
                 orderingMethod: OrderingMethod = OrderingMethod.CholmodNesdisParallel, refine_tol: float = 1e-10,
                 refine_maxit: int = 50, small_front_max: int = 0, tensor_cores: int = 0, relax: bool = True,
                 use_graphs: bool = False, nd_reuse_period: int = 0,
                 relax_zeros: int = 128, relax_ratio: float = 0.01, nd_leaf_size: int = 120, seed: int = 12345,
                 stream: int | None = None, solve_chain: int = 0, factor_group: int = 0, solve_subtrees: int = 0):
        self._lib = _lib.load()
        self.singlePrecision = bool(singlePrecision)
        self.orderingMethod = OrderingMethod(orderingMethod)
        self._base_opts = dict(
            precision=_lib.MFS_PREC_FP32 if singlePrecision else _lib.MFS_PREC_FP64, device=device,
            refine=int(refine), refine_tol=refine_tol, refine_maxit=refine_maxit, small_front_max=small_front_max,
            use_graphs=int(use_graphs), nd_reuse_period=int(nd_reuse_period),
            tensor_cores=tensor_cores, relax=int(relax), relax_zeros=relax_zeros, relax_ratio=relax_ratio,
            nd_leaf_size=nd_leaf_size, seed=seed, solve_chain=solve_chain, factor_group=factor_group,
            solve_subtrees=solve_subtrees)
        opts = _lib.default_options(**self._base_opts)
        # nested dissection, or minimum degree when the adaptive choice switches to it
        self.adaptiveOrdering = AdaptiveOrderingSelection(OrderingMethod.CholmodNesdisParallel, OrderingMethod.AMD)
        opts.ordering = int(OrderingMethod.CholmodNesdisParallel if self.orderingMethod == OrderingMethod.Adaptive
                            else self.orderingMethod)
        if stream is not None:
            opts.stream = C.c_void_p(stream)
        self._h = C.c_void_p()
        _lib.check(self._lib.mfs_create(C.byref(self._h), C.byref(opts)), None, "mfs_create failed")
        self._opts = opts
        self._fixed = np.zeros(0, dtype=np.int64)
        self._n_full = 0
        self._n_reduced = 0
        self._bs = 3
        self._maps = None
        self._stash_meta = None
        self._axlen = 0

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.mfs_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------- sizes
    def _type(self) -> int:
        t = C.c_int32(0)
        self._lib.mfs_info(self._h, None, None, None, None, None, C.byref(t))
        return int(t.value)

    def hasFactorization(self, sys: CholeskySys = CholeskySys.A) -> bool:
        need = FactorizationType.Numeric if sys in (CholeskySys.A, CholeskySys.L, CholeskySys.Lt) \
            else FactorizationType.Symbolic
        return self._type() >= need

    def hasNumericFactorization(self) -> bool:
        return self._type() >= FactorizationType.Numeric

    def checkPosDef(self) -> bool:
        return self.hasNumericFactorization()

    def _assert(self, t: FactorizationType):
        if self._type() < t:
            raise RuntimeError(("Numeric" if t == FactorizationType.Numeric else "Symbolic") +
                               " factorization does not exist")

    def m_reduced(self) -> int:
        self._assert(FactorizationType.Symbolic)
        return self._n_reduced

    def n_reduced(self) -> int:
        return self.m_reduced()

    def m(self) -> int:
        return self.n_reduced() + len(self._fixed)

    def n(self) -> int:
        return self.m()

    def hasFixedVars(self) -> bool:
        return len(self._fixed) > 0

    def getFixedVars(self) -> list[int]:
        return [int(v) for v in self._fixed]

    def provider(self) -> CholeskyProvider:
        if self.orderingMethod == OrderingMethod.Adaptive:
            return CholeskyProvider.CatamariAdaptive
        return CholeskyProvider.B200Native if self.orderingMethod == OrderingMethod.Native else CholeskyProvider.B200

    def wantsSymbolicFactorizationRecompute(self) -> bool:
        """Adaptive ordering: whether to redo the analysis now with the other method
        (CatamariFactorizer.hh:114-117)."""
        return self.orderingMethod == OrderingMethod.Adaptive and self.adaptiveOrdering.should_trigger_recompute()

    def _adaptive_record(self, what: str) -> None:
        if self.orderingMethod != OrderingMethod.Adaptive:
            return
        st = self.stats()
        if what == "numeric":
            self.adaptiveOrdering.record_numeric(st["factor_ms"] * 1e-3)
        else:
            self.adaptiveOrdering.record_solve(st["solve_ms"] * 1e-3)

    def preferInPlaceSolve(self) -> bool:
        return True

    def supportsPrePermutation(self) -> bool:
        return True

    # ----------------------------------------------------------- symbolic
    def factorizeSymbolic(self, mat, pinnedVars=(), user_perm=None, supernode_sizes=None):
        """Symbolic analysis. `user_perm` (User ordering): new->old over reduced block
        variables; `supernode_sizes` (Native/User): a partition to use verbatim."""
        H = _as_hessian(mat)
        pins = np.ascontiguousarray(np.asarray(list(pinnedVars), dtype=np.int64))
        up = None
        if self.orderingMethod == OrderingMethod.User:
            if user_perm is None:
                raise ValueError("User ordering requires user_perm")
            up = np.ascontiguousarray(np.asarray(user_perm, dtype=np.int64))
        sns = None if supernode_sizes is None else np.ascontiguousarray(np.asarray(supernode_sizes, dtype=np.int64))
        # the ordering choice takes effect here, at symbolic analysis
        adaptive = self.orderingMethod == OrderingMethod.Adaptive
        method = self.adaptiveOrdering.update_selection() if adaptive else self.orderingMethod
        self._opts.ordering = int(method)
        _lib.check(self._lib.mfs_set_options(self._h, C.byref(self._opts)), self._h, "set options")
        t0 = time.perf_counter()
        st = self._lib.mfs_symbolic(self._h, H.numBlocks, _lib.i64ptr(H.Ap), _lib.i64ptr(H.Ai), H.bs,
                                    _lib.i64ptr(pins) if pins.size else None, int(pins.size), _lib.i64ptr(up),
                                    _lib.i64ptr(sns), 0 if sns is None else int(sns.size))
        if adaptive and st == _lib.MFS_OK:
            self.adaptiveOrdering.record_symbolic(time.perf_counter() - t0, self.getFactorNNZ())
        if st != _lib.MFS_OK:
            self._fixed = np.zeros(0, dtype=np.int64)
            _lib.check(st, self._h, "symbolic factorization failed")
        self._fixed = np.unique(pins)
        self._bs = H.bs
        self._axlen = H.nz * H.bs * H.bs
        n_full, n_red = C.c_int64(), C.c_int64()
        self._lib.mfs_info(self._h, C.byref(n_full), C.byref(n_red), None, None, None, None)
        self._n_full, self._n_reduced = int(n_full.value), int(n_red.value)
        self._maps = None

    # ------------------------------------------------------------ numeric
    def _values(self, mat) -> np.ndarray:
        H = _as_hessian(mat)
        if H.Ax is None:
            raise ValueError("matrix has no values")
        return np.ascontiguousarray(H.Ax, dtype=np.float64)

    def factorizeNumeric(self, mat, isInTryCatch: bool = False):
        self._assert(FactorizationType.Symbolic)
        Ax = self._values(mat)
        _lib.check(self._lib.mfs_numeric(self._h, _lib.dptr(Ax), None, 0.0, 0), self._h, "numeric failed")
        self._adaptive_record("numeric")

    def factorizeNumericWithShift(self, A, sigma: float, B=None, isInTryCatch: bool = False):
        self._assert(FactorizationType.Symbolic)
        Ax = self._values(A)
        Bx = None
        if B is not None:
            HB, HA = _as_hessian(B), _as_hessian(A)
            if (HB.numBlocks != HA.numBlocks or HB.bs != HA.bs or not np.array_equal(HB.Ap, HA.Ap)
                    or not np.array_equal(HB.Ai, HA.Ai) or HB.Ax is None or HB.Ax.size != HA.Ax.size):
                raise ValueError("Shift matrix must have the same sparsity and value layout as A")
            Bx = self._values(B)
        _lib.check(self._lib.mfs_numeric(self._h, _lib.dptr(Ax), _lib.dptr(Bx), float(sigma), 0), self._h,
                   "numeric failed")
        self._adaptive_record("numeric")

    def factorize(self, mat, fixedVars=(), isInTryCatch: bool = False):
        self.factorizeSymbolic(mat, fixedVars)
        self.factorizeNumeric(mat)

    # ----------------------------------------------------------- assembly
    def setElements(self, conn: np.ndarray):
        """Element stencils (numElems x 4 node indices) for on-device assembly."""
        conn = np.ascontiguousarray(conn, dtype=np.int64)
        _lib.check(self._lib.mfs_assembly_setup(self._h, conn.shape[0], _lib.i64ptr(conn)), self._h,
                   "assembly setup failed")
        self._nelem = conn.shape[0]

    def assemble(self, Ke: np.ndarray, return_values: bool = True):
        """Assemble sum_e Ke_e on the GPU; the values stay resident for factorizeAssembled()."""
        Ke = np.ascontiguousarray(Ke, dtype=np.float64)
        out = np.empty(self._ax_len(), dtype=np.float64) if return_values else None
        _lib.check(self._lib.mfs_assemble(self._h, _lib.dptr(Ke), _lib.dptr(out), 0), self._h, "assemble failed")
        return out

    def factorizeAssembled(self, sigma: float = 0.0):
        _lib.check(self._lib.mfs_numeric(self._h, None, None, float(sigma), 0), self._h, "numeric failed")
        self._adaptive_record("numeric")

    def _ax_len(self) -> int:
        return self._axlen

    # -------------------------------------------------------------- maps
    def _row_maps(self):
        if self._maps is None:
            n = self._n_full
            rr = np.full(n, -1, dtype=np.int64)
            mask = np.ones(n, dtype=bool)
            mask[self._fixed] = False
            rr[mask] = np.arange(int(mask.sum()))
            iperm = self.getInversePermutation()
            perm = np.empty_like(iperm)
            perm[iperm] = np.arange(iperm.size)
            prr = np.where(rr >= 0, perm[np.maximum(rr, 0)], -1)
            self._maps = (rr, prr)
        return self._maps

    def removeFixedEntries(self, x: np.ndarray, permute: bool = False) -> np.ndarray:
        x = np.asarray(x, dtype=float)
        if x.shape[0] != self.n():
            raise RuntimeError("Invalid x size")
        rr, prr = self._row_maps()
        m = prr if permute else rr
        out = np.zeros((self.n_reduced(),) + x.shape[1:])
        keep = m >= 0
        out[m[keep]] = x[keep]
        return out

    def extractFullSolution(self, xr: np.ndarray, permute: bool = False) -> np.ndarray:
        xr = np.asarray(xr, dtype=float)
        if xr.shape[0] != self.n_reduced():
            raise RuntimeError("Invalid xReduced size")
        rr, prr = self._row_maps()
        m = prr if permute else rr
        out = np.zeros((self.n(),) + xr.shape[1:])
        keep = m >= 0
        out[keep] = xr[m[keep]]
        return out

    # ------------------------------------------------------------- solves
    def _solve(self, B: np.ndarray, mode: int) -> np.ndarray:
        self._assert(FactorizationType.Numeric)
        B = np.asarray(B, dtype=np.float64)
        vec = B.ndim == 1
        Bm = B.reshape(B.shape[0], -1)
        X = np.asfortranarray(Bm.copy())
        nrhs = X.shape[1]
        _lib.check(self._lib.mfs_solve(self._h, _lib.dptr(X), _lib.dptr(X), nrhs, X.shape[0], mode), self._h,
                   "solve failed")
        self._adaptive_record("solve")
        return X[:, 0].copy() if vec else np.ascontiguousarray(X)

    def solve(self, b: np.ndarray, sys: CholeskySys = CholeskySys.A) -> np.ndarray:
        if sys != CholeskySys.A:
            raise RuntimeError("Alternative CholeskySys not yet wrapped for Catamari")
        self._assert(FactorizationType.Numeric)
        if np.asarray(b).shape[0] != self.m():
            raise RuntimeError("CholeskyFactorizerBase::solve: incorrect b size")
        return self._solve(b, _lib.MFS_SOLVE_FULL)

    def solveMultiRHS(self, B: np.ndarray) -> np.ndarray:
        self._assert(FactorizationType.Numeric)
        B = np.asarray(B, dtype=float)
        if B.shape[0] != self.m():
            raise RuntimeError("Incorrect RHS size")
        if B.ndim != 2 or B.shape[1] < 1:
            raise RuntimeError("Must specify at least one rhs.")
        return self._solve(B, _lib.MFS_SOLVE_FULL)

    def solveRawReduced(self, b: np.ndarray, sys: CholeskySys = CholeskySys.A,
                        alreadyPermuted: bool = False) -> np.ndarray:
        if sys != CholeskySys.A:
            raise RuntimeError("Alternative CholeskySys not yet wrapped for Catamari")
        mode = _lib.MFS_SOLVE_REDUCED_PERMUTED if alreadyPermuted else _lib.MFS_SOLVE_REDUCED
        return self._solve(b, mode)

    def solveRawReducedInPlace(self, bx: np.ndarray, sys: CholeskySys = CholeskySys.A,
                               alreadyPermuted: bool = False) -> None:
        bx[...] = self.solveRawReduced(bx, sys, alreadyPermuted)

    def apply(self, x: np.ndarray) -> np.ndarray:
        """y = H x on the GPU (full-size vectors; pinned rows of y are zero)."""
        x = np.asarray(x, dtype=np.float64)
        vec = x.ndim == 1
        X = np.asfortranarray(x.reshape(x.shape[0], -1).copy())
        _lib.check(self._lib.mfs_apply(self._h, _lib.dptr(X), _lib.dptr(X), X.shape[1], X.shape[0],
                                       _lib.MFS_SOLVE_FULL), self._h, "apply failed")
        return X[:, 0].copy() if vec else np.ascontiguousarray(X)

    # ------------------------------------------------------ introspection
    def getFactorNNZ(self) -> int:
        self._assert(FactorizationType.Symbolic)
        v = C.c_int64()
        self._lib.mfs_info(self._h, None, None, C.byref(v), None, None, None)
        return int(v.value)

    def getFlopEstimate(self) -> float:
        self._assert(FactorizationType.Symbolic)
        v = C.c_double()
        self._lib.mfs_info(self._h, None, None, None, C.byref(v), None, None)
        return float(v.value)

    def getInversePermutation(self) -> np.ndarray:
        self._assert(FactorizationType.Symbolic)
        out = np.zeros(self._n_reduced, dtype=np.int64)
        _lib.check(self._lib.mfs_inverse_permutation(self._h, _lib.i64ptr(out)), self._h, "no permutation")
        return out

    def ndOrdering(self) -> NDOrdering | None:
        if self._type() < FactorizationType.Symbolic:
            return None
        nc, nm = C.c_int64(), C.c_int64()
        self._lib.mfs_nd_ordering(self._h, C.byref(nc), C.byref(nm), None, None)
        if nc.value == 0:
            return None
        cp = np.zeros(nc.value, dtype=np.int64)
        cm = np.zeros(nm.value, dtype=np.int64)
        self._lib.mfs_nd_ordering(self._h, C.byref(nc), C.byref(nm), _lib.i64ptr(cp), _lib.i64ptr(cm))
        return NDOrdering(cp, cm, self._vb())

    def _vb(self) -> int:
        nsn, nst, vb = C.c_int64(), C.c_int64(), C.c_int32()
        self._lib.mfs_supernodes(self._h, C.byref(nsn), C.byref(nst), C.byref(vb), None, None, None, None, None)
        return int(vb.value)

    def supernodes(self) -> dict:
        """Supernode partition, assembly tree, structures and child_rel_indices."""
        nsn, nst, vb = C.c_int64(), C.c_int64(), C.c_int32()
        _lib.check(self._lib.mfs_supernodes(self._h, C.byref(nsn), C.byref(nst), C.byref(vb), None, None, None,
                                            None, None), self._h)
        s = int(nsn.value)
        out = {k: np.zeros(n, dtype=np.int64) for k, n in
               (("sn_start", s + 1), ("parent", s), ("struct_ptr", s + 1), ("struct_rows", nst.value),
                ("rel", nst.value))}
        self._lib.mfs_supernodes(self._h, C.byref(nsn), C.byref(nst), C.byref(vb), _lib.i64ptr(out["sn_start"]),
                                 _lib.i64ptr(out["parent"]), _lib.i64ptr(out["struct_ptr"]),
                                 _lib.i64ptr(out["struct_rows"]), _lib.i64ptr(out["rel"]))
        out["vb"] = int(vb.value)
        return out

    def conversionPlan(self, device_built: bool = False) -> dict:
        """The block conversion plan (CatamariConversionPlan.hh:402-541); device_built:
        the copy built on the GPU for the numeric factorization."""
        fn = self._lib.mfs_conversion_plan_device if device_built else self._lib.mfs_conversion_plan
        nv, ne = C.c_int64(), C.c_int64()
        _lib.check(fn(self._h, C.byref(nv), C.byref(ne), None, None), self._h)
        offs = np.zeros(2 * nv.value + 1, dtype=np.int64)
        ent = np.zeros(4 * ne.value, dtype=np.int64)
        _lib.check(fn(self._h, C.byref(nv), C.byref(ne), _lib.i64ptr(offs), _lib.i64ptr(ent)), self._h)
        return {"columnOffsets": offs, "entries": ent.reshape(-1, 4)}

    def factorValues(self) -> np.ndarray:
        fs = C.c_int64()
        _lib.check(self._lib.mfs_factor_values(self._h, C.byref(fs), None), self._h)
        out = np.zeros(fs.value)
        _lib.check(self._lib.mfs_factor_values(self._h, C.byref(fs), _lib.dptr(out)), self._h)
        return out

    def stats(self) -> dict:
        st = _lib.Stats()
        self._lib.mfs_get_stats(self._h, C.byref(st))
        return {name: getattr(st, name) for name, _ in _lib.Stats._fields_}

    # --------------------------------------------------------------- stash
    def stashFactorization(self):
        _lib.check(self._lib.mfs_stash(self._h), self._h)
        self._stash_meta = (self._fixed, self._n_full, self._n_reduced, self._bs, self._axlen)

    def hasStashedFactorization(self) -> bool:
        v = C.c_int32()
        self._lib.mfs_has_stash(self._h, C.byref(v))
        return bool(v.value)

    def swapStashedFactorization(self):
        _lib.check(self._lib.mfs_swap_stash(self._h), self._h)
        cur = (self._fixed, self._n_full, self._n_reduced, self._bs, self._axlen)
        if self._stash_meta is not None:
            self._fixed, self._n_full, self._n_reduced, self._bs, self._axlen = self._stash_meta
        self._stash_meta = cur
        self._maps = None

    def clearStashedFactorization(self):
        self._lib.mfs_clear_stash(self._h)

    def clearFactors(self):
        self._lib.mfs_clear_factors(self._h)
        self._maps = None


def make_cholesky_factorizer(provider: CholeskyProvider = CholeskyProvider.B200, singlePrecision: bool = False,
                             **kw) -> B200Factorizer:
    """Factory hook (make_cholesky_factorizer.cc:54-123): the B200 providers map to this library."""
    if provider in (CholeskyProvider.B200Native, CholeskyProvider.CatamariNative):
        kw.setdefault("orderingMethod", OrderingMethod.Native)
    elif provider in (CholeskyProvider.CatamariAMD,):
        kw.setdefault("orderingMethod", OrderingMethod.AMD)
    elif provider in (CholeskyProvider.CatamariAdaptive,):
        kw.setdefault("orderingMethod", OrderingMethod.Adaptive)
    elif provider in (CholeskyProvider.B200, CholeskyProvider.CatamariNesdisParallel, CholeskyProvider.Catamari,
                      CholeskyProvider.CatamariNesdis):
        kw.setdefault("orderingMethod", OrderingMethod.CholmodNesdisParallel)
    else:
        raise RuntimeError(f"provider {provider} is not available in this build")
    return B200Factorizer(singlePrecision, **kw)
