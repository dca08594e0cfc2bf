"""B200-native numeric path for MeshFEMSparse block-CSC Hessians.

Element assembly, supernodal Cholesky factorization and multi-RHS triangular
solves on one GPU, behind the reference's BlockCSCHessian / factorizer API.
"""
from .hessian import BlockCSCHessian, ScalarCSC, SystemAssembler
from .factorizer import (B200Factorizer, CholeskyProvider, CholeskySys, NDOrdering, OrderingMethod,
                         make_cholesky_factorizer)

__all__ = [
    "BlockCSCHessian", "ScalarCSC", "SystemAssembler", "B200Factorizer", "CholeskyProvider", "CholeskySys",
    "NDOrdering", "OrderingMethod", "make_cholesky_factorizer",
]
