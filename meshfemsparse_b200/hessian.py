"""Host-side block-CSC Hessian container and pattern builder.

Mirrors the data layout and host API of the reference's
``BlockCSCHessian<OptimizationVarStructure<N>, ContiguousBlocks=true>``
(src/lib/MeshFEMSparse/BlockCSCHessian.hh:560-571, 798-1454) and of
``SystemAssembler<N>::blockSparsityPattern`` (SystemAssembler.hh:252-465):

* ``Ap``/``Ai`` are the upper-triangular *block* pattern (int64, rows sorted per
  column, the diagonal last);
* ``Ax`` holds ``bs*bs`` scalars per stored block, each block column-major and
  contiguous, block ``k`` at ``Ax[bs*bs*k]`` (``scalarOffsetForColumn(bj) =
  bs*bs*Ap[bj]``, BlockCSCHessian.hh:75-82); diagonal blocks are stored in full
  but only their upper triangle is meaningful (:1408-1425).

The container methods here (``toScalar``, ``apply`` ...) are host utilities of
the matrix type, exactly as in the reference; the GPU numeric path lives behind
``B200Factorizer``.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class ScalarCSC:
    """Scalar upper-triangular CSC matrix (the reference's SuiteSparseMatrix with
    symmetry_mode == UPPER_TRIANGLE)."""
    n: int
    Ap: np.ndarray
    Ai: np.ndarray
    Ax: np.ndarray | None = None

    @property
    def nz(self) -> int:
        return int(self.Ap[-1])

    def entries(self):
        """Yield (i, j) of every stored entry in storage order."""
        for j in range(self.n):
            for k in range(self.Ap[j], self.Ap[j + 1]):
                yield int(self.Ai[k]), j

    def to_dense(self) -> np.ndarray:
        A = np.zeros((self.n, self.n))
        cols = np.repeat(np.arange(self.n), np.diff(self.Ap))
        A[self.Ai, cols] = self.Ax
        A = A + np.triu(A, 1).T
        return A

    def apply(self, x: np.ndarray) -> np.ndarray:
        cols = np.repeat(np.arange(self.n), np.diff(self.Ap))
        y = np.zeros_like(x, dtype=float)
        np.add.at(y, self.Ai, self.Ax[:, None] * x[cols] if x.ndim == 2 else self.Ax * x[cols])
        off = self.Ai != cols
        if x.ndim == 2:
            np.add.at(y, cols[off], self.Ax[off][:, None] * x[self.Ai[off]])
        else:
            np.add.at(y, cols[off], self.Ax[off] * x[self.Ai[off]])
        return y


class BlockCSCHessian:
    """Upper block-CSC Hessian with contiguous bs x bs blocks."""

    def __init__(self, n_blocks: int, Ap, Ai, bs: int = 3, Ax=None):
        self.bs = int(bs)
        self.numBlocks = int(n_blocks)
        self.Ap = np.ascontiguousarray(Ap, dtype=np.int64)
        self.Ai = np.ascontiguousarray(Ai, dtype=np.int64)
        self.Ax = None if Ax is None else np.ascontiguousarray(Ax, dtype=np.float64)
        if self.Ap.shape[0] != self.numBlocks + 1:
            raise ValueError("Ap must have numBlocks+1 entries")

    # ----------------------------------------------------------- basic sizes
    @property
    def m(self) -> int:
        return self.bs * self.numBlocks

    @property
    def n(self) -> int:
        return self.bs * self.numBlocks

    @property
    def nz(self) -> int:
        return int(self.Ap[-1])

    def scalarNNZ(self) -> int:
        return self.bs * self.bs * self.nz

    def isSparsityOnly(self) -> bool:
        return self.Ax is None

    def setZero(self):
        self.Ax = np.zeros(self.scalarNNZ())
        return self

    def copy(self) -> "BlockCSCHessian":
        return BlockCSCHessian(self.numBlocks, self.Ap.copy(), self.Ai.copy(), self.bs,
                               None if self.Ax is None else self.Ax.copy())

    def data(self) -> np.ndarray:
        return self.Ax

    # ------------------------------------------------------------- offsets
    def findEntry(self, bi: int, bj: int) -> int:
        lo, hi = int(self.Ap[bj]), int(self.Ap[bj + 1])
        k = lo + int(np.searchsorted(self.Ai[lo:hi], bi))
        if k >= hi or self.Ai[k] != bi:
            return -1
        return k

    def scalarOffsetForColumn(self, bj: int) -> int:
        return self.bs * self.bs * int(self.Ap[bj])

    def scalarColStride(self, bj: int) -> int:
        return self.bs

    def locForBlock(self, bi: int, bj: int) -> int:
        k = self.findEntry(bi, bj)
        if k < 0:
            raise KeyError((bi, bj))
        return self.bs * self.bs * k

    def locForScalar(self, i: int, j: int) -> int:
        if i > j:
            i, j = j, i
        bs = self.bs
        return self.locForBlock(i // bs, j // bs) + (j % bs) * bs + (i % bs)

    def addNZScalar(self, i: int, j: int, v: float):
        if self.Ax is None:
            self.setZero()
        self.Ax[self.locForScalar(i, j)] += v

    def addDiag(self, d):
        if self.Ax is None:
            self.setZero()
        d = np.broadcast_to(np.asarray(d, dtype=float), (self.n,))
        for i in range(self.n):
            self.Ax[self.locForScalar(i, i)] += d[i]

    def setIdentity(self):
        self.setZero()
        self.addDiag(1.0)
        return self

    def trace(self) -> float:
        return float(sum(self.Ax[self.locForScalar(i, i)] for i in range(self.n)))

    def addWithSubSparsity(self, b: "BlockCSCHessian", alpha: float = 1.0) -> "BlockCSCHessian":
        """self += alpha * b where b's block pattern is contained in self's (the
        numeric matrix enlarged into a cached pattern; reference
        BlockCSCHessian::addWithSubSparsityFast, BlockCSCHessian.hh:1222-1262).
        Raises ValueError on incompatible blocks or a block of b outside self."""
        if b.bs != self.bs or b.numBlocks != self.numBlocks:
            raise ValueError("addWithSubSparsity: incompatible variable block structure")
        if b.isSparsityOnly():
            return self
        if self.isSparsityOnly():
            self.setZero()
        bcols = np.repeat(np.arange(b.numBlocks, dtype=np.int64), np.diff(b.Ap))
        # position of each of b's blocks in self: search its row among self's column
        key_self = np.repeat(np.arange(self.numBlocks, dtype=np.int64), np.diff(self.Ap)) * self.numBlocks + self.Ai
        key_b = bcols * b.numBlocks + b.Ai
        pos = np.searchsorted(key_self, key_b)
        if key_b.size and (np.any(pos >= key_self.size) or np.any(key_self[np.minimum(pos, key_self.size - 1)] != key_b)):
            raise ValueError("addWithSubSparsity: the added matrix has a block outside this pattern")
        bb = self.bs * self.bs
        dst = self.Ax.reshape(-1, bb)
        dst[pos] += alpha * b.Ax.reshape(-1, bb)
        return self

    # -------------------------------------------------- scalar conversions
    def dataOffsetsForScalarCSCDataOffsets(self) -> np.ndarray:
        """For every entry of the scalar upper CSC (toScalar order), its offset in Ax."""
        bs = self.bs
        offs = []
        for bj in range(self.numBlocks):
            for c in range(bs):
                for k in range(self.Ap[bj], self.Ap[bj + 1]):
                    bi = int(self.Ai[k])
                    rmax = c if bi == bj else bs - 1
                    for r in range(rmax + 1):
                        offs.append(bs * bs * k + c * bs + r)
        return np.asarray(offs, dtype=np.int64)

    # ------------------------------------------------------- binary format
    # The reference's on-disk format (BlockCSCHessian.cc:11-100), always written in
    # the non-contiguous block layout: header size_t blockSize, size_t numBlocks,
    # int64 m, n (= numBlocks), nz (blocks), snz (scalars in Ax, 0 when sparsity
    # only), uint32 symmetry mode (1 = upper triangle); then Ap (n + 1), Ai (nz)
    # as int64 and Ax (snz) as double. In that layout each scalar column of a block
    # column lists the bs rows of every off-diagonal block, then rows 0..c of the
    # diagonal block (upper triangle only): the scalar upper-CSC value order.
    _SYM_UPPER = 1

    def _noncontiguous_offsets(self) -> np.ndarray:
        """Offset in this (contiguous) Ax of every value of the non-contiguous layout, in order."""
        bs, nb, nz = self.bs, self.numBlocks, self.nz
        bj = np.repeat(np.arange(nb, dtype=np.int64), np.diff(self.Ap))
        last = self.Ap[1:] - 1
        if nb and (np.any(np.diff(self.Ap) <= 0) or np.any(self.Ai[last] != np.arange(nb))):
            raise ValueError("every block column must end with its diagonal block")
        diag = self.Ai == bj
        K = np.repeat(np.arange(nz, dtype=np.int64), bs * bs)
        C = np.tile(np.repeat(np.arange(bs, dtype=np.int64), bs), nz)
        R = np.tile(np.tile(np.arange(bs, dtype=np.int64), bs), nz)
        keep = ~diag[K] | (R <= C)
        K, C, R = K[keep], C[keep], R[keep]
        order = np.lexsort((R, K, C, bj[K]))
        return (bs * bs * K + C * bs + R)[order]

    def dumpBinaryToStream(self, f) -> None:
        """BlockCSCHessianBase::dumpBinaryToStream (BlockCSCHessian.cc:11-40)."""
        offs = self._noncontiguous_offsets()
        snz = 0 if self.Ax is None else int(offs.size)
        f.write(struct.pack("<QQ", self.bs, self.numBlocks))
        f.write(struct.pack("<qqqqI", self.numBlocks, self.numBlocks, self.nz, snz, self._SYM_UPPER))
        f.write(self.Ap.astype("<i8").tobytes())
        f.write(self.Ai.astype("<i8").tobytes())
        if snz:
            f.write(self.Ax[offs].astype("<f8").tobytes())

    def dumpBinaryToFile(self, path) -> None:
        with open(path, "wb") as f:
            self.dumpBinaryToStream(f)

    dumpBinary = dumpBinaryToFile

    @staticmethod
    def constructFromBinaryStream(f) -> "BlockCSCHessian":
        """BlockCSCHessianBase::constructFromBinaryStream / readBinaryFromStream
        (BlockCSCHessian.cc:42-100): returns the contiguous-block form; the strict
        lower triangle of each diagonal block (not stored) mirrors its upper triangle."""
        def read(nbytes):
            b = f.read(nbytes)
            if len(b) != nbytes:
                raise ValueError("truncated BlockCSC binary stream")
            return b
        bs, nb = struct.unpack("<QQ", read(16))
        if bs not in (1, 2, 3):
            raise ValueError("constructFromBinaryStream: uninstantiated block size")
        m, n, nz, snz, sym = struct.unpack("<qqqqI", read(36))
        if sym not in (0, 1, 2):
            raise ValueError(f"Invalid symmetry_mode: {sym}")
        if m != nb or n != nb:
            raise ValueError("block counts in the header disagree")
        Ap = np.frombuffer(read(8 * (n + 1)), dtype="<i8").astype(np.int64)
        Ai = np.frombuffer(read(8 * nz), dtype="<i8").astype(np.int64)
        H = BlockCSCHessian(int(nb), Ap, Ai, int(bs))
        if snz:
            vals = np.frombuffer(read(8 * snz), dtype="<f8").astype(np.float64)
            offs = H._noncontiguous_offsets()
            if offs.size != snz:
                raise ValueError("constructFromBinaryStream: scalarNNZ mismatch")
            Ax = np.zeros(H.scalarNNZ())
            Ax[offs] = vals
            bj = np.repeat(np.arange(H.numBlocks), np.diff(H.Ap))
            dk = np.nonzero(H.Ai == bj)[0]
            blocks = Ax.reshape(-1, bs, bs)                   # [k][c][r]: column-major blocks
            d = blocks[dk]
            lower = np.tril_indices(bs, -1)                    # (c, r) with r < c ... mirrored below
            d[:, lower[1], lower[0]] = d[:, lower[0], lower[1]]
            blocks[dk] = d
            H.Ax = Ax
        return H

    @staticmethod
    def constructFromBinaryFile(path) -> "BlockCSCHessian":
        with open(path, "rb") as f:
            return BlockCSCHessian.constructFromBinaryStream(f)

    def toScalar(self, sparsityOnly: bool = False) -> ScalarCSC:
        bs = self.bs
        n = self.n
        Ap = np.zeros(n + 1, dtype=np.int64)
        Ai = []
        for bj in range(self.numBlocks):
            for c in range(bs):
                j = bj * bs + c
                for k in range(self.Ap[bj], self.Ap[bj + 1]):
                    bi = int(self.Ai[k])
                    rmax = c if bi == bj else bs - 1
                    Ai.extend(bi * bs + r for r in range(rmax + 1))
                Ap[j + 1] = len(Ai)
        Ai = np.asarray(Ai, dtype=np.int64)
        Ax = None
        if not sparsityOnly and self.Ax is not None:
            Ax = self.Ax[self.dataOffsetsForScalarCSCDataOffsets()]
        return ScalarCSC(n, Ap, Ai, Ax)

    @staticmethod
    def fromScalar(S: ScalarCSC, bs: int) -> "BlockCSCHessian":
        """Compress a scalar upper pattern with uniform bs x bs blocks (BlockCSCHessian.hh:1456-1481)."""
        if S.n % bs:
            raise ValueError("size not divisible by the block size")
        nb = S.n // bs
        cols = [set() for _ in range(nb)]
        for i, j in S.entries():
            cols[j // bs].add(i // bs)
        Ap = np.zeros(nb + 1, dtype=np.int64)
        Ai = []
        for bj in range(nb):
            rows = sorted(cols[bj] | {bj})
            Ai.extend(rows)
            Ap[bj + 1] = len(Ai)
        H = BlockCSCHessian(nb, Ap, np.asarray(Ai, dtype=np.int64), bs)
        H.setZero()
        if S.Ax is not None:
            for (i, j), v in zip(S.entries(), S.Ax):
                H.Ax[H.locForScalar(i, j)] += v
        return H

    # ----------------------------------------------------- host products
    def to_scipy_full(self):
        """Full symmetric scipy.sparse matrix (test/analysis helper)."""
        import scipy.sparse as sp
        S = self.toScalar()
        cols = np.repeat(np.arange(S.n), np.diff(S.Ap))
        A = sp.csc_matrix((S.Ax, (S.Ai, cols)), shape=(S.n, S.n))
        return A + sp.triu(A, 1).T

    def apply(self, x: np.ndarray) -> np.ndarray:
        return self.toScalar().apply(np.asarray(x, dtype=float))

    def evalQuadraticForm(self, x: np.ndarray) -> float:
        x = np.asarray(x, dtype=float)
        return float(x @ self.apply(x))

    # --------------------------------------------------------- binary I/O
    # Layout of BlockCSCHessianBase::dumpBinaryToStream (BlockCSCHessian.cc:255-310):
    # header (block size, numBlocks, m, n, nz, scalar nz, symmetry mode) followed by
    # Ap, Ai (int64) and the scalar Ax array in the non-contiguous (scalar CSC) order.
    _MAGIC = b"MFSBCSC1"

    def dumpBinary(self, path: str):
        S = self.toScalar()
        with open(path, "wb") as fh:
            fh.write(self._MAGIC)
            fh.write(struct.pack("<7q", self.bs, self.numBlocks, self.m, self.n, self.nz, S.nz, 1))
            fh.write(self.Ap.astype("<i8").tobytes())
            fh.write(self.Ai.astype("<i8").tobytes())
            ax = S.Ax if S.Ax is not None else np.zeros(0)
            fh.write(np.asarray(ax, dtype="<f8").tobytes())

    @classmethod
    def readBinary(cls, path: str) -> "BlockCSCHessian":
        with open(path, "rb") as fh:
            if fh.read(8) != cls._MAGIC:
                raise ValueError("not a block-CSC Hessian file")
            bs, nb, m, n, nz, snz, sym = struct.unpack("<7q", fh.read(56))
            Ap = np.frombuffer(fh.read(8 * (nb + 1)), dtype="<i8").astype(np.int64)
            Ai = np.frombuffer(fh.read(8 * nz), dtype="<i8").astype(np.int64)
            ax = np.frombuffer(fh.read(), dtype="<f8")
        H = cls(nb, Ap, Ai, bs)
        if ax.size:
            H.setZero()
            H.Ax[H.dataOffsetsForScalarCSCDataOffsets()] = ax
        return H


class SystemAssembler:
    """Pattern construction for uniform block size ``bs`` (SystemAssembler<N>)."""

    def __init__(self, numBlockVars: int, bs: int = 3):
        self.numBlockVars = int(numBlockVars)
        self.bs = int(bs)

    def blockSparsityPattern(self, elements) -> BlockCSCHessian:
        conn = np.ascontiguousarray(np.asarray(elements, dtype=np.int64))
        if conn.ndim != 2:
            raise ValueError("elements must be (numElems, nodesPerElement)")
        Ap, Ai = _lib.build_pattern(self.numBlockVars, conn)
        return BlockCSCHessian(self.numBlockVars, Ap, Ai, self.bs)
