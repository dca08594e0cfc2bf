"""Record and replay factorization sequences in the reference's on-disk format.

`MatrixRecorder` mirrors the reference's recorder (Solvers/MatrixRecorder.hh:22-107):
while recording, every symbolic factorization writes
``symbolic_mat_<id>_from_update_<u>.bin`` plus ``pinned_vars_<id>.txt`` and every
numeric factorization writes ``numeric_mat_<id>.bin``. Ids are zero-padded to
four digits and shared by both kinds, so a numeric matrix follows the pattern it
belongs to. The .bin files use the BlockCSC binary format
(`BlockCSCHessian.dumpBinaryToFile`).

`replay` drives such a directory through this library's factorizer. It
reanalyses at each symbolic file, factors each numeric file, and optionally
solves a seeded right-hand side and checks the residual. Sequences recorded by
the reference (a MeshFEM Newton run) therefore run unchanged on the GPU path.
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np

from .hessian import BlockCSCHessian


class MatrixRecorder:
    def __init__(self):
        self.path = ""
        self.numeric = self.symbolic = self.dynamic = False
        self.resetIDs()

    # -- configuration (MatrixRecorder.hh:24-44)
    def recordMatrices(self, directory_path: str, symbolic: bool = True, numeric: bool = True,
                       dynamic: bool = False) -> None:
        if not directory_path:
            raise RuntimeError("MatrixRecorder: Must pass a nonempty path")
        if not (symbolic or numeric):
            raise RuntimeError("MatrixRecorder: Must record at least one type of matrix (symbolic or numeric)")
        self.path = str(directory_path)
        self.symbolic, self.numeric, self.dynamic = bool(symbolic), bool(numeric), bool(dynamic)
        self.resetIDs()

    def stopRecordingMatrices(self) -> None:
        self.path = ""

    def recordingMatrices(self) -> bool:
        return bool(self.path)

    def resetIDs(self) -> None:
        self.matrixId = 0
        self.numSparsityUpdateCalls = 0
        self.dynamicSparsityCounter = 0

    def countSparsityUpdateCall(self) -> None:
        self.numSparsityUpdateCalls += 1

    # -- file names (MatrixRecorder.hh:36-39, 87-92)
    @staticmethod
    def idString(i: int) -> str:
        return str(i).rjust(4, "0")

    @classmethod
    def symbolicMatrixFileName(cls, i: int, suffix: str = "") -> str:
        return f"symbolic_mat_{cls.idString(i)}{suffix}.bin"

    @classmethod
    def numericMatrixFileName(cls, i: int) -> str:
        return f"numeric_mat_{cls.idString(i)}.bin"

    @classmethod
    def pinnedVarsFileName(cls, i: int) -> str:
        return f"pinned_vars_{cls.idString(i)}.txt"

    # -- recording (MatrixRecorder.hh:47-73)
    def _next_id(self) -> int:
        i = self.matrixId
        self.matrixId += 1
        return i

    def recordNumeric(self, mat: BlockCSCHessian) -> None:
        if not self.recordingMatrices() or not self.numeric:
            return
        mat.dumpBinaryToFile(Path(self.path) / self.numericMatrixFileName(self._next_id()))

    def recordStaticSparsity(self, mat: BlockCSCHessian) -> None:
        if not self.recordingMatrices() or not self.symbolic:
            return
        mat.dumpBinaryToFile(Path(self.path) / "static_sparsity_pattern.bin")

    def recordSymbolic(self, mat: BlockCSCHessian, pinnedVars) -> None:
        if not self.recordingMatrices() or not self.symbolic:
            return
        i = self._next_id()
        suffix = f"_from_update_{self.numSparsityUpdateCalls - 1}"
        mat.dumpBinaryToFile(Path(self.path) / self.symbolicMatrixFileName(i, suffix))
        with open(Path(self.path) / self.pinnedVarsFileName(i), "w") as f:
            for v in pinnedVars:
                f.write(f"{int(v)}\n")


_SYM = re.compile(r"symbolic_mat_(\d+)(_from_update_-?\d+)?\.bin$")
_NUM = re.compile(r"numeric_mat_(\d+)\.bin$")


def recorded_sequence(directory) -> list[tuple[str, int, Path]]:
    """The recorded events in id order: ("symbolic" | "numeric", id, file)."""
    events = []
    for p in Path(directory).iterdir():
        m = _SYM.match(p.name)
        if m:
            events.append(("symbolic", int(m.group(1)), p))
            continue
        m = _NUM.match(p.name)
        if m:
            events.append(("numeric", int(m.group(1)), p))
    return sorted(events, key=lambda e: e[1])


def replay(directory, factorizer, solve: bool = True, seed: int = 0, shift_ratio: float | None = None,
           sparsity_cache: float | None = None) -> list[dict]:
    """Run a recorded sequence through `factorizer` (a B200Factorizer). Each numeric
    step returns its relative residual when `solve` is set (a seeded N(0,1) RHS, pins
    zero). With `shift_ratio`, each numeric step factors H + (shift_ratio * trace(H) / n) I,
    as the reference's benchmark driver does with 1e-8 (benchmark_linear_systems.cc:298-302);
    the residual is then against H + shift I.

    With `sparsity_cache` (the entry budget ratio), patterns pass through a SparsityLRU
    as in the reference's contact-sequence driver (benchmark_sparsity_lru.cc:100-150): a
    symbolic file whose entries the cache already holds reuses the last symbolic
    factorization (its record has "symbolic_factorization": False), otherwise the
    factorizer analyses the cache's enlarged pattern; every numeric matrix is added into
    the cached pattern before it is factored."""
    from .sparsity_lru import SparsityLRU

    out = []
    pins = np.zeros(0, dtype=np.int64)
    rng = np.random.default_rng(seed)
    lru = None
    for kind, i, path in recorded_sequence(directory):
        H = BlockCSCHessian.constructFromBinaryFile(path)
        if kind == "symbolic":
            pv = Path(directory) / MatrixRecorder.pinnedVarsFileName(i)
            pins = np.loadtxt(pv, dtype=np.int64, ndmin=1) if pv.exists() and pv.stat().st_size else \
                np.zeros(0, dtype=np.int64)
            rec = {"id": i, "kind": kind, "n": H.n, "blocks": H.nz}
            if sparsity_cache is None:
                factorizer.factorizeSymbolic(H, pins)
            else:
                if lru is None:
                    lru = SparsityLRU(H.numBlocks, H.Ap, H.Ai, budget_ratio=float(sparsity_cache))
                    needs = True
                else:
                    needs = lru.update(H.numBlocks, H.Ap, H.Ai) != 0
                if needs:
                    factorizer.factorizeSymbolic(BlockCSCHessian(H.numBlocks, lru.Ap, lru.Ai, H.bs), pins)
                rec.update(symbolic_factorization=bool(needs), cached_blocks=int(lru.Ap[-1]))
            out.append(rec)
            continue
        Hf = H
        if lru is not None:
            Hf = BlockCSCHessian(H.numBlocks, lru.Ap, lru.Ai, H.bs).setZero().addWithSubSparsity(H)
        sigma = 0.0
        if shift_ratio is not None:
            sigma = float(shift_ratio) * H.trace() / H.n
            factorizer.factorizeNumericWithShift(Hf, sigma)
        else:
            factorizer.factorizeNumeric(Hf)
        rec = {"id": i, "kind": kind, "n": H.n, "shift": sigma}
        if solve:
            b = rng.normal(size=H.n)
            b[pins] = 0.0
            x = factorizer.solve(b)
            keep = np.ones(H.n, dtype=bool)
            keep[pins] = False
            r = (b - H.apply(x) - sigma * x)[keep]
            rec["residual"] = float(np.linalg.norm(r) / np.linalg.norm(b[keep]))
        out.append(rec)
    return out
