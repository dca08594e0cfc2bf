"""BlockCSC binary format (BlockCSCHessian.cc:11-100) and the matrix recorder /
replay (Solvers/MatrixRecorder.hh), on CPU."""
import io
import struct

import numpy as np
import pytest

from meshfemsparse_b200 import BlockCSCHessian
from meshfemsparse_b200.recorder import MatrixRecorder, recorded_sequence, replay

from helpers import path_hessian, random_stencil_hessian


@pytest.mark.parametrize("bs", [1, 2, 3])
def test_binary_round_trip_and_layout(bs):
    H = random_stencil_hessian(11, bs=bs)
    buf = io.BytesIO()
    H.dumpBinaryToStream(buf)
    raw = buf.getvalue()
    S = H.toScalar()
    blockSize, nb = struct.unpack("<QQ", raw[:16])
    m, n, nz, snz, sym = struct.unpack("<qqqqI", raw[16:52])
    assert (blockSize, nb, m, n, nz, sym) == (bs, H.numBlocks, H.numBlocks, H.numBlocks, H.nz, 1)
    # the non-contiguous layout stores exactly the scalar upper CSC values, in order
    assert snz == S.nz
    assert len(raw) == 52 + 8 * (n + 1) + 8 * nz + 8 * snz
    vals = np.frombuffer(raw[52 + 8 * (n + 1 + nz):], dtype="<f8")
    assert np.array_equal(vals, S.Ax)
    G = BlockCSCHessian.constructFromBinaryStream(io.BytesIO(raw))
    assert np.array_equal(G.Ap, H.Ap) and np.array_equal(G.Ai, H.Ai)
    assert np.array_equal(G.toScalar().Ax, S.Ax)
    x = np.random.default_rng(0).normal(size=H.n)
    assert np.allclose(G.apply(x), H.apply(x), rtol=0, atol=1e-12)


def test_sparsity_only_and_errors():
    H = path_hessian(6)
    P = BlockCSCHessian(H.numBlocks, H.Ap, H.Ai, H.bs)
    buf = io.BytesIO()
    P.dumpBinaryToStream(buf)
    G = BlockCSCHessian.constructFromBinaryStream(io.BytesIO(buf.getvalue()))
    assert G.isSparsityOnly() and np.array_equal(G.Ai, H.Ai)
    with pytest.raises(ValueError):
        BlockCSCHessian.constructFromBinaryStream(io.BytesIO(buf.getvalue()[:40]))
    bad = bytearray(buf.getvalue())
    bad[48:52] = struct.pack("<I", 7)
    with pytest.raises(ValueError, match="symmetry_mode"):
        BlockCSCHessian.constructFromBinaryStream(io.BytesIO(bytes(bad)))


class _Recording:
    """Duck-typed factorizer that logs the calls replay makes."""

    def __init__(self):
        self.calls = []

    def factorizeSymbolic(self, H, pins):
        self.calls.append(("symbolic", H.nz, list(pins)))

    def factorizeNumeric(self, H):
        self.calls.append(("numeric", float(H.Ax.sum())))

    def factorizeNumericWithShift(self, H, sigma):
        self.calls.append(("shifted", float(sigma)))


def test_recorder_names_and_replay_order(tmp_path):
    rec = MatrixRecorder()
    rec.recordMatrices(str(tmp_path))
    H = path_hessian(8)
    rec.countSparsityUpdateCall()
    rec.recordSymbolic(H, [0, 1, 2])
    rec.recordNumeric(H)
    H2 = H.copy()
    H2.Ax *= 2.0
    rec.recordNumeric(H2)
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["numeric_mat_0001.bin", "numeric_mat_0002.bin", "pinned_vars_0000.txt",
                     "symbolic_mat_0000_from_update_0.bin"]
    assert [k for k, _, _ in recorded_sequence(tmp_path)] == ["symbolic", "numeric", "numeric"]
    f = _Recording()
    replay(tmp_path, f, solve=False)
    assert f.calls[0] == ("symbolic", H.nz, [0, 1, 2])
    assert f.calls[1][0] == "numeric" and f.calls[2][1] == pytest.approx(2.0 * f.calls[1][1])
    g = _Recording()
    out = replay(tmp_path, g, solve=False, shift_ratio=1e-8)
    assert g.calls[1][0] == "shifted" and g.calls[1][1] == pytest.approx(1e-8 * H.trace() / H.n)
    assert out[1]["shift"] == g.calls[1][1]
    rec.stopRecordingMatrices()
    rec.recordNumeric(H)                   # not recording: nothing written
    assert len(list(tmp_path.iterdir())) == 4
