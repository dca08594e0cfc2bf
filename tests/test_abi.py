"""The C-ABI library loads and exports every entry point declared in include/*.h (no GPU needed)."""
import ctypes
import re
from pathlib import Path

from meshfemsparse_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names.update(re.findall(r"^\s*mfs_status\s+(mfs_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mfs_symbolic" in syms and "mfs_numeric" in syms and "mfs_solve" in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_symbols()) == set(_lib.EXPORTED)


def test_default_options_and_host_only_handle():
    lib = _lib.load()
    o = _lib.default_options()
    assert o.relax == 1 and o.relax_zeros == 128 and abs(o.relax_ratio - 0.01) < 1e-15
    o.device = -1
    h = ctypes.c_void_p()
    assert lib.mfs_create(ctypes.byref(h), ctypes.byref(o)) == _lib.MFS_OK
    # numeric on an analysis-only handle is refused, not crashed
    assert lib.mfs_numeric(h, None, None, 0.0, 0) != _lib.MFS_OK
    assert lib.mfs_destroy(h) == _lib.MFS_OK


def test_gemm_hook_checks_accesses_before_launch():
    """The GEMM test hook validates every access against the array lengths on the
    host and refuses before touching a device (so this runs without a GPU)."""
    import numpy as np
    t = np.array([[0, 0, 0, 128, 128, 128, 128, 128, 64, 0, 0, 0]], dtype=np.int64)
    import pytest
    with pytest.raises(ValueError):
        _lib.debug_gemm(0, _lib.MFS_PREC_FP32, 1, t, 1, 100, 1, 100, 1, 100)
    bad_ld = np.array([[0, 0, 0, 130, 128, 128, 128, 128, 64, 0, 0, 0]], dtype=np.int64)
    with pytest.raises(ValueError):
        _lib.debug_gemm(0, _lib.MFS_PREC_FP32, 1, bad_ld, 1, 1 << 20, 1, 1 << 20, 1, 1 << 20)
