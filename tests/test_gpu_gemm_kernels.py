"""The factorization's Schur-update GEMM kernels against a host FP64 product.

Crafted operands go through the test hook ``mfs_debug_gemm`` (one launch of the
kernel the factorization uses), the way ``tests/test_catamari_solve_kernels.cc``
checks catamari's dense kernels against dense references. Cases cover edge tiles
(m, n, k not multiples of the 128 x 256 x 32 tile), both tcgen05 tile widths
(bn = 128 when at most 128 columns are left, 256 otherwise), every 16-byte
alignment shift of the A and B operands, the lower-triangle mask, several tasks in
one launch, and the row solve's (mode 1) rounding of its A operand and result.
The mode-0 cases run on both tcgen05 kernels: operands staged by cp.async
(kernel 1) and by TMA through tensor maps (kernel 4); FP16 operands (kernel 5)
have their own cases.

Tolerances:
* tcgen05 single-pass TF32, mode 0 (C -= A B^T on TF32-exact operands, as the
  factorization's L21 blocks are): the product of two TF32 values is exact in FP32,
  so the only error is FP32 accumulation: elementwise within (k + 2) 2^-21 times
  S = |C| + |A||B|^T (the standard bound with 4x room for the tensor cores'
  accumulation order), and normwise within 1e-6 of ||S||. A misplaced row, column
  or k index moves an element by about S / k, far above both.
* mode 1 (C = A B^T, A rounded to TF32 in the kernel, result stored rounded to
  TF32): within 2^-11 relative per element plus the accumulation bound, and every
  output is a TF32 value.
* split 3xTF32 (mma.sync): FP32-level, 1e-5 normwise on arbitrary FP32 operands.
* FP64 (DMMA): 1e-13 normwise.
Elements outside the written block (guard rows and columns, the strict upper
triangle of lower tasks) must be unchanged.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from meshfemsparse_b200 import _lib

pytestmark = pytest.mark.gpu


def tf32_rna(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to TF32 (10 explicit mantissa bits), nearest, ties away from zero."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u.astype(np.uint64) + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return r.view(np.float32)


def column_block(arr, off, ld, rows, cols):
    """View of the column-major block (rows x cols) at element offset `off` with leading dimension `ld`."""
    idx = off + np.arange(rows)[:, None] + ld * np.arange(cols)[None, :]
    return arr[idx]


FIELDS = ["a_off", "b_off", "c_off", "lda", "ldb", "ldc", "m", "n", "k", "lower", "mode", "scale_exp"]


def run_case(tasks, a_len, b_len, c_len, dtype, kernel, seed, tf32_exact=True):
    """tasks: list of dicts with a_off b_off c_off lda ldb ldc m n k lower mode scale_exp.
    Returns (A, B, C_before, C_after) host arrays (A and B FP16 for kernel 5)."""
    rng = np.random.default_rng(seed)
    op = np.float16 if kernel == 5 else dtype
    A = rng.uniform(-1, 1, a_len).astype(op)
    B = rng.uniform(-1, 1, b_len).astype(op)
    C0 = rng.uniform(-1, 1, c_len).astype(dtype)
    if op == np.float32 and tf32_exact:
        A, B = tf32_rna(A), tf32_rna(B)
    dev = "cuda:0"
    tA, tB, tC = (torch.from_numpy(v.copy()).to(dev) for v in (A, B, C0))
    tk = np.array([[t[f] for f in FIELDS] for t in tasks], dtype=np.int64)
    prec = _lib.MFS_PREC_FP32 if dtype == np.float32 else _lib.MFS_PREC_FP64
    _lib.debug_gemm(0, prec, kernel, tk, tA.data_ptr(), a_len, tB.data_ptr(), b_len, tC.data_ptr(), c_len)
    torch.cuda.synchronize()
    return A, B, C0, tC.cpu().numpy()


def expected(tasks, A, B, C0, a_round=None):
    """FP64 reference of every task applied to C0 (tasks write disjoint blocks), the
    elementwise accumulation scale, and the mask of written elements."""
    ref = C0.astype(np.float64).copy()
    scale = np.abs(C0.astype(np.float64))
    written = np.zeros(C0.shape, dtype=bool)
    for t in tasks:
        m, n, k = t["m"], t["n"], t["k"]
        Ab = column_block(A, t["a_off"], t["lda"], m, k).astype(np.float64)
        if a_round is not None:
            Ab = a_round(Ab.astype(np.float32)).astype(np.float64)
        Bb = column_block(B, t["b_off"], t["ldb"], n, k).astype(np.float64)
        sc = 2.0 ** t.get("scale_exp", 0)
        P = sc * (Ab @ Bb.T)
        S = sc * (np.abs(Ab) @ np.abs(Bb).T)
        idx = t["c_off"] + np.arange(m)[:, None] + t["ldc"] * np.arange(n)[None, :]
        mask = np.ones((m, n), dtype=bool)
        if t["lower"]:
            mask = np.arange(m)[:, None] >= np.arange(n)[None, :]
        cur = ref[idx]
        new = cur - P if t["mode"] == 0 else P
        ref[idx[mask]] = new[mask]
        sc = scale[idx]
        sc = sc + S if t["mode"] == 0 else S
        scale[idx[mask]] = sc[mask]
        written[idx[mask]] = True
    return ref, scale, written


def task(a_off, b_off, c_off, lda, ldb, ldc, m, n, k, lower=0, mode=0, scale_exp=0):
    return dict(a_off=a_off, b_off=b_off, c_off=c_off, lda=lda, ldb=ldb, ldc=ldc, m=m, n=n, k=k, lower=lower,
                mode=mode, scale_exp=scale_exp)


def lens(tasks):
    a = max(t["a_off"] + (t["k"] - 1) * t["lda"] + t["m"] for t in tasks)
    b = max(t["b_off"] + (t["k"] - 1) * t["ldb"] + t["n"] for t in tasks)
    c = max(t["c_off"] + (t["n"] - 1) * t["ldc"] + t["m"] for t in tasks)
    return a + 64, b + 64, c + 4 * max(t["ldc"] for t in tasks)


def check_mode0(tasks, A, B, C0, C, k_max):
    ref, scale, written = expected(tasks, A, B, C0)
    err = np.abs(C.astype(np.float64) - ref)
    bound = (k_max + 2) * 2.0 ** -21 * scale
    assert np.all(err[written] <= bound[written]), float(np.max(err[written] / np.maximum(bound[written], 1e-300)))
    assert np.linalg.norm(err[written]) <= 1e-6 * np.linalg.norm(scale[written])
    assert np.array_equal(C[~written], C0[~written]), "an element outside the task blocks changed"


SHIFTS = [(0, 0), (1, 3), (2, 1), (3, 2), (5, 7), (7, 4)]
TCGEN05 = [1, 4]


@pytest.mark.parametrize("kernel", TCGEN05)
@pytest.mark.parametrize("da,db", SHIFTS)
@pytest.mark.parametrize("m,n,k", [(300, 200, 77), (129, 100, 512), (37, 300, 1), (520, 129, 96)])
def test_tcgen05_update_edges_and_shifts(m, n, k, da, db, kernel):
    """mode 0, rectangular: edge tiles in m, n and k; n + db <= 128 takes the 128-wide
    tile, wider blocks the 256-wide one; every operand shift."""
    lda = (m + da + 7) // 8 * 8 + 8
    ldb = (n + db + 7) // 8 * 8 + 8
    ldc = m + 5
    t = [task(16 + da, 8 + db, 3, lda, ldb, ldc, m, n, k)]
    a_len, b_len, c_len = lens(t)
    A, B, C0, C = run_case(t, a_len, b_len, c_len, np.float32, kernel, seed=m * 7 + n + k + da * 3 + db)
    check_mode0(t, A, B, C0, C, k)


@pytest.mark.parametrize("kernel", TCGEN05)
@pytest.mark.parametrize("n,da", [(333, 0), (333, 2), (100, 1), (256, 3), (300, 6)])
def test_tcgen05_syrk_lower(n, da, kernel):
    """SYRK of a diagonal block (A and B the same panel rows): only the lower
    triangle is written, tiles above the diagonal exit early."""
    k = 200
    ld = (n + da + 7) // 8 * 8
    t = [task(8 + da, 8 + da, 0, ld, ld, n + 2, n, n, k, lower=1)]
    a_len, _, c_len = lens(t)
    rng = np.random.default_rng(n + da)
    A = tf32_rna(rng.uniform(-1, 1, a_len).astype(np.float32))
    C0 = rng.uniform(-1, 1, c_len).astype(np.float32)
    dev = "cuda:0"
    tA, tC = torch.from_numpy(A.copy()).to(dev), torch.from_numpy(C0.copy()).to(dev)
    tk = np.array([[t[0][f] for f in FIELDS]], dtype=np.int64)
    _lib.debug_gemm(0, _lib.MFS_PREC_FP32, kernel, tk, tA.data_ptr(), a_len, tA.data_ptr(), a_len, tC.data_ptr(),
                    c_len)
    C = tC.cpu().numpy()
    check_mode0(t, A, A, C0, C, k)


@pytest.mark.parametrize("kernel", TCGEN05)
@pytest.mark.parametrize("m,n,da", [(700, 300, 1), (1000, 512, 0), (257, 129, 3), (500, 250, 7)])
def test_tcgen05_trailing_update_lower(m, n, da, kernel):
    """A front's trailing update: rows below the block (m > n), lower mask, the
    operand rows start db = da rows into their 16-byte chunk."""
    k = 128
    ld = 1024 + 4
    t = [task(8 + da, 8 + da, 11, ld, ld, ld, m, n, k, lower=1)]
    a_len, b_len, c_len = lens(t)
    A, B, C0, C = run_case(t, a_len, b_len, c_len, np.float32, kernel, seed=m + n + da)
    check_mode0(t, A, B, C0, C, k)


@pytest.mark.parametrize("kernel", TCGEN05)
def test_tcgen05_several_tasks_one_launch(kernel):
    """Tasks of different shapes in one launch (the tile prefix and the task search)."""
    ts = [task(0, 0, 0, 528, 528, 400, 300, 250, 64),
          task(2, 1, 400 * 250, 528, 528, 200, 150, 90, 33, lower=0),
          task(3, 3, 400 * 250 + 200 * 90, 528, 528, 520, 520, 260, 130, lower=1),
          task(6, 5, 400 * 250 + 200 * 90 + 520 * 260, 528, 528, 100, 77, 60, 17, lower=0)]
    a_len, b_len, c_len = lens(ts)
    A, B, C0, C = run_case(ts, a_len, b_len, c_len, np.float32, kernel, seed=5)
    check_mode0(ts, A, B, C0, C, 130)


@pytest.mark.parametrize("m,n,da", [(500, 128, 0), (333, 128, 3), (61, 72, 2), (1024, 100, 1), (400, 128, 6)])
def test_tcgen05_row_solve_rounding(m, n, da):
    """mode 1 (the row solve X := X inv(L)^T): the FP32 A operand is rounded to TF32
    in the kernel, B (the stored inverse) is TF32-exact, the result is stored rounded
    to TF32."""
    k = n
    lda = (m + da + 7) // 8 * 8
    ldb = (n + 3) // 4 * 4
    t = [task(da, 0, 7, lda, ldb, m + 9, m, n, k, mode=1)]
    a_len, b_len, c_len = lens(t)
    rng = np.random.default_rng(m + n)
    A = rng.uniform(-1, 1, a_len).astype(np.float32)              # arbitrary FP32
    B = tf32_rna(rng.uniform(-1, 1, b_len).astype(np.float32))
    C0 = rng.uniform(-1, 1, c_len).astype(np.float32)
    dev = "cuda:0"
    tA, tB, tC = (torch.from_numpy(v.copy()).to(dev) for v in (A, B, C0))
    tk = np.array([[t[0][f] for f in FIELDS]], dtype=np.int64)
    _lib.debug_gemm(0, _lib.MFS_PREC_FP32, 1, tk, tA.data_ptr(), a_len, tB.data_ptr(), b_len, tC.data_ptr(), c_len)
    C = tC.cpu().numpy()
    ref, scale, written = expected(t, A, B, C0, a_round=tf32_rna)
    got = C.astype(np.float64)
    err = np.abs(got - ref)
    bound = 2.0 ** -11 * np.abs(ref) + (k + 2) * 2.0 ** -21 * scale
    assert np.all(err[written] <= bound[written])
    assert np.array_equal(tf32_rna(C[written]), C[written]), "row-solve output is not TF32-exact"
    assert np.array_equal(C[~written], C0[~written])


def test_mma_split3_fp32_accuracy():
    """The split 3xTF32 kernel keeps FP32-level accuracy on arbitrary FP32 operands."""
    t = [task(1, 2, 0, 404, 260, 310, 300, 250, 200)]
    a_len, b_len, c_len = lens(t)
    A, B, C0, C = run_case(t, a_len, b_len, c_len, np.float32, 3, seed=11, tf32_exact=False)
    ref, scale, written = expected(t, A, B, C0)
    prod = (ref - C0.astype(np.float64))[written]
    assert np.linalg.norm((C.astype(np.float64) - ref)[written]) <= 1e-5 * np.linalg.norm(prod)
    assert np.array_equal(C[~written], C0[~written])


@pytest.mark.parametrize("lower", [0, 1])
def test_dmma_fp64(lower):
    t = [task(3, 5, 1, 301, 299, 305, 290, 290 if lower else 170, 75, lower=lower)]
    a_len, b_len, c_len = lens(t)
    A, B, C0, C = run_case(t, a_len, b_len, c_len, np.float64, 0, seed=12 + lower)
    ref, scale, written = expected(t, A, B, C0)
    prod = (ref - C0)[written]
    assert np.linalg.norm((C - ref)[written]) <= 1e-13 * np.linalg.norm(prod)
    assert np.array_equal(C[~written], C0[~written])


@pytest.mark.parametrize("lower", [0, 1])
@pytest.mark.parametrize("m,n,k,da,db,e", [(300, 200, 77, 3, 5, 0), (520, 256, 512, 7, 7, 6), (129, 100, 64, 0, 2, -9)])
def test_tcgen05_fp16_operands(m, n, k, da, db, e, lower):
    """kind::f16 with TMA (kernel 5): FP16 A and B, FP32 C, C -= 2^e A B^T. The product
    of two FP16 values is exact in FP32; the error is FP32 accumulation only."""
    if lower:
        n = min(n, m)
        db = da
    lda = (m + da + 7) // 8 * 8 + 8
    ldb = (n + db + 7) // 8 * 8
    t = [task(8 + da, 16 + db, 5, lda, ldb, m + 3, m, n, k, lower=lower, scale_exp=e)]
    a_len, b_len, c_len = lens(t)
    A, B, C0, C = run_case(t, a_len, b_len, c_len, np.float32, 5, seed=m + n + k + lower)
    check_mode0(t, A, B, C0, C, k)


def split_fp16(x: np.ndarray):
    """hi = rn16(x), lo = rn16(2^11 (x - hi)): the split-FP16 operand pair."""
    hi = x.astype(np.float16)
    lo = ((x.astype(np.float64) - hi.astype(np.float64)) * 2048.0).astype(np.float16)
    return hi, lo


@pytest.mark.parametrize("lower", [0, 1])
@pytest.mark.parametrize("m,n,k,da,db,e", [(300, 200, 77, 3, 5, 0), (520, 256, 512, 7, 7, 6), (129, 100, 64, 0, 2, -9)])
def test_tcgen05_split_fp16_operands(m, n, k, da, db, e, lower):
    """Split FP16 with TMA (kernel 6): A = hi + 2^-11 lo, B likewise (each FP16), three
    MMAs per k slice (hi hi into one accumulator, hi lo + lo hi into another), C -=
    2^e (hi hi + 2^-11 (hi lo + lo hi)). Against the FP64 product of the operands'
    exact values the only errors are the dropped lo lo term (2^-22 relative) and FP32
    accumulation: normwise within 4e-6 of ||S||, FP32-level."""
    if lower:
        n = min(n, m)
        db = da
    lda = (m + da + 7) // 8 * 8 + 8
    ldb = (n + db + 7) // 8 * 8
    t = [task(8 + da, 16 + db, 5, lda, ldb, m + 3, m, n, k, lower=lower, scale_exp=e)]
    a_len, b_len, c_len = lens(t)
    a_len = (a_len + 7) // 8 * 8                # the lo halves start 16-byte aligned
    b_len = (b_len + 7) // 8 * 8
    rng = np.random.default_rng(m + n + k + lower + 99)
    Ax = rng.uniform(-1, 1, a_len)
    Bx = rng.uniform(-1, 1, b_len)
    Ah, Al = split_fp16(Ax)
    Bh, Bl = split_fp16(Bx)
    A_val = Ah.astype(np.float64) + Al.astype(np.float64) / 2048.0
    B_val = Bh.astype(np.float64) + Bl.astype(np.float64) / 2048.0
    C0 = rng.uniform(-1, 1, c_len).astype(np.float32)
    dev = "cuda:0"
    tA = torch.from_numpy(np.concatenate([Ah, Al])).to(dev)
    tB = torch.from_numpy(np.concatenate([Bh, Bl])).to(dev)
    tC = torch.from_numpy(C0.copy()).to(dev)
    tk = np.array([[t[0][f] for f in FIELDS]], dtype=np.int64)
    _lib.debug_gemm(0, _lib.MFS_PREC_FP32, 6, tk, tA.data_ptr(), 2 * a_len, tB.data_ptr(), 2 * b_len,
                    tC.data_ptr(), c_len)
    C = tC.cpu().numpy()
    ref, scale, written = expected(t, A_val, B_val, C0)
    err = np.abs(C.astype(np.float64) - ref)
    assert np.linalg.norm(err[written]) <= 4e-6 * np.linalg.norm(scale[written])
    # the split is far more accurate than the hi operands alone
    ref_hi, _, _ = expected(t, Ah.astype(np.float64), Bh.astype(np.float64), C0)
    assert np.linalg.norm(err[written]) < 0.05 * np.linalg.norm((ref_hi - ref)[written])
    assert np.array_equal(C[~written], C0[~written])


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("m,n,da,db", [(500, 128, 0, 0), (333, 128, 3, 0), (61, 72, 2, 1), (1024, 200, 1, 3)])
def test_tcgen05_split_tf32(m, n, da, db, mode):
    """Split TF32 on tcgen05 (kernel 7, the row solves of tensor_cores 6): arbitrary FP32
    operands split in shared memory into TF32 hi + lo, three MMAs; FP32-level accuracy
    (normwise 1e-5 of the product), for updates (mode 0) and row solves (mode 1, whose
    FP32 result is stored unrounded)."""
    k = n
    lda = (m + da + 7) // 8 * 8
    ldb = (n + db + 7) // 8 * 8
    t = [task(da, db, 7, lda, ldb, m + 9, m, n, k, mode=mode)]
    a_len, b_len, c_len = lens(t)
    A, B, C0, C = run_case(t, a_len, b_len, c_len, np.float32, 7, seed=m + n + mode, tf32_exact=False)
    ref, scale, written = expected(t, A, B, C0)
    prod = (ref - (C0.astype(np.float64) if mode == 0 else 0.0))[written]
    assert np.linalg.norm((C.astype(np.float64) - ref)[written]) <= 1e-5 * np.linalg.norm(prod)
    assert np.array_equal(C[~written], C0[~written])
