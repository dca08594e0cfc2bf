"""GPU construction of the pattern-dependent structures, bit-exact with the host's.

* Block pattern from element stencils (SystemAssembler.hh:252-465):
  mfs_build_pattern_device against mfs_build_pattern, on tet cubes (the benchmark's
  64^3 cube included), random stencils with repeated nodes, and other stencil sizes.
* Block conversion plan (CatamariConversionPlan.hh:402-541): the plan the numeric
  factorization uses, built on the GPU, against the analysis' host plan, entry for
  entry (bucket offsets, destinations, sources, leading dimensions, flags).
* Element -> slot map: assembly through it is bit-exact with the oracle (the
  assembly tests), and invalid elements are refused.
"""
import numpy as np
import pytest
import torch

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, _lib, fem

from helpers import cube_problem, random_stencil_hessian

pytestmark = pytest.mark.gpu


def gpu_pattern(nvars, conn):
    conn = np.ascontiguousarray(conn, dtype=np.int64)
    nelem, npe = conn.shape
    dconn = torch.from_numpy(conn.reshape(-1).copy()).cuda()
    Ap = torch.zeros(nvars + 1, dtype=torch.int64, device="cuda")
    nnz = _lib.build_pattern_device(nvars, dconn.data_ptr(), nelem, npe, Ap.data_ptr(), None)
    Ai = torch.zeros(max(nnz, 1), dtype=torch.int64, device="cuda")
    nnz2 = _lib.build_pattern_device(nvars, dconn.data_ptr(), nelem, npe, Ap.data_ptr(), Ai.data_ptr())
    assert nnz2 == nnz
    return Ap.cpu().numpy(), Ai.cpu().numpy()[:nnz]


@pytest.mark.parametrize("k", [1, 3, 8])
def test_pattern_tet_cube(k):
    nodes, tets = fem.tet_cube(k, jitter=0.0, seed=1)
    Ap, Ai = _lib.build_pattern(nodes.shape[0], tets)
    gAp, gAi = gpu_pattern(nodes.shape[0], tets)
    assert np.array_equal(Ap, gAp) and np.array_equal(Ai, gAi)


def test_pattern_benchmark_cube_64():
    nodes, tets = fem.tet_cube(64, jitter=0.0, seed=2)
    Ap, Ai = _lib.build_pattern(nodes.shape[0], tets)
    gAp, gAi = gpu_pattern(nodes.shape[0], tets)
    assert np.array_equal(Ap, gAp) and np.array_equal(Ai, gAi)


@pytest.mark.parametrize("npe", [1, 2, 4, 7])
@pytest.mark.parametrize("seed", range(3))
def test_pattern_random_stencils_with_repeats(npe, seed):
    rng = np.random.default_rng(seed)
    nvars = 50
    conn = rng.integers(0, nvars, size=(200, npe))
    conn[::7, 0] = conn[::7, -1]                      # repeated nodes in some stencils
    Ap, Ai = _lib.build_pattern(nvars, conn)
    gAp, gAi = gpu_pattern(nvars, conn)
    assert np.array_equal(Ap, gAp) and np.array_equal(Ai, gAi)


def test_pattern_rejects_out_of_range():
    with pytest.raises(ValueError):
        gpu_pattern(5, np.array([[0, 1, 2, 5]]))


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("case", ["cube7", "cube12_pinned", "stencil"])
def test_conversion_plan_built_on_gpu(case, single):
    if case == "stencil":
        H = random_stencil_hessian(3, bs=3)
        pins = [0, 1, 2]
    else:
        H, tets, Ke, pins, nodes = cube_problem(7 if case == "cube7" else 12)
    f = B200Factorizer(single, refine=single)
    f.factorizeSymbolic(H, pins)
    host = f.conversionPlan()
    dev = f.conversionPlan(device_built=True)
    assert np.array_equal(host["columnOffsets"], dev["columnOffsets"])
    assert np.array_equal(host["entries"], dev["entries"])
    # and the factorization driven by it solves
    f.factorizeNumeric(H)
    b = H.apply(np.ones(H.n))
    x = f.solve(b)
    keep = np.ones(H.n, bool)
    keep[pins] = False
    A = H.to_scipy_full()[keep][:, keep]
    assert np.linalg.norm(A @ x[keep] - b[keep]) <= 1e-10 * np.linalg.norm(b[keep])


def test_slot_map_refuses_invalid_elements():
    nodes, tets = fem.tet_cube(2, jitter=0.0, seed=1)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    f = B200Factorizer()
    f.factorizeSymbolic(H, fem.bottom_pins(nodes))
    bad = tets.copy()
    bad[3, 2] = nodes.shape[0]
    with pytest.raises(ValueError):
        f.setElements(bad)
    far = tets.copy()
    far[0] = [0, 1, nodes.shape[0] - 1, nodes.shape[0] - 2]   # a block the pattern does not hold
    with pytest.raises(ValueError):
        f.setElements(far)
