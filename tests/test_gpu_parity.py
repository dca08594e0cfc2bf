"""GPU kernels against the CPU oracle on the same seeded inputs.

* K1 element assembly: bit-exact (both sum every slot in element order).
* K2 injection + K3-K5 factorization: panels within 1e-12 relative of the
  oracle's multifrontal FP64 factor (summation order can differ by FMA
  contraction), FP32 within 1e-5.
* K6 solves and K7 SpMV: within 1e-12 relative of the oracle / host product.
"""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, OrderingMethod, fem
from oracle import pyoracle

from helpers import cube_problem, grid_forest, path_hessian, random_stencil_hessian

pytestmark = pytest.mark.gpu


def gpu_and_oracle(H, pins, single=False, **kw):
    f = B200Factorizer(single, **kw)
    f.factorizeSymbolic(H, pins)
    f.factorizeNumeric(H)
    sn = f.supernodes()
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    ref = pyoracle.inject(plan["entries"], sn["vb"], H.bs, H.Ax, int(pan[-1]))
    assert pyoracle.mf_factor(sn, ref, 0) == -1
    return f, sn, ref, f.factorValues()


def rel_err(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("seed", range(4))
@pytest.mark.parametrize("small", [0, 8])
def test_factor_panels_random_stencils(seed, small):
    H = random_stencil_hessian(seed, bs=3)
    f, sn, ref, got = gpu_and_oracle(H, [0, 1, 2], small_front_max=small)
    assert rel_err(got, ref) <= 1e-12


@pytest.mark.parametrize("k", [4, 7])
@pytest.mark.parametrize("small", [0, 16, 64])
def test_factor_panels_cube(k, small):
    H, tets, Ke, pins, nodes = cube_problem(k)
    f, sn, ref, got = gpu_and_oracle(H, pins, small_front_max=small)
    assert rel_err(got, ref) <= 1e-11
    rng = np.random.default_rng(k)
    B = rng.normal(size=(f.n_reduced(), 4))
    X = f.solveRawReduced(B, alreadyPermuted=True)
    Xref = pyoracle.mf_solve(sn, ref, B)
    assert np.linalg.norm(X - Xref) <= 1e-11 * np.linalg.norm(Xref)


@pytest.mark.parametrize("small", [0, 16])
@pytest.mark.parametrize("tc,tol", [(2, 1e-4), (6, 1e-4), (1, 3e-2), (3, 3e-2), (4, 3e-2), (5, 3e-2)])
def test_factor_panels_single_precision(small, tc, tol):
    """FP32 factor: split Schur updates (3xTF32 on mma.sync: tc=2; hi/lo FP16 on tcgen05:
    tc=6) keep FP32-level error; single-pass TF32 (tcgen05: tc=1, mma.sync: tc=3) and
    FP16 (tc=5) are looser."""
    H, tets, Ke, pins, nodes = cube_problem(5)
    f, sn, ref, got = gpu_and_oracle(H, pins, single=True, small_front_max=small, tensor_cores=tc,
                                     refine=tc in (5, 6))
    assert rel_err(got, ref) <= tol


@pytest.mark.parametrize("single", [False, True])
def test_tiled_path_large_fronts(single):
    """A cube whose top fronts exceed the tile sizes: several POTRF/inverse steps,
    multi-tile panel solves, lower-masked diagonal tiles."""
    H, tets, Ke, pins, nodes = cube_problem(9)
    f, sn, ref, got = gpu_and_oracle(H, pins, single=single, small_front_max=32)
    assert rel_err(got, ref) <= (1e-4 if single else 1e-11)


@pytest.mark.parametrize("single", [False, True])
def test_large_cube_many_panel_tiles(single):
    """k=24 cube: large fronts whose panel tasks span several CTA waves (the diagonal
    block is read by every CTA of a task while the factored copy is written elsewhere)."""
    H, tets, Ke, pins, nodes = cube_problem(24)
    f = B200Factorizer(single, tensor_cores=2)
    f.factorizeSymbolic(H, pins)
    f.factorizeNumeric(H)
    sn = f.supernodes()
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    ref = pyoracle.inject(plan["entries"], sn["vb"], H.bs, H.Ax, int(pan[-1]))
    pyoracle.load_blas()
    assert pyoracle.mf_factor(sn, ref, 8) == -1
    got = f.factorValues()
    assert rel_err(got, ref) <= (1e-4 if single else 1e-11)


@pytest.mark.parametrize("k", [2, 4])
def test_assembly_bit_exact(k):
    nodes, tets = fem.tet_cube(k, jitter=0.1, seed=7)
    from meshfemsparse_b200 import SystemAssembler
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    Ke = fem.linear_elastic_hessians(nodes, tets, np.linspace(0.5, 2.0, tets.shape[0]), 0.3)
    ref = pyoracle.assemble(H.numBlocks, H.Ap, H.Ai, tets, Ke)
    f = B200Factorizer()
    f.factorizeSymbolic(H, fem.bottom_pins(nodes))
    f.setElements(tets)
    got = f.assemble(Ke)
    assert np.array_equal(got, ref)
    # the assembled values stay resident: factor them without a host round trip
    f.factorizeAssembled()
    H.Ax = ref
    b = H.apply(np.ones(H.n))
    x = f.solve(b)
    keep = np.ones(H.n, bool)
    keep[fem.bottom_pins(nodes)] = False
    A = H.to_scipy_full()[keep][:, keep]
    assert np.linalg.norm(A @ x[keep] - b[keep]) <= 1e-10 * np.linalg.norm(b[keep])


def test_assembly_golden_fixture():
    from pathlib import Path
    z = np.load(Path(__file__).parent / "golden" / "assembly_k2.npz")
    from meshfemsparse_b200 import BlockCSCHessian
    H = BlockCSCHessian(z["nodes"].shape[0], z["Ap"], z["Ai"], 3)
    f = B200Factorizer()
    f.factorizeSymbolic(H, [])
    f.setElements(z["tets"])
    assert np.array_equal(f.assemble(z["Ke"]), z["Ax"])


@pytest.mark.parametrize("bs", [1, 2, 3])
def test_apply_matches_host(bs):
    H = path_hessian(12, bs)
    pins = [0] if bs == 1 else list(range(bs))
    f = B200Factorizer()
    f.factorize(H, pins)
    x = np.random.default_rng(bs).normal(size=(H.n, 2))
    x[pins] = 0
    y = f.apply(x)
    ref = H.apply(x)
    ref[pins] = 0
    assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)


def test_deterministic_reruns():
    H, tets, Ke, pins, nodes = cube_problem(6)
    f = B200Factorizer(small_front_max=32)
    f.factorize(H, pins)
    a = f.factorValues()
    b = H.apply(np.ones(H.n))
    x1 = f.solve(b)
    f.factorizeNumeric(H)
    assert np.array_equal(a, f.factorValues())
    assert np.array_equal(x1, f.solve(b))


def test_fp32_refined_reaches_1e_minus_10():
    H, tets, Ke, pins, nodes = cube_problem(8)
    f = B200Factorizer(True, refine=True, refine_tol=1e-10)
    f.factorize(H, pins)
    rng = np.random.default_rng(3)
    b = rng.normal(size=(H.n, 4))
    b[pins] = 0
    x = f.solveMultiRHS(b)
    keep = np.ones(H.n, bool)
    keep[pins] = False
    A = H.to_scipy_full()[keep][:, keep]
    r = A @ x[keep] - b[keep]
    assert np.max(np.linalg.norm(r, axis=0) / np.linalg.norm(b[keep], axis=0)) <= 1e-10
    assert f.stats()["refine_iterations"] >= 1


@pytest.mark.parametrize("tc", [0, 1, 4, 5, 6])
def test_bench_path_tcgen05_factor_k24(tc):
    """The benchmark's own FP32 path at k = 24 (45,000 DOFs): refined FP32 with
    tensor_cores 0 (automatic: 6), 1 (tcgen05 TF32, cp.async operands), 4 (tcgen05
    TF32, TMA-fed Schur updates), 5 (tcgen05 FP16 operands scaled per front) and 6
    (split FP16 on tcgen05, FP32-level products).
    * every panel entry within 3e-2 of the FP64 oracle factor, relative to its
      largest entry (single-pass TF32 Schur updates);
    * backward error of the TF32 factor ||L L^T x - A x|| / ||A x|| <= 1e-2 for a
      random x (an indexing error in a Schur-update tile gives O(1));
    * refinement reaches 1e-10 within 12 iterations with no perturbed pivot;
    * the split mode (0 and 6) within 1e-4 entrywise, 1e-5 backward error and 6
      iterations."""
    H, tets, Ke, pins, nodes = cube_problem(24)
    f = B200Factorizer(True, refine=True, tensor_cores=tc)
    f.factorizeSymbolic(H, pins)
    f.factorizeNumeric(H)
    sn = f.supernodes()
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    injected = pyoracle.inject(plan["entries"], sn["vb"], H.bs, H.Ax, int(pan[-1]))
    ref = injected.copy()
    pyoracle.load_blas()
    assert pyoracle.mf_factor(sn, ref, 8) == -1
    got = f.factorValues()
    split = tc in (0, 6)                       # FP32-level Schur-update products
    assert rel_err(got, ref) <= (1e-4 if split else 3e-2)
    n = f.n_reduced()
    L = pyoracle.panels_to_csc(sn, got, n)
    Al = pyoracle.panels_to_csc(sn, injected, n)
    import scipy.sparse as sp
    A = Al + Al.T - sp.diags(Al.diagonal())
    x = np.random.default_rng(24).normal(size=n)
    Ax = A @ x
    assert np.linalg.norm(L @ (L.T @ x) - Ax) <= (1e-5 if split else 1e-2) * np.linalg.norm(Ax)
    assert f.stats()["perturbed_pivots"] == 0
    rng = np.random.default_rng(5)
    b = rng.normal(size=(H.n, 4))
    b[pins] = 0
    X = f.solveMultiRHS(b)
    keep = np.ones(H.n, bool)
    keep[pins] = False
    Af = H.to_scipy_full()[keep][:, keep]
    r = Af @ X[keep] - b[keep]
    assert np.max(np.linalg.norm(r, axis=0) / np.linalg.norm(b[keep], axis=0)) <= 1e-10
    assert f.stats()["refine_iterations"] <= (6 if split else 12)


def test_config1_exact():
    """The plain FP64 parity case as stated: 20^3 hexes -> 48,000 jittered tets,
    linear elastic E = 1, nu = 0.3, z = 0 pinned, one N(0,1) right-hand side.
    GPU assembly bit-exact with the oracle, the FP64 factor entrywise within 1e-11
    of the oracle's, the solve within 1e-11 of the oracle's solve, and the relative
    residual within 1e-10."""
    from meshfemsparse_b200 import workloads
    wl = workloads.config1()
    assert wl.tets.shape[0] == 48000 and wl.nodes.shape[0] == 9261
    f = B200Factorizer(False)
    f.factorizeSymbolic(wl.H, wl.pins)
    assert f.n_reduced() == 26460
    f.setElements(wl.tets)
    Ax = f.assemble(wl.Ke)
    Ax_ref = pyoracle.assemble(wl.H.numBlocks, wl.H.Ap, wl.H.Ai, wl.tets, wl.Ke)
    assert np.array_equal(Ax, Ax_ref)
    f.factorizeAssembled()
    sn = f.supernodes()
    plan = f.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    ref = pyoracle.inject(plan["entries"], sn["vb"], 3, Ax_ref, int(pan[-1]))
    pyoracle.load_blas()
    assert pyoracle.mf_factor(sn, ref, 8) == -1
    got = f.factorValues()
    assert rel_err(got, ref) <= 1e-11
    b = wl.rhs[:, 0]
    x = f.solve(b)
    bp = f.removeFixedEntries(b, permute=True)
    x_ref = f.extractFullSolution(pyoracle.mf_solve(sn, ref, bp), permute=True)
    assert np.linalg.norm(x - x_ref) <= 1e-11 * np.linalg.norm(x_ref)
    wl.H.Ax = Ax_ref
    keep = np.ones(wl.H.n, bool)
    keep[wl.pins] = False
    A = wl.H.to_scipy_full()[keep][:, keep]
    assert np.linalg.norm(A @ x[keep] - b[keep]) <= 1e-10 * np.linalg.norm(b[keep])
    assert np.all(x[wl.pins] == 0.0)
