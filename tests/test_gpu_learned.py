"""Learned preconditioner on the GPU: loss and gradient of the network kernels
against the CPU oracle, PCG with the learned and the Jacobi preconditioner, the
Cholesky fallback, and what training gains over the untrained (Jacobi) method."""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, _lib, fem
from meshfemsparse_b200.learned import LearnedPreconditioner, pcg_solve
from oracle import learned_oracle as lo
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def cube(k: int, seed: int, log_e=(np.log(0.2), np.log(5.0))):
    nodes, tets = fem.tet_cube(k, jitter=0.1, seed=seed)
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(*log_e, size=tets.shape[0]))
    Ke = fem.linear_elastic_hessians(nodes, tets, E, 0.3)
    return nodes, tets, Ke, fem.bottom_pins(nodes)


def factorizer(k: int, seed: int):
    nodes, tets, Ke, pins = cube(k, seed)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    f = B200Factorizer()
    f.factorizeSymbolic(H, pins)
    f.setElements(tets)
    H.Ax = f.assemble(Ke)
    return f, H, pins, tets


def oracle_graph(f, H, pins):
    iperm = f.getInversePermutation()
    A = pyoracle.reduced_permuted_dense(H, pins, iperm)
    prr = pyoracle.scalar_perm_map(f.n(), pins, iperm)
    pairs = []
    for bj in range(H.numBlocks):
        for k in range(H.Ap[bj], H.Ap[bj + 1]):
            pi, pj = prr[3 * H.Ai[k]], prr[3 * bj]
            if pi >= 0 and pj >= 0:
                pairs.append((pi // 3, pj // 3))
    return lo.Graph(A.shape[0] // 3, np.array(pairs), A), A


def rel_residual(f, B, X):
    R = B - f.apply(X)
    return np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)


def test_loss_and_gradient_match_oracle():
    f, H, pins, _ = factorizer(3, 0)
    g, A = oracle_graph(f, H, pins)
    net = LearnedPreconditioner(seed=3)
    rng = np.random.default_rng(5)
    w = (rng.normal(size=net.n) * 0.05).astype(np.float32)
    net.set_weights(w)
    assert np.array_equal(net.get_weights(), w)
    B = rng.normal(size=(A.shape[0], 2))
    X = np.linalg.solve(A, B)
    loss, grad = net.loss_grad(f, B, X, mode=_lib.MFS_SOLVE_REDUCED_PERMUTED)
    lref, gref = lo.loss_grad(lo.bf16_round(w), g, B, X)
    # FP32 network arithmetic against the float64 oracle on the same BF16 weights
    assert abs(loss - lref) <= 1e-4 * abs(lref)
    assert np.linalg.norm(grad - gref) <= 2e-3 * np.linalg.norm(gref)
    off, _ = lo.layout()
    for name, (o, r, c) in off.items():
        gs, rs = grad[o:o + r * c], gref[o:o + r * c]
        assert np.linalg.norm(gs - rs) <= 5e-3 * np.linalg.norm(rs) + 1e-6 * np.linalg.norm(gref), name


def test_untrained_network_is_jacobi_pcg():
    f, H, pins, _ = factorizer(4, 1)
    rng = np.random.default_rng(2)
    B = rng.normal(size=(f.n(), 2))
    B[pins] = 0.0
    net = LearnedPreconditioner(seed=0)           # head weights zero: G = I
    Xj, itj, fbj = pcg_solve(f, B, None, maxit=2000, tol=1e-10)
    Xn, itn, fbn = pcg_solve(f, B, net, maxit=2000, tol=1e-10)
    assert not fbj and not fbn
    assert itj == itn
    assert rel_residual(f, B, Xj).max() <= 1e-10
    assert np.abs(Xj - Xn).max() <= 1e-9 * np.abs(Xj).max()


def test_fallback_to_cholesky():
    f, H, pins, _ = factorizer(4, 2)
    rng = np.random.default_rng(3)
    B = rng.normal(size=(f.n(), 3))
    B[pins] = 0.0
    X, it, fb = pcg_solve(f, B, None, maxit=2, tol=1e-10)
    assert fb and it == 2
    assert rel_residual(f, B, X).max() <= 1e-10
    assert np.abs(X[pins]).max() == 0.0


def test_training_reduces_pcg_iterations():
    """Pairs from the FP64 factor on several Hessians of one pattern; the trained
    preconditioner needs fewer PCG iterations than Jacobi on a held-out Hessian."""
    k = 6
    nodes, tets, _, pins = cube(k, 0)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    f = B200Factorizer()
    f.factorizeSymbolic(H, pins)
    f.setElements(tets)
    rng = np.random.default_rng(7)
    data = []
    for seed in range(1, 7):
        Ke = cube(k, seed)[2]
        Ax = f.assemble(Ke)
        f.factorizeNumeric(_with_values(H, Ax))
        B = rng.normal(size=(f.n(), 4))
        B[pins] = 0.0
        data.append((Ax, B, f.solveMultiRHS(B)))
    net = LearnedPreconditioner(seed=11)
    losses = []
    for step in range(300):
        Ax, B, X = data[step % len(data)]
        losses.append(net.train_step(f, B, X, lr=2e-3, Ax=Ax))
    assert np.mean(losses[-30:]) < np.mean(losses[:30])
    Ke = cube(k, 99)[2]
    Ax = f.assemble(Ke)
    B = rng.normal(size=(f.n(), 2))
    B[pins] = 0.0
    _, it_jacobi, fb0 = pcg_solve(f, B, None, Ax=Ax, maxit=3000, tol=1e-10)
    X, it_learned, fb1 = pcg_solve(f, B, net, Ax=Ax, maxit=3000, tol=1e-10)
    assert not fb0 and not fb1
    print(f"PCG iterations to 1e-10: Jacobi {it_jacobi}, learned {it_learned}")
    assert it_learned < it_jacobi
    R = B - _apply_dense(H, Ax, X)
    R[pins] = 0.0
    assert (np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)).max() <= 1e-9


def _with_values(H, Ax):
    H.Ax = np.asarray(Ax)
    return H


def _apply_dense(H, Ax, X):
    H.Ax = np.asarray(Ax)
    return H.to_scipy_full() @ X
