"""The benchmark workloads at reduced sizes, on the GPU: a batch of uneven
independent meshes solved as one system (config 3), the two-material
high-contrast case with 32 right-hand sides (config 5), and a short Newton load
ramp with the learned preconditioner (config 4)."""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, workloads
from meshfemsparse_b200.learned import LearnedPreconditioner, pcg_solve
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def residual(wl, X):
    H = wl.H
    H.Ax = wl.Ax
    keep = np.ones(wl.n_full, dtype=bool)
    keep[wl.pins] = False
    R = (wl.rhs - H.to_scipy_full() @ X)[keep]
    return (np.linalg.norm(R, axis=0) / np.linalg.norm(wl.rhs[keep], axis=0)).max()


def assembled(wl, single=False, refine=False, tc=0):
    f = B200Factorizer(single, refine=refine, tensor_cores=tc)
    f.factorizeSymbolic(wl.H, wl.pins)
    f.setElements(wl.tets)
    wl.Ax = f.assemble(wl.Ke)
    f.factorizeAssembled()
    return f


def test_batched_uneven_meshes_match_oracle_and_single_instances():
    wl = workloads.config3(count=6, seed=3, dof_range=(800, 6000))
    f64 = assembled(wl)
    X64 = f64.solveMultiRHS(wl.rhs)
    assert residual(wl, X64) <= 1e-11
    # the FP64 factor equals the oracle's numeric factor on the same ordering
    sn, plan = f64.supernodes(), f64.conversionPlan()
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    ref = pyoracle.inject(plan["entries"], sn["vb"], 3, wl.Ax, int(pan[-1]))
    assert pyoracle.mf_factor(sn, ref, 0) == -1
    got = f64.factorValues()
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()
    # FP32 factor + FP64 refinement reaches the target on every instance at once
    f32 = assembled(wl, single=True, refine=True)
    X32 = f32.solveMultiRHS(wl.rhs)
    assert residual(wl, X32) <= 1e-10
    assert np.abs(X32 - X64).max() <= 1e-8 * np.abs(X64).max()


def test_batch_instances_are_independent():
    """Solving the batch gives each instance's own solution."""
    wl = workloads.config3(count=4, seed=5, dof_range=(800, 4000))
    Xb = assembled(wl).solveMultiRHS(wl.rhs)
    sides = wl.info["sides"]
    node0 = 0
    for k in sides[:2]:
        nn = (k + 1) ** 3
        sl = slice(3 * node0, 3 * (node0 + nn))
        # reassemble this instance alone from the batch's own element data
        tets = wl.tets[(wl.tets >= node0).all(1) & (wl.tets < node0 + nn).all(1)] - node0
        Ke = wl.Ke[(wl.tets >= node0).all(1) & (wl.tets < node0 + nn).all(1)]
        pins = wl.pins[(wl.pins >= 3 * node0) & (wl.pins < 3 * (node0 + nn))] - 3 * node0
        sub = workloads.Workload("one", wl.nodes[node0:node0 + nn], tets, Ke, pins, wl.nrhs,
                                 workloads.SystemAssembler(nn).blockSparsityPattern(tets), wl.rhs[sl])
        Xs = assembled(sub).solveMultiRHS(sub.rhs)
        assert np.abs(Xs - Xb[sl]).max() <= 1e-10 * np.abs(Xs).max()
        node0 += nn


@pytest.mark.parametrize("tc", [0, 5])
def test_two_material_contrast_32_rhs(tc):
    """1e3 stiffness contrast, 32 right-hand sides (the solves sweep L21 with eight of
    them at a time): FP32 + refinement with split FP16 Schur updates (tc 0, automatic)
    and with single FP16 operands scaled per front (tc 5) reach 1e-10."""
    wl = workloads.config5(k=10, seed=5)
    assert wl.nrhs == 32
    f32 = assembled(wl, single=True, refine=True, tc=tc)
    X = f32.solveMultiRHS(wl.rhs)
    st = f32.stats()
    assert residual(wl, X) <= 1e-10
    assert 1 <= st["refine_iterations"] <= 50
    X64 = assembled(wl).solveMultiRHS(wl.rhs)
    assert residual(wl, X64) <= 1e-10


def test_contrast_escalates_low_precision_factor():
    """1e3 contrast, k=32: the automatic mode (split FP16 products) reaches 1e-10 with
    no perturbed pivot and no escalation, in `it6` iterations. The single-pass FP16
    factorization (tc 5) needs more; capped at `it6` its refinement stalls, so the
    handle redoes the factorization with split FP16 products (tc 6), which reach the
    target within the same cap, and keeps them for the next factorization of the
    pattern. (With earlier orderings tc 5 also perturbed pivots here; the cap makes the
    stall, and so the escalation, independent of that.)"""
    wl = workloads.config5(k=32, seed=5)
    auto = assembled(wl, single=True, refine=True, tc=0)
    assert residual(wl, auto.solveMultiRHS(wl.rhs)) <= 1e-10
    st6 = auto.stats()
    assert st6["split_escalations"] == 0 and st6["perturbed_pivots"] == 0
    it6 = st6["refine_iterations"]
    del auto
    f32 = B200Factorizer(True, refine=True, tensor_cores=5, refine_maxit=it6)
    f32.factorizeSymbolic(wl.H, wl.pins)
    f32.setElements(wl.tets)
    f32.assemble(wl.Ke)
    f32.factorizeAssembled()
    X = f32.solveMultiRHS(wl.rhs)
    st = f32.stats()
    assert st["split_escalations"] >= 1
    assert st["refine_iterations"] <= it6
    assert residual(wl, X) <= 1e-10
    f32.factorizeAssembled()
    assert f32.stats()["split_escalations"] == st["split_escalations"]
    assert f32.stats()["perturbed_pivots"] == 0


def test_newton_ramp_with_learned_pcg():
    seq = workloads.newton_sequence(k=6, final_hessians=False)
    wl = seq.wl
    f = B200Factorizer(True, refine=True)
    f.factorizeSymbolic(wl.H, wl.pins)
    f.setElements(wl.tets)
    fx = B200Factorizer()
    fx.factorizeSymbolic(wl.H, wl.pins)
    fx.setElements(wl.tets)
    rng = np.random.default_rng(0)
    keep = np.ones(wl.n_full, dtype=bool)
    keep[wl.pins] = False
    net = LearnedPreconditioner(seed=1)
    pairs = []
    for i in range(4):
        Ax = fx.assemble(seq.hessians(float(rng.uniform(0, 0.2)), seed=100 + i))
        wl.H.Ax = Ax
        fx.factorizeNumeric(wl.H)
        B = rng.normal(size=(wl.n_full, 4))
        B[~keep] = 0.0
        pairs.append((Ax, B, fx.solveMultiRHS(B)))
    for step in range(120):
        Ax, B, X = pairs[step % 4]
        net.train_step(f, B, X, lr=2e-3, Ax=Ax)
    for t in (10, 20, 30):
        Ke = seq.hessians(seq.strain(t))
        Ax = f.assemble(Ke)
        X, it, fell_back = pcg_solve(f, wl.rhs, net, maxit=200, tol=1e-10)
        wl.Ax = Ax
        wl.Ke = Ke
        assert residual(wl, X) <= 1e-10, (t, it, fell_back)
