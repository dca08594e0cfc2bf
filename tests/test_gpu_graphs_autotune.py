"""CUDA-graph replay of the factorization and the autotuner, on the GPU, with a
small batch of uneven meshes (the batched workload's shape)."""
import numpy as np
import pytest

from meshfemsparse_b200 import B200Factorizer, autotune, workloads

pytestmark = pytest.mark.gpu


def _setup(wl, **kw):
    f = B200Factorizer(**kw)
    f.factorizeSymbolic(wl.H, wl.pins)
    f.setElements(wl.tets)
    return f


@pytest.mark.parametrize("single", [False, True])
def test_graph_replay_equals_direct_launches(single):
    wl = workloads.config3(count=5, seed=7, dof_range=(800, 5000))
    rng = np.random.default_rng(0)
    Ke2 = wl.Ke * rng.uniform(0.5, 2.0, size=(wl.Ke.shape[0], 1, 1))
    ref = _setup(wl, singlePrecision=single, refine=single)
    gr = _setup(wl, singlePrecision=single, refine=single, use_graphs=True)
    # alternating values: direct run, capture, replays (two assembly buffers -> two graphs)
    for Ke in (wl.Ke, Ke2, wl.Ke, Ke2, wl.Ke):
        for f in (ref, gr):
            f.assemble(Ke, return_values=False)
            f.factorizeAssembled()
        assert np.array_equal(ref.factorValues(), gr.factorValues())
        X0, X1 = ref.solveMultiRHS(wl.rhs), gr.solveMultiRHS(wl.rhs)
        assert np.array_equal(X0, X1)


def test_autotune_on_batch(tmp_path):
    wl = workloads.config3(count=4, seed=9, dof_range=(800, 4000))
    r = autotune.tune(wl.H, wl.pins, wl.tets, wl.Ke, wl.rhs, single=True, refine=True, cutoffs=(96, 160),
                      repeats=1, cache=tmp_path / "t.json")
    assert (r["small_front_max"], r["tensor_cores"]) in {(c, t) for c in (96, 160) for t in (5, 6)}
    assert all(c["ms"] > 0 for c in r["candidates"])
    f = _setup(wl, singlePrecision=True, refine=True, small_front_max=r["small_front_max"],
               tensor_cores=r["tensor_cores"])
    H = wl.H
    H.Ax = f.assemble(wl.Ke)
    f.factorizeAssembled()
    X = f.solveMultiRHS(wl.rhs)
    keep = np.ones(wl.n_full, dtype=bool)
    keep[wl.pins] = False
    R = (wl.rhs - H.to_scipy_full() @ X)[keep]
    assert (np.linalg.norm(R, axis=0) / np.linalg.norm(wl.rhs[keep], axis=0)).max() <= 1e-10
    assert autotune.tune(wl.H, wl.pins, wl.tets, wl.Ke, wl.rhs, cache=tmp_path / "t.json")["cached"]
