"""Synthetic workload generators (CPU): shapes, pins, block-diagonal batches, the
load ramp's displacement and the SPD projection of its element Hessians."""
import numpy as np

from meshfemsparse_b200 import fem, workloads


def test_cube_counts_and_pins():
    wl = workloads.config1(k=4)
    assert wl.nodes.shape == (125, 3) and wl.tets.shape == (6 * 64, 4)
    assert len(wl.pins) == 3 * 25                      # all three DOFs of the z = 0 nodes
    assert np.all(wl.rhs[wl.pins] == 0.0)


def test_batch_is_block_diagonal():
    wl = workloads.config3(count=5, seed=1, dof_range=(200, 3000))
    sizes = [(k + 1) ** 3 for k in wl.info["sides"]]
    owner = np.repeat(np.arange(len(sizes)), sizes)
    H = wl.H
    for bj in range(H.numBlocks):
        rows = H.Ai[H.Ap[bj]:H.Ap[bj + 1]]
        assert np.all(owner[rows] == owner[bj])


def test_two_material_contrast():
    wl = workloads.config5(k=6, seed=2)
    assert wl.nrhs == 32
    # element stiffness scales with E: the two materials differ by 1e3
    s = np.array([np.trace(k) for k in wl.Ke])
    ratio = np.percentile(s, 99) / np.percentile(s, 1)
    assert 300 < ratio < 3e4


def test_load_ramp_displacement_and_hessians():
    seq = workloads.newton_sequence(k=3, final_hessians=False)
    nodes = seq.wl.nodes
    u = workloads.compression_displacement(nodes, seq.strain(seq.steps), seed=4)
    bottom = nodes[:, 2] == 0.0
    assert np.abs(u[bottom]).max() == 0.0
    top = nodes[:, 2] == 1.0
    assert np.allclose(u[top, 2].mean(), -0.2, atol=0.02)
    Ke = seq.hessians(seq.strain(15))
    assert Ke.shape == (seq.wl.tets.shape[0], 12, 12)
    assert np.allclose(Ke, Ke.transpose(0, 2, 1))
    assert np.linalg.eigvalsh(Ke).min() >= 1e-8 * 0.999
    assert seq.strain(0) == 0.0 and seq.strain(30) == 0.2
