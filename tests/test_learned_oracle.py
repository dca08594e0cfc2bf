"""CPU checks of the learned-preconditioner oracle: its gradient against central
finite differences, the BF16 rounding it applies to the weights, and the
parameter layout against the library's."""
import numpy as np

from meshfemsparse_b200 import learned
from oracle import learned_oracle as lo


def random_block_spd(nv: int, density: float, seed: int):
    rng = np.random.default_rng(seed)
    pairs = np.array([(i, j) for i in range(nv) for j in range(i) if rng.random() < density])
    n = 3 * nv
    M = np.zeros((n, n))
    for i, j in pairs:
        blk = rng.normal(size=(3, 3)) * 0.3
        M[3 * i:3 * i + 3, 3 * j:3 * j + 3] = blk
        M[3 * j:3 * j + 3, 3 * i:3 * i + 3] = blk.T
    for i in range(nv):
        b = rng.normal(size=(3, 3)) * 0.2
        M[3 * i:3 * i + 3, 3 * i:3 * i + 3] = b + b.T
    M += np.eye(n) * (np.abs(np.linalg.eigvalsh(M)).max() + 1.0)
    return pairs, M


def test_oracle_gradient_matches_finite_differences():
    pairs, M = random_block_spd(12, 0.3, 0)
    g = lo.Graph(12, pairs, M)
    _, P = lo.layout()
    rng = np.random.default_rng(1)
    w = rng.normal(size=P) * 0.1
    B = rng.normal(size=(M.shape[0], 2))
    X = np.linalg.solve(M, B)
    loss, grad = lo.loss_grad(w, g, B, X)
    assert np.isfinite(loss) and loss > 0
    off, _ = lo.layout()
    idx = np.concatenate([rng.choice(P, 40, replace=False),
                          [off["ve"][0] + 3, off["vd"][0] + 5, off["vh"][0] + 7, off["w0"][0] + 11]])
    h = 1e-6
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (lo.loss_grad(wp, g, B, X)[0] - lo.loss_grad(wm, g, B, X)[0]) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-4 * abs(fd) + 1e-7, (k, fd, grad[k])


def test_identity_head_is_jacobi():
    """Zero head weights give G = I, so M^{-1} = D^{-1}."""
    pairs, M = random_block_spd(8, 0.4, 2)
    g = lo.Graph(8, pairs, M)
    _, P = lo.layout()
    w = np.zeros(P)
    G, _ = lo.forward(w, g)
    assert np.allclose(lo.g_matrix(g, G), np.eye(M.shape[0]))


def test_bf16_rounding():
    """BF16 keeps 7 mantissa bits: the step at 1.0 is 2^-7; ties round to even."""
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, 1.0 + 3 * 2 ** -8, -2.5, 0.0],
                 dtype=np.float32)
    r = lo.bf16_round(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                        # tie, rounds to the even neighbour
    assert r[2] == 1.0                        # below the tie
    assert r[3] == 1.0 + 2 ** -7              # above the tie
    assert r[4] == 1.0 + 2 * 2 ** -7          # tie between 1 + 2^-7 (odd) and 1 + 2^-6 (even)
    assert r[5] == -2.5 and r[6] == 0.0


def test_layout_matches_library():
    _, total = lo.layout()
    assert learned.param_count() == total == 30894
