"""CPU oracle of the learned preconditioner (K8): forward pass, loss and
gradient of the message-passing network in float64 numpy. TEST INFRASTRUCTURE
ONLY — imported by tests/, never by the product path.

The reference has no learned preconditioner; this restates the network of
meshfemsparse_b200/csrc/kernels_learned.cu from its definition:

  Hs = D^{-1/2} H D^{-1/2}; per block entry (i, j) of row i: Hs_ij (3 x 3, row-major),
  a_ij = ||Hs_ij||_F (j != i);
  x_i = [Hs_ii (9), sum_j a_ij, max_j a_ij, deg_i / 16, 0, 0, 0, 0]
  layer l: h' = relu(W_l [h_i; s_i; e_i; 1]) (+ h_i for l > 0), s_i = sum_j a_ij h_j,
           e_i = sum_{j != i} Hs_ij
  head:    q_i = V_h [h_i; 1] = [P_i | Q_i | R_i];  G_ij = P_i + Q_j + V_e [Hs_ij; 1] (i > j);
           G_ii = [[exp o0, 0, 0], [o1, exp o2, 0], [o3, o4, exp o5]], o = R_i + V_d [Hs_ii; 1],
           exponents clamped to [-8, 8]
  loss:    mean_r e_r^T Hs e_r / (x_r^T b_r), e = G^T G (D^{-1/2} b) - D^{1/2} x.

Parameters are one flat array in the layout of lpc_layout(): W_0 (64 x 42),
W_1..W_3 (64 x 138), V_h (24 x 65), V_e (9 x 10), V_d (6 x 10), row-major.
The GPU kernels read the weights rounded to BF16; `bf16_round` reproduces that.
"""
from __future__ import annotations

import numpy as np

HID, LAYERS, NIN, NHEAD = 64, 4, 16, 24


def layout():
    off, o = {}, 0
    for l in range(LAYERS):
        din = NIN if l == 0 else HID
        off[f"w{l}"] = (o, HID, 2 * din + 10)
        o += HID * (2 * din + 10)
    off["vh"] = (o, NHEAD, HID + 1)
    o += NHEAD * (HID + 1)
    off["ve"] = (o, 9, 10)
    o += 90
    off["vd"] = (o, 6, 10)
    o += 60
    return off, o


def unpack(w):
    off, _ = layout()
    return {k: w[o:o + r * c].reshape(r, c) for k, (o, r, c) in off.items()}


def pack(parts):
    off, total = layout()
    out = np.zeros(total)
    for k, (o, r, c) in off.items():
        out[o:o + r * c] = parts[k].reshape(-1)
    return out


def bf16_round(w: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest even) -> float64."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


class Graph:
    """Block rows of the permuted reduced matrix: rows sorted by column."""

    def __init__(self, nv: int, pairs: np.ndarray, A: np.ndarray):
        pairs = np.unique(np.vstack([pairs, pairs[:, ::-1], np.stack([np.arange(nv)] * 2, 1)]), axis=0)
        order = np.lexsort((pairs[:, 1], pairs[:, 0]))
        pairs = pairs[order]
        self.nv = nv
        self.row, self.col = pairs[:, 0], pairs[:, 1]
        self.ptr = np.searchsorted(self.row, np.arange(nv + 1))
        self.diag = np.array([self.ptr[i] + np.searchsorted(self.col[self.ptr[i]:self.ptr[i + 1]], i)
                              for i in range(nv)])
        key = {(int(a), int(b)): e for e, (a, b) in enumerate(pairs)}
        self.mirror = np.array([key[(int(b), int(a))] for a, b in pairs])
        self.blocks = np.stack([A[3 * a:3 * a + 3, 3 * b:3 * b + 3] for a, b in pairs])   # nnz x 3 x 3
        self.A = A
        self.lower = self.col < self.row
        self.off = self.col != self.row


def features(g: Graph):
    d = np.diag(g.A).copy()
    dinv = np.where(d > 0, 1.0 / np.sqrt(np.where(d > 0, d, 1.0)), 1.0)
    eh = g.blocks * dinv.reshape(-1, 3)[g.row][:, :, None] * dinv.reshape(-1, 3)[g.col][:, None, :]
    eh = eh.reshape(-1, 9)
    ea = np.where(g.off, np.sqrt((eh ** 2).sum(1)), 0.0)
    esum = np.zeros((g.nv, 9))
    np.add.at(esum, g.row[g.off], eh[g.off])
    x0 = np.zeros((g.nv, NIN))
    x0[:, :9] = eh[g.diag]
    np.add.at(x0[:, 9], g.row, ea)
    amax = np.zeros(g.nv)
    np.maximum.at(amax, g.row, ea)
    x0[:, 10] = amax
    x0[:, 11] = np.diff(g.ptr) / 16.0
    return dinv, eh, ea, esum, x0


def _agg(g, ea, h):
    s = np.zeros_like(h)
    np.add.at(s, g.row, ea[:, None] * h[g.col])
    return s


def forward(w, g: Graph):
    P = unpack(w)
    dinv, eh, ea, esum, x0 = features(g)
    hs, ss, us, pres = [x0], [], [], []
    h = x0
    for l in range(LAYERS):
        s = _agg(g, ea, h)
        u = np.hstack([h, s, esum, np.ones((g.nv, 1))])
        pre = u @ P[f"w{l}"].T
        hn = np.maximum(pre, 0.0) + (h if l > 0 else 0.0)
        ss.append(s), us.append(u), pres.append(pre), hs.append(hn)
        h = hn
    uh = np.hstack([h, np.ones((g.nv, 1))])
    q = uh @ P["vh"].T
    G = np.zeros((len(g.row), 9))
    L = g.lower
    ue = np.hstack([eh, np.ones((len(g.row), 1))])
    G[L] = q[g.row[L], :9] + q[g.col[L], 9:18] + ue[L] @ P["ve"].T
    o = q[:, 18:24] + ue[g.diag] @ P["vd"].T
    c = np.clip(o, -8, 8)
    Gd = np.zeros((g.nv, 9))
    Gd[:, 0], Gd[:, 3], Gd[:, 4] = np.exp(c[:, 0]), o[:, 1], np.exp(c[:, 2])
    Gd[:, 6], Gd[:, 7], Gd[:, 8] = o[:, 3], o[:, 4], np.exp(c[:, 5])
    G[g.diag] = Gd
    cache = dict(P=P, dinv=dinv, eh=eh, ea=ea, esum=esum, hs=hs, us=us, pres=pres, uh=uh, q=q, o=o, ue=ue)
    return G, cache


def g_matrix(g: Graph, G) -> np.ndarray:
    """Dense lower block-triangular G from the per-entry blocks."""
    M = np.zeros((3 * g.nv, 3 * g.nv))
    for e in np.nonzero(g.col <= g.row)[0]:
        i, j = g.row[e], g.col[e]
        M[3 * i:3 * i + 3, 3 * j:3 * j + 3] = G[e].reshape(3, 3)
    return M


def loss_grad(w, g: Graph, B, X):
    """Loss and gradient (flat, layout()) for pairs B, X (n x nrhs, permuted reduced)."""
    G, c = forward(w, g)
    P, dinv = c["P"], c["dinv"]
    Gm = g_matrix(g, G)
    nr = B.shape[1]
    Hs = dinv[:, None] * g.A * dinv[None, :]
    bs, xs = dinv[:, None] * B, X / dinv[:, None]
    z = Gm @ bs
    e = Gm.T @ z - xs
    qv = Hs @ e
    nrm = np.einsum("ir,ir->r", X, B)
    loss = float(np.mean(np.einsum("ir,ir->r", e, qv) / nrm))
    gy = 2.0 * qv / (nr * nrm[None, :])
    gz = Gm @ gy
    dG = np.zeros_like(G)
    for e_ in np.nonzero(g.col <= g.row)[0]:
        i, j = g.row[e_], g.col[e_]
        dG[e_] = (z[3 * i:3 * i + 3] @ gy[3 * j:3 * j + 3].T + gz[3 * i:3 * i + 3] @ bs[3 * j:3 * j + 3].T).reshape(9)
    grads = {k: np.zeros_like(v) for k, v in P.items()}
    L = g.lower
    dq = np.zeros((g.nv, NHEAD))
    np.add.at(dq[:, :9], g.row[L], dG[L])
    np.add.at(dq[:, 9:18], g.col[L], dG[L])
    grads["ve"] = dG[L].T @ c["ue"][L]
    o = c["o"]
    dd = dG[g.diag]
    Gd = G[g.diag]
    m0, m2, m5 = (np.abs(o[:, k]) < 8 for k in (0, 2, 5))
    dout = np.stack([dd[:, 0] * Gd[:, 0] * m0, dd[:, 3], dd[:, 4] * Gd[:, 4] * m2, dd[:, 6], dd[:, 7],
                     dd[:, 8] * Gd[:, 8] * m5], 1)
    dq[:, 18:24] = dout
    grads["vd"] = dout.T @ c["ue"][g.diag]
    grads["vh"] = dq.T @ c["uh"]
    dh = dq @ P["vh"][:, :HID]
    for l in range(LAYERS - 1, -1, -1):
        din = NIN if l == 0 else HID
        dpre = dh * (c["pres"][l] > 0)
        grads[f"w{l}"] = dpre.T @ c["us"][l]
        du = dpre @ P[f"w{l}"]
        dhn = du[:, :din] + (dh if l > 0 else 0.0)
        ds = du[:, din:2 * din]
        dhn = dhn + _agg(g, c["ea"], ds)
        dh = dhn
    return loss, pack(grads)
