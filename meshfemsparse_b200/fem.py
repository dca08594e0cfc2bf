"""Synthetic finite-element inputs: tetrahedralised cubes and P1 element Hessians.

The reference receives element Hessians from MeshFEM (not part of the
reference tree); these generators produce the same kind of input from the
continuum-mechanics formulas so that the numeric path can be exercised on the
named mesh shapes. They are inputs, not parity targets.

* ``tet_cube(k)``: unit cube, k^3 hexes, each split into 6 tets along the
  (0,0,0)-(1,1,1) diagonal (Kuhn/Freudenthal split); node (i,j,l) has index
  i + (k+1)*(j + (k+1)*l).
* ``linear_elastic_hessians``: P1 stiffness V * B^T C B (12x12, dof 3a+i).
* ``neo_hookean_hessians``: compressible Neo-Hookean
  psi = mu/2 (I1 - 3) - mu ln J + lambda/2 (ln J)^2, Hessian at a deformed
  state, projected to SPD per element by clamping eigenvalues at ``clamp``.
"""
from __future__ import annotations

import itertools
import math

import numpy as np


def lame(E, nu):
    E = np.asarray(E, dtype=float)
    nu = np.asarray(nu, dtype=float)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return lam, mu


def tet_cube(k: int, jitter: float = 0.0, seed: int = 0):
    """Nodes (N,3) and tets (6k^3, 4) of the unit cube; interior nodes jittered by U(+-jitter*h)."""
    h = 1.0 / k
    g = np.arange(k + 1) * h
    X = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1)       # [i,j,l,3]
    nodes = X.transpose(2, 1, 0, 3).reshape(-1, 3)                      # index i + (k+1)(j + (k+1) l)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        idx = np.arange(nodes.shape[0])
        i = idx % (k + 1)
        j = (idx // (k + 1)) % (k + 1)
        l = idx // (k + 1) ** 2
        interior = (i > 0) & (i < k) & (j > 0) & (j < k) & (l > 0) & (l < k)
        nodes = nodes.copy()
        nodes[interior] += rng.uniform(-jitter * h, jitter * h, size=(int(interior.sum()), 3))
    K1 = k + 1
    ii, jj, ll = np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij")
    base = (ii + K1 * (jj + K1 * ll)).transpose(2, 1, 0).reshape(-1)
    step = np.array([1, K1, K1 * K1])
    tets = []
    for perm in itertools.permutations(range(3)):
        v0 = base
        v1 = v0 + step[perm[0]]
        v2 = v1 + step[perm[1]]
        v3 = v2 + step[perm[2]]
        # orientation on the reference hex: fix to positive volume
        e = np.eye(3)
        p1 = e[perm[0]]
        p2 = p1 + e[perm[1]]
        p3 = p2 + e[perm[2]]
        vol = np.linalg.det(np.stack([p1, p2, p3]))
        tets.append(np.stack([v0, v1, v2, v3] if vol > 0 else [v0, v2, v1, v3], axis=1))
    tets = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)
    return nodes, tets


def bottom_pins(nodes: np.ndarray, tol: float = 1e-12) -> np.ndarray:
    """Scalar dof indices of every node with z == 0 (all three components)."""
    bn = np.nonzero(np.abs(nodes[:, 2]) < tol)[0]
    return (3 * bn[:, None] + np.arange(3)[None, :]).reshape(-1).astype(np.int64)


def face_pins(nodes: np.ndarray, axis: int, value: float, tol: float = 1e-12) -> np.ndarray:
    bn = np.nonzero(np.abs(nodes[:, axis] - value) < tol)[0]
    return (3 * bn[:, None] + np.arange(3)[None, :]).reshape(-1).astype(np.int64)


def shape_gradients(nodes: np.ndarray, tets: np.ndarray):
    """Gradients of the 4 barycentric shape functions (ne,4,3) and volumes (ne,)."""
    X = nodes[tets]                                   # ne,4,3
    Dm = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)   # columns
    det = np.linalg.det(Dm)
    if np.any(det <= 0):
        raise ValueError("inverted or degenerate tetrahedron")
    Dinv = np.linalg.inv(Dm)                          # rows = grad N1..N3
    g = np.empty((tets.shape[0], 4, 3))
    g[:, 1:] = Dinv
    g[:, 0] = -Dinv.sum(axis=1)
    return g, det / 6.0


def linear_elastic_hessians(nodes, tets, E=1.0, nu=0.3) -> np.ndarray:
    """(ne, 12, 12) row-major P1 linear-elasticity stiffness matrices."""
    g, V = shape_gradients(nodes, tets)
    ne = tets.shape[0]
    lam, mu = lame(np.broadcast_to(E, (ne,)), np.broadcast_to(nu, (ne,)))
    gg = np.einsum("eai,ebi->eab", g, g)
    K = (lam[:, None, None, None, None] * np.einsum("eai,ebj->eaibj", g, g)
         + mu[:, None, None, None, None] * np.einsum("eaj,ebi->eaibj", g, g))
    K += (mu[:, None, None] * gg)[:, :, None, :, None] * np.eye(3)[None, None, :, None, :]
    K *= V[:, None, None, None, None]
    return np.ascontiguousarray(K.reshape(ne, 12, 12))


def fourier_displacement(nodes: np.ndarray, amplitude: float = 0.05, modes: int = 3, seed: int = 0):
    """Smooth displacement amplitude * mean_m d_m sin(2 pi k_m . X + phi_m) with seeded modes."""
    rng = np.random.default_rng(seed)
    u = np.zeros_like(nodes)
    for _ in range(modes):
        kvec = rng.integers(0, 2, size=3)
        if not kvec.any():
            kvec[rng.integers(0, 3)] = 1
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        phi = rng.uniform(0, 2 * math.pi)
        u += d[None, :] * np.sin(2 * math.pi * nodes @ kvec + phi)[:, None]
    return amplitude * u / modes


def neo_hookean_hessians(nodes, tets, u, E, nu, clamp: float = 1e-8, device: str | None = None) -> np.ndarray:
    """SPD-projected compressible Neo-Hookean element Hessians at displacement u (N,3)."""
    import torch
    g, V = shape_gradients(nodes, tets)
    ne = tets.shape[0]
    lam, mu = lame(np.broadcast_to(E, (ne,)), np.broadcast_to(nu, (ne,)))
    dev = torch.device(device) if device else torch.device("cpu")
    out = np.empty((ne, 12, 12))
    chunk = 1 << 16
    for s in range(0, ne, chunk):
        e = slice(s, min(ne, s + chunk))
        G = torch.as_tensor(g[e], device=dev)                               # m,4,3  (a, J)
        x = torch.as_tensor((nodes + u)[tets[e]], device=dev)               # m,4,3  (a, i)
        F = torch.einsum("mai,maJ->miJ", x, G)
        J = torch.linalg.det(F)
        if bool((J <= 0).any()):
            raise ValueError("inverted element in the deformed state")
        Finv = torch.linalg.inv(F)                                          # (J,i) layout: Finv[m,J,i]
        lnJ = torch.log(J)
        lm = torch.as_tensor(lam[e], device=dev)
        mm = torch.as_tensor(mu[e], device=dev)
        I3 = torch.eye(3, device=dev, dtype=F.dtype)
        # A[i,J,k,L] = mu d_ik d_JL + (mu - lam lnJ) Finv[J,k] Finv[L,i] + lam Finv[J,i] Finv[L,k]
        A = (mm[:, None, None, None, None] * torch.einsum("ik,JL->iJkL", I3, I3)[None]
             + (mm - lm * lnJ)[:, None, None, None, None] * torch.einsum("mJk,mLi->miJkL", Finv, Finv)
             + lm[:, None, None, None, None] * torch.einsum("mJi,mLk->miJkL", Finv, Finv))
        K = torch.einsum("maJ,miJkL,mbL->maibk", G, A, G).reshape(-1, 12, 12)
        K = K * torch.as_tensor(V[e], device=dev)[:, None, None]
        K = 0.5 * (K + K.transpose(1, 2))
        # SPD projection on the host (batched syevd from the CUDA math library
        # rejects these batch shapes on some driver/library combinations)
        Kc = K.cpu()
        w, Q = torch.linalg.eigh(Kc)
        w = torch.clamp(w, min=clamp)
        Kc = (Q * w[:, None, :]) @ Q.transpose(1, 2)
        Kc = 0.5 * (Kc + Kc.transpose(1, 2))
        out[e] = Kc.numpy()
    return out


def spherical_inclusions(centroids: np.ndarray, fraction: float = 0.3, seed: int = 0, radius=(0.05, 0.15)):
    """Boolean mask of elements whose centroid lies in a seeded random set of spheres
    covering about `fraction` of the unit cube."""
    rng = np.random.default_rng(seed)
    inside = np.zeros(centroids.shape[0], dtype=bool)
    while inside.mean() < fraction:
        c = rng.uniform(0, 1, size=3)
        r = rng.uniform(*radius)
        inside |= np.sum((centroids - c) ** 2, axis=1) <= r * r
    return inside


def element_centroids(nodes, tets):
    return nodes[tets].mean(axis=1)


def free_dofs(n_nodes: int, pins: np.ndarray) -> np.ndarray:
    mask = np.ones(3 * n_nodes, dtype=bool)
    mask[pins] = False
    return np.nonzero(mask)[0]
