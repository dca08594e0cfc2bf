"""Synthetic workloads of the benchmark configurations (seeded; no datasets).

1  20^3 hex cube -> 48,000 P1 tets, interior jitter +-0.1h, linear elastic E=1 nu=0.3,
   z=0 pinned, 1 RHS N(0,1), FP64.
2  64^3 cube -> 1,572,864 tets, compressible Neo-Hookean, per-element E log-uniform
   [0.1, 10], nu=0.35, Hessians at u = 0.05 * (3 seeded Fourier modes), per-element
   eigenvalue clamp 1e-8, 4 RHS.
3  256 independent cubes, side log-uniform so DOFs span 1k..50k, linear elastic with
   per-mesh E log-uniform [0.5, 2], nu U[0.25, 0.45], 8 RHS each (one block-diagonal system).
4  48^3 cube, Neo-Hookean E log-uniform [0.1, 10], nu=0.4; 30 load steps of a top-face
   compression ramp to 20% (fixed pattern, drifting values).
5  96^3 cube, linear elastic two-material 1e3 contrast by random spherical inclusions
   (30% volume fraction), nu=0.3, 32 RHS.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import fem
from .hessian import BlockCSCHessian, SystemAssembler


@dataclass
class Workload:
    name: str
    nodes: np.ndarray
    tets: np.ndarray
    Ke: np.ndarray
    pins: np.ndarray
    nrhs: int
    H: BlockCSCHessian
    rhs: np.ndarray                 # (n_full, nrhs), zero on pins
    info: dict = field(default_factory=dict)

    @property
    def n_full(self) -> int:
        return 3 * self.nodes.shape[0]


def _rhs(n_full: int, pins: np.ndarray, nrhs: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    b = rng.normal(size=(n_full, nrhs))
    b[pins] = 0.0
    return b


def config1(k: int = 20, seed: int = 1) -> Workload:
    nodes, tets = fem.tet_cube(k, jitter=0.1, seed=seed)
    Ke = fem.linear_elastic_hessians(nodes, tets, 1.0, 0.3)
    pins = fem.bottom_pins(nodes)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    return Workload(f"cube{k}_linear_elastic", nodes, tets, Ke, pins, 1, H, _rhs(3 * nodes.shape[0], pins, 1, seed + 100),
                    dict(k=k, tets=int(tets.shape[0]), material="linear elastic E=1 nu=0.3"))


def config2(k: int = 64, seed: int = 2, device: str | None = None) -> Workload:
    nodes, tets = fem.tet_cube(k, jitter=0.0, seed=seed)
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=tets.shape[0]))
    u = fem.fourier_displacement(nodes, amplitude=0.05, modes=3, seed=seed)
    Ke = fem.neo_hookean_hessians(nodes, tets, u, E, 0.35, clamp=1e-8, device=device)
    pins = fem.bottom_pins(nodes)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    return Workload(f"cube{k}_neo_hookean", nodes, tets, Ke, pins, 4, H, _rhs(3 * nodes.shape[0], pins, 4, seed + 100),
                    dict(k=k, tets=int(tets.shape[0]), material="Neo-Hookean E~logU[0.1,10] nu=0.35"))


def config5(k: int = 96, seed: int = 5) -> Workload:
    nodes, tets = fem.tet_cube(k, jitter=0.0, seed=seed)
    inc = fem.spherical_inclusions(fem.element_centroids(nodes, tets), 0.3, seed=seed)
    E = np.where(inc, 1e3, 1.0)
    Ke = fem.linear_elastic_hessians(nodes, tets, E, 0.3)
    pins = fem.bottom_pins(nodes)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    return Workload(f"cube{k}_two_material", nodes, tets, Ke, pins, 32, H, _rhs(3 * nodes.shape[0], pins, 32, seed + 100),
                    dict(k=k, tets=int(tets.shape[0]), material="linear elastic, 1e3 contrast inclusions"))


def config3(count: int = 256, seed: int = 3, dof_range=(1000, 50000)) -> Workload:
    """Block-diagonal batch of independent cubes of uneven size."""
    rng = np.random.default_rng(seed)
    # free DOFs of a side-k cube with z=0 pinned: 3 k (k+1)^2
    kmin = next(k for k in range(2, 100) if 3 * k * (k + 1) ** 2 >= dof_range[0])
    kmax = max(k for k in range(2, 100) if 3 * k * (k + 1) ** 2 <= dof_range[1])
    ks = np.round(np.exp(rng.uniform(math.log(kmin), math.log(kmax), size=count))).astype(int)
    all_nodes, all_tets, all_Ke, all_pins = [], [], [], []
    off = 0
    for m, k in enumerate(ks):
        nodes, tets = fem.tet_cube(int(k), jitter=0.1, seed=seed + m)
        E = math.exp(rng.uniform(math.log(0.5), math.log(2.0)))
        nu = rng.uniform(0.25, 0.45)
        all_Ke.append(fem.linear_elastic_hessians(nodes, tets, E, nu))
        all_tets.append(tets + off)
        all_pins.append(fem.bottom_pins(nodes) + 3 * off)
        all_nodes.append(nodes)
        off += nodes.shape[0]
    nodes = np.concatenate(all_nodes)
    tets = np.concatenate(all_tets)
    Ke = np.concatenate(all_Ke)
    pins = np.concatenate(all_pins)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    return Workload(f"batch{count}_cubes", nodes, tets, Ke, pins, 8, H, _rhs(3 * nodes.shape[0], pins, 8, seed + 100),
                    dict(count=count, sides=ks.tolist(), tets=int(tets.shape[0])))


def compression_displacement(nodes: np.ndarray, strain: float, nu: float = 0.4, seed: int = 0,
                             amplitude: float = 0.01) -> np.ndarray:
    """Top-face compression by `strain` (z=0 fixed): u = s [nu (x-1/2) z, nu (y-1/2) z, -z]
    plus a seeded smooth perturbation that grows with the load and vanishes at z=0. A
    stand-in for the equilibrium states of the load ramp (the Hessians are inputs)."""
    z = nodes[:, 2]
    u = np.zeros_like(nodes)
    u[:, 0] = nu * strain * (nodes[:, 0] - 0.5) * z
    u[:, 1] = nu * strain * (nodes[:, 1] - 0.5) * z
    u[:, 2] = -strain * z
    pert = fem.fourier_displacement(nodes, amplitude=amplitude, modes=3, seed=seed)
    return u + (strain / 0.2) * pert * z[:, None]


@dataclass
class NewtonSequence:
    """Config 4: one mesh and material, Hessians that drift with the load on a fixed pattern."""
    wl: Workload
    E: np.ndarray
    nu: float
    steps: int
    max_strain: float
    seed: int

    def strain(self, t: int) -> float:
        return self.max_strain * t / self.steps

    def hessians(self, strain: float, seed: int | None = None, device: str | None = None) -> np.ndarray:
        u = compression_displacement(self.wl.nodes, strain, 0.4, self.seed if seed is None else seed)
        return fem.neo_hookean_hessians(self.wl.nodes, self.wl.tets, u, self.E, self.nu, clamp=1e-8, device=device)


def newton_sequence(k: int = 48, seed: int = 4, steps: int = 30, device: str | None = None,
                    final_hessians: bool = True) -> NewtonSequence:
    """48^3 cube, Neo-Hookean E log-uniform [0.1, 10], nu = 0.4, `steps` load steps of a
    top-face compression ramp to 20%; one right-hand side per Newton step."""
    nodes, tets = fem.tet_cube(k, jitter=0.0, seed=seed)
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(math.log(0.1), math.log(10.0), size=tets.shape[0]))
    pins = fem.bottom_pins(nodes)
    H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
    wl = Workload(f"cube{k}_neo_hookean_compression", nodes, tets, np.zeros((0, 12, 12)), pins, 1, H,
                  _rhs(3 * nodes.shape[0], pins, 1, seed + 100),
                  dict(k=k, tets=int(tets.shape[0]), material="Neo-Hookean E~logU[0.1,10] nu=0.4",
                       load_steps=steps, max_strain=0.2))
    seq = NewtonSequence(wl, E, 0.4, steps, 0.2, seed)
    if final_hessians:
        wl.Ke = seq.hessians(seq.strain(steps), device=device)
    return seq


def config4(k: int = 48, seed: int = 4, device: str | None = None) -> Workload:
    return newton_sequence(k, seed, device=device).wl


def build(cfg: int, k: int | None = None, device: str | None = None) -> Workload:
    if cfg == 1:
        return config1(k or 20)
    if cfg == 2:
        return config2(k or 64, device=device)
    if cfg == 3:
        return config3()
    if cfg == 4:
        return config4(k or 48, device=device)
    if cfg == 5:
        return config5(k or 96)
    raise ValueError(f"unknown configuration {cfg}")
