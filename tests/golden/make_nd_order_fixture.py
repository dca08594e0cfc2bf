"""Writes nd_order_regression.npz: the inverse permutations the host analysis gives for
two jittered cubes (sides 6 and 12, bottom pins) and a batch of four meshes. A
regression pin of this library's own ordering (not a reference artefact): changes meant
to be pure speedups of the nested dissection must leave it unchanged.

    python tests/golden/make_nd_order_fixture.py
"""
from pathlib import Path

import numpy as np

from meshfemsparse_b200 import B200Factorizer, SystemAssembler, fem, workloads


def orders():
    out = {}
    for k in (6, 12):
        nodes, tets = fem.tet_cube(k, jitter=0.1, seed=k)
        H = SystemAssembler(nodes.shape[0]).blockSparsityPattern(tets)
        f = B200Factorizer(device=-1)
        f.factorizeSymbolic(H, fem.bottom_pins(nodes))
        out[f"cube{k}"] = f.getInversePermutation()
    wl = workloads.config3(count=4, seed=7, dof_range=(800, 3000))
    f = B200Factorizer(device=-1)
    f.factorizeSymbolic(wl.H, wl.pins)
    out["batch4"] = f.getInversePermutation()
    return out


if __name__ == "__main__":
    np.savez_compressed(Path(__file__).with_name("nd_order_regression.npz"), **orders())
