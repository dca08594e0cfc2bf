"""Writes the golden fixtures used by the CPU tests.

known_answers.json: the integer known answers the reference's own tests pin for
this path (they hold no stored matrices or vectors):
  * factor nnz 43 with relaxation / 31 fundamental-only for the interleaved
    5-block native-ordering example (tests/test_native_ordering.cc:123-153);
  * child_rel_indices / num_child_diag_indices of a 3-supernode chain with
    sizes [d, 2d, d], degrees [2d, d, 0], structures {d, 3d} and {3d}
    (tests/test_catamari_factorizer.cc:299-343);
  * the MultiplyLowerBlock update with padded RHS columns
    (tests/test_catamari_solve_kernels.cc:33-51).
assembly_k2.npz: the oracle's sequential assembly of a 2x2x2 tet cube
(jitter 0.1, seed 3, E=1, nu=0.3), pinned so later oracle edits are caught.
Run: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

known = {
    "native_relaxed_example": {
        "block_size": 2, "num_blocks": 5, "edges": [[0, 3], [1, 2], [2, 4], [3, 4]],
        "factor_nnz_relaxed": 43, "factor_nnz_fundamental": 31,
        "source": "tests/test_native_ordering.cc:123-153",
    },
    "child_rel_indices": {
        "cases": [{"d": d, "sizes": [d, 2 * d, d], "degrees": [2 * d, d, 0],
                   "structure": [[d, 3 * d], [3 * d], []], "parents": [1, 2, -1],
                   "child_rel_indices": [0, 2 * d, 0], "num_child_diag_indices": [d, d, 0]}
                  for d in (1, 2, 3)],
        "source": "tests/test_catamari_factorizer.cc:299-343",
    },
    "multiply_lower_block": {
        "indices": [2], "lower_block": [2.0], "supernode_start": 1, "num_rhs": 3, "ld": 4,
        "rhs": [9, 1, 5, 99, 8, 3, 11, 99, 7, -2, 0, 99],
        "expected": [9, 1, 3, 99, 8, 3, 5, 99, 7, -2, 4, 99],
        "source": "tests/test_catamari_solve_kernels.cc:33-51",
    },
}

if __name__ == "__main__":
    with open(os.path.join(HERE, "known_answers.json"), "w") as fh:
        json.dump(known, fh, indent=1)
    from meshfemsparse_b200 import fem
    from oracle import pyoracle
    nodes, tets = fem.tet_cube(2, jitter=0.1, seed=3)
    Ap, Ai = pyoracle.build_pattern(nodes.shape[0], tets)
    Ke = fem.linear_elastic_hessians(nodes, tets, 1.0, 0.3)
    Ax = pyoracle.assemble(nodes.shape[0], Ap, Ai, tets, Ke)
    np.savez_compressed(os.path.join(HERE, "assembly_k2.npz"), nodes=nodes, tets=tets, Ke=Ke, Ap=Ap, Ai=Ai, Ax=Ax)
    print("wrote fixtures")
