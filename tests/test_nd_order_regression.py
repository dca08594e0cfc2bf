"""The host ordering is deterministic and unchanged by performance work: the inverse
permutations of tests/golden/nd_order_regression.npz (written by make_nd_order_fixture.py,
a regression pin of this library's own output) are reproduced exactly."""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))

from make_nd_order_fixture import orders   # noqa: E402


def test_orders_match_the_pinned_ones():
    pinned = np.load(HERE / "golden" / "nd_order_regression.npz")
    got = orders()
    assert set(pinned.files) == set(got)
    for k in pinned.files:
        assert np.array_equal(pinned[k], got[k]), k
