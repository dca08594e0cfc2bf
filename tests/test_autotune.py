"""Autotuner selection and on-disk cache (no GPU: the timing is injected)."""
from meshfemsparse_b200 import autotune

from helpers import grid_forest


def test_picks_fastest_and_caches(tmp_path):
    H = grid_forest(6)
    pins = [0, 1, 2]
    calls = []

    def fake(cut, tc):
        calls.append((cut, tc))
        return abs(cut - 128) + (0.5 if tc == 6 else 0.0)

    cache = tmp_path / "tune.json"
    r = autotune.tune(H, pins, None, None, None, single=True, refine=True, cache=cache, measure=fake)
    assert (r["small_front_max"], r["tensor_cores"]) == (128, 5) and not r["cached"]
    assert len(calls) == len(autotune.CUTOFFS_FP32) * 2
    r2 = autotune.tune(H, pins, None, None, None, single=True, refine=True, cache=cache, measure=fake)
    assert r2["cached"] and r2["small_front_max"] == 128 and len(calls) == len(autotune.CUTOFFS_FP32) * 2
    # another precision or other pins is another key
    r3 = autotune.tune(H, pins, None, None, None, single=False, refine=False, cache=cache, measure=fake)
    assert not r3["cached"] and r3["tensor_cores"] == 0
    r4 = autotune.tune(H, [3, 4, 5], None, None, None, single=True, refine=True, cache=cache, measure=fake)
    assert not r4["cached"]


def test_choose_form_keeps_the_faster_precision(tmp_path):
    H = grid_forest(5)
    fast64 = lambda single, cut, tc: (10.0 if single else 5.0) + cut / 1000.0
    r = autotune.choose_form(H, [0], None, None, None, cache=tmp_path / "a.json", measure=fast64)
    assert not r["singlePrecision"] and not r["refine"] and r["small_front_max"] == 64
    fast32 = lambda single, cut, tc: (3.0 if single else 5.0) + tc / 10.0
    r = autotune.choose_form(H, [1], None, None, None, cache=tmp_path / "b.json", measure=fast32)
    assert r["singlePrecision"] and r["refine"] and r["tensor_cores"] == 5


def test_schedule_shapes_are_tuned_when_asked(tmp_path):
    """factor_group and solve_subtrees join the search when more than one value is given,
    as another cache entry; a plain tune reports the defaults (0)."""
    H = grid_forest(6)
    calls = []

    def fake(cut, tc, group=None, sub=None):
        calls.append((cut, tc, group, sub))
        return abs(cut - 128) + (0.5 if tc == 6 else 0.0) + (0.0 if group == 8 else 0.3) + \
            (0.0 if sub == 12000 else 0.2)

    cache = tmp_path / "tune.json"
    plain = autotune.tune(H, [0], None, None, None, cache=cache, measure=fake)
    assert plain["factor_group"] == 0 and plain["solve_subtrees"] == 0
    assert all(c[2] is None for c in calls)
    calls.clear()
    r = autotune.tune(H, [0], None, None, None, cache=cache, measure=fake, factor_groups=(4, 8),
                      solve_subtrees=(0, 12000))
    assert not r["cached"] and (r["small_front_max"], r["tensor_cores"]) == (128, 5)
    assert (r["factor_group"], r["solve_subtrees"]) == (8, 12000)
    assert len(calls) == len(autotune.CUTOFFS_FP32) * 2 * 2 * 2
    again = autotune.tune(H, [0], None, None, None, cache=cache, measure=fake, factor_groups=(4, 8),
                          solve_subtrees=(0, 12000))
    assert again["cached"] and again["factor_group"] == 8
